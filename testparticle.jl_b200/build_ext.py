"""Build libtpb200.so (the CUDA library behind include/tp_abi.h) in-tree.

Every translation unit is compiled for sm_100a only.  The float64 kernels
(boris_fp64.cu, gc_fp64.cu, hybrid.cu, detect.cu) are compiled with -fmad=false so that their
arithmetic follows the reference's operation order; the float32 kernels use
contraction.  Objects are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libtpb200.so"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}"]
NO_FMAD = {"boris_fp64.cu", "gc_fp64.cu", "hybrid.cu", "detect.cu"}
SOURCES = ["runtime.cu", "pack.cu", "boris_fp64.cu", "boris_fp32c.cu", "gc_fp64.cu", "gc_fp32.cu", "adjoint.cu",
           "noalloc.cu", "hybrid.cu", "detect.cu"]


def _nvcc() -> str:
    cand = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "bin" / "nvcc"
    return str(cand) if cand.exists() else "nvcc"


def _headers() -> list[Path]:
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))


def _compile(src: str, verbose_ptxas: bool) -> Path:
    s = CSRC / src
    o = BUILD / (src + ".o")
    newest = max([s.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    if o.exists() and o.stat().st_mtime >= newest and not verbose_ptxas:
        return o
    cmd = [_nvcc(), *ARCH, *COMMON, "-c", str(s), "-o", str(o)]
    cmd.append("-fmad=false" if src in NO_FMAD else "-fmad=true")
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas:
        sys.stderr.write(r.stderr)
    return o


def build(verbose_ptxas: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), SOURCES))
    newest = max(o.stat().st_mtime for o in objs)
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [_nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv))
