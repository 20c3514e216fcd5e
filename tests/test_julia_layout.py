"""The Julia binding's descriptor structs against the C header, byte for byte.

Julia is not installed here, so the binding in
testparticle.jl_b200/julia/TestParticleB200/src/TestParticleB200.jl cannot
run.  What a wrong binding would get wrong first is the memory layout of the
descriptors it passes by reference to ccall.  Julia lays out an isbits struct
like C (natural alignment, fields in order), so this test parses each
`struct Tp*Desc` of the binding, computes that layout, and compares every
field's name, offset and size, and the struct's size, with what gcc reports
for the matching struct of include/tp_abi.h (offsetof / sizeof).
"""
from __future__ import annotations

import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
JL = ROOT / "testparticle.jl_b200" / "julia" / "TestParticleB200" / "src" / "TestParticleB200.jl"
HDR = ROOT / "include" / "tp_abi.h"

PAIRS = [("TpFieldDesc", "tp_field_desc"), ("TpTermDesc", "tp_term_desc"), ("TpRunDesc", "tp_run_desc"),
         ("TpGCDesc", "tp_gc_desc"), ("TpAdjDesc", "tp_adj_desc")]

PRIM = {"Int32": (4, 4), "Int64": (8, 8), "Float64": (8, 8), "Cint": (4, 4), "Cdouble": (8, 8)}


def _julia_structs(src: str) -> dict:
    out = {}
    for m in re.finditer(r"^struct (Tp\w+)[^\n]*\n(.*?)^end", src, re.S | re.M):
        fields = []
        for line in m.group(2).splitlines():
            line = line.split("#", 1)[0]
            for part in line.split(";"):
                part = part.strip()
                if "::" in part:
                    name, typ = (x.strip() for x in part.split("::", 1))
                    fields.append((name, typ))
        out[m.group(1)] = fields
    return out


def _jl_size_align(typ: str, structs: dict, memo: dict):
    if typ in PRIM:
        return PRIM[typ]
    if typ.startswith("Ptr{") or typ == "Ptr":
        return 8, 8
    m = re.fullmatch(r"NTuple\{(\d+),\s*(.+)\}", typ)
    if m:
        s, a = _jl_size_align(m.group(2), structs, memo)
        return int(m.group(1)) * s, a
    if typ in structs:
        lay = _jl_layout(typ, structs, memo)
        return lay["size"], lay["align"]
    raise AssertionError(f"unknown Julia field type {typ}")


def _jl_layout(name: str, structs: dict, memo: dict) -> dict:
    if name in memo:
        return memo[name]
    off, align, fields = 0, 1, []
    for fname, typ in structs[name]:
        s, a = _jl_size_align(typ, structs, memo)
        off = (off + a - 1) // a * a
        fields.append((fname, off, s))
        off += s
        align = max(align, a)
    lay = {"fields": fields, "size": (off + align - 1) // align * align, "align": align}
    memo[name] = lay
    return lay


def _c_members(hdr: str, cname: str) -> list:
    m = re.search(r"typedef struct " + cname + r" \{(.*?)\} " + cname + ";", hdr, re.S)
    assert m, cname
    body = re.sub(r"/\*.*?\*/", "", m.group(1), flags=re.S)
    names = []
    for stmt in body.split(";"):
        stmt = " ".join(stmt.split())
        if not stmt:
            continue
        # "type a, b[3]" or "const T* x[3]": declarators after the type
        first, *rest = stmt.split(",")
        decl0 = first.split()[-1].lstrip("*")
        for d in [decl0] + [r.strip().lstrip("*") for r in rest]:
            names.append(re.sub(r"\[.*\]", "", d))
    return names


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    hdr = HDR.read_text()
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "tp_abi.h"', "int main(void) {"]
    members = {}
    for _, c in PAIRS:
        members[c] = _c_members(hdr, c)
        lines.append(f'printf("S {c} %zu\\n", sizeof({c}));')
        for f in members[c]:
            lines.append(f'printf("F {c} {f} %zu %zu\\n", offsetof({c}, {f}), sizeof((({c}*)0)->{f}));')
    lines += ["return 0;", "}"]
    d = tmp_path_factory.mktemp("layout")
    (d / "l.c").write_text("\n".join(lines))
    subprocess.run([gcc, "-std=c99", f"-I{HDR.parent}", "-o", str(d / "l"), str(d / "l.c")], check=True)
    out = subprocess.run([str(d / "l")], check=True, capture_output=True, text=True).stdout
    lay = {c: {"fields": [], "size": None} for _, c in PAIRS}
    for line in out.splitlines():
        k = line.split()
        if k[0] == "S":
            lay[k[1]]["size"] = int(k[2])
        else:
            lay[k[1]]["fields"].append((k[2], int(k[3]), int(k[4])))
    return lay


@pytest.mark.parametrize("jl,c", PAIRS)
def test_julia_descriptor_matches_header(c_layout, jl, c):
    structs = _julia_structs(JL.read_text())
    assert jl in structs, f"{jl} not found in the Julia binding"
    lay = _jl_layout(jl, structs, {})
    cl = c_layout[c]
    assert [f[0] for f in lay["fields"]] == [f[0] for f in cl["fields"]], "field names / order differ"
    assert lay["fields"] == cl["fields"], "field offsets or sizes differ"
    assert lay["size"] == cl["size"]


def test_integration_doc_lists_the_run_descriptor_in_full():
    """The TpRunDesc listing a maintainer would copy from INTEGRATION.md."""
    doc = (ROOT / "INTEGRATION.md").read_text()
    m = re.search(r"struct TpRunDesc.*?\nend", doc, re.S)
    assert m
    structs = _julia_structs(m.group(0) + "\n")
    full = _julia_structs(JL.read_text())
    assert structs["TpRunDesc"] == full["TpRunDesc"]
