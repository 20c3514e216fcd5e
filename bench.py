#!/usr/bin/env python
"""Benchmark of the particle-push hot path on B200 (one JSON line on rank 0).

Workload (default): the gridded-Boris configuration -- 1e6 protons in a 128^3
periodic turbulent E/B field (float32 nodes, trilinear), dt = T_gyro(B0)/50,
1e4 time steps, saves every 1000 steps.  One bench step is one complete solve
of that workload (1e10 particle-steps) with the initial states already in HBM;
`value` is particle-steps/s of the FP32-compensated push, the FP64 drop-in
path and the FP32C error against it are reported beside it.  `e2e` is the
same solve through the public API (solve() with host arrays: the upload of the
initial states and the download of every saved state are inside the timing).

--impl reference times the CPU restatement of the reference's EnsembleThreads
path (oracle/, OpenMP on all host cores) on a bounded sample of the same
workload: the reference itself is Julia, which is not available here.

Multi-GPU: particles are independent; each rank runs its own replica of the
workload (weak scaling, no collective on the data path); the time is the max
over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import __graft_entry__ as ge  # noqa: E402

BYTES_PER_PARTICLE_STEP = 192  # 8 trilinear corners x (E, B) x 3 float32
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def _peaks():
    try:
        p = json.loads(PEAKS_FILE.read_text())
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _workload(tp, name: str, n: int, nt: int = 10_000):
    if name == "config2":
        return tp.workloads.config2(n=n, nt=nt, ssi=min(1000, nt))
    if name == "config3":
        return tp.workloads.config3(n=n, nt=nt, ssi=min(1000, nt))
    if name == "config1":
        w = tp.workloads.config1(n=n)
        if nt != 10_000:
            w.tspan = (0.0, nt * w.dt)
        return w
    raise SystemExit(f"unknown workload {name}")


def _alg(tp, name):
    return tp.MultistepBoris4(2) if name == "config3" else tp.Boris()


def cpu_rate(tp, orc, w, alg, sample: int, nthreads: int = 0):
    """Particle-steps/s of the oracle's OpenMP ensemble on the first `sample` particles."""
    sub = tp.TraceProblem(w.u0[:, :sample].copy(), w.tspan, tp.prepare(w.E, w.B, species=w.species))
    dt = w.dt if np.ndim(w.dt) == 0 else np.asarray(w.dt)[:sample]
    tend = None if w.tend is None else np.asarray(w.tend)[:sample]
    plan = tp.plan_boris(sub, alg, tp.EnsembleB200(), dt=dt, tend=tend, savestepinterval=w.savestepinterval,
                         isoutside=w.isoutside)
    t0 = time.perf_counter()
    r = orc.boris_run(plan.desc, plan.E, plan.B, plan.u0, plan.dt_i, plan.tend_i, nthreads=nthreads)
    el = time.perf_counter() - t0
    return float(r.nsteps.sum()) / el, el, int(r.nsteps.sum())


def run_reference(args):
    world, rank, _ = _dist()
    if rank != 0:
        return
    tp = ge.load_package()
    orc = ge.load_oracle()
    w = _workload(tp, args.workload, args.sample, args.nt)
    alg = _alg(tp, args.workload)
    cores = orc.max_threads()
    rates = []
    for k in range(args.warmup + args.steps):
        rate, el, ps = cpu_rate(tp, orc, w, alg, args.sample)
        if k >= args.warmup:
            rates.append((rate, el, ps))
    tot_ps = sum(r[2] for r in rates)
    tot_t = sum(r[1] for r in rates)
    value = tot_ps / tot_t
    line = {
        "impl": "reference", "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot_t / len(rates), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded SplitMix64)",
        "config": {"workload": w.name, "particles_per_step": args.sample, "time_steps": w.nt,
                   "precision": "fp64 (reference order)"},
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores, "kind": "port",
                         "sample": f"{args.sample} of the workload's particles x {w.nt} steps per step; "
                                   "C++ restatement of the reference EnsembleThreads path (Julia absent)"},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="config2", choices=["config1", "config2", "config3"])
    ap.add_argument("--particles", type=int, default=1_000_000)
    ap.add_argument("--sample", type=int, default=4000, help="particles of the CPU legs")
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--nt", type=int, default=10_000, help="time steps (reduced only for profiling)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    tp = ge.load_package()
    ctx = tp.Context.get(local)
    w = _workload(tp, args.workload, args.particles, args.nt)
    alg = _alg(tp, args.workload)
    n = w.n
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    def plan(prec):
        prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
        return tp.plan_boris(prob, alg, tp.EnsembleB200(device=local, precision=prec), dt=w.dt, tend=w.tend,
                             savestepinterval=w.savestepinterval, isoutside=w.isoutside)

    p32, p64 = plan("fp32c"), plan("fp64")
    nslots = ctx.slots(p32.desc, n, p32.dt_i, p32.tend_i)
    W = 6
    u0_d = torch.from_numpy(p32.u0).to(dev)
    dti_d = None if p32.dt_i is None else torch.from_numpy(p32.dt_i).to(dev)
    tend_d = None if p32.tend_i is None else torch.from_numpy(p32.tend_i).to(dev)
    t_out = torch.empty((nslots, n), dtype=torch.float64, device=dev)
    u_out = torch.empty((nslots, W, n), dtype=torch.float64, device=dev)
    nsaved = torch.empty(n, dtype=torch.int32, device=dev)
    retc = torch.empty(n, dtype=torch.int8, device=dev)
    nsteps = torch.empty(n, dtype=torch.int64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2

    def ptr(t):
        return None if t is None else t.data_ptr()

    def launch(p):
        ctx.boris_run_device(p.desc, p.E, p.B, ptr(u0_d), ptr(dti_d), ptr(tend_d), n, nslots, ptr(t_out),
                             ptr(u_out), ptr(nsaved), ptr(retc), ptr(nsteps), ptr(status), sptr)

    def timed(p, k, warm):
        for _ in range(warm):
            launch(p)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        evs = []
        for _ in range(k):
            flush.zero_()  # L2 flush between timed iterations (outside the events)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            launch(p)
            b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ms = [a.elapsed_time(b) for a, b in evs]
        tot = torch.tensor([sum(ms)], dtype=torch.float64, device=dev)
        if dist:
            dist.all_reduce(tot, op=dist.ReduceOp.MAX)
        if int(status.item()) != 0:
            raise SystemExit(f"kernel status {int(status.item())}")
        return float(tot.item()), ms

    # ---- FP32C (headline), clocks sampled during the timed region
    sampler = ClockSampler(local)
    status.zero_()
    launch(p32)  # first call builds the interleaved field table
    torch.cuda.synchronize()
    sampler.start()
    tot32, ms32 = timed(p32, args.steps, args.warmup)
    clocks = sampler.stop()
    ps_step = float(nsteps.sum().item())
    fs32 = _final_states(tp, t_out, u_out, nsaved, n)

    # ---- FP64 drop-in path on the same workload
    status.zero_()
    tot64, ms64 = timed(p64, max(args.fp64_steps, 1), 1)
    ps64 = float(nsteps.sum().item())
    fs64 = _final_states(tp, t_out, u_out, nsaved, n)
    err = _rel_err(fs32, fs64)
    # the same float64 solve started 1 ulp away: how fast neighbouring orbits
    # separate in this field (chaotic flows separate at any precision)
    u0_saved = u0_d.clone()
    u0_d.mul_(1.0 + 2.0 ** -52)
    launch(p64)
    torch.cuda.synchronize()
    fs64b = _final_states(tp, t_out, u_out, nsaved, n)
    u0_d.copy_(u0_saved)
    chaos = _rel_err(fs64b, fs64)

    value = world * ps_step * args.steps / (tot32 * 1e-3)
    value64 = world * ps64 * max(args.fp64_steps, 1) / (tot64 * 1e-3)
    kernel_s = tot32 * 1e-3 / args.steps
    peak, peak_kind = _peaks()
    achieved = BYTES_PER_PARTICLE_STEP * ps_step / kernel_s / 1e9

    # ---- end to end through the public API (host arrays in, packed host results out)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    e2e_t = []
    h2d = d2h = 0
    for k in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sol = tp.solve(prob, alg, tp.EnsembleB200(device=local, precision="fp32c"), dt=w.dt, tend=w.tend,
                       savestepinterval=w.savestepinterval, isoutside=w.isoutside)
        el = time.perf_counter() - t0
        if k > 0:
            e2e_t.append(el)
        h2d = w.u0.nbytes + (0 if w.tend is None else np.asarray(w.tend).nbytes) + \
            (0 if np.ndim(w.dt) == 0 else np.asarray(w.dt).nbytes)
        d2h = sol.t_all.nbytes + sol.u_all.nbytes + sol.nsaved.nbytes + sol.retcodes.nbytes + sol.nsteps.nbytes
    e2e_value = None
    if e2e_t:
        e2e_time = max(e2e_t)
        if dist:
            tt = torch.tensor([e2e_time], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e2e_time = float(tt.item())
        e2e_value = world * float(sol.nsteps.sum()) / e2e_time

    line = None
    if rank == 0:
        cpu = None
        if not args.no_cpu:
            orc = ge.load_oracle()
            rate, el, ps = cpu_rate(tp, orc, w, alg, args.sample)
            cpu = {"value": rate, "unit": "particle-steps/s", "cores": orc.max_threads(), "kind": "port",
                   "sample": f"{args.sample} particles x {w.nt} steps of the same workload, FP64 reference "
                             f"order, {el:.1f} s (C++ restatement of the reference EnsembleThreads path)"}
        line = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot32 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+compensated",
            "data": "synthetic (seeded SplitMix64)",
            "config": {"workload": w.name, "particles": n, "time_steps": w.nt,
                       "savestepinterval": w.savestepinterval, "precision": "fp32c",
                       "inputs_in_hbm": True, "l2": "flushed between timed steps (256 MB write)",
                       "parallelism": f"replicas x{world}"},
            "fp64": {"value": value64, "unit": "particle-steps/s", "ms_per_step": tot64 / args.fp64_steps,
                     "speedup_fp32c_over_fp64": value / value64},
            "fp32c_error_vs_fp64": _err_summary(err),
            "fp64_vs_fp64_1ulp_start": _err_summary(chaos),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "note": f"{BYTES_PER_PARTICLE_STEP} algorithmic B/particle-step; peak {peak_kind}; "
                                 "the 50 MB field table is L2-resident, so frac > 1 is possible"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": args.steps,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def _rel_err(a, b):
    """|x_a - x_b| / |x_b| of final positions, finite entries only."""
    e = np.linalg.norm(a[:, :3] - b[:, :3], axis=1) / np.linalg.norm(b[:, :3], axis=1)
    return e[np.isfinite(e)]


def _err_summary(e):
    if e.size == 0:
        return None
    return {"final_position_rel_median": float(np.median(e)), "p90": float(np.quantile(e, 0.9)),
            "p99": float(np.quantile(e, 0.99)), "max": float(e.max())}


def _final_states(tp, t_out, u_out, nsaved, n):
    ns = nsaved.to("cpu").numpy().astype(np.int64)
    u = u_out.to("cpu").numpy()
    idx = np.clip(ns - 1, 0, u.shape[0] - 1)
    return u[idx, :, np.arange(n)]


if __name__ == "__main__":
    main()
