#!/usr/bin/env python
"""Benchmark of the particle-push hot path on B200 (one JSON line on rank 0).

Workload (default): the Earth-dipole ensemble -- 1e6 protons, kinetic energy
log-uniform 10 keV - 10 MeV, isotropic pitch angles, L uniform in [3, 7],
MultistepBoris4(n=2) at dt_i = 0.02 T_gyro(|B(r0)|), 1e4 steps, termination
at 1 and 15 R_E, saves every 1000 steps.  One bench step is one complete
solve of that workload (up to 1e10 particle-steps) with the initial states
already in HBM; `value` is particle-steps/s of the FP32-compensated push
(float rotation factors, compensated float positions, float64 field and
velocity).  Beside it: the plain FP64 drop-in path on the same workload, the
FP32C final-position error against it, and how far float64 runs started a
float32 ulp (and a float64 ulp) away separate -- the orbits' own
sensitivity, which classifies them into regular and chaotic ones.  `e2e` is
the same solve through the public API (solve() with host arrays: the upload
of the initial states, dt and tspan, and the download of every saved state
are inside the timing).  `--workload config2` makes the gridded turbulent
field (128^3, 1e6 protons, 1e4 Boris steps) the headline instead; by default
it is a leg.

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

# gridded workload (config 2): algorithmic bytes of one particle-step, 8
# trilinear corners x (E, B) x 3 float32, and the DRAM bytes per particle-step
# of k_fixed32c measured by ncu (1.683 GB over 2e8 particle-steps; the 67 MB
# field table is L2-resident)
BYTES_PER_PARTICLE_STEP = 192
TRAFFIC_PER_PARTICLE_STEP = 8.4
# dipole workload (config 3, MultistepBoris4(2)): algorithmic flops of one
# particle-step (the rotation 121, the dipole 29), and the warp instructions
# one warp-step of k_fixed32c<MULTI, queue, analytic> issues and the DRAM
# bytes per particle-step, both measured by ncu on 262144 protons x 200 steps
FLOPS_PER_PARTICLE_STEP_DIPOLE = 150
INST_PER_WARP_STEP_DIPOLE = 340.8
TRAFFIC_PER_PARTICLE_STEP_DIPOLE = 0.32
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
SMS = 148
ISSUE_PER_SM_CLOCK = 4  # one warp instruction per clock on each of the four SM sub-partitions


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


def max_over_ranks(dist, value: float, device) -> float:
    """The job's time is its slowest rank's: the maximum of `value` over ranks
    (every rank calls this at the same point; identity without a process group)."""
    if not dist:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, units_per_rank: float, seconds: float) -> float:
    """Whole-job throughput of `world` replicas that each processed
    `units_per_rank` units, the slowest finishing after `seconds`."""
    return world * float(units_per_rank) / float(seconds)


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


class DeviceRun:
    """Device buffers of one full-orbit workload, launched through tp_boris_run_device."""

    def __init__(self, tp, torch, ctx, plan, dev, stream):
        self.tp, self.torch, self.ctx = tp, torch, ctx
        self.n = n = plan.u0.shape[0]
        self.nslots = ctx.slots(plan.desc, n, plan.dt_i, plan.tend_i)
        if self.nslots < 0:
            raise SystemExit("bench runs need a bounded number of saves (set step_cap for adaptive runs)")
        W = 6 + 6 * bool(plan.desc.save_fields) + 4 * bool(plan.desc.save_work)
        f = lambda a: None if a is None else torch.from_numpy(a).to(dev)  # noqa: E731
        self.u0, self.dt_i, self.tend_i = f(plan.u0), f(plan.dt_i), f(plan.tend_i)
        self.t_out = torch.empty((self.nslots, n), dtype=torch.float64, device=dev)
        self.u_out = torch.empty((self.nslots, W, n), dtype=torch.float64, device=dev)
        self.nsaved = torch.empty(n, dtype=torch.int32, device=dev)
        self.retc = torch.empty(n, dtype=torch.int8, device=dev)
        self.nsteps = torch.empty(n, dtype=torch.int64, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.stream = stream

    def launch(self, plan):
        p = lambda t: None if t is None else t.data_ptr()  # noqa: E731
        self.ctx.boris_run_device(plan.desc, plan.E, plan.B, p(self.u0), p(self.dt_i), p(self.tend_i), self.n,
                                  self.nslots, p(self.t_out), p(self.u_out), p(self.nsaved), p(self.retc),
                                  p(self.nsteps), p(self.status), self.stream.cuda_stream)

    def check(self):
        st = int(self.status.item())
        if st != 0:
            raise SystemExit(f"kernel status {st}")

    def final_states(self):
        ns = self.nsaved.to("cpu").numpy().astype(np.int64)
        u = self.u_out.to("cpu").numpy()
        idx = np.clip(ns - 1, 0, u.shape[0] - 1)
        return u[idx, :, np.arange(self.n)]

    def particle_steps(self):
        return float(self.nsteps.sum().item())


def timed(torch, dist, dev, run, plan, k, warm, flush):
    """k launches bracketed by barrier + synchronize; device time (ms), max over ranks."""
    for _ in range(warm):
        run.launch(plan)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    evs = []
    for _ in range(k):
        flush.zero_()  # L2 flush between timed iterations (outside the events)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(run.stream)
        run.launch(plan)
        b.record(run.stream)
        evs.append((a, b))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    tot = max_over_ranks(dist, sum(a.elapsed_time(b) for a, b in evs), dev)
    run.check()
    return tot


def _plan(tp, w, alg, prec, device, step_cap=0):
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    return tp.plan_boris(prob, alg, tp.EnsembleB200(device=device, precision=prec), dt=w.dt, tend=w.tend,
                         savestepinterval=w.savestepinterval, isoutside=w.isoutside, step_cap=step_cap)


def leg_dipole(tp, torch, ctx, dist, dev, stream, flush, world, n, nt, multistep=True):
    """Dipole ensemble (config 3): AdaptiveBoris(0.1) (and MultistepBoris4(n=2)
    when it is not the headline), FP32C vs FP64."""
    w = tp.workloads.config3(n=n, nt=nt, ssi=min(1000, nt))
    out = {"workload": w.name, "particles": n, "time_steps": nt}
    cases = [("adaptive_0.1", tp.AdaptiveBoris(0.1), nt)]
    if multistep:
        cases.insert(0, ("multistep4_n2", tp.MultistepBoris4(2), 0))
    for name, alg, cap in cases:
        p32, p64 = _plan(tp, w, alg, "fp32c", ctx.device, cap), _plan(tp, w, alg, "fp64", ctx.device, cap)
        shapes = {k: ctx.autotune(pl.desc, pl.E, pl.B, pl.u0, max_steps=200) for k, pl in (("fp32c", p32),
                                                                                          ("fp64", p64))}
        run = DeviceRun(tp, torch, ctx, p32, dev, stream)
        ms32 = timed(torch, dist, dev, run, p32, 1, 1, flush)
        ps32 = run.particle_steps()
        fs32, rc32 = run.final_states(), run.retc.cpu().numpy()
        ms64 = timed(torch, dist, dev, run, p64, 1, 1, flush)
        ps64 = run.particle_steps()
        fs64, rc64 = run.final_states(), run.retc.cpu().numpy()
        # float64 started 1 ulp away: the orbits' own sensitivity
        u0_saved = run.u0.clone()
        run.u0.mul_(1.0 + 2.0 ** -52)
        run.launch(p64)
        torch.cuda.synchronize()
        fs64b, rc64b = run.final_states(), run.retc.cpu().numpy()
        run.u0.copy_(u0_saved)
        ok = (rc32 == 1) & (rc64 == 1)
        okb = (rc64b == 1) & (rc64 == 1)
        v32, v64 = whole_job_rate(world, ps32, ms32 * 1e-3), whole_job_rate(world, ps64, ms64 * 1e-3)
        out[name] = {"fp32c": v32, "fp64": v64, "speedup_fp32c_over_fp64": v32 / v64,
                     "unit": "particle-steps/s", "fp32c_error_vs_fp64": _err_summary(_rel_err(fs32[ok], fs64[ok])),
                     "fp64_vs_fp64_1ulp_start": _err_summary(_rel_err(fs64b[okb], fs64[okb])),
                     "both_success_fraction": float(ok.mean()), "autotune": shapes}
    return out


def leg_adjoint(tp, torch, ctx, dev, stream, flush, n=1 << 18, nt=4096, K=0, reps=3, compare_k=64):
    """Discrete adjoint of Boris in the gridded field (config 5): forward with
    checkpoints, backward, and the plain FP32C push of the same workload, each
    timed on the device.  K = 0 takes the library's automatic segment length
    (2 steps: the one-kernel backward); the same problem with `compare_k`-step
    segments (two kernels per segment) is timed beside it."""
    w = tp.workloads.config5(n=n, nt=nt)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    # targets: the float64 endpoints (library FP64 path) plus seeded offsets
    sol64 = tp.solve(prob, tp.Boris(), tp.EnsembleB200(device=ctx.device, precision="fp64"), dt=w.dt,
                     savestepinterval=10 ** 9, save_start=False)
    x_target = torch.from_numpy(sol64.final_states()[:, :3] + w.extra["target_offset"]).to(dev)
    del sol64
    s = stream.cuda_stream
    nodes = int(np.prod(w.B.data.shape[1:]))
    gE = torch.empty(3 * nodes, dtype=torch.float64, device=dev)
    gB = torch.empty_like(gE)
    gp = torch.empty(6, dtype=torch.float64, device=dev)

    def device_ms(fn, *args):
        fn(*args)  # warm-up (first backward allocates the records and tables)
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(reps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn(*args)
            b.record(stream)
            torch.cuda.synchronize()
            tot += a.elapsed_time(b)
        return tot / reps

    def run_tape(k):
        plan = tp.plan_adjoint(prob, tp.EnsembleB200(device=ctx.device, precision="fp32c"), dt=w.dt,
                               checkpoint_every=k)
        u0 = torch.from_numpy(plan.u0).to(dev)
        uf = torch.empty_like(u0)
        gu = torch.empty_like(u0)
        tape = ctx.adjoint_forward_device(plan.desc, plan.E, plan.B, u0.data_ptr(), n, uf.data_ptr(), s)
        torch.cuda.synchronize()
        ms_f = device_ms(lambda: tape.rerun_device(u0.data_ptr(), uf.data_ptr(), s))
        g = torch.zeros_like(uf)
        g[:, :3] = 2.0 * (uf[:, :3] - x_target) / n
        loss = float(((uf[:, :3] - x_target) ** 2).sum().item() / n)
        ms_b = device_ms(lambda: tape.backward_device(g.data_ptr(), gu.data_ptr(), gE.data_ptr(), gB.data_ptr(),
                                                      gp.data_ptr(), s))
        out = {"checkpoint_every": tape.segments()[0], "forward_ms": ms_f, "backward_ms": ms_b,
               "tape_device_bytes": tape.info()[0], "loss": loss,
               "grad_x0_norm": float(torch.linalg.vector_norm(gu[:, :3]).item()),
               "dL_dB0": 4.0e5 * float(gp[1].item()) + float(gp[5].item())}
        tape.close()
        return out

    main = run_tape(K)
    other = run_tape(compare_k)
    # the plain FP32C push of the same workload (no checkpoints, final save only)
    pp = tp.plan_boris(prob, tp.Boris(), tp.EnsembleB200(device=ctx.device, precision="fp32c"), dt=w.dt,
                       savestepinterval=10 ** 9, save_start=False)
    run = DeviceRun(tp, torch, ctx, pp, dev, stream)
    ms_p = device_ms(run.launch, pp)
    run.check()
    ps = float(n) * nt
    ms_f, ms_b = main["forward_ms"], main["backward_ms"]
    return {"workload": w.name, "particles": n, "time_steps": nt, **main, "plain_fp32c_push_ms": ms_p,
            "forward": {"value": ps / (ms_f * 1e-3), "unit": "particle-steps/s"},
            "backward": {"value": ps / (ms_b * 1e-3), "unit": "particle-steps/s"},
            "adjoint_over_forward": ms_b / ms_f, "adjoint_over_plain_push": ms_b / ms_p,
            "forward_plus_backward_ms": ms_f + ms_b,
            f"segments_of_{compare_k}": {k: other[k] for k in ("checkpoint_every", "forward_ms", "backward_ms",
                                                             "tape_device_bytes", "loss")}}


def leg_gc(tp, n):
    """Guiding centres in the dipole (config 4): RK4 over 5 bounce periods, RK45, FP64 vs float32 RHS."""
    w = tp.workloads.config4(n)
    prob = tp.TraceGCProblem(w.y0, (0.0, 1.0), (w.q, w.q2m, w.mu, w.E, w.B))
    out = {"workload": w.name, "particles": n}
    res = {}
    for prec in ("fp64", "fp32"):
        for alg, kw in (("rk4", dict(dt=w.tau_b / 200)), ("rk45", dict(abstol=1e-9, reltol=1e-6))):
            s = tp.solve(prob, tp.EnsembleB200(precision=prec), alg=alg, tend=5 * w.tau_b, savestepinterval=100000,
                         save_everystep=False, maxiters=1_000_000, **kw)
            res[(prec, alg)] = s
            out[f"{alg}_{prec}"] = {"value": s.particle_steps() / s.elapsedTime, "unit": "particle-steps/s",
                                    "device_s": s.elapsedTime}
    # mu through gc_to_full then full_to_gc (prepare_gc) at the final states:
    # mu is a constant parameter of the guiding-centre equations, so this is
    # the drift the conversion pair reports at the end of the run
    half = n // 2

    def mu_roundtrip(final):
        rel = np.empty(n)
        for lo, hi, sp in ((0, half, tp.Electron), (half, n, tp.Proton)):
            pd = tp.prepare(w.E, w.B, species=sp)
            xv = tp.gc_to_full(final[lo:hi].T, pd, w.mu[lo:hi])
            _, mu2 = tp.full_to_gc(xv, pd)
            rel[lo:hi] = np.abs(mu2 - w.mu[lo:hi]) / w.mu[lo:hi]
        return float(np.median(rel))

    for prec in ("fp64", "fp32"):
        out[f"rk4_{prec}"]["mu_roundtrip_rel_median"] = mu_roundtrip(res[(prec, "rk4")].final_states())
    # energy 1/2 m v_par^2 + mu |B| at the end, float32 RHS against float64 (same algorithm)
    for alg in ("rk4", "rk45"):
        a, b = res[("fp32", alg)].final_states(), res[("fp64", alg)].final_states()
        def energy(s):
            B = np.linalg.norm(tp.workloads.dipole_B(s[:, :3], (0.0, 0.0, -8.0e22)), axis=1)
            return 0.5 * w.m * s[:, 3] ** 2 + w.mu * B
        e0 = energy(w.y0.T)
        e64, e32 = energy(b), energy(a)
        out[f"{alg}_energy_drift_fp64_median"] = float(np.median(np.abs(e64 - e0) / e0))
        out[f"{alg}_fp32rhs_vs_fp64"] = {"energy_rel_median": float(np.median(np.abs(e32 - e64) / e64)),
                                         "position": _err_summary(_rel_err(a, b))}
    return out


def leg_next_rows(tp, n=1 << 20, nt=1000):
    """Throughput of the rows beyond the drop-in path (device time of solve()):
    cubic and nearest-node grids and a field time series on the config-2 box,
    the dipole sampled on a spherical grid, the adaptive hybrid in a magnetic
    bottle, and the virtual detectors over saved trajectories."""
    import math
    out = {}
    w = tp.workloads.config2(n=n, nt=nt, ssi=nt)
    dx = 1.0e5
    g = np.arange(128) * dx
    Ea, Ba, _L = tp.workloads.turbulent_grid(128, dx, 5.0e-9)

    def rate(sol):
        return sol.particle_steps() / sol.elapsedTime

    for order in (3, 0):
        E = tp.build_interpolator(Ea, g, g, g, order, tp.PeriodicBC("exclusive"))
        B = tp.build_interpolator(Ba, g, g, g, order, tp.PeriodicBC("exclusive"))
        prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(E, B))
        r = {}
        for prec in ("fp32c", "fp64"):
            r[prec] = rate(tp.solve(prob, tp.Boris(), tp.EnsembleB200(precision=prec), dt=w.dt,
                                    savestepinterval=nt))
        out[f"config2_order{order}"] = {**r, "unit": "particle-steps/s", "particles": n, "time_steps": nt}
    # a 4-snapshot time series of the config-2 fields (linear in time)
    times = np.linspace(0.0, float(w.tspan[1]), 4)

    def loader(Af):
        return lambda i: tp.build_interpolator(Af * (0.7 + 0.1 * i), g, g, g, 1, tp.PeriodicBC("exclusive"))

    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(tp.LazyTimeInterpolator(times, loader(Ea)),
                                                     tp.LazyTimeInterpolator(times, loader(Ba))))
    out["config2_series4"] = {prec: rate(tp.solve(prob, tp.Boris(), tp.EnsembleB200(precision=prec), dt=w.dt,
                                                  savestepinterval=nt)) for prec in ("fp32c", "fp64")}
    out["config2_series4"]["unit"] = "particle-steps/s"
    # the Earth dipole on a 64 x 64 x 96 spherical grid (linear), config-3 particles
    w3 = tp.workloads.config3(n=n, nt=nt, ssi=nt)
    r_ = np.geomspace(0.8 * tp.Re, 20.0 * tp.Re, 64)
    th = np.linspace(0.0, math.pi, 64)
    ph = np.linspace(0.0, 2 * math.pi, 96)
    R, T, _P = np.meshgrid(r_, th, ph, indexing="ij")
    k = tp.MU0_OVER_4PI * 8.0e22 / R ** 3
    A = np.zeros((3,) + R.shape)
    A[0] = -2.0 * k * np.cos(T)
    A[1] = -k * np.sin(T)
    Bs = tp.build_interpolator(tp.StructuredGrid, A.astype(np.float32), r_, th, ph)
    prob = tp.TraceProblem(w3.u0, w3.tspan, tp.prepare(tp.ZeroField(), Bs))
    out["config3_spherical_grid"] = {
        prec: rate(tp.solve(prob, tp.Boris(), tp.EnsembleB200(precision=prec), dt=w3.dt, tend=w3.tend,
                            savestepinterval=nt, isoutside=w3.isoutside)) for prec in ("fp32c", "fp64")}
    out["config3_spherical_grid"]["unit"] = "particle-steps/s"
    # adaptive hybrid in the bottle of test_hybrid.jl, 2^18 protons, 30 gyroperiods
    B0, alpha = 1.0e-4, 1.0e-2
    Tg = 2 * math.pi / (tp.qi / tp.mi * B0)
    rng = np.random.default_rng(3)
    nh = 1 << 18
    u0 = np.zeros((6, nh))
    u0[:3] = rng.normal(0.0, 0.5, (3, nh))
    vp = rng.uniform(2.0e4, 8.0e4, nh)
    phs = rng.uniform(0, 2 * math.pi, nh)
    u0[3], u0[4], u0[5] = vp * np.cos(phs), vp * np.sin(phs), rng.uniform(-1.2e5, 1.2e5, nh)
    prob = tp.TraceHybridProblem(u0, (0.0, 30 * Tg), tp.prepare(tp.ZeroField(), tp.QuadraticField.bottle(B0, alpha)))
    sh = tp.solve(prob, tp.AdaptiveHybrid(threshold=0.1, dtmax=Tg, dtmin=1e-4 * Tg, check_interval=100),
                  savestepinterval=1000)
    out["hybrid_bottle"] = {"value": rate(sh), "unit": "particle-steps/s", "particles": nh,
                            "steps_mean": float(sh.nsteps.mean())}
    # detectors over the saves of a config-2 FP64 run (1e6 x 11 saves)
    ws = tp.workloads.config2(n=n, nt=nt, ssi=nt // 10)
    sol = tp.solve(tp.TraceProblem(ws.u0, ws.tspan, tp.prepare(ws.E, ws.B)), tp.Boris(), dt=ws.dt,
                   savestepinterval=nt // 10)
    L = 128 * dx
    surfs = [tp.Disk(tp.Plane((L / 2, L / 2, L / 2), (1.0, 0.0, 0.0)), L / 4), tp.Sphere((L / 2, L / 2, L / 2), L / 3)]
    t0 = time.perf_counter()
    nf, _vf = tp.get_particle_fluxes(sol, surfs, 1.0)
    el = time.perf_counter() - t0
    segs = float(np.maximum(sol.nsaved - 1, 0).sum()) * len(surfs)
    out["detectors_config2_saves"] = {"segment_surface_checks_per_s": segs / el, "wall_s": el,
                                      "includes": "host -> device copy of the saved trajectories",
                                      "n_flux": [float(x) for x in nf]}
    return out


def profile_case(tp, case, device):
    """Small untimed runs of the adaptive, guiding-centre and general-grid kernels, for ncu captures."""
    if case == "adaptive":
        w = tp.workloads.config3(n=262144, nt=200, ssi=200)
        prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
        for prec in ("fp32c", "fp64"):
            tp.solve(prob, tp.AdaptiveBoris(0.1), tp.EnsembleB200(device=device, precision=prec),
                     savestepinterval=200, isoutside=w.isoutside, tend=w.tend, step_cap=200)
    elif case == "grids":
        w = tp.workloads.config2(n=262144, nt=100, ssi=100)
        dx = 1.0e5
        g = np.arange(128) * dx
        Ea, Ba, _L = tp.workloads.turbulent_grid(128, dx, 5.0e-9)
        for order in (3, 0):
            E = tp.build_interpolator(Ea, g, g, g, order, tp.PeriodicBC("exclusive"))
            B = tp.build_interpolator(Ba, g, g, g, order, tp.PeriodicBC("exclusive"))
            prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(E, B))
            for prec in ("fp32c", "fp64"):
                tp.solve(prob, tp.Boris(), tp.EnsembleB200(device=device, precision=prec), dt=w.dt,
                         savestepinterval=100)
    else:
        w = tp.workloads.config4(1 << 18)
        prob = tp.TraceGCProblem(w.y0, (0.0, 1.0), (w.q, w.q2m, w.mu, w.E, w.B))
        for alg, kw in (("rk4", dict(dt=w.tau_b / 200)), ("rk45", dict(abstol=1e-9, reltol=1e-6))):
            for prec in ("fp64", "fp32"):
                tp.solve(prob, tp.EnsembleB200(device=device, precision=prec), alg=alg, tend=w.tau_b,
                         savestepinterval=100000, save_everystep=False, maxiters=1_000_000, **kw)


def _device_err(a, b, torch):
    """|x_a - x_b| / |x_b| per save slot and particle (slots, n), on the device."""
    return (torch.linalg.vector_norm(a - b, dim=1) / torch.linalg.vector_norm(b, dim=1))


def _quantiles(e):
    e = e[np.isfinite(e)]
    if e.size == 0:
        return None
    q = np.quantile(e, [0.5, 0.9, 0.99, 0.999])
    return {"p50": float(q[0]), "p90": float(q[1]), "p99": float(q[2]), "p999": float(q[3]), "max": float(e.max()),
            "orbits": int(e.size)}


def orbit_errors(torch, run, p32, p64):
    """FP32C against FP64 on the same workload, and the orbits' own sensitivity.

    Runs FP32C, FP64 and FP64 from three perturbed starts (each component
    rounded to float32; all scaled by 1 + 2^-23, one float32 ulp; scaled by
    1 + 2^-52, one float64 ulp) into the same device buffers, and compares the
    saved positions.  An orbit is "regular" when the float32-ulp starts stay
    within 1e-6 (round) and 1e-5 (scale) of the float64 orbit at every save:
    there the float32 arithmetic itself is what the error measures.
    """
    def saves(plan):
        run.launch(plan)
        torch.cuda.synchronize()
        run.check()
        return run.u_out[:, :3, :].clone(), run.retc.clone()

    x32, rc32 = saves(p32)
    x64, rc64 = saves(p64)
    ok = (rc32 == 1) & (rc64 == 1)
    e32 = _device_err(x32, x64, torch)
    del x32
    u0 = run.u0.clone()
    seps = {}
    for name, pert in (("f32ulp_round", lambda u: u.float().double()), ("f32ulp_scale", lambda u: u * (1.0 + 2.0 ** -23)),
                       ("f64ulp_scale", lambda u: u * (1.0 + 2.0 ** -52))):
        run.u0.copy_(pert(u0))
        xp, rcp = saves(p64)
        ok &= rcp == 1
        seps[name] = _device_err(xp, x64, torch)
        del xp
    run.u0.copy_(u0)
    okc = ok.cpu().numpy()
    fin = e32[-1].cpu().numpy()[okc]
    out = {"fp32c_error_vs_fp64": _quantiles(fin), "orbits_compared": int(okc.sum()),
           "fp64_vs_fp64": {k: _quantiles(v[-1].cpu().numpy()[okc]) for k, v in seps.items()}}
    r_max = seps["f32ulp_round"].amax(dim=0).cpu().numpy()[okc]
    s_max = seps["f32ulp_scale"].amax(dim=0).cpu().numpy()[okc]
    reg = (r_max < 1e-6) & (s_max < 1e-5)
    out["regular_orbits"] = {"classifier": "float64 runs started a float32 ulp away stay within 1e-6 (components "
                                           "rounded) and 1e-5 (scaled by 1 + 2^-23) at every save",
                             "fraction": float(reg.mean()), "fp32c_error": _quantiles(fin[reg])}
    reg1 = r_max < 1e-6
    out["regular_orbits_round_only"] = {"classifier": "components rounded to float32: within 1e-6 at every save",
                                        "fraction": float(reg1.mean()), "fp32c_error": _quantiles(fin[reg1])}
    sep = seps["f32ulp_scale"][-1].cpu().numpy()[okc]
    ratio = fin / np.maximum(sep, 1e-300)
    out["fp32c_error_over_f32ulp_scale_separation"] = {k: float(v) for k, v in zip(
        ("p50", "p90", "p99"), np.quantile(ratio, [0.5, 0.9, 0.99]))}
    return out


def headline_run(tp, torch, ctx, dist, dev, stream, flush, world, local, args, w, alg):
    """Timed FP32C and FP64 solves of workload w, errors, and the end-to-end solve."""
    p32, p64 = _plan(tp, w, alg, "fp32c", local), _plan(tp, w, alg, "fp64", local)
    tune = None if args.no_autotune else {
        "fp32c": ctx.autotune(p32.desc, p32.E, p32.B, p32.u0, max_steps=200),
        "fp64": ctx.autotune(p64.desc, p64.E, p64.B, p64.u0, max_steps=200)}
    run = DeviceRun(tp, torch, ctx, p32, dev, stream)
    sampler = ClockSampler(local)
    run.launch(p32)  # first call builds any field tables
    torch.cuda.synchronize()
    sampler.start()
    tot32 = timed(torch, dist, dev, run, p32, args.steps, args.warmup, flush)
    clocks = sampler.stop()
    ps_step = run.particle_steps()
    k64 = max(args.fp64_steps, 1)
    tot64 = timed(torch, dist, dev, run, p64, k64, 1, flush)
    ps64 = run.particle_steps()
    errs = orbit_errors(torch, run, p32, p64)
    value = whole_job_rate(world, ps_step * args.steps, tot32 * 1e-3)
    value64 = whole_job_rate(world, ps64 * k64, tot64 * 1e-3)

    # end to end through the public API (host arrays in, packed host results out)
    prob = tp.TraceProblem(w.u0, w.tspan, tp.prepare(w.E, w.B, species=w.species))
    e2e_t = []
    h2d = d2h = 0
    sol = None
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
        e2e_time = max_over_ranks(dist, max(e2e_t), dev)
        e2e_value = whole_job_rate(world, float(sol.nsteps.sum()), e2e_time)
    del sol
    return {"value": value, "value64": value64, "tot32": tot32, "tot64": tot64, "k64": k64, "ps_step": ps_step,
            "clocks": clocks, "tune": tune, "errors": errs, "e2e": e2e_value, "h2d": h2d, "d2h": d2h, "n": run.n}


def gridded_roofline(r, world, args, peak, peak_kind):
    kernel_s = r["tot32"] * 1e-3 / args.steps
    achieved = BYTES_PER_PARTICLE_STEP * r["ps_step"] / kernel_s / 1e9
    sm_clock = (r["clocks"].get("sm_mhz") or 1965.0) * 1e6
    l1_ceiling = SMS * sm_clock / 8  # one L1 wavefront per SM clock, 8 corner lines per particle-step
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": TRAFFIC_PER_PARTICLE_STEP * r["ps_step"],
            "note": f"{BYTES_PER_PARTICLE_STEP} algorithmic B/particle-step; peak {peak_kind}; the field table is "
                    f"L2-resident (DRAM {TRAFFIC_PER_PARTICLE_STEP} B/particle-step by ncu), so the binding "
                    "ceiling is the L1 wavefront one beside this"}
    l1 = {"value": l1_ceiling, "unit": "particle-steps/s", "frac": r["value"] / world / l1_ceiling,
          "note": "148 SMs x SM clock / 8 corner lines per particle-step"}
    return roof, l1


def dipole_roofline(r, world, args):
    """Instruction-issue ceiling of the dipole push: no field memory and no
    contraction, so neither HBM nor the tensor cores bound it."""
    kernel_s = r["tot32"] * 1e-3 / args.steps
    sm_clock = (r["clocks"].get("sm_mhz") or 1965.0) * 1e6
    peak = SMS * ISSUE_PER_SM_CLOCK * sm_clock
    warp_steps = r["ps_step"] / 32.0
    achieved = INST_PER_WARP_STEP_DIPOLE * warp_steps / kernel_s
    return {"bound": "issue", "achieved": achieved, "peak": peak, "unit": "warp-instructions/s",
            "frac": achieved / peak, "traffic": TRAFFIC_PER_PARTICLE_STEP_DIPOLE * r["ps_step"],
            "flops": {"per_particle_step": FLOPS_PER_PARTICLE_STEP_DIPOLE,
                      "achieved_tflops": FLOPS_PER_PARTICLE_STEP_DIPOLE * r["ps_step"] / kernel_s / 1e12},
            "note": f"{INST_PER_WARP_STEP_DIPOLE:.0f} warp instructions per warp-step (ncu, 262144 x 200 steps) x "
                    "warp-steps / kernel time, against 148 SMs x 4 issue slots x the sampled SM clock; "
                    "MEASURED_PEAKS.json holds no FP32 or FP64 peak, so the flop rate is stated without a "
                    "fraction; DRAM traffic (inputs and saves only) by ncu"}


def leg_gridded(tp, torch, ctx, dist, dev, stream, flush, world, local, args, peak, peak_kind):
    """The gridded turbulent field (config 2): FP32C and FP64 Boris, 1e6 x 1e4."""
    w = _workload(tp, "config2", args.particles, args.nt)
    r = headline_run(tp, torch, ctx, dist, dev, stream, flush, world, local, args, w, tp.Boris())
    roof, l1 = gridded_roofline(r, world, args, peak, peak_kind)
    return {"workload": w.name, "particles": r["n"], "time_steps": w.nt,
            "fp32c": r["value"], "fp64": r["value64"], "unit": "particle-steps/s",
            "speedup_fp32c_over_fp64": r["value"] / r["value64"], "errors": r["errors"],
            "roofline": roof, "l1_wavefront_ceiling": l1, "e2e": r["e2e"], "autotune": r["tune"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="config3", choices=["config1", "config2", "config3"])
    ap.add_argument("--particles", type=int, default=1_000_000)
    ap.add_argument("--sample", type=int, default=0,
                    help="particles of the CPU legs (default: about 10-20 s of host work at 16 cores)")
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-legs", action="store_true", help="skip the gridded / adaptive / guiding-centre / adjoint legs")
    ap.add_argument("--nt", type=int, default=10_000, help="time steps (reduced only for profiling)")
    ap.add_argument("--adjoint-only", action="store_true", help="run only the adjoint leg (profiling)")
    ap.add_argument("--next-rows", action="store_true",
                    help="also time the general grids, field series, hybrid and detectors")
    ap.add_argument("--no-autotune", action="store_true", help="default launch shapes (profiling)")
    ap.add_argument("--profile-case", choices=["adaptive", "gc", "grids"], default=None,
                    help="run one small untimed case for an ncu capture: AdaptiveBoris(0.1) in the dipole "
                         "(262144 protons, 200 steps, FP32C then FP64) or guiding centres in the dipole "
                         "(2^18 particles, one bounce period, RK4 then RK45, FP64 then float32 RHS) or the "
                         "config-2 field on cubic then nearest-node grids (262144 protons, 100 steps, FP32C "
                         "then FP64)")
    ap.add_argument("--adj-n", type=int, default=1 << 18)
    ap.add_argument("--adj-nt", type=int, default=4096)
    ap.add_argument("--adj-k", type=int, default=0, help="checkpoint interval of the adjoint leg (0: automatic)")
    args = ap.parse_args()
    if args.sample <= 0:
        # oracle rates at 16 threads: ~1.5e8 (gridded Boris) and ~1.3e8
        # (dipole Multistep) particle-steps/s: about 10 s of host work
        args.sample = {"config2": 150_000, "config3": 150_000}.get(args.workload, 1000)
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
    if args.profile_case:
        profile_case(tp, args.profile_case, local)
        return
    if args.adjoint_only:
        dev = torch.device("cuda", local)
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
        leg = leg_adjoint(tp, torch, ctx, dev, torch.cuda.current_stream(), flush, n=args.adj_n, nt=args.adj_nt,
                          K=args.adj_k)
        if rank == 0:
            print(json.dumps({"adjoint_only": leg}), flush=True)
        return
    w = _workload(tp, args.workload, args.particles, args.nt)
    alg = _alg(tp, args.workload)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    peak, peak_kind = _peaks()

    r = headline_run(tp, torch, ctx, dist, dev, stream, flush, world, local, args, w, alg)
    value, value64 = r["value"], r["value64"]
    if args.workload == "config2":
        roof, l1 = gridded_roofline(r, world, args, peak, peak_kind)
        extra_roof = {"l1_wavefront_ceiling": l1}
    else:
        roof, extra_roof = dipole_roofline(r, world, args), {}

    legs = {}
    if not args.no_legs:
        if args.workload != "config2":
            legs["gridded_config2"] = leg_gridded(tp, torch, ctx, dist, dev, stream, flush, world, local, args,
                                                  peak, peak_kind)
        legs["dipole_config3"] = leg_dipole(tp, torch, ctx, dist, dev, stream, flush, world, 1_000_000, args.nt,
                                            multistep=args.workload != "config3")
        if rank == 0:
            legs["guiding_centre_config4"] = leg_gc(tp, 1 << 20)
        legs["adjoint_config5"] = leg_adjoint(tp, torch, ctx, dev, stream, flush)
    if args.next_rows and rank == 0:
        legs["next_rows"] = leg_next_rows(tp)

    if rank == 0:
        cpu = None
        if not args.no_cpu:
            orc = ge.load_oracle()
            rate, el, ps = cpu_rate(tp, orc, w, alg, args.sample)
            cpu = {"value": rate, "unit": "particle-steps/s", "cores": orc.max_threads(), "kind": "port",
                   "sample": f"{args.sample} particles x {w.nt} steps of the same workload, FP64 reference "
                             f"order, {el:.1f} s (C++ restatement of the reference EnsembleThreads path)"}
        alg_name = "MultistepBoris4(n=2)" if args.workload == "config3" else "Boris()"
        line = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["tot32"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+compensated",
            "data": "synthetic (seeded SplitMix64)",
            "config": {"workload": w.name, "algorithm": alg_name, "particles": r["n"], "time_steps": w.nt,
                       "savestepinterval": w.savestepinterval, "precision": "fp32c",
                       "inputs_in_hbm": True, "l2": "flushed between timed steps (256 MB write)",
                       "parallelism": f"replicas x{world}"},
            "fp64": {"value": value64, "unit": "particle-steps/s", "ms_per_step": r["tot64"] / r["k64"],
                     "speedup_fp32c_over_fp64": value / value64},
            **r["errors"],
            "roofline": roof, **extra_roof,
            "cpu_baseline": cpu,
            "e2e": {"value": r["e2e"], "unit": "particle-steps/s", "h2d_bytes_per_step": int(r["h2d"]),
                    "d2h_bytes_per_step": int(r["d2h"])},
            "gpu_launches": args.steps,
            "autotune": r["tune"],
            "clocks": r["clocks"],
            "legs": legs,
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


if __name__ == "__main__":
    main()
