#!/usr/bin/env python
"""Benchmark of the AMOEBA induced-dipole polarization path on B200.

Workload: the 96,000-water (288,000-atom) synthetic box (142.3 A, PME grid
120^3, alpha 0.5446, cutoff 7.0 + 0.5 A buffer), one step = one single-point
polarization solve: list build + permanent field (direct + PME) + PCG to
tolerance + polarization energy.  The headline is the mixed-precision form
(FP32 pair fields and PME, FP64 CG scalars); both forms stop at the CG_TOL below; the plain FP64 form
on the same box, the dipole error of mixed versus FP64, p50/p99 latency, the
end-to-end host-buffer call and the CPU baseline are reported beside it.

Contract: one JSON line on rank 0.  N>1 (torchrun): independent replicas, one
box per GPU (weak scaling), time = max over ranks.
"""
import argparse
import math
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

# Independent systems (batches, served requests) run on many streams and as
# parallel graph branches; the default of 8 hardware work queues would run
# at most 8 of them at a time.  Read when the CUDA context is created.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def load_package():
    import importlib.util
    name = "tinker_hp_b200"
    if name in sys.modules:
        return sys.modules[name]
    d = os.path.join(ROOT, "tinker-hp_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    m = importlib.util.module_from_spec(spec)
    sys.modules[name] = m
    spec.loader.exec_module(m)
    return m


METRIC = "induced-dipole solves/s & p99 latency, mixed vs FP64 on one B200 at 1e-5 D RMS"
WORKLOADS = {
    # name: (waters, cfg index for seeds)
    "water-288k": (96000, 2),
    "water-96k": (32000, 2),
    "water-32k": (10800, 1),
    "water-1944": (648, 0),
}
DEBYE = 4.80321
# CG stop threshold (Tinker's poleps, internal e*A units) for both forms: the
# dipole error against the fully converged FP64 answer tracks it (about 4x in
# Debye, identical in both forms) and stays at 3-4e-6 D on every box measured,
# inside the 1e-5 D acceptance; 2e-6 lands at 1.05-1.17e-5 D on some boxes
CG_TOL = 1e-6


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms during the
    timed region (one background nvidia-smi process, stopped by its PID)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        import tempfile
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.out.close()
        rows = []
        if self.path and os.path.exists(self.path):
            with open(self.path) as f:
                rows = [[c.strip() for c in line.split(",")] for line in f if line.strip()]
            os.unlink(self.path)

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if len(r) > 2 and num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if len(r) > 2 and num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def allreduce_max(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline_oracle(ws_sys, max_seconds, threads, tol=CG_TOL):
    """The oracle (C++ FP64 restatement of the reference) on the host cores,
    one full single-point solve of the same box."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    orc = O.Oracle(ws_sys, poleps=tol, nthreads=threads)
    st, _, _ = orc.mlistcell()
    if st != 0:
        raise RuntimeError(f"oracle list status {st}")
    res = orc.solve()
    e, _ = orc.epolar(res["uind"])
    dt = time.perf_counter() - t0
    return dt, res, e


def cpu_model():
    """The host CPU's model name (Linux /proc/cpuinfo)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_one_core_sample(ws_sys, n_iter, tol=CG_TOL):
    """One core: the oracle's list build, then two solves stopped after 1 and
    3 CG iterations; their difference gives the cost of one iteration, from
    which a full solve of n_iter iterations is assembled (list + front +
    n_iter iterations).  About 25 s of one core at 288,000 atoms."""
    from oracle import oracle as O
    out = {}
    for politer in (1, 3):
        orc = O.Oracle(ws_sys, poleps=tol, nthreads=1, politer=politer)
        t0 = time.perf_counter()
        st, _, _ = orc.mlistcell()
        t_list = time.perf_counter() - t0
        if st != 0:
            raise RuntimeError(f"oracle list status {st}")
        t0 = time.perf_counter()
        orc.solve()
        out[politer] = (t_list, time.perf_counter() - t0)
        orc.close()
    t_list = min(out[1][0], out[3][0])
    t_iter = max(0.0, (out[3][1] - out[1][1]) / 2.0)
    t_front = max(0.0, out[1][1] - t_iter)
    t_solve = t_list + t_front + n_iter * t_iter
    return {"value": 1.0 / t_solve, "unit": "solves/s", "cores": 1, "kind": "port",
            "sample": f"one core: list {t_list:.2f} s, front (E0) {t_front:.2f} s, {t_iter:.2f} s per CG "
                      f"iteration x {n_iter} (from solves stopped after 1 and 3 iterations)"}


def run_reference(args, ws_n, rank, world):
    """--impl reference: the CPU restatement of the reference's v1.2 path
    (the Fortran reference cannot be built here), all host threads."""
    if rank != 0:
        return
    thp = load_package()
    nw, cfg = WORKLOADS[args.workload]
    ws = thp.water.make_water_box(nw, cfg=cfg)
    threads = os.cpu_count() or 1
    budget = 150.0
    times = []
    warm = min(args.warmup, 1)
    t_start = time.perf_counter()
    for _ in range(warm):
        dt, _, _ = cpu_baseline_oracle(ws, budget, threads)
    steps = 0
    for _ in range(args.steps):
        dt, res, e = cpu_baseline_oracle(ws, budget, threads)
        times.append(dt)
        steps += 1
        if time.perf_counter() - t_start > budget:
            break
    tot = sum(times)
    value = steps / tot
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": 1000.0 * tot / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{args.workload} ({ws.n} atoms, box {ws.box[0]:.2f} A, grid {ws.nfft[0]}^3)",
                       "cg_tol": CG_TOL, "iterations": res["niter"]},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port",
                             "cpu_model": cpu_model(),
                             "sample": f"{steps} full FP64 solves of the {ws.n}-atom box (C++ restatement of "
                                       f"v1.2, OpenMP {threads} threads); the Fortran reference needs gfortran+MPI, "
                                       "absent on this image"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def batched_throughput(lib, systems, copies, steps, warmup=2, precision=None):
    """Batched form: `copies` resident contexts per system solved together by
    thp_solve_batch (each on its own stream); host-timed over whole batches.
    Mixed form unless `precision` says otherwise."""
    prec = lib.MIXED if precision is None else precision
    ctxs = [lib.Context(ws, precision=prec, poleps=CG_TOL) for ws in systems for _ in range(copies)]
    for _ in range(warmup):
        lib.solve_batch(ctxs)
    t0 = time.perf_counter()
    iters = []
    for _ in range(steps):
        infos = lib.solve_batch(ctxs)
        iters += [f["niter"] for f in infos]
    dt = time.perf_counter() - t0
    for c in ctxs:
        c.close()
    return {"solves": len(ctxs) * steps, "seconds": dt, "solves_per_s": len(ctxs) * steps / dt,
            "ms_per_batch": 1000.0 * dt / steps, "median_iters": float(np.median(iters))}


def batch_plan_throughput(lib, systems, steps, precision=None):
    """Batched form through a batch plan (thp_batch_*): the CG iterations of
    all systems as batched persistent kernels in one graph.  The first solves
    tune the launch shape (untimed); host-timed over whole batches."""
    prec = lib.MIXED if precision is None else precision
    ctxs = [lib.Context(ws, precision=prec, poleps=CG_TOL) for ws in systems]
    plan = lib.Batch(ctxs)
    tuning_solves = 0
    while plan.tuning() is None and tuning_solves < 16:
        plan.solve()
        tuning_solves += 1
    plan.solve()
    t0 = time.perf_counter()
    iters = []
    for _ in range(steps):
        infos = plan.solve()
        iters += [f["niter"] for f in infos]
    dt = time.perf_counter() - t0
    tuned = plan.tuning()
    plan.close()
    for c in ctxs:
        c.close()
    return {"solves": len(ctxs) * steps, "seconds": dt, "solves_per_s": len(ctxs) * steps / dt,
            "ms_per_batch": 1000.0 * dt / steps, "median_iters": float(np.median(iters)),
            "tuning_solves": tuning_solves, "tuned": tuned}


def serving_run(lib, thp, count, workers=8):
    """Serving form: seeded Poisson stream (200 req/s, 1k-60k atoms, 30 %
    repeats perturbed by 0.01 A RMS) through the native request loop with a
    120 GB device budget."""
    from tinker_hp_b200 import serve
    reqs = serve.poisson_stream(count)
    srv = serve.Server(precision=lib.MIXED, poleps=CG_TOL, budget_bytes=120 << 30, workers=workers)
    srv.run(reqs[: min(8, len(reqs))], realtime=False)  # warm the kernels
    srv.close()
    srv = serve.Server(precision=lib.MIXED, poleps=CG_TOL, budget_bytes=120 << 30, workers=workers, max_resident=16)
    out = srv.run(reqs, realtime=True, warm=24)
    stats = srv.stats()
    srv.close()
    summ = serve.summarize(out)
    summ["contexts"] = {k: stats[k] for k in ("created", "reused", "evicted", "resident", "pooled")}
    summ["max_resident"] = 16
    summ["warm_pool"] = "24 contexts sized for the largest system, created at start-up before the stream"
    summ.update({"requests": len(reqs), "rate_req_per_s": 200.0, "workers": workers,
                 "atoms": "1,000-60,000 log-uniform", "repeats": "30 % (0.01 A RMS perturbation, warm start)"})
    return summ


def served_repeats(lib, boxes0, precision, count=20, perturb=0.01, seed=5011):
    """Served repeats of resident systems: after a cold first request per
    system, each request carries one system's coordinates with a fresh
    Gaussian perturbation of `perturb` A RMS (as the repeats of the serving
    stream).  The server keeps each system's list (reused while no atom has
    moved half the 0.5 A buffer since the build) and its last dipoles (the
    warm start).  With one system one request is in flight at a time; with
    several, all requests are submitted at once (systems interleaved), one
    worker per system, and requests of different systems overlap on the
    device.  Returns the throughput, latencies and the dipole error of the
    last request against an FP64 solve of its coordinates to 1e-8."""
    import torch
    from tinker_hp_b200 import serve

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy()
        t[...] = a
        return t

    rng = np.random.default_rng(seed)
    nsys = len(boxes0)
    reqs = []  # (system, box, pinned xyz, pinned uind)
    for q in range(count):
        k = q % nsys
        ws = boxes0[k]
        b = ws.with_positions(ws.positions() + rng.normal(0.0, perturb / np.sqrt(3.0), size=(ws.n, 3)))
        reqs.append((k, b, [pinned(np.asarray(a, dtype=np.float64)) for a in (b.x, b.y, b.z)],
                     pinned(np.zeros((ws.n, 3)))))
    srv = serve.Server(precision=precision, poleps=CG_TOL, budget_bytes=120 << 30, workers=nsys,
                       max_resident=nsys + 1)
    for k, ws in enumerate(boxes0):
        srv.register(f"box{k}", ws)
    for t in [srv.submit(f"box{k}", ws)[0] for k, ws in enumerate(boxes0)]:
        srv.wait(t)
    res = []
    t0 = time.perf_counter()
    if nsys == 1:
        for k, b, xyz, ui in reqs:
            ticket, _ = srv.submit(f"box{k}", b, xyz=xyz, uind=ui)
            res.append(srv.wait(ticket))
    else:
        tickets = [srv.submit(f"box{k}", b, xyz=xyz, uind=ui)[0] for k, b, xyz, ui in reqs]
        res = [srv.wait(t) for t in tickets]
    wall = time.perf_counter() - t0
    srv.close()
    _, last, _, ulast = reqs[-1]
    ref = lib.Context(last, precision=lib.FP64, poleps=1e-8)
    ref.solve()
    ue, _ = ref.dipoles()
    ref.close()
    err = float(np.sqrt(np.mean(np.sum((ulast - ue) ** 2, axis=1))) * DEBYE)
    lat = [r.latency_ms for r in res]
    sol = [r.solve_ms for r in res]
    return {"systems": nsys, "requests": count, "solves_per_s": count / wall,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "solve_p50_ms": float(np.percentile(sol, 50)), "mean_iters": float(np.mean([r.niter for r in res])),
            "warm_fraction": float(np.mean([bool(r.warm) for r in res])), "dipole_rms_D_vs_fp64_1e-8": err,
            "perturbation": f"{perturb} A RMS per request around its box",
            "host_buffers": "pinned coordinates in, pinned dipoles out"}


def md_run(lib, thp, nsteps=20, predictor=None):
    """Config 1 dynamics: 10,800 waters (32,400 atoms), FP64, velocity Verlet
    at 1 fs from Maxwell velocities at 300 K (seed 3001), each solve started
    from the previous step's dipoles or from a predictor.  The polarization
    gradient is the only force, which is attractive, so unbonded water
    collapses after some 60 fs: the run is kept to the first 20 fs."""
    ws = thp.water.make_water_box(10800, cfg=1)
    mass = thp.water.masses(ws)
    vel = thp.water.maxwell_velocities(mass, 300.0, seed=3001)
    ctx = lib.Context(ws, precision=lib.FP64, poleps=1e-6)
    if predictor:
        ctx.set_predictor(getattr(lib, f"PRED_{predictor}"))
    ctx.md_verlet(2, 0.001, mass, vel)  # warm the kernels and graphs
    ctx.close()
    ctx = lib.Context(ws, precision=lib.FP64, poleps=1e-6)
    if predictor:
        ctx.set_predictor(getattr(lib, f"PRED_{predictor}"))
    t0 = time.perf_counter()
    _, en, it = ctx.md_verlet(nsteps, 0.001, mass, vel)
    wall = time.perf_counter() - t0
    ctx.close()
    ms = wall / nsteps * 1e3
    return {"steps": nsteps, "ms_per_step": ms, "ns_per_day": 1e-6 * 86400.0 / (ms * 1e-3),
            "guess": predictor or "previous step", "mean_iters": float(np.mean(it)),
            "iters": [int(x) for x in it], "energy_drift_rel": float(abs(en[-1, 2] - en[0, 2]) / abs(en[0, 1])),
            "atoms": ws.n, "dt_fs": 1.0}


def empole_run(lib, ws, reps=10):
    """Permanent-multipole energy and gradient (empole1c) of the box, FP64 and
    mixed: wall time per call through the C-ABI with the list already built
    (each call: rotpole, multipole spread + FFTs + 20-term gather, the pair
    terms, energy, and the gradient into a pinned host array)."""
    import torch
    out = {}
    res = {}
    for name, prec in (("fp64", lib.FP64), ("mixed", lib.MIXED)):
        ctx = lib.Context(ws, precision=prec)
        buf = torch.empty((ws.n, 3), dtype=torch.float64, pin_memory=True).numpy()
        ctx.empole1(out=buf)
        ctx.empole1(out=buf)
        t0 = time.perf_counter()
        for _ in range(reps):
            em, dem = ctx.empole1(out=buf)
        dt = (time.perf_counter() - t0) / reps
        res[name] = (em, dem.copy())
        out[name] = {"ms_per_call": dt * 1e3, "em_kcal_mol": em}
        ctx.close()
    (e64, d64), (em, dm) = res["fp64"], res["mixed"]
    out["mixed_energy_err_kcal_mol"] = em - e64
    out["mixed_force_rms_rel_err"] = float(np.sqrt(np.mean(np.sum((dm - d64) ** 2, axis=1)))
                                           / np.sqrt(np.mean(np.sum(d64 ** 2, axis=1))))
    out["atoms"] = ws.n
    return out


def solve_roofline(n, nfft, n_it, ms_mixed, hbm_gbs, ms_fp64=None):
    """Whole-solve roofline of the polarization path from the per-unit work
    table of the path (flops and bytes per atom, per list entry, per
    interacting pair, per grid point):
      W = a6 + a11 + a4 + a10 + (n_it + 1) (a3 + a5 + CG),
    roofline time = sum over the terms of max(bytes / HBM, flops / FLOP peak),
    achieved = roofline time / measured time.  Pair and list counts use the
    water-box constants P = 71.8 N interacting half-pairs and L = 88.4 N list
    half-entries (7.0 / 7.5 A); candidates of the list build 712 per atom.
    The HBM peak is measured; the FP32 / FP64 vector FLOP peaks are nominal
    (75 / 37 TFLOP/s), as none is measured here.  The mixed form halves the
    per-atom and grid bytes (not the list)."""
    K3 = float(nfft[0] * nfft[1] * nfft[2])
    P, L = 71.8 * n, 88.4 * n
    log2k3 = math.log2(K3)

    def terms(mixed):
        h = 0.5 if mixed else 1.0
        return {
            "a3_matvec_real": (120.0 * P, h * 136.0 * n + 4.0 * L),
            "a5_matvec_recip": (3500.0 * n + 10.0 * K3 * log2k3 + 6.0 * K3, h * (128.0 * K3 + 96.0 * n)),
            "cg_vectors": (60.0 * n, h * 624.0 * n),
            "a4_efld0_direct": (220.0 * P, h * 184.0 * n + 4.0 * L),
            "a10_efld0_recip": (3500.0 * n + 10.0 * K3 * log2k3 + 6.0 * K3, h * (128.0 * K3 + 96.0 * n)),
            "a6_bsplines": (300.0 * n, h * 504.0 * n),
            "a11_list": (30.0 * 712.0 * n, 24.0 * n + 4.0 * L),
        }

    out = {"n_it": n_it, "hbm_gbs": hbm_gbs, "flop_peaks_tflops": {"fp32": 75.0, "fp64": 37.0},
           "flop_peak_kind": "nominal", "hbm_kind": "measured"}
    for name, mixed, ms in (("mixed", True, ms_mixed), ("fp64", False, ms_fp64)):
        if ms is None or not hbm_gbs:
            continue
        fpk = (75.0 if mixed else 37.0) * 1e12
        t = 0.0
        for key, (fl, by) in terms(mixed).items():
            reps = (n_it + 1) if key in ("a3_matvec_real", "a5_matvec_recip", "cg_vectors") else 1
            t += reps * max(by / (hbm_gbs * 1e9), fl / fpk)
        out[name] = {"roofline_ms": t * 1e3, "measured_ms": ms, "achieved": t * 1e3 / ms}
    return out


def nonbonded_run(lib, ws, reps=10, perturb=0.01, seed=5021):
    """All the AMOEBA non-bonded terms built here, per step as in dynamics:
    new positions (a 0.01 A RMS displacement of the box), a polarization
    solve warm-started from the previous dipoles, its gradient, the
    permanent-multipole and the van der Waals energies and gradients (mixed
    form; gradients into pinned host arrays).  Wall time per step."""
    import torch
    rng = np.random.default_rng(seed)
    ctx = lib.Context(ws, precision=lib.MIXED, poleps=CG_TOL)
    pin = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64).pin_memory().numpy()
    g = torch.empty((ws.n, 3), dtype=torch.float64, pin_memory=True).numpy()
    pos0 = ws.positions()
    frames = [[pin(p[:, 0]), pin(p[:, 1]), pin(p[:, 2])]
              for p in (pos0 + rng.normal(0.0, perturb, pos0.shape) for _ in range(reps + 2))]
    iters = []

    def step(f):
        ctx.set_positions(*f)
        r = ctx.solve(lib.GUESS_PREVIOUS)
        ctx.gradient(out=g)
        ctx.empole1(out=g)
        ctx.ehal1(out=g)
        return r["niter"]

    step(frames[0])
    step(frames[1])
    t0 = time.perf_counter()
    for f in frames[2:]:
        iters.append(step(f))
    dt = (time.perf_counter() - t0) / reps
    ctx.close()
    return {"ms_per_step": dt * 1e3, "mean_iters": float(np.mean(iters)), "atoms": ws.n,
            "terms": "polarization solve (warm) + gradient, empole1, ehal1; mixed form"}


def ehal_run(lib, ws, reps=10):
    """Buffered 14-7 van der Waals energy and gradient (ehal1c) of the box,
    FP64 and mixed: wall time per call through the C-ABI with the vdW list in
    place (each call: reduced sites, the displacement check, the pair terms
    over the list, the gradient into a pinned host array)."""
    import torch
    out = {"atoms": ws.n, "cutoff_A": ws.vdw["vdwcut"]}
    res = {}
    for name, prec in (("fp64", lib.FP64), ("mixed", lib.MIXED)):
        ctx = lib.Context(ws, precision=prec)
        buf = torch.empty((ws.n, 3), dtype=torch.float64, pin_memory=True).numpy()
        ctx.ehal1(out=buf)
        ctx.ehal1(out=buf)
        t0 = time.perf_counter()
        for _ in range(reps):
            ev, dev = ctx.ehal1(out=buf)
        dt = (time.perf_counter() - t0) / reps
        res[name] = (ev, dev.copy())
        out[name] = {"ms_per_call": dt * 1e3, "ev_kcal_mol": ev}
        ctx.close()
    (e64, d64), (em, dm) = res["fp64"], res["mixed"]
    out["mixed_energy_rel_err"] = (em - e64) / e64
    out["mixed_force_rms_rel_err"] = float(np.sqrt(np.mean(np.sum((dm - d64) ** 2, axis=1)))
                                           / np.sqrt(np.mean(np.sum(d64 ** 2, axis=1))))
    return out


def timed_solves(ctx, lib, steps, warmup, rebuild=True, guess=None):
    """Device-resident solves; per-step device time from CUDA events."""
    import torch
    guess = lib.GUESS_DIRECT if guess is None else guess
    for _ in range(warmup):
        if rebuild:
            ctx.invalidate_list()
        ctx.solve(guess)
    torch.cuda.synchronize()
    lat = []
    niters = []
    for _ in range(steps):
        if rebuild:
            ctx.invalidate_list()
        r = ctx.solve(guess)
        lat.append(r["ms"])
        niters.append(r["niter"])
    torch.cuda.synchronize()
    return lat, niters


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="water-288k", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched and serving measurements")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, None, rank, world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch
    torch.cuda.set_device(local)
    thp = load_package()
    from tinker_hp_b200 import lib
    lib.load()
    nw, cfg = WORKLOADS[args.workload]
    ws = thp.water.make_water_box(nw, cfg=cfg)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    # mixed form (headline)
    mixed = lib.Context(ws, precision=lib.MIXED, poleps=CG_TOL, device=local)
    mixed.set_stream(stream.cuda_stream)
    fp64 = None if args.no_fp64 else lib.Context(ws, precision=lib.FP64, poleps=CG_TOL, device=local)
    if fp64 is not None:
        fp64.set_stream(stream.cuda_stream)

    # accuracy of mixed against FP64 on the GPU (tight FP64 reference)
    acc = {}
    if fp64 is not None:
        ref64 = lib.Context(ws, precision=lib.FP64, poleps=1e-8, device=local)
        ref64.set_stream(stream.cuda_stream)
        r_ref = ref64.solve()
        u_ref, _ = ref64.dipoles()
        r_m = mixed.solve()
        u_m, _ = mixed.dipoles()
        r_d = fp64.solve()
        u_d, _ = fp64.dipoles()
        acc = {"mixed_dipole_rms_D": float(np.sqrt(np.mean(np.sum((u_m - u_ref) ** 2, 1))) * DEBYE),
               "fp64_dipole_rms_D": float(np.sqrt(np.mean(np.sum((u_d - u_ref) ** 2, 1))) * DEBYE),
               "mixed_vs_fp64_same_tol_rms_D": float(np.sqrt(np.mean(np.sum((u_m - u_d) ** 2, 1))) * DEBYE),
               "reference": "FP64 GPU solve converged to poleps 1e-8",
               "mixed_epol_rel": abs(r_m["epol"] - r_ref["epol"]) / abs(r_ref["epol"]),
               "fp64_epol_rel": abs(r_d["epol"] - r_ref["epol"]) / abs(r_ref["epol"]),
               "epol_kcal": r_ref["epol"], "iters_mixed": r_m["niter"], "iters_fp64": r_d["niter"]}
        ref64.close()
        del ref64

    clocks = ClockSampler(local)
    # ---- timed region: mixed, device-resident inputs
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    for _ in range(args.warmup):
        mixed.invalidate_list()
        mixed.solve()
    barrier(world)
    torch.cuda.synchronize()
    ev0.record(stream)
    lat = []
    niter = []
    for _ in range(args.steps):
        mixed.invalidate_list()
        r = mixed.solve()
        lat.append(r["ms"])
        niter.append(r["niter"])
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    t_mixed = allreduce_max(ev0.elapsed_time(ev1), world)
    clk = clocks.stop()
    # roofline of the real-space row: its launches are event-timed in a
    # separate pass (the event-timed path runs without the device-side loop
    # graph, so it stays out of the timed region above)
    mixed.profile(1)
    work_launches = 0
    for _ in range(3):
        mixed.invalidate_list()
        work_launches += mixed.solve()["niter"] + 1  # the initial matvec and one per iteration
    mv_ms, mv_launches = mixed.profile(0)
    # launches enqueued after the stop flag return at entry (a few us each);
    # the average is taken over the launches that did the work
    mv_launches = max(1, min(mv_launches, work_launches))

    # ---- FP64 form on the same box
    fp64_line = None
    if fp64 is not None:
        lat64, nit64 = timed_solves(fp64, lib, max(3, args.steps // 2), 3)
        t64 = allreduce_max(float(np.sum(lat64)), world)
        fp64_line = {"value": world * len(lat64) / (t64 / 1000.0), "unit": "solves/s",
                     "ms_per_step": t64 / len(lat64), "p50_ms": float(np.percentile(lat64, 50)),
                     "p99_ms": float(np.percentile(lat64, 99)), "iterations": int(np.median(nit64))}

    # ---- end to end through the host-buffer C-ABI call, from and into
    # pinned host memory
    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy()
        t[...] = a
        return t

    rp = pinned(mixed.rpole())
    x, y, z = (pinned(np.asarray(a, dtype=np.float64)) for a in (ws.x, ws.y, ws.z))
    outs = (pinned(np.zeros((ws.n, 3))), pinned(np.zeros((ws.n, 3))))
    for _ in range(2):
        mixed.solve_host(x, y, z, rp, out=outs)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_steps = max(3, args.steps // 2)
    for _ in range(e2e_steps):
        mixed.solve_host(x, y, z, rp, out=outs)  # positions+rpole H2D, solve, dipoles D2H (synchronous)
    torch.cuda.synchronize()
    t_e2e = allreduce_max(time.perf_counter() - t0, world)
    n = ws.n
    h2d = n * 3 * 8 + n * 13 * 8
    d2h = n * 6 * 8

    peaks, peak_kind = measured_peaks()
    # roofline of the real-space row of the mixed CG matvec (the PME branch runs beside it on
    # another stream; the combine is its own kernel): algorithmic bytes per launch, the FP64 a3 figure 136 N + 4 L with per-atom data
    # halved in the mixed form: 68 N (positions, polarity, mu in, field out) + 4 L (half list,
    # 88.4 entries per atom at 7.5 A)
    L_entries = 88.4 * n
    alg_bytes = 68.0 * n + 4.0 * L_entries
    avg_ms = mv_ms / max(mv_launches, 1)
    achieved = alg_bytes / (avg_ms * 1e-3) / 1e9
    # DRAM bytes per launch (read + write) from one ncu capture of this kernel on the 96,000-atom
    # box (182.1 MB per launch), scaled by the atom count: the traffic is the streamed pair entries
    # (index and two FP32 coefficients, 12 B per directed pair) plus per-atom data, both
    # proportional to n
    traffic = 182.1e6 * n / 96000.0
    roof = {"bound": "hbm", "kernel": "k_real_row<mixed> (real-space row of the CG matvec)",
            "limiter": "L1 data pipe (73 % of cycles) and the latency of the dependent stream and partner "
                       "loads; DRAM at 40 % (ncu, 96k-atom capture)",
            "achieved": achieved, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
            "frac": achieved / peaks.get("hbm_gbs"), "peak_kind": peak_kind, "traffic": traffic,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, 96k-atom capture scaled by n",
            "avg_launch_ms": avg_ms, "launches": mv_launches, "alg_bytes_per_launch": alg_bytes}

    solve_roof = solve_roofline(n, ws.nfft, int(np.median(niter)), t_mixed / args.steps, peaks.get("hbm_gbs"),
                                fp64_line["ms_per_step"] if fp64_line else None)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            th = os.cpu_count() or 1
            dt, res_c, e_c = cpu_baseline_oracle(ws, 120, th, CG_TOL)
            cpu = {"value": 1.0 / dt, "unit": "solves/s", "cores": th, "kind": "port",
                   "cpu_model": cpu_model(),
                   "sample": f"1 full FP64 solve of the {n}-atom box by the C++ restatement of v1.2 "
                             f"({res_c['niter']} CG iterations, {dt:.1f} s)"}
            try:
                cpu["one_core"] = cpu_one_core_sample(ws, res_c["niter"])
            except Exception as ex:  # the all-core figure stands without it
                cpu["one_core"] = {"value": None, "sample": f"failed: {ex}"}
        except Exception as ex:  # the GPU number stands without it
            cpu = {"value": None, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"failed: {ex}"}

    extras = {}
    if not args.no_extras:
        b2 = batched_throughput(lib, [ws], 2, max(2, args.steps // 6))
        b4 = batched_throughput(lib, [ws], 4, max(2, args.steps // 10))
        b2_64 = batched_throughput(lib, [ws], 2, max(2, args.steps // 6), precision=lib.FP64)
        extras["batched_288k"] = {"copies_2": b2, "copies_4": b4, "fp64_copies_2": b2_64}
        batch64 = thp.water.make_batch(64, seed=4003)
        extras["batch_64_boxes"] = batched_throughput(lib, batch64, 1, 3)
        extras["batch_64_boxes"]["atoms"] = f"{sum(w.n for w in batch64)} over 64 boxes (300-6000 each)"
        extras["batch_64_boxes_plan"] = batch_plan_throughput(lib, batch64, 5)
        extras["batch_64_boxes_plan_fp64"] = batch_plan_throughput(lib, batch64, 5, precision=lib.FP64)
        extras["serving"] = serving_run(lib, thp, 120)
        ws2 = thp.water.make_water_box(nw, cfg=cfg, seed_lattice=7001, seed_orient=7002)
        extras["served_288k_repeats"] = {"mixed": served_repeats(lib, [ws], lib.MIXED),
                                         "fp64": served_repeats(lib, [ws], lib.FP64),
                                         "mixed_2_systems": served_repeats(lib, [ws, ws2], lib.MIXED, count=24),
                                         "fp64_2_systems": served_repeats(lib, [ws, ws2], lib.FP64, count=24)}
        extras["md_config1"] = {"previous": md_run(lib, thp), "aspc": md_run(lib, thp, predictor="ASPC")}
        extras["empole1"] = empole_run(lib, ws)
        extras["ehal1"] = ehal_run(lib, ws)
        extras["nonbonded_step"] = nonbonded_run(lib, ws)
        if fp64 is not None:
            best = max(b2["solves_per_s"], b4["solves_per_s"])
            plain64 = world * len(lat64) / (t64 / 1000.0)
            extras["batched_288k"]["speedup_vs_fp64_plain"] = best / plain64
            sr = extras["served_288k_repeats"]
            sr["mixed_vs_fp64_plain"] = sr["mixed"]["solves_per_s"] / plain64
            sr["mixed_vs_fp64_served"] = sr["mixed"]["solves_per_s"] / sr["fp64"]["solves_per_s"]
            sr["mixed_2_systems_vs_fp64_plain"] = sr["mixed_2_systems"]["solves_per_s"] / plain64
            sr["mixed_2_systems_vs_fp64_2_systems"] = (sr["mixed_2_systems"]["solves_per_s"]
                                                       / sr["fp64_2_systems"]["solves_per_s"])

    steps = args.steps
    value = world * steps / (t_mixed / 1000.0)
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": t_mixed / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {nw} waters, {n} atoms, box {ws.box[0]:.2f} A, PME "
                               f"{ws.nfft[0]}^3 order 5, alpha {ws.aewald:.4f}, cutoff 7.0+0.5 A",
                   "form": "mixed (FP32 pair fields/PME/CG vectors, FP64 CG scalars)", "cg_tol": CG_TOL,
                   "parallelism": f"replicas x{world}", "l2": "inputs > L2 (pair stream ~0.5 GB per matvec)",
                   "iterations": int(np.median(niter))},
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "fp64": fp64_line, "accuracy": acc, "extras": extras,
        "speedup_mixed_vs_fp64": (value / fp64_line["value"]) if fp64_line else None,
        "e2e": {"value": world * e2e_steps / t_e2e, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "host_buffers": "pinned (positions, rpole in; uind, uinp out)"},
        "roofline": roof, "solve_roofline": solve_roof, "cpu_baseline": cpu, "clocks": clk,
        "gpu_launches": None,
    }
    # compact summaries last, so that a truncated record still ends with them
    if extras and fp64_line:
        sr = extras["served_288k_repeats"]
        bt = extras["batched_288k"]
        line["target_3x"] = {
            "goal": "mixed batched/served solves/s >= 3x plain FP64 solves/s, 288k box, <= 1e-5 D",
            "like_for_like": {
                "cold_mixed_vs_cold_fp64": value / fp64_line["value"],
                "batched_mixed_vs_batched_fp64": bt["copies_2"]["solves_per_s"] / bt["fp64_copies_2"]["solves_per_s"],
                "served_mixed_vs_served_fp64": sr["mixed_vs_fp64_served"],
                "served_2_systems_mixed_vs_fp64": sr["mixed_2_systems_vs_fp64_2_systems"]},
            "served_mixed_vs_plain_fp64": {
                "one_system": sr["mixed_vs_fp64_plain"], "two_systems": sr["mixed_2_systems_vs_fp64_plain"],
                "note": "warm-started served mixed (0.01 A repeats) against cold single FP64 solves"},
            "batched_mixed_vs_plain_fp64": bt["speedup_vs_fp64_plain"]}
    if extras:
        sv = extras["serving"]
        line["serving"] = {k: sv[k] for k in ("solves_per_s", "p50_ms", "p99_ms", "requests", "rate_req_per_s",
                                              "mean_setup_ms", "mean_solve_ms", "completed", "failed")}
    # kernels of this library per timed step (cuFFT's not counted; the
    # positions do not move, so rotpole does not run):
    #   re-sort 11: dipoles and last E0 out of sorted order (2), cell count,
    #     scan (3), fill, sort, special pairs to sorted numbering, dipoles and
    #     last E0 back (2);
    #   sorted gather 1; list 1; E_direct + pair stream 1; multipole spread,
    #     qfac, multipole gather 3;
    #   CG start 6: direct guess, row records, real row, dipole spread, qfac,
    #     combine;
    #   7 per iteration (device-side loop): row records, real row, dipole
    #     spread, qfac, combine, update, loop condition;
    #   Epol 1.
    it = int(np.median(niter))
    per_step = 11 + 1 + 1 + 1 + 3 + 6 + 7 * it + 1
    line["gpu_launches"] = per_step * steps
    if rank == 0:
        print(json.dumps(line), flush=True)
    mixed.close()
    if fp64 is not None:
        fp64.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
