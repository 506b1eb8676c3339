"""Continuous-batching server for single-point polarization solves.

Requests (water boxes of any size) arrive over time.  The server:
  * admits a request when a worker slot is free and the system's device
    footprint (thp_footprint) fits the memory budget next to the resident
    systems, evicting idle least-recently-used systems when needed;
  * keeps each system resident (topology, parameters, lists, last dipoles)
    so a repeat of a system with moved coordinates is warm-started from its
    previous dipoles (THP_GUESS_PREVIOUS);
  * runs admitted requests on worker threads, each system on its own CUDA
    stream, so requests that arrive while others are on the GPU overlap with
    them on the device (the ctypes calls release the GIL).
Latency is completion time minus arrival time.
"""
import dataclasses
import heapq
import threading
import time
from collections import OrderedDict

import numpy as np

from . import lib as L
from . import water


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float          # seconds after stream start
    key: str                # system identity (repeats share it)
    ws: object              # water.WaterSystem with this request's coordinates
    repeat: bool = False


@dataclasses.dataclass
class Result:
    rid: int
    key: str
    arrival: float
    start: float
    end: float
    niter: int
    epol: float
    uind: np.ndarray
    status: int
    repeat: bool

    @property
    def latency(self):
        return self.end - self.arrival


def poisson_stream(count, rate=200.0, nmin=1000, nmax=60000, repeat_frac=0.3, perturb=0.01, seed=5004,
                   base_cfg=4):
    """Seeded request stream: exponential inter-arrival times (mean 1/rate),
    sizes log-uniform in [nmin, nmax] atoms (whole waters), a fraction of
    requests repeating an earlier system with a Gaussian perturbation of
    `perturb` A RMS on every coordinate."""
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs, systems = [], []
    for rid in range(count):
        t += rng.exponential(1.0 / rate)
        if systems and rng.random() < repeat_frac:
            key, ws0 = systems[rng.integers(len(systems))]
            pos = ws0.positions() + rng.normal(0.0, perturb / np.sqrt(3.0), size=(ws0.n, 3))
            reqs.append(Request(rid, t, key, ws0.with_positions(pos), True))
        else:
            nw = max(1, int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax))) / 3.0)))
            edge = max(water.box_edge(nw), water.min_box_edge())
            ws = water.make_water_box(nw, edge=edge, seed_lattice=seed * 1000 + 2 * rid,
                                      seed_orient=seed * 1000 + 2 * rid + 1)
            key = f"sys{rid}"
            systems.append((key, ws))
            reqs.append(Request(rid, t, key, ws, False))
    return reqs


class Server:
    """Admission, residency and worker pool (see module docstring)."""

    def __init__(self, precision=L.MIXED, poleps=1e-6, budget_bytes=120 << 30, workers=8, device=0,
                 context_factory=None, footprint_fn=None):
        self.precision = precision
        self.poleps = poleps
        self.budget = budget_bytes
        self.workers = workers
        self.device = device
        self._make = context_factory or (lambda ws: L.Context(ws, precision=precision, poleps=poleps,
                                                              device=device))
        self._footprint = footprint_fn or (lambda ws: L.footprint(ws, precision))
        self.resident = OrderedDict()  # key -> [ctx, bytes, busy]
        self.used = 0
        self.lock = threading.Condition()
        self.results = []

    # -- residency ---------------------------------------------------------
    def _acquire(self, req):
        """Blocks until the system is resident and idle; returns its context."""
        need = self._footprint(req.ws)
        if need > self.budget:
            raise L.ThpError(L.THP_E_OOM_ADMISSION, f"request {req.rid} needs {need} bytes")
        with self.lock:
            while True:
                ent = self.resident.get(req.key)
                if ent is not None:
                    if not ent[2]:
                        ent[2] = True
                        self.resident.move_to_end(req.key)
                        return ent[0], False
                    self.lock.wait()
                    continue
                if self.used + need <= self.budget:
                    self.used += need
                    self.resident[req.key] = [None, need, True]
                    break
                victim = next((k for k, e in self.resident.items() if not e[2]), None)
                if victim is None:
                    self.lock.wait()
                    continue
                ctx, nbytes, _ = self.resident.pop(victim)
                self.used -= nbytes
                ctx.close()
        try:
            ctx = self._make(req.ws)
        except Exception:
            with self.lock:
                self.used -= need
                self.resident.pop(req.key, None)
                self.lock.notify_all()
            raise
        with self.lock:
            self.resident[req.key][0] = ctx
        return ctx, True

    def _release(self, key):
        with self.lock:
            ent = self.resident.get(key)
            if ent is not None:
                ent[2] = False
            self.lock.notify_all()

    # -- serving ----------------------------------------------------------
    def _work(self, req, t0):
        start = time.perf_counter() - t0
        ctx, fresh = self._acquire(req)
        try:
            if not fresh:
                ctx.set_positions(req.ws.x, req.ws.y, req.ws.z)
            guess = L.GUESS_DIRECT if fresh else L.GUESS_PREVIOUS
            r = ctx.solve(guess, allow_unconverged=True)
            uind, _ = ctx.dipoles()
            st = r["status"]
        except L.ThpError as e:  # quarantine: the request fails, the server keeps going
            r, uind, st = {"niter": 0, "epol": float("nan")}, None, e.status
        finally:
            self._release(req.key)
        end = time.perf_counter() - t0
        return Result(req.rid, req.key, req.arrival, start, end, r["niter"], r["epol"], uind, st, req.repeat)

    def run(self, requests, realtime=True):
        """Serve the stream; returns results in completion order."""
        import concurrent.futures as cf
        reqs = sorted(requests, key=lambda q: q.arrival)
        t0 = time.perf_counter()
        out = []
        with cf.ThreadPoolExecutor(max_workers=self.workers) as ex:
            futs = []
            for q in reqs:
                if realtime:
                    delay = q.arrival - (time.perf_counter() - t0)
                    if delay > 0:
                        time.sleep(delay)
                futs.append(ex.submit(self._work, q, t0))
            for f in cf.as_completed(futs):
                out.append(f.result())
        self.results = out
        return out

    def close(self):
        with self.lock:
            for ctx, _, _ in self.resident.values():
                if ctx is not None:
                    ctx.close()
            self.resident.clear()
            self.used = 0


def summarize(results):
    ok = [r for r in results if r.status in (L.THP_OK, L.THP_E_NOT_CONVERGED)]
    lat = np.array([r.latency for r in ok]) * 1e3
    span = max(r.end for r in results) - min(r.arrival for r in results)
    return {"completed": len(ok), "failed": len(results) - len(ok), "solves_per_s": len(ok) / span,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_iters": float(np.mean([r.niter for r in ok])),
            "repeat_iters": float(np.mean([r.niter for r in ok if r.repeat])) if any(r.repeat for r in ok) else None}
