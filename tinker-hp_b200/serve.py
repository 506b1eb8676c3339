"""Serving of single-point polarization solves over the native request loop.

The loop itself is C++ (thp_server_* in csrc/server.cu): admission by device
footprint against a memory budget, residency of each system's topology,
parameters, list and last dipoles (a repeat is warm-started), worker threads
that drive the GPU with one stream per system, and a pool of idle contexts
that new systems are re-targeted onto instead of allocating and freeing
device memory.  This module feeds it a request stream in real time and
collects the results; latency is measured inside the loop, from submission to
the dipoles in the caller's buffer.
"""
import ctypes as C
import dataclasses
import time

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
    arrival: float          # seconds after stream start, when it was submitted
    queue_ms: float
    latency_ms: float
    niter: int
    epol: float
    uind: np.ndarray
    status: int
    repeat: bool
    warm: bool
    setup_ms: float = 0.0
    solve_ms: float = 0.0

    @property
    def latency(self):
        return self.latency_ms * 1e-3

    @property
    def end(self):
        return self.arrival + self.latency


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
    """Python face of thp_server (see module docstring)."""

    def __init__(self, precision=L.MIXED, poleps=1e-6, politer=500, budget_bytes=120 << 30, workers=8, device=0,
                 max_resident=16):
        cfg = L.ThpServerConfig(precision, poleps, politer, device, budget_bytes, workers, max_resident)
        h = C.c_void_p()
        st = L.load().thp_server_create(C.byref(cfg), C.byref(h))
        if st:
            raise L.ThpError(st, "thp_server_create")
        self.h = h
        self.keys = {}
        self._live = {}  # ticket -> buffers the native loop reads or fills

    def register(self, key, ws):
        keep = []
        sysd = L.system_struct(ws, keep)
        code = self.keys.setdefault(key, len(self.keys) + 1)
        st = L.load().thp_server_register(self.h, code, C.byref(sysd))
        if st:
            raise L.ThpError(st, "thp_server_register")
        return code

    def submit(self, key, ws, xyz=None, uind=None):
        """Queues one solve; returns (ticket, uind buffer).  The coordinate
        and dipole buffers are the loop's until wait() returns: given ones
        (`xyz` = three C-contiguous float64 [n] arrays, `uind` [n,3], e.g.
        pinned) are used as they are, otherwise copies are made and kept."""
        code = self.keys.get(key) or self.register(key, ws)
        if xyz is None:
            xyz = [np.ascontiguousarray(a, dtype=np.float64) for a in (ws.x, ws.y, ws.z)]
        if uind is None:
            uind = np.zeros((ws.n, 3))
        t = C.c_ulonglong()
        st = L.load().thp_server_submit(self.h, code, *(L._p(a) for a in xyz), L._p(uind), None, C.byref(t))
        if st:
            raise L.ThpError(st, "thp_server_submit")
        self._live[t.value] = (xyz, uind)
        return t.value, uind

    def warm(self, count):
        """Pre-creates `count` pooled contexts for the largest registered system."""
        st = L.load().thp_server_warm(self.h, int(count))
        if st:
            raise L.ThpError(st, "thp_server_warm")

    def wait(self, ticket, timeout_ms=None):
        """The request's thp_result.  With timeout_ms, raises ThpError with
        THP_E_TIMEOUT when it has not finished by then; the ticket (and its
        buffers) stay live for a later wait."""
        r = L.ThpResult()
        if timeout_ms is None:
            st = L.load().thp_server_wait(self.h, ticket, C.byref(r))
        else:
            st = L.load().thp_server_wait_for(self.h, ticket, float(timeout_ms), C.byref(r))
            if st == L.THP_E_TIMEOUT:
                raise L.ThpError(st, "thp_server_wait_for")
        self._live.pop(ticket, None)
        if st:
            raise L.ThpError(st, "thp_server_wait")
        return r

    def pause(self, paused=True):
        """Holds (True) or releases (False) the queue: paused workers take no
        new request."""
        st = L.load().thp_server_pause(self.h, 1 if paused else 0)
        if st:
            raise L.ThpError(st, "thp_server_pause")

    def run(self, requests, realtime=True, warm=0):
        """Serve the stream (submitting each request at its arrival time when
        realtime); returns one Result per request.  Registration (and `warm`
        pooled contexts) happen before the clock starts, as at a server's
        start-up."""
        reqs = sorted(requests, key=lambda q: q.arrival)
        for q in reqs:
            if q.key not in self.keys:
                self.register(q.key, q.ws)
        if warm:
            self.warm(warm)
        t0 = time.perf_counter()
        pending = []
        for q in reqs:
            if realtime:
                delay = q.arrival - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
            submitted = time.perf_counter() - t0
            ticket, uind = self.submit(q.key, q.ws)
            pending.append((q, submitted, ticket, uind))
        out = []
        for q, submitted, ticket, uind in pending:
            r = self.wait(ticket)
            out.append(Result(q.rid, q.key, submitted, r.queue_ms, r.latency_ms, r.niter, r.epol,
                              uind if r.status == L.THP_OK else None, r.status, q.repeat, bool(r.warm),
                              r.setup_ms, r.solve_ms))
        return out

    def stats(self):
        s = L.ThpServerStats()
        L.load().thp_server_query(self.h, C.byref(s))
        return {k: getattr(s, k) for k, _ in L.ThpServerStats._fields_}

    def close(self):
        if getattr(self, "h", None):
            L.load().thp_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def summarize(results):
    ok = [r for r in results if r.status == L.THP_OK]
    lat = np.array([r.latency_ms for r in ok])
    span = max(r.end for r in results) - min(r.arrival for r in results)
    return {"completed": len(ok), "failed": len(results) - len(ok), "solves_per_s": len(ok) / span,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_iters": float(np.mean([r.niter for r in ok])),
            "repeat_iters": float(np.mean([r.niter for r in ok if r.repeat])) if any(r.repeat for r in ok) else None,
            "warm_fraction": float(np.mean([r.warm for r in ok])),
            "mean_setup_ms": float(np.mean([r.setup_ms for r in ok])),
            "mean_solve_ms": float(np.mean([r.solve_ms for r in ok]))}
