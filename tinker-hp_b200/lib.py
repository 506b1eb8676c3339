"""ctypes binding of libthp.so (the C-ABI declared in include/thp.h).

This is the host-side mirror of the reference's polarization interface for
Python callers (tests, benchmarks, the batch and serving layers).  There is no
fallback path: if libthp.so is missing or cannot load, every call raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libthp.so")

THP_OK = 0
THP_E_INVALID = 1
THP_E_LIST_OVERFLOW = 2
THP_E_NOT_CONVERGED = 3
THP_E_NAN = 4
THP_E_CUDA = 5
THP_E_TIMEOUT = 6
THP_E_OOM_ADMISSION = 7
THP_E_BOX_TOO_SMALL = 8
THP_E_NO_DEVICE = 9
THP_E_STATE = 10
NOALLOC_MAX_ATOMS = 4194304

FP64 = 0
MIXED = 1

GUESS_DIRECT = 0
GUESS_PREVIOUS = 1
GUESS_HOST = 2
GUESS_PREDICT = 3
PRED_NONE, PRED_ASPC, PRED_GEAR, PRED_LSQR = 0, 1, 2, 3

CONN_NAMES = ("i12", "i13", "i14", "i15", "ip11", "ip12", "ip13", "ip14")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class ThpConfig(C.Structure):
    _fields_ = [("n", C.c_int), ("box", C.c_double * 3), ("aewald", C.c_double), ("ewaldcut", C.c_double),
                ("lbuffer", C.c_double), ("nfft", C.c_int * 3), ("bsorder", C.c_int), ("politer", C.c_int),
                ("poleps", C.c_double), ("precision", C.c_int), ("max_neighbors", C.c_int), ("device", C.c_int)]


class ThpSolveInfo(C.Structure):
    _fields_ = [("niter", C.c_int), ("converged", C.c_int), ("resnrm", C.c_double), ("epol", C.c_double),
                ("ene", C.c_double * 2), ("ms_total", C.c_double)]


class ThpSystem(C.Structure):
    _fields_ = [("cfg", ThpConfig), ("polarity", _dp), ("thole", _dp), ("pdamp", _dp),
                ("conn_off", C.POINTER(_ip)), ("conn_idx", C.POINTER(_ip)), ("scales", _dp), ("pole", _dp),
                ("zaxis", _ip), ("xaxis", _ip), ("axt", _ip)]


class ThpServerConfig(C.Structure):
    _fields_ = [("precision", C.c_int), ("poleps", C.c_double), ("politer", C.c_int), ("device", C.c_int),
                ("budget_bytes", C.c_size_t), ("workers", C.c_int), ("max_resident", C.c_int)]


class ThpResult(C.Structure):
    _fields_ = [("status", C.c_int), ("niter", C.c_int), ("warm", C.c_int), ("epol", C.c_double),
                ("queue_ms", C.c_double), ("latency_ms", C.c_double), ("wait_ms", C.c_double),
                ("setup_ms", C.c_double), ("solve_ms", C.c_double)]


class ThpServerStats(C.Structure):
    _fields_ = [("completed", C.c_long), ("failed", C.c_long), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("resident", C.c_int), ("pooled", C.c_int), ("created", C.c_long), ("reused", C.c_long),
                ("evicted", C.c_long), ("bytes", C.c_size_t)]


class ThpError(RuntimeError):
    def __init__(self, status, what):
        self.status = status
        super().__init__(f"{what}: status {status} ({status_string(status)})")


_lib = None


def load():
    """Load libthp.so (raises if it is absent: the CUDA path is the only path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} not built; run tinker-hp_b200/build.py")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    sig = {
        "thp_ctx_create": ([C.POINTER(ThpConfig), C.POINTER(vp)], C.c_int),
        "thp_ctx_destroy": ([vp], C.c_int),
        "thp_ctx_reset": ([vp, C.POINTER(ThpConfig)], C.c_int),
        "thp_ctx_footprint": ([vp], C.c_size_t),
        "thp_set_stream": ([vp, vp], C.c_int),
        "thp_set_params": ([vp, _dp, _dp, _dp], C.c_int),
        "thp_set_connectivity": ([vp, C.POINTER(_ip), C.POINTER(_ip), _dp], C.c_int),
        "thp_set_positions": ([vp, _dp, _dp, _dp], C.c_int),
        "thp_set_rpole": ([vp, _dp], C.c_int),
        "thp_set_frames": ([vp, _dp, _ip, _ip, _ip], C.c_int),
        "thp_set_guess": ([vp, _dp], C.c_int),
        "thp_set_predictor": ([vp, C.c_int], C.c_int),
        "thp_nblist": ([vp], C.c_int),
        "thp_invalidate_list": ([vp], C.c_int),
        "thp_profile": ([vp, C.c_int, _dp, _ip], C.c_int),
        "thp_solve": ([vp, C.c_int, C.POINTER(ThpSolveInfo)], C.c_int),
        "thp_get_dipoles": ([vp, _dp, _dp], C.c_int),
        "thp_get_gradient": ([vp, _dp, _dp], C.c_int),
        "thp_get_gradient_device": ([vp, vp], C.c_int),
        "thp_set_virial": ([vp, C.c_int], C.c_int),
        "thp_get_virial": ([vp, C.c_int, _dp], C.c_int),
        "thp_get_empole_virial": ([vp, C.c_int, _dp], C.c_int),
        "thp_get_ehal_virial": ([vp, _dp], C.c_int),
        "thp_bind_virial": ([vp, _dp], C.c_int),
        "thp_md_verlet": ([vp, C.c_int, C.c_double, _dp, _dp, _dp, _ip], C.c_int),
        "thp_get_positions": ([vp, _dp, _dp, _dp], C.c_int),
        "thp_get_field": ([vp, _dp], C.c_int),
        "thp_get_rpole": ([vp, _dp], C.c_int),
        "thp_get_nblist": ([vp, C.c_int, _ip, _ip], C.c_int),
        "thp_tmatxb": ([vp, C.c_int, C.c_int, _dp, _dp], C.c_int),
        "thp_efld0_direct": ([vp, C.c_int, _dp], C.c_int),
        "thp_efld0_recip": ([vp, _dp], C.c_int),
        "thp_tmatxbrecip": ([vp, C.c_int, _dp, _dp], C.c_int),
        "thp_solve_batch": ([C.POINTER(vp), C.c_int, C.c_int, C.POINTER(ThpSolveInfo)], C.c_int),
        "thp_batch_create": ([C.POINTER(vp), C.c_int, C.POINTER(vp)], C.c_int),
        "thp_batch_solve": ([vp, C.c_int, C.POINTER(ThpSolveInfo)], C.c_int),
        "thp_batch_tuning": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)], C.c_int),
        "thp_batch_profile": ([vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int)], C.c_int),
        "thp_batch_destroy": ([vp], C.c_int),
        "thp_solve_host": ([vp, _dp, _dp, _dp, _dp, _dp, _dp, C.POINTER(ThpSolveInfo)], C.c_int),
        "thp_footprint": ([C.POINTER(ThpConfig)], C.c_size_t),
        "thp_status_string": ([C.c_int], C.c_char_p),
        "thp_bind_state": ([vp, _dp, _dp, _dp, _dp, _dp, _dp, _ip, _ip, C.c_int, _dp], C.c_int),
        "thp_last_error": ([], C.c_int),
        "thp_bind_gradient": ([vp, _dp], C.c_int),
        "thp_set_mpole_scales": ([vp, _dp], C.c_int),
        "thp_set_vdw": ([vp, _ip, C.c_int, _dp, _ip, _dp, _dp, C.c_double, C.c_double, C.c_double, C.c_double],
                        C.c_int),
        "thp_ehal1": ([vp, _dp, _dp], C.c_int),
        "thp_get_vlist": ([vp, C.c_int, _ip, _ip], C.c_int),
        "thp_bind_vlist": ([vp, _ip, _ip, C.c_int], C.c_int),
        "thp_bind_vdw": ([vp, _dp, _dp], C.c_int),
        "ehal1_": ([], None),
        "thp_empole1": ([vp, _dp, _dp], C.c_int),
        "thp_bind_mpole": ([vp, _dp, _dp], C.c_int),
        "empole1_": ([], None),
        "thp_bind_grid": ([vp, _dp], C.c_int),
        "grid_uind_sites_": ([_ip, _ip, _dp, _dp, _dp], None),
        "fphi_uind_sites_": ([_ip, _ip, _dp, _dp, _dp, _dp], None),
        "grid_uind_site_": ([_ip, _ip, _dp, _dp, _dp], None),
        "fphi_uind_site_": ([_ip, _ip, _dp, _dp, _dp], None),
        "thp_epolar_noalloc": ([C.c_int, vp, vp, vp, vp], C.c_int),
        "thp_server_create": ([C.POINTER(ThpServerConfig), C.POINTER(vp)], C.c_int),
        "thp_server_register": ([vp, C.c_ulonglong, C.POINTER(ThpSystem)], C.c_int),
        "thp_server_submit": ([vp, C.c_ulonglong, _dp, _dp, _dp, _dp, _dp, C.POINTER(C.c_ulonglong)], C.c_int),
        "thp_server_wait": ([vp, C.c_ulonglong, C.POINTER(ThpResult)], C.c_int),
        "thp_server_wait_for": ([vp, C.c_ulonglong, C.c_double, C.POINTER(ThpResult)], C.c_int),
        "thp_server_pause": ([vp, C.c_int], C.c_int),
        "thp_server_warm": ([vp, C.c_int], C.c_int),
        "thp_server_query": ([vp, C.POINTER(ThpServerStats)], C.c_int),
        "thp_server_destroy": ([vp], C.c_int),
        "newinduce_pme2_": ([], None),
        "tmatxb_pme_": ([_ip, _ip, _dp, _dp], None),
        "efld0_direct_": ([_ip, _dp], None),
        "efld0_recip_": ([_dp], None),
        "tmatxbrecip_": ([_dp, _dp, _ip, _dp, _dp], None),
        "mlistcell_": ([], None),
        "vlistcell_": ([], None),
        "epolar_": ([], None),
        "epolar1_": ([], None),
        "inducepcg_pme2_": ([vp, _ip, _ip, _dp, _dp, _dp], None),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def status_string(st):
    try:
        return load().thp_status_string(st).decode()
    except Exception:
        return "?"


def _p(a, t=_dp):
    return None if a is None else a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def config_for(ws, precision=FP64, poleps=1e-6, politer=500, device=0, max_neighbors=0):
    cfg = ThpConfig()
    cfg.n = ws.n
    for d in range(3):
        cfg.box[d] = ws.box[d]
        cfg.nfft[d] = ws.nfft[d]
    cfg.aewald = ws.aewald
    cfg.ewaldcut = ws.ewaldcut
    cfg.lbuffer = ws.lbuffer
    cfg.bsorder = ws.bsorder
    cfg.politer = politer
    cfg.poleps = poleps
    cfg.precision = precision
    cfg.max_neighbors = max_neighbors
    cfg.device = device
    return cfg


def footprint(ws, precision=FP64):
    return int(load().thp_footprint(C.byref(config_for(ws, precision))))


def solve_batch(contexts, guess=GUESS_DIRECT, allow_unconverged=False):
    """Solve several resident systems together (thp_solve_batch)."""
    L = load()
    n = len(contexts)
    hs = (C.c_void_p * n)(*[c.h for c in contexts])
    infos = (ThpSolveInfo * n)()
    st = L.thp_solve_batch(hs, n, guess, infos)
    if st != THP_OK and not (allow_unconverged and st == THP_E_NOT_CONVERGED):
        raise ThpError(st, "thp_solve_batch")
    return [{"niter": f.niter, "converged": bool(f.converged), "resnrm": f.resnrm, "epol": f.epol,
             "ene": tuple(f.ene), "ms": f.ms_total} for f in infos]


def _infos(infos):
    return [{"niter": f.niter, "converged": bool(f.converged), "resnrm": f.resnrm, "epol": f.epol,
             "ene": tuple(f.ene), "ms": f.ms_total} for f in infos]


class Batch:
    """A batch plan (thp_batch_*): the CG iterations of a fixed set of small
    resident systems run as batched persistent kernels in one CUDA graph.  The
    contexts must stay alive (and not be re-targeted) while the plan is used."""

    def __init__(self, contexts):
        L = load()
        self.contexts = list(contexts)
        n = len(self.contexts)
        hs = (C.c_void_p * n)(*[c.h for c in self.contexts])
        h = C.c_void_p()
        st = L.thp_batch_create(hs, n, C.byref(h))
        if st != THP_OK:
            raise ThpError(st, "thp_batch_create")
        self.h = h

    def solve(self, guess=GUESS_DIRECT, allow_unconverged=False):
        n = len(self.contexts)
        infos = (ThpSolveInfo * n)()
        st = load().thp_batch_solve(self.h, guess, infos)
        if st != THP_OK and not (allow_unconverged and st == THP_E_NOT_CONVERGED):
            raise ThpError(st, "thp_batch_solve")
        return _infos(infos)

    def tuning(self):
        """The autotuner's kept launch shape, or None while it is still tuning."""
        b, a, ms = C.c_int(), C.c_int(), C.c_double()
        st = load().thp_batch_tuning(self.h, C.byref(b), C.byref(a), C.byref(ms))
        if st == THP_E_STATE:
            return None
        if st != THP_OK:
            raise ThpError(st, "thp_batch_tuning")
        return {"blocks_per_sm": b.value, "matvec_atoms": a.value, "ms_per_solve": ms.value}

    KERNELS = ("spread", "fft_forward", "qfac", "fft_inverse", "matvec", "update")

    def profile(self, enable=None):
        """enable True/False switches the eager, per-kernel-timed loop on/off
        (resetting the accumulators); returns the accumulated ms per kernel
        and the iterations timed so far."""
        ms = (C.c_double * len(self.KERNELS))()
        it = C.c_int()
        mode = -1 if enable is None else (1 if enable else 0)
        st = load().thp_batch_profile(self.h, mode, ms, C.byref(it))
        if st != THP_OK:
            raise ThpError(st, "thp_batch_profile")
        return dict(zip(self.KERNELS, list(ms))), it.value

    def close(self):
        if getattr(self, "h", None):
            load().thp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def scales_array(ws):
    s = ws.scales
    return _f64(list(s["p_scale"]) + list(s["pi_scale"]) + list(s["d_scale"]) + list(s["u_scale"]))


class Context:
    """One system resident on the GPU (wraps thp_ctx)."""

    def __init__(self, ws, precision=FP64, poleps=1e-6, politer=500, device=0, frames=True, rpole=None,
                 max_neighbors=0):
        L = load()
        self.cfg = config_for(ws, precision, poleps, politer, device, max_neighbors)
        h = C.c_void_p()
        self._check(L.thp_ctx_create(C.byref(self.cfg), C.byref(h)), "thp_ctx_create")
        self.h = h
        self._setup(ws, frames, rpole)

    def retarget(self, ws, frames=True, rpole=None, max_neighbors=0):
        """Serve another system with this context (thp_ctx_reset): buffers
        that are large enough and an unchanged FFT plan are kept."""
        self.cfg = config_for(ws, self.cfg.precision, self.cfg.poleps, self.cfg.politer, self.cfg.device,
                              max_neighbors)
        self._check(load().thp_ctx_reset(self.h, C.byref(self.cfg)), "thp_ctx_reset")
        self._setup(ws, frames, rpole)

    def footprint(self):
        return load().thp_ctx_footprint(self.h)

    def _setup(self, ws, frames, rpole):
        L = load()
        self.ws = ws
        self.n = ws.n
        self._keep = []
        self._check(L.thp_set_params(self.h, _p(_f64(ws.polarity)), _p(_f64(ws.thole)), _p(_f64(ws.pdamp))),
                    "thp_set_params")
        offs = (_ip * 8)()
        idxs = (_ip * 8)()
        for q, name in enumerate(CONN_NAMES):
            off, idx = ws.conn[name]
            off, idx = _i32(off), _i32(idx if len(idx) else np.zeros(1, np.int32))
            self._keep += [off, idx]
            offs[q] = _p(off, _ip)
            idxs[q] = _p(idx, _ip)
        self._check(L.thp_set_connectivity(self.h, offs, idxs, _p(scales_array(ws))), "thp_set_connectivity")
        self._check(L.thp_set_mpole_scales(self.h, _p(_f64(ws.scales["m_scale"]))), "thp_set_mpole_scales")
        if getattr(ws, "vdw", None) is not None and 2.0 * (ws.vdw["vdwcut"] + ws.lbuffer) <= min(ws.box):
            self.set_vdw(ws.vdw)
        self.set_positions(ws.x, ws.y, ws.z)
        if rpole is not None:
            self.set_rpole(rpole)
        elif frames:
            self._check(L.thp_set_frames(self.h, _p(_f64(ws.pole)), _p(_i32(ws.zaxis), _ip),
                                         _p(_i32(ws.xaxis), _ip), _p(_i32(ws.axt), _ip)), "thp_set_frames")

    def _check(self, st, what):
        if st not in (THP_OK,):
            raise ThpError(st, what)
        return st

    def close(self):
        if getattr(self, "h", None):
            load().thp_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        self._check(load().thp_set_stream(self.h, C.c_void_p(stream_ptr)), "thp_set_stream")

    def set_positions(self, x, y, z):
        self._x, self._y, self._z = _f64(x), _f64(y), _f64(z)
        self._check(load().thp_set_positions(self.h, _p(self._x), _p(self._y), _p(self._z)), "thp_set_positions")

    def set_rpole(self, rpole):
        self._check(load().thp_set_rpole(self.h, _p(_f64(rpole))), "thp_set_rpole")

    def set_predictor(self, mode):
        self._check(load().thp_set_predictor(self.h, int(mode)), "thp_set_predictor")

    def set_guess(self, mu):
        self._check(load().thp_set_guess(self.h, _p(_f64(mu))), "thp_set_guess")

    def nblist(self):
        self._check(load().thp_nblist(self.h), "thp_nblist")

    def invalidate_list(self):
        self._check(load().thp_invalidate_list(self.h), "thp_invalidate_list")

    def profile(self, enable):
        """Start (enable=1) or stop event recording around the real-space CG matvec row;
        returns (total ms, launches) recorded since the last call."""
        ms = C.c_double()
        cnt = C.c_int()
        self._check(load().thp_profile(self.h, int(enable), C.byref(ms), C.byref(cnt)), "thp_profile")
        return ms.value, cnt.value

    def solve(self, guess=GUESS_DIRECT, allow_unconverged=False):
        info = ThpSolveInfo()
        st = load().thp_solve(self.h, guess, C.byref(info))
        if st != THP_OK and not (allow_unconverged and st == THP_E_NOT_CONVERGED):
            raise ThpError(st, "thp_solve")
        return {"niter": info.niter, "converged": bool(info.converged), "resnrm": info.resnrm, "epol": info.epol,
                "ene": tuple(info.ene), "ms": info.ms_total, "status": st}

    def dipoles(self):
        uind = np.zeros((self.n, 3))
        uinp = np.zeros((self.n, 3))
        self._check(load().thp_get_dipoles(self.h, _p(uind), _p(uinp)), "thp_get_dipoles")
        return uind, uinp

    def gradient(self, out=None):
        """(Epol, dEpol/dx [n,3] kcal/mol/A) for the dipoles of the last solve;
        `out` (a C-contiguous float64 [n,3] array, e.g. pinned) receives it."""
        dep = np.zeros((self.n, 3)) if out is None else out
        assert dep.shape == (self.n, 3) and dep.dtype == np.float64 and dep.flags["C_CONTIGUOUS"]
        ep = C.c_double()
        self._check(load().thp_get_gradient(self.h, _p(dep), C.byref(ep)), "thp_get_gradient")
        return ep.value, dep

    def set_virial(self, on=True):
        """Later gradient and empole1 calls also compute their virials."""
        self._check(load().thp_set_virial(self.h, 1 if on else 0), "thp_set_virial")

    def virial(self, form=0):
        """vir [3,3] (kcal/mol) of the last gradient call made with the virial
        on; form 1 adds the reciprocal and self torques' frame-atom terms."""
        v = np.zeros((3, 3))
        self._check(load().thp_get_virial(self.h, int(form), _p(v)), "thp_get_virial")
        return v

    def empole_virial(self, form=0):
        """vir [3,3] (kcal/mol) of the last empole1 call made with the virial
        on; form 1 adds the reciprocal torques' frame-atom terms."""
        v = np.zeros((3, 3))
        self._check(load().thp_get_empole_virial(self.h, int(form), _p(v)), "thp_get_empole_virial")
        return v

    def ehal_virial(self):
        """vir [3,3] (kcal/mol) of the last ehal1 call made with the virial on."""
        v = np.zeros((3, 3))
        self._check(load().thp_get_ehal_virial(self.h, _p(v)), "thp_get_ehal_virial")
        return v

    def set_vdw(self, v):
        """van der Waals description (water.water_vdw layout)."""
        nc = int(v["nclass"])
        tab = np.ascontiguousarray(np.stack([np.asarray(v[k], dtype=np.float64).reshape(nc, nc)
                                             for k in ("radmin", "eps", "radmin4", "eps4")]))
        keep = [_i32(v["cls"]), _i32(v["ired"]), _f64(v["kred"]), tab, _f64(v["v_scale"])]
        self._keep += keep
        self._check(load().thp_set_vdw(self.h, _p(keep[0], _ip), nc, _p(keep[3]), _p(keep[1], _ip), _p(keep[2]),
                                       _p(keep[4]), float(v["vdwcut"]), float(v["vdwtaper"]), float(v["ghal"]),
                                       float(v["dhal"])), "thp_set_vdw")

    def ehal1(self, out=None):
        """(Ev, dEv/dx [n,3] kcal/mol/A): buffered 14-7 van der Waals energy
        and gradient at the current positions (ehal1c)."""
        dev = np.zeros((self.n, 3)) if out is None else out
        assert dev.shape == (self.n, 3) and dev.dtype == np.float64 and dev.flags["C_CONTIGUOUS"]
        ev = C.c_double()
        self._check(load().thp_ehal1(self.h, C.byref(ev), _p(dev)), "thp_ehal1")
        return ev.value, dev

    def vdw_pairs(self, maxvlst=1200):
        """Sorted (i, k) pairs of the vdW half list (vlistcell) as [P,2]."""
        nv = np.zeros(self.n, np.int32)
        vl = np.zeros(self.n * maxvlst, np.int32)
        self._check(load().thp_get_vlist(self.h, maxvlst, _p(nv, _ip), _p(vl, _ip)), "thp_get_vlist")
        vl = vl.reshape(self.n, maxvlst)
        rows = np.repeat(np.arange(self.n), nv)
        cols = vl[np.arange(maxvlst)[None, :] < nv[:, None]]
        p = np.stack([rows, cols], axis=1)
        return p[np.lexsort((p[:, 1], p[:, 0]))]

    def empole1(self, out=None):
        """(Em, dEm/dx [n,3] kcal/mol/A): permanent-multipole energy and
        gradient at the current positions (empole1c); `out` (a C-contiguous
        float64 [n,3] array, e.g. pinned) receives the gradient."""
        dem = np.zeros((self.n, 3)) if out is None else out
        assert dem.shape == (self.n, 3) and dem.dtype == np.float64 and dem.flags["C_CONTIGUOUS"]
        em = C.c_double()
        self._check(load().thp_empole1(self.h, C.byref(em), _p(dem)), "thp_empole1")
        return em.value, dem

    def md_verlet(self, nsteps, dt, mass, vel):
        """Velocity-Verlet NVE steps on the device (dt in ps).  Returns
        (velocities [n,3], energies [nsteps,3] = epol/kinetic/total, CG
        iterations [nsteps]); positions() gives the advanced positions."""
        vel = np.ascontiguousarray(vel, dtype=np.float64).copy()
        en = np.zeros((nsteps, 3))
        it = np.zeros(nsteps, np.int32)
        self._check(load().thp_md_verlet(self.h, nsteps, dt, _p(_f64(mass)), _p(vel), _p(en), _p(it, _ip)),
                    "thp_md_verlet")
        return vel, en, it

    def positions(self):
        x, y, z = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        self._check(load().thp_get_positions(self.h, _p(x), _p(y), _p(z)), "thp_get_positions")
        return np.stack([x, y, z], axis=1)

    def field(self):
        ef = np.zeros((self.n, 2, 3))
        self._check(load().thp_get_field(self.h, _p(ef)), "thp_get_field")
        return ef

    def rpole(self):
        rp = np.zeros((self.n, 13))
        self._check(load().thp_get_rpole(self.h, _p(rp)), "thp_get_rpole")
        return rp

    def nblist_half(self, maxelst=1200):
        nelst = np.zeros(self.n, np.int32)
        elst = np.zeros((self.n, maxelst), np.int32)
        self._check(load().thp_get_nblist(self.h, maxelst, _p(nelst, _ip), _p(elst, _ip)), "thp_get_nblist")
        return nelst, elst

    def pairs(self, maxelst=1200):
        nelst, elst = self.nblist_half(maxelst)
        rows = np.repeat(np.arange(self.n), nelst)
        mask = np.arange(elst.shape[1])[None, :] < nelst[:, None]
        p = np.stack([rows, elst[mask]], axis=1)
        return p[np.lexsort((p[:, 1], p[:, 0]))]

    def tmatxb(self, mu, dodiag=True):
        mu = _f64(mu)
        out = np.zeros_like(mu)
        self._check(load().thp_tmatxb(self.h, mu.shape[1], int(dodiag), _p(mu), _p(out)), "thp_tmatxb")
        return out

    def efld0_direct(self, nrhs=2):
        ef = np.zeros((self.n, nrhs, 3))
        self._check(load().thp_efld0_direct(self.h, nrhs, _p(ef)), "thp_efld0_direct")
        return ef

    def efld0_recip(self):
        cphi = np.zeros((self.n, 10))
        self._check(load().thp_efld0_recip(self.h, _p(cphi)), "thp_efld0_recip")
        return cphi

    def tmatxbrecip(self, mu):
        mu = _f64(mu)
        out = np.zeros_like(mu)
        self._check(load().thp_tmatxbrecip(self.h, mu.shape[1], _p(mu), _p(out)), "thp_tmatxbrecip")
        return out

    def solve_host(self, x, y, z, rpole=None, out=None):
        """One call on host buffers: positions in, dipoles and energy out.
        `out` = (uind, uinp) C-contiguous float64 [n,3] arrays to fill (for
        example views of pinned memory, which the copies DMA into)."""
        if out is None:
            uind = np.zeros((self.n, 3))
            uinp = np.zeros((self.n, 3))
        else:
            uind, uinp = out
            for a in out:
                if a.dtype != np.float64 or a.shape != (self.n, 3) or not a.flags.c_contiguous:
                    raise ValueError("out arrays must be C-contiguous float64 [n, 3]")
        info = ThpSolveInfo()
        st = load().thp_solve_host(self.h, _p(_f64(x)), _p(_f64(y)), _p(_f64(z)),
                                   None if rpole is None else _p(_f64(rpole)), _p(uind), _p(uinp),
                                   C.byref(info))
        if st not in (THP_OK, THP_E_NOT_CONVERGED):
            raise ThpError(st, "thp_solve_host")
        return uind, uinp, {"niter": info.niter, "converged": bool(info.converged), "epol": info.epol,
                            "ms": info.ms_total}


def system_struct(ws, keep):
    """thp_system for a water.WaterSystem; `keep` collects the arrays the
    pointers refer to (they must live until the call that copies them)."""
    sysd = ThpSystem()
    sysd.cfg = config_for(ws)
    arr = {k: _f64(getattr(ws, k)) for k in ("polarity", "thole", "pdamp", "pole")}
    ax = {k: _i32(getattr(ws, k)) for k in ("zaxis", "xaxis", "axt")}
    sc = scales_array(ws)
    offs, idxs = (_ip * 8)(), (_ip * 8)()
    for q, name in enumerate(CONN_NAMES):
        off, idx = ws.conn[name]
        off, idx = _i32(off), _i32(idx if len(idx) else np.zeros(1, np.int32))
        keep += [off, idx]
        offs[q], idxs[q] = _p(off, _ip), _p(idx, _ip)
    keep += list(arr.values()) + list(ax.values()) + [sc, offs, idxs]
    sysd.polarity, sysd.thole, sysd.pdamp, sysd.pole = (_p(arr[k]) for k in ("polarity", "thole", "pdamp", "pole"))
    sysd.zaxis, sysd.xaxis, sysd.axt = (_p(ax[k], _ip) for k in ("zaxis", "xaxis", "axt"))
    sysd.scales = _p(sc)
    sysd.conn_off = C.cast(offs, C.POINTER(_ip))
    sysd.conn_idx = C.cast(idxs, C.POINTER(_ip))
    return sysd
