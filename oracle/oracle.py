"""ctypes loader for the CPU FP64 oracle -- TEST INFRASTRUCTURE, NOT THE PRODUCT.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this module.  It wraps oracle/libthp_oracle.so (built by oracle/Makefile), the
C++ restatement of the Tinker-HP v1.2 polarization path.  Parity status:
unpinned by the reference (no golden vectors exist for this path); pinned by
self-consistency tests in tests/test_oracle.py.
"""

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libthp_oracle.so")

CONN_NAMES = ("i12", "i13", "i14", "i15", "ip11", "ip12", "ip13", "ip14")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class OrSystem(C.Structure):
    _fields_ = [
        ("n", C.c_int),
        ("xbox", C.c_double), ("ybox", C.c_double), ("zbox", C.c_double),
        ("x", _dp), ("y", _dp), ("z", _dp),
        ("rpole", _dp), ("polarity", _dp), ("thole", _dp), ("pdamp", _dp),
        ("conn_off", _ip * 8), ("conn_idx", _ip * 8),
        ("p_scale", C.c_double * 4), ("pi_scale", C.c_double * 4),
        ("d_scale", C.c_double * 4), ("u_scale", C.c_double * 4),
        ("aewald", C.c_double), ("ewaldcut", C.c_double), ("lbuffer", C.c_double),
        ("vdwcut", C.c_double),
        ("nfft1", C.c_int), ("nfft2", C.c_int), ("nfft3", C.c_int), ("bsorder", C.c_int),
        ("politer", C.c_int), ("poleps", C.c_double), ("nthreads", C.c_int),
        ("m_scale", C.c_double * 4),
    ]


class OrVdw(C.Structure):
    _fields_ = [
        ("nclass", C.c_int), ("cls", _ip), ("radmin", _dp), ("eps", _dp), ("radmin4", _dp), ("eps4", _dp),
        ("ired", _ip), ("kred", _dp), ("v_scale", C.c_double * 4), ("vdwcut", C.c_double),
        ("vdwtaper", C.c_double), ("ghal", C.c_double), ("dhal", C.c_double),
    ]


class OrSolveInfo(C.Structure):
    _fields_ = [("niter", C.c_int), ("converged", C.c_int), ("resnrm", C.c_double),
                ("ene", C.c_double * 2)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.or_create.restype = C.c_void_p
        L.or_create.argtypes = [C.POINTER(OrSystem)]
        L.or_destroy.argtypes = [C.c_void_p]
        L.or_mlistcell.argtypes = [C.c_void_p, C.c_int, _ip, _ip]
        L.or_efld0_direct.argtypes = [C.c_void_p, _dp]
        L.or_tmatxb_pme.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp]
        L.or_efld0_recip.argtypes = [C.c_void_p, _dp]
        L.or_tmatxbrecip.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        L.or_newinduce_pme2.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, C.POINTER(OrSolveInfo)]
        L.or_epolar.restype = C.c_double
        L.or_epolar.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        L.or_epolar1.argtypes = [C.c_void_p, _dp, _dp, _ip, _ip, _ip, _dp, _dp, _dp, _dp]
        L.or_empole1.argtypes = [C.c_void_p, _ip, _ip, _ip, _dp, _dp, _dp, _dp]
        L.or_ehal1.argtypes = [C.c_void_p, C.POINTER(OrVdw), _dp, _dp, _dp]
        L.or_rotpole.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _ip, _ip, _ip, _dp]
        L.or_grid_uind_sites.argtypes = [C.c_void_p, C.c_int, _ip, _dp, _dp, _dp]
        L.or_fphi_uind_sites.argtypes = [C.c_void_p, C.c_int, _ip, _dp, _dp, _dp, _dp]
        L.or_ewaldcof.restype = C.c_double
        L.or_ewaldcof.argtypes = [C.c_double]
        L.or_erfc.restype = C.c_double
        L.or_erfc.argtypes = [C.c_double]
        L.or_fft3d.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_int]
        _lib = L
    return _lib


def _p(a, t=_dp):
    return a.ctypes.data_as(t) if a is not None else None


def rotpole(ws):
    """Global-frame multipoles [n,13] for a water.WaterSystem (rotpole.f:17)."""
    n = ws.n
    rp = np.zeros((n, 13))
    pole = np.ascontiguousarray(ws.pole, dtype=np.float64)
    lib().or_rotpole(n, _p(ws.x), _p(ws.y), _p(ws.z), _p(pole), _p(ws.zaxis, _ip), _p(ws.xaxis, _ip),
                     _p(ws.axt, _ip), _p(rp))
    return rp


def fft3d(grid, sign):
    """In-place unnormalised complex FFT of a [n3,n2,n1] complex128 array."""
    g = np.ascontiguousarray(grid, dtype=np.complex128).copy()
    n3, n2, n1 = g.shape
    lib().or_fft3d(g.ctypes.data_as(_dp), n1, n2, n3, sign)
    return g


class Oracle:
    """One system on the CPU oracle. Vectors use the reference's (3,nrhs,n)
    interleave: shape [n, nrhs, 3]."""

    MAXELST = 1200  # MOD_sizes.f:58

    def __init__(self, ws, rpole=None, politer=500, poleps=1e-6, nthreads=1, vdwcut=9.0):
        self.ws = ws
        self.rpole = np.ascontiguousarray(rotpole(ws) if rpole is None else rpole, dtype=np.float64)
        self._keep = []
        s = OrSystem()
        s.n = ws.n
        s.xbox, s.ybox, s.zbox = ws.box
        self._x = np.ascontiguousarray(ws.x, dtype=np.float64)
        self._y = np.ascontiguousarray(ws.y, dtype=np.float64)
        self._z = np.ascontiguousarray(ws.z, dtype=np.float64)
        self._pol = np.ascontiguousarray(ws.polarity, dtype=np.float64)
        self._thl = np.ascontiguousarray(ws.thole, dtype=np.float64)
        self._pd = np.ascontiguousarray(ws.pdamp, dtype=np.float64)
        s.x, s.y, s.z = _p(self._x), _p(self._y), _p(self._z)
        s.rpole = _p(self.rpole)
        s.polarity, s.thole, s.pdamp = _p(self._pol), _p(self._thl), _p(self._pd)
        for q, name in enumerate(CONN_NAMES):
            off, idx = ws.conn[name]
            off = np.ascontiguousarray(off, dtype=np.int32)
            idx = np.ascontiguousarray(idx if len(idx) else np.zeros(1, np.int32), dtype=np.int32)
            self._keep += [off, idx]
            s.conn_off[q] = _p(off, _ip)
            s.conn_idx[q] = _p(idx, _ip)
        for key in ("p_scale", "pi_scale", "d_scale", "u_scale", "m_scale"):
            arr = getattr(s, key)
            for q in range(4):
                arr[q] = ws.scales[key][q]
        s.aewald, s.ewaldcut, s.lbuffer, s.vdwcut = ws.aewald, ws.ewaldcut, ws.lbuffer, vdwcut
        s.nfft1, s.nfft2, s.nfft3 = ws.nfft
        s.bsorder = ws.bsorder
        s.politer, s.poleps, s.nthreads = politer, poleps, nthreads
        self.sys = s
        self.ctx = lib().or_create(C.byref(s))
        self.nelst = None
        self.elst = None

    def close(self):
        if self.ctx:
            lib().or_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def mlistcell(self, maxelst=None):
        maxelst = maxelst or self.MAXELST
        n = self.ws.n
        nelst = np.zeros(n, np.int32)
        elst = np.zeros(n * maxelst, np.int32)
        st = lib().or_mlistcell(self.ctx, maxelst, _p(nelst, _ip), _p(elst, _ip))
        self.nelst, self.elst = nelst, elst.reshape(n, maxelst)
        return st, nelst, self.elst

    def pairs(self):
        """Sorted (i, k) half-list pairs as an [P,2] int array."""
        rows = np.repeat(np.arange(self.ws.n), self.nelst)
        mask = np.arange(self.elst.shape[1])[None, :] < self.nelst[:, None]
        cols = self.elst[mask]
        p = np.stack([rows, cols], axis=1)
        return p[np.lexsort((p[:, 1], p[:, 0]))]

    def efld0_direct(self):
        ef = np.zeros((self.ws.n, 2, 3))
        lib().or_efld0_direct(self.ctx, _p(ef))
        return ef

    def tmatxb(self, mu, dodiag=True):
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        efi = np.zeros_like(mu)
        lib().or_tmatxb_pme(self.ctx, mu.shape[1], int(dodiag), _p(mu), _p(efi))
        return efi

    def efld0_recip(self):
        cphi = np.zeros((self.ws.n, 10))
        lib().or_efld0_recip(self.ctx, _p(cphi))
        return cphi

    def tmatxbrecip(self, mu):
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        out = np.zeros_like(mu)
        lib().or_tmatxbrecip(self.ctx, mu.shape[1], _p(mu), _p(out))
        return out

    def solve(self, mu_guess=None):
        n = self.ws.n
        uind = np.zeros((n, 3))
        uinp = np.zeros((n, 3))
        ef = np.zeros((n, 2, 3))
        info = OrSolveInfo()
        g = None if mu_guess is None else np.ascontiguousarray(mu_guess, dtype=np.float64)
        st = lib().or_newinduce_pme2(self.ctx, _p(g), _p(uind), _p(uinp), _p(ef), C.byref(info))
        if st != 0:
            raise RuntimeError(f"oracle solve failed with status {st}")
        return {"uind": uind, "uinp": uinp, "ef": ef, "niter": info.niter,
                "converged": bool(info.converged), "resnrm": info.resnrm, "ene": tuple(info.ene)}

    def epolar1(self, uind, uinp, virial=False):
        """Energy and gradient dE/dx [n,3] (kcal/mol/A), epolar1c; with
        virial=True also the internal virial vir(3,3) (kcal/mol) as the
        reference accumulates it and the frame-atom virial of the
        reciprocal and self torques it leaves out (their sum is the strain
        derivative of the energy)."""
        uind = np.ascontiguousarray(uind, dtype=np.float64)
        uinp = np.ascontiguousarray(uinp, dtype=np.float64)
        dep = np.zeros((self.ws.n, 3))
        ep = C.c_double()
        ws = self.ws
        vir = np.zeros((3, 3)) if virial else None
        vfr = np.zeros((3, 3)) if virial else None
        st = lib().or_epolar1(self.ctx, _p(uind), _p(uinp), _p(np.ascontiguousarray(ws.zaxis, np.int32), _ip),
                              _p(np.ascontiguousarray(ws.xaxis, np.int32), _ip),
                              _p(np.ascontiguousarray(ws.axt, np.int32), _ip), _p(dep), C.byref(ep), _p(vir),
                              _p(vfr))
        if st != 0:
            raise RuntimeError(f"oracle epolar1 status {st}")
        if virial:
            return ep.value, dep, vir, vfr
        return ep.value, dep

    def empole1(self, virial=False):
        """Permanent-multipole energy and gradient, empole1c: returns
        (em, dem [n,3], parts) with parts = (real, recip, self) kcal/mol; with
        virial=True also the internal virial vir(3,3) (kcal/mol) as the
        reference accumulates it and the frame-atom virial of the reciprocal
        torques it leaves out (their sum is the strain derivative)."""
        dem = np.zeros((self.ws.n, 3))
        parts = np.zeros(4)
        ws = self.ws
        vir = np.zeros((3, 3)) if virial else None
        vfr = np.zeros((3, 3)) if virial else None
        st = lib().or_empole1(self.ctx, _p(np.ascontiguousarray(ws.zaxis, np.int32), _ip),
                              _p(np.ascontiguousarray(ws.xaxis, np.int32), _ip),
                              _p(np.ascontiguousarray(ws.axt, np.int32), _ip), _p(dem), _p(parts), _p(vir),
                              _p(vfr))
        if st != 0:
            raise RuntimeError(f"oracle empole1 status {st}")
        if virial:
            return parts[0], dem, tuple(parts[1:]), vir, vfr
        return parts[0], dem, tuple(parts[1:])

    def ehal1(self, vdw=None, virial=False):
        """Buffered 14-7 energy and gradient (ehal1c): (ev, dev [n,3]); with
        virial=True also the pairs' internal virial vir(3,3) (kcal/mol)."""
        v = self.ws.vdw if vdw is None else vdw
        keep = [np.ascontiguousarray(v["cls"], np.int32), np.ascontiguousarray(v["radmin"], np.float64),
                np.ascontiguousarray(v["eps"], np.float64), np.ascontiguousarray(v["radmin4"], np.float64),
                np.ascontiguousarray(v["eps4"], np.float64), np.ascontiguousarray(v["ired"], np.int32),
                np.ascontiguousarray(v["kred"], np.float64)]
        sv = OrVdw()
        sv.nclass = int(v["nclass"])
        sv.cls, sv.radmin, sv.eps, sv.radmin4, sv.eps4 = (_p(keep[0], _ip), _p(keep[1]), _p(keep[2]),
                                                          _p(keep[3]), _p(keep[4]))
        sv.ired, sv.kred = _p(keep[5], _ip), _p(keep[6])
        for q in range(4):
            sv.v_scale[q] = v["v_scale"][q]
        sv.vdwcut, sv.vdwtaper, sv.ghal, sv.dhal = v["vdwcut"], v["vdwtaper"], v["ghal"], v["dhal"]
        dev = np.zeros((self.ws.n, 3))
        ev = C.c_double()
        vir = np.zeros((3, 3)) if virial else None
        st = lib().or_ehal1(self.ctx, C.byref(sv), _p(dev), C.byref(ev), _p(vir))
        if st != 0:
            raise RuntimeError(f"oracle ehal1 status {st}")
        if virial:
            return ev.value, dev, vir
        return ev.value, dev

    def grid_uind_sites(self, sites, fuind, fuinp, grid):
        """grid_uind_site for 0-based `sites`: adds into a copy of the complex
        grid [n3,n2,n1] and returns it."""
        sites = np.ascontiguousarray(sites, dtype=np.int32)
        g = np.ascontiguousarray(grid, dtype=np.complex128).copy()
        st = lib().or_grid_uind_sites(self.ctx, len(sites), _p(sites, _ip), _p(np.ascontiguousarray(fuind, float)),
                                      _p(np.ascontiguousarray(fuinp, float)), g.ctypes.data_as(_dp))
        if st != 0:
            raise RuntimeError("oracle grid_uind_sites: bad site")
        return g

    def fphi_uind_sites(self, sites, grid):
        """fphi_uind_site for 0-based `sites` on a complex grid [n3,n2,n1]:
        (fdip_phi1 [ns,10], fdip_phi2 [ns,10], fdip_sum_phi [ns,20])."""
        sites = np.ascontiguousarray(sites, dtype=np.int32)
        g = np.ascontiguousarray(grid, dtype=np.complex128)
        p1, p2, sm = np.zeros((len(sites), 10)), np.zeros((len(sites), 10)), np.zeros((len(sites), 20))
        st = lib().or_fphi_uind_sites(self.ctx, len(sites), _p(sites, _ip), g.ctypes.data_as(_dp), _p(p1), _p(p2),
                                      _p(sm))
        if st != 0:
            raise RuntimeError("oracle fphi_uind_sites: bad site")
        return p1, p2, sm

    def epolar(self, uind):
        uind = np.ascontiguousarray(uind, dtype=np.float64)
        er, ek, es = C.c_double(), C.c_double(), C.c_double()
        e = lib().or_epolar(self.ctx, _p(uind), C.byref(er), C.byref(ek), C.byref(es))
        return e, {"real": er.value, "recip": ek.value, "self": es.value}


# kpolar.f:405-425
GEAR = (6.0, -15.0, 20.0, -15.0, 6.0, -1.0, 0.0)
ASPC = (22.0 / 7.0, -55.0 / 14.0, 55.0 / 21.0, -22.0 / 21.0, 5.0 / 21.0, -1.0 / 42.0, 0.0)
MAXUALT = 7  # MOD_uprior.f:33


def predict(history, mode):
    """ulspred (newinduce_pme2.f:910-1010) and the guess of :165-178:
    history is a list of [n,2,3] solutions, newest first, of length 7."""
    m = len(history)
    if mode in ("ASPC", "GEAR"):
        b = ASPC if mode == "ASPC" else GEAR
        bd = bp = np.array(b[: m - 1])
    else:  # least-squares fit of the newest solution on the six before it
        coef = []
        for r in (0, 1):
            a = np.array([h[:, r, :].ravel() for h in history])
            c = a @ a.T
            coef.append(np.linalg.solve(c[1:, 1:], c[0, 1:]))
        bd, bp = coef
    g = np.zeros_like(history[0])
    for k in range(m - 1):
        g[:, 0, :] += bd[k] * history[k][:, 0, :]
        g[:, 1, :] += bp[k] * history[k][:, 1, :]
    return g


def verlet(ws, vel, mass, dt, nsteps, poleps=1e-8, predictor=None):
    """Velocity-Verlet NVE with the polarization gradient as the only force
    (verlet.f:17-200; a = -convert * dE/dx / m, units.f:76).  Each solve
    starts from the direct guess, or, with a predictor ("ASPC", "GEAR",
    "LSQR"), from its extrapolation once seven solutions are stored.  Returns
    (positions [n,3], velocities [n,3], energies [nsteps,3] =
    epol/kinetic/total, CG iterations [nsteps])."""
    convert = 418.4
    m = np.asarray(mass, dtype=np.float64)[:, None]
    v = np.array(vel, dtype=np.float64)
    pos = ws.positions().copy()
    history = []

    def grad(p):
        w = ws.with_positions(p)
        o = Oracle(w, poleps=poleps)
        if o.mlistcell()[0] != 0:
            raise RuntimeError("oracle list overflow")
        guess = predict(history, predictor) if predictor and len(history) == MAXUALT else None
        r = o.solve(guess)
        if predictor:
            history.insert(0, np.stack([r["uind"], r["uinp"]], axis=1))
            del history[MAXUALT:]
        ep, dep = o.epolar1(r["uind"], r["uinp"])
        o.close()
        return ep, dep, r["niter"]

    _, g, _ = grad(pos)
    out = np.zeros((nsteps, 3))
    its = np.zeros(nsteps, dtype=int)
    for s in range(nsteps):
        v += -convert * g / m * (0.5 * dt)
        pos += v * dt
        ep, g, its[s] = grad(pos)
        v += -convert * g / m * (0.5 * dt)
        ek = 0.5 * np.sum(m * v * v) / convert
        out[s] = (ep, ek, ep + ek)
    return pos, v, out, its
