"""Batched per-site PME routines (grid_uind_sites_, fphi_uind_sites_) and the
reference-signature per-site stubs against the oracle's restatement of
grid_uind_site (pmestuff.f:280) and fphi_uind_site (pmestuff.f:746), FP64, on
the caller's grid qgrid(2,n1,n2,n3).  Tolerance 1e-12 of the largest value."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
I = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))


@pytest.fixture(scope="module")
def setup(thp):
    from tinker_hp_b200 import lib
    L = lib.load()
    ws = thp.water.make_water_box(216, cfg=0)
    ctx = lib.Context(ws)
    xyz = [np.ascontiguousarray(a) for a in (ws.x, ws.y, ws.z)]
    assert L.thp_bind_state(ctx.h, P(xyz[0]), P(xyz[1]), P(xyz[2]), None, None, None, None, None, 0, None) == 0
    return L, ws, ctx, O.Oracle(ws), xyz


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_grid_uind_sites_adds_like_reference(setup):
    L, ws, ctx, orc, _ = setup
    rng = np.random.default_rng(21)
    n1, n2, n3 = ws.nfft
    sites = np.sort(rng.choice(ws.n, size=300, replace=False)).astype(np.int32)
    fuind = rng.standard_normal((300, 3))
    fuinp = rng.standard_normal((300, 3))
    grid0 = rng.standard_normal((n3, n2, n1)) + 1j * rng.standard_normal((n3, n2, n1))
    want = orc.grid_uind_sites(sites, fuind, fuinp, grid0)
    got = np.ascontiguousarray(grid0.copy())
    f1 = (sites + 1).astype(np.int32)
    L.grid_uind_sites_(C.byref(C.c_int(300)), I(f1), P(fuind), P(fuinp), P(got.view(np.float64)))
    assert L.thp_last_error() == 0
    assert rel(got - grid0, want - grid0) < 1e-12
    # the reference signature, one site
    one = np.ascontiguousarray(grid0.copy())
    L.grid_uind_site_(C.byref(C.c_int(int(f1[7]))), C.byref(C.c_int(1)), P(np.ascontiguousarray(fuind[7])),
                      P(np.ascontiguousarray(fuinp[7])), P(one.view(np.float64)))
    assert L.thp_last_error() == 0
    want1 = orc.grid_uind_sites(sites[7:8], fuind[7:8], fuinp[7:8], grid0)
    assert rel(one - grid0, want1 - grid0) < 1e-12


def test_fphi_uind_sites_matches_reference(setup):
    L, ws, ctx, orc, _ = setup
    rng = np.random.default_rng(22)
    n1, n2, n3 = ws.nfft
    grid = np.ascontiguousarray(rng.standard_normal((n3, n2, n1)) + 1j * rng.standard_normal((n3, n2, n1)))
    sites = np.arange(0, ws.n, 3, dtype=np.int32)
    w1, w2, ws_ = orc.fphi_uind_sites(sites, grid)
    ns = len(sites)
    p1, p2, sm = np.zeros((ns, 10)), np.zeros((ns, 10)), np.zeros((ns, 20))
    f1 = (sites + 1).astype(np.int32)
    L.fphi_uind_sites_(C.byref(C.c_int(ns)), I(f1), P(grid.view(np.float64)), P(p1), P(p2), P(sm))
    assert L.thp_last_error() == 0
    assert rel(p1, w1) < 1e-12 and rel(p2, w2) < 1e-12 and rel(sm, ws_) < 1e-12
    assert np.all(p1[:, 0] == 0) and np.all(p2[:, 0] == 0)
    # per-site stub reads the bound grid
    assert L.thp_bind_grid(ctx.h, P(grid.view(np.float64))) == 0
    q1, q2, qs = np.zeros(10), np.zeros(10), np.zeros(20)
    L.fphi_uind_site_(C.byref(C.c_int(int(f1[5]))), C.byref(C.c_int(1)), P(q1), P(q2), P(qs))
    assert L.thp_last_error() == 0
    assert rel(q1, w1[5]) < 1e-12 and rel(qs, ws_[5]) < 1e-12


def test_site_numbers_are_checked(setup):
    L, ws, ctx, orc, _ = setup
    n1, n2, n3 = ws.nfft
    grid = np.zeros(2 * n1 * n2 * n3)
    bad = np.array([0], np.int32)  # Fortran numbers start at 1
    f = np.zeros(3)
    L.grid_uind_sites_(C.byref(C.c_int(1)), I(bad), P(f), P(f), P(grid))
    assert L.thp_last_error() == 1  # THP_E_INVALID
    assert not grid.any()
