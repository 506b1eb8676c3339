"""Permanent-multipole energy and gradient (empole1c) of the CUDA path against
the CPU oracle.

The oracle's empole1 is pinned by finite differences, classical Ewald sums,
alpha invariance and the two-water vacuum limit (tests/test_oracle.py).  FP64
form: energy within 1e-12 of the sum of the real, reciprocal and self parts'
magnitudes (the total is their small difference: at 32,400 atoms it is 3e-4
of them), gradient within 1e-9 of its largest component.  Mixed form (FP32 unscaled pairs and grid; FP64 scaled pairs,
reciprocal sums and self term): energy within 1e-8 of the sum of the parts'
magnitudes, force RMS error within 1e-5 of the force RMS (measured: 1e-9 and
2e-6).
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib(thp):
    from tinker_hp_b200 import lib as L
    L.load()
    return L


@pytest.fixture(scope="module", params=[216, 648], ids=["216w", "648w"])
def case(request, thp):
    ws = thp.water.make_water_box(request.param, cfg=0)
    orc = O.Oracle(ws)
    assert orc.mlistcell()[0] == 0
    return ws, orc.empole1()


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def parts_scale(parts):
    return sum(abs(p) for p in parts)


def test_empole1_fp64_matches_oracle(lib, case):
    ws, (em_ref, dem_ref, parts) = case
    ctx = lib.Context(ws)
    em, dem = ctx.empole1()
    assert abs(em - em_ref) < 1e-12 * parts_scale(parts), (em, em_ref)
    assert rel(dem, dem_ref) < 1e-9, rel(dem, dem_ref)


def test_empole1_mixed_error(lib, case):
    ws, (em_ref, dem_ref, parts) = case
    ctx = lib.Context(ws, precision=lib.MIXED)
    em, dem = ctx.empole1()
    scale_e = sum(abs(p) for p in parts)
    err = np.sqrt(np.mean(np.sum((dem - dem_ref) ** 2, axis=1)))
    scale = np.sqrt(np.mean(np.sum(dem_ref ** 2, axis=1)))
    print(f"mixed empole: energy error {em - em_ref:.3e} of parts {scale_e:.3e}; "
          f"force RMS error {err:.3e} of RMS {scale:.3e} ({err / scale:.2e})")
    assert abs(em - em_ref) < 1e-8 * scale_e, (em, em_ref)
    assert err < 1e-5 * scale, (err, scale)


def test_empole1_after_solve_and_moves(lib, thp):
    # a solve between calls and displacements below and above the list
    # buffer: the list is reused or rebuilt as for a solve, the multipoles are
    # re-rotated, and the result follows the oracle at each geometry
    ws = thp.water.make_water_box(216, cfg=0)
    ctx = lib.Context(ws)
    ctx.solve()
    rng = np.random.default_rng(11)
    for amp in (0.0, 0.05, 0.6):
        pos = ws.positions() + rng.normal(0.0, amp, (ws.n, 3)) if amp else ws.positions()
        w2 = ws.with_positions(pos)
        ctx.set_positions(w2.x, w2.y, w2.z)
        em, dem = ctx.empole1()
        orc = O.Oracle(w2)
        assert orc.mlistcell()[0] == 0
        em_ref, dem_ref, parts = orc.empole1()
        assert abs(em - em_ref) < 1e-12 * parts_scale(parts), (amp, em, em_ref)
        assert rel(dem, dem_ref) < 1e-9, (amp, rel(dem, dem_ref))


def test_empole1_large_box(lib, thp):
    # 10,800 waters (32,400 atoms, 60^3 grid): many cells and blocks
    ws = thp.water.make_water_box(10800, cfg=1)
    orc = O.Oracle(ws)
    assert orc.mlistcell()[0] == 0
    em_ref, dem_ref, parts = orc.empole1()
    em, dem = lib.Context(ws).empole1()
    assert abs(em - em_ref) < 1e-12 * parts_scale(parts), (em, em_ref, parts)
    assert rel(dem, dem_ref) < 1e-9, rel(dem, dem_ref)


def test_empole1_fortran_dropin(lib, thp):
    ws = thp.water.make_water_box(216, cfg=0)
    orc = O.Oracle(ws)
    assert orc.mlistcell()[0] == 0
    em_ref, dem_ref, parts = orc.empole1()
    L = lib.load()
    ctx = lib.Context(ws)
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (ws.x, ws.y, ws.z))
    rpole = np.ascontiguousarray(orc.rpole)
    uind, uinp = np.zeros((ws.n, 3)), np.zeros((ws.n, 3))
    em = np.zeros(1)
    dem = np.full((ws.n, 3), 7.0)  # overwritten, as empole1c zeroes dem
    st = L.thp_bind_state(ctx.h, x.ctypes.data_as(C.POINTER(C.c_double)), y.ctypes.data_as(C.POINTER(C.c_double)),
                          z.ctypes.data_as(C.POINTER(C.c_double)), rpole.ctypes.data_as(C.POINTER(C.c_double)),
                          uind.ctypes.data_as(C.POINTER(C.c_double)), uinp.ctypes.data_as(C.POINTER(C.c_double)),
                          None, None, 0, None)
    assert st == 0
    assert L.thp_bind_mpole(ctx.h, em.ctypes.data_as(C.POINTER(C.c_double)),
                            dem.ctypes.data_as(C.POINTER(C.c_double))) == 0
    L.empole1_()
    assert L.thp_last_error() == 0
    assert abs(em[0] - em_ref) < 1e-12 * parts_scale(parts)
    assert rel(dem, dem_ref) < 1e-9


def test_empole1_needs_frames(lib, thp):
    ws = thp.water.make_water_box(216, cfg=0)
    ctx = lib.Context(ws, frames=False, rpole=O.rotpole(ws))
    with pytest.raises(lib.ThpError) as e:
        ctx.empole1()
    assert e.value.status == lib.THP_E_STATE


def _with_extra_14_15(ws, rng):
    """The box with artificial 1-4 and 1-5 relations between oxygens of
    nearby molecules (symmetric), so the m4/m5 scales and the vdW 1-4
    parameters take part (water itself has only 1-2 and 1-3 pairs)."""
    import dataclasses
    pos = ws.positions()
    L = np.asarray(ws.box)
    ox = np.arange(0, ws.n, 3)
    rows14 = [[] for _ in range(ws.n)]
    rows15 = [[] for _ in range(ws.n)]
    for a in ox[: len(ox) // 2]:
        d = pos[ox] - pos[a]
        d -= L * np.round(d / L)
        r = np.sqrt(np.einsum("ij,ij->i", d, d))
        near = [int(b) for b in ox[np.argsort(r)[1:3]]]
        for rows, b in ((rows14, near[0]), (rows15, near[1])):
            if b not in rows[a] and b not in rows14[a] and b not in rows15[a]:
                rows[a].append(b)
                rows[b].append(a)

    def csr(rows):
        off = np.zeros(ws.n + 1, np.int32)
        off[1:] = np.cumsum([len(r) for r in rows])
        return off, np.array([v for r in rows for v in sorted(r)], dtype=np.int32)

    conn = dict(ws.conn)
    conn["i14"], conn["i15"] = csr(rows14), csr(rows15)
    v = dict(ws.vdw)
    v["radmin4"] = np.asarray(v["radmin"]) * 0.9
    v["eps4"] = np.asarray(v["eps"]) * 0.5
    v["v_scale"] = (0.0, 0.0, 0.7, 0.9)
    sc = dict(ws.scales)
    sc["m_scale"] = (0.0, 0.0, 0.4, 0.8)
    return dataclasses.replace(ws, conn=conn, vdw=v, scales=sc)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_scaled_14_15_pairs_match_oracle(lib, thp, precision):
    ws = _with_extra_14_15(thp.water.make_water_box(648, cfg=0), np.random.default_rng(2))
    orc = O.Oracle(ws)
    assert orc.mlistcell()[0] == 0
    em_ref, dem_ref, parts = orc.empole1()
    ev_ref, dev_ref = orc.ehal1()
    ctx = lib.Context(ws, precision=lib.FP64 if precision == "fp64" else lib.MIXED)
    em, dem = ctx.empole1()
    ev, dev = ctx.ehal1()
    if precision == "fp64":
        assert abs(em - em_ref) < 1e-12 * parts_scale(parts), (em, em_ref)
        assert rel(dem, dem_ref) < 1e-9
        assert abs(ev - ev_ref) < 1e-10 * abs(ev_ref), (ev, ev_ref)
        assert rel(dev, dev_ref) < 1e-9
    else:
        assert abs(em - em_ref) < 1e-8 * parts_scale(parts), (em, em_ref)
        assert abs(ev - ev_ref) < 1e-5 * abs(ev_ref), (ev, ev_ref)
    # and the scaled pairs matter: the unmodified box gives other energies
    base = lib.Context(thp.water.make_water_box(648, cfg=0))
    assert abs(base.empole1()[0] - em_ref) > 1e-3 and abs(base.ehal1()[0] - ev_ref) > 1e-3
