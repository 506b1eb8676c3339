"""Buffered 14-7 van der Waals energy and gradient (ehal1c) of the CUDA path
against the CPU oracle (itself pinned by a textbook-form direct sum and finite
differences in tests/test_oracle.py).  FP64 form: energy within 1e-10
relative, gradient within 1e-9 of its largest component.  Mixed form (FP32
pair terms from FP32 wrapped sites, FP64 accumulation): energy within 1e-5
relative, force RMS error within 1e-5 of the force RMS."""
import ctypes as C
import dataclasses

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib(thp):
    from tinker_hp_b200 import lib as L
    L.load()
    return L


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nw,edge", [(216, 20.0), (648, None)], ids=["216w", "648w"])
def test_ehal1_matches_oracle(lib, thp, precision, nw, edge):
    ws = thp.water.make_water_box(nw, cfg=0, edge=edge)
    ev_ref, dev_ref = O.Oracle(ws).ehal1()
    ctx = lib.Context(ws, precision=lib.FP64 if precision == "fp64" else lib.MIXED)
    ev, dev = ctx.ehal1()
    if precision == "fp64":
        assert abs(ev - ev_ref) < 1e-10 * abs(ev_ref), (ev, ev_ref)
        assert rel(dev, dev_ref) < 1e-9, rel(dev, dev_ref)
    else:
        err = np.sqrt(np.mean(np.sum((dev - dev_ref) ** 2, axis=1)))
        scale = np.sqrt(np.mean(np.sum(dev_ref ** 2, axis=1)))
        print(f"mixed ehal: energy error {(ev - ev_ref) / ev_ref:.2e} relative; force RMS error {err / scale:.2e}")
        assert abs(ev - ev_ref) < 1e-5 * abs(ev_ref), (ev, ev_ref)
        assert err < 1e-5 * scale, (err, scale)


def test_ehal1_large_box_and_moves(lib, thp):
    # 32,400 atoms: cell reach over many cells; then whole-molecule
    # displacements below and above the list buffer (the cell sort is kept,
    # then rebuilt); molecules move rigidly so the reduced sites stay on
    # their bonds
    ws = thp.water.make_water_box(10800, cfg=1)
    ctx = lib.Context(ws)
    rng = np.random.default_rng(3)
    for amp in (0.0, 0.1, 0.6):
        shift = np.repeat(rng.normal(0.0, amp, (ws.nw, 3)), 3, axis=0)
        w2 = ws.with_positions(ws.positions() + shift) if amp else ws
        ctx.set_positions(w2.x, w2.y, w2.z)
        ev, dev = ctx.ehal1()
        ev_ref, dev_ref = O.Oracle(w2).ehal1()
        assert abs(ev - ev_ref) < 1e-10 * abs(ev_ref), (amp, ev, ev_ref)
        assert rel(dev, dev_ref) < 1e-9, (amp, rel(dev, dev_ref))


def test_ehal1_fortran_dropin(lib, thp):
    ws = thp.water.make_water_box(648, cfg=0)
    ev_ref, dev_ref = O.Oracle(ws).ehal1()
    L = lib.load()
    ctx = lib.Context(ws)
    dp = C.POINTER(C.c_double)
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (ws.x, ws.y, ws.z))
    rp = np.ascontiguousarray(O.rotpole(ws))
    u1, u2 = np.zeros((ws.n, 3)), np.zeros((ws.n, 3))
    assert L.thp_bind_state(ctx.h, x.ctypes.data_as(dp), y.ctypes.data_as(dp), z.ctypes.data_as(dp),
                            rp.ctypes.data_as(dp), u1.ctypes.data_as(dp), u2.ctypes.data_as(dp), None, None, 0,
                            None) == 0
    ev = np.zeros(1)
    dev = np.full((ws.n, 3), 5.0)  # overwritten, as ehal1c zeroes dev
    assert L.thp_bind_vdw(ctx.h, ev.ctypes.data_as(dp), dev.ctypes.data_as(dp)) == 0
    L.ehal1_()
    assert L.thp_last_error() == 0
    assert abs(ev[0] - ev_ref) < 1e-10 * abs(ev_ref)
    assert rel(dev, dev_ref) < 1e-9


def test_ehal1_refuses_a_reduction_beyond_the_reach(lib, thp):
    # H sites reduced to half their bond (0.48 A shift): the pair search's
    # cell reach assumes at most 0.3 A, so the call reports it
    ws = thp.water.make_water_box(648, cfg=0)
    v = dict(ws.vdw)
    v["kred"] = np.where(v["cls"] == 0, 0.0, 0.5)
    ctx = lib.Context(dataclasses.replace(ws, vdw=v))
    with pytest.raises(lib.ThpError) as e:
        ctx.ehal1()
    assert e.value.status == lib.THP_E_INVALID


def _vdw_pairs_bruteforce(ws):
    v = ws.vdw
    pos = ws.positions()
    par = pos[v["ired"]]
    red = v["kred"][:, None] * (pos - par) + par
    L = np.asarray(ws.box)
    vbuf2 = (v["vdwcut"] + ws.lbuffer) ** 2
    out = []
    for i in range(ws.n - 1):
        x = red[i] - red[i + 1:]
        x -= L * np.round(x / L)
        r2 = np.einsum("ij,ij->i", x, x)
        k = np.nonzero(r2 <= vbuf2)[0] + i + 1
        out.append(np.stack([np.full(len(k), i), k], axis=1))
    return np.concatenate(out)


def test_vdw_list_is_vlistcell_pair_set(lib, thp):
    ws = thp.water.make_water_box(648, cfg=0)
    ctx = lib.Context(ws)
    got = ctx.vdw_pairs()
    ref = _vdw_pairs_bruteforce(ws)
    assert len(got) == len(ref) and np.array_equal(got, ref[np.lexsort((ref[:, 1], ref[:, 0]))])


def test_vlistcell_dropin_fills_the_vdw_list(lib, thp):
    ws = thp.water.make_water_box(648, cfg=0)
    L = lib.load()
    ctx = lib.Context(ws)
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (ws.x, ws.y, ws.z))
    rp = np.ascontiguousarray(O.rotpole(ws))
    u1, u2 = np.zeros((ws.n, 3)), np.zeros((ws.n, 3))
    assert L.thp_bind_state(ctx.h, x.ctypes.data_as(dp), y.ctypes.data_as(dp), z.ctypes.data_as(dp),
                            rp.ctypes.data_as(dp), u1.ctypes.data_as(dp), u2.ctypes.data_as(dp), None, None, 0,
                            None) == 0
    maxv = 1200
    nv = np.zeros(ws.n, np.int32)
    vl = np.zeros((ws.n, maxv), np.int32)
    assert L.thp_bind_vlist(ctx.h, nv.ctypes.data_as(ip), vl.ctypes.data_as(ip), maxv) == 0
    L.vlistcell_()
    assert L.thp_last_error() == 0
    rows = np.repeat(np.arange(ws.n), nv)
    cols = vl[np.arange(maxv)[None, :] < nv[:, None]] - 1  # 1-based in the bound list
    got = np.stack([rows, cols], axis=1)
    got = got[np.lexsort((got[:, 1], got[:, 0]))]
    ref = _vdw_pairs_bruteforce(ws)
    assert np.array_equal(got, ref[np.lexsort((ref[:, 1], ref[:, 0]))])


def test_retargeted_context_and_shared_buffers(lib, thp):
    # one context re-targeted from a small box to a larger one (the buffers
    # sized by n are regrown) and then to a mid-size one (they are reused):
    # the results follow the oracle; the polarization gradient is unchanged
    # by interleaved empole1/ehal1 calls (they share the gradient buffers)
    small = thp.water.make_water_box(648, cfg=0)
    big = thp.water.make_water_box(10800, cfg=1)
    mid = thp.water.make_water_box(4000, cfg=0)
    ctx = lib.Context(small)
    ctx.ehal1()
    ctx.empole1()
    for ws in (big, mid):
        ctx.retarget(ws)
        orc = O.Oracle(ws)
        assert orc.mlistcell()[0] == 0
        ev, dev = ctx.ehal1()
        ev_ref, dev_ref = orc.ehal1()
        assert abs(ev - ev_ref) < 1e-10 * abs(ev_ref), (ws.n, ev, ev_ref)
        assert rel(dev, dev_ref) < 1e-9
        em, dem = ctx.empole1()
        em_ref, dem_ref, parts = orc.empole1()
        assert abs(em - em_ref) < 1e-12 * sum(abs(p) for p in parts), (ws.n, em, em_ref)
        assert rel(dem, dem_ref) < 1e-9
    assert ctx.solve()["converged"]
    ep0, g0 = ctx.gradient()
    ctx.empole1()
    ctx.ehal1()
    ep1, g1 = ctx.gradient()
    # the same up to the order of the PME spread's FP64 atomics (~1e-15)
    assert ep0 == ep1 and rel(g1, g0) < 1e-12, rel(g1, g0)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_sites_without_radius_take_no_part(lib, thp, precision):
    # hydrogens without a vdW radius are not vdW sites (kvdw.f:592-598), even
    # though the cubic-mean rule gives their pairs with oxygen a nonzero Rmin
    ws = thp.water.make_water_box(648, cfg=0)
    P = thp.params
    rad = [P.WATER_VDW["O"][0], 0.0]
    eps = [P.WATER_VDW["O"][1], P.WATER_VDW["H"][1]]
    radmin, epsm, radmin4, eps4 = P.vdw_pair_tables(rad, eps)
    v = dict(ws.vdw, radmin=np.array(radmin), eps=np.array(epsm), radmin4=np.array(radmin4), eps4=np.array(eps4))
    assert v["radmin"][0][1] > 0.0
    w2 = dataclasses.replace(ws, vdw=v)
    ev_ref, dev_ref = O.Oracle(w2).ehal1()
    ev_oo, _ = O.Oracle(dataclasses.replace(ws, vdw=dict(v, kred=np.zeros(ws.n)))).ehal1()
    assert abs(ev_ref - ev_oo) < 1e-9 * abs(ev_oo)  # only O-O pairs remain, whatever the H reduction
    ctx = lib.Context(w2, precision=lib.FP64 if precision == "fp64" else lib.MIXED)
    ev, dev = ctx.ehal1()
    tol = 1e-10 if precision == "fp64" else 1e-5
    assert abs(ev - ev_ref) < tol * abs(ev_ref), (ev, ev_ref)
    assert np.abs(dev[1::3]).max() == 0.0 and np.abs(dev[2::3]).max() == 0.0  # no force on the H atoms


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ehal1_virial_matches_oracle(lib, thp, precision):
    # ehal1c's pair virial over the reduced sites (ehal1.f:431-446) against
    # the oracle's, which the strain derivative of its energy pins
    # (tests/test_oracle.py::test_ehal1_virial_matches_strain_derivative):
    # FP64 within 1e-10 of the largest component, mixed (FP32 pair terms)
    # within 1e-5
    ws = thp.water.make_water_box(216, cfg=0, edge=20.0)
    _, _, vir_ref = O.Oracle(ws).ehal1(virial=True)
    ctx = lib.Context(ws, precision=lib.FP64 if precision == "fp64" else lib.MIXED)
    ctx.set_virial(True)
    ctx.ehal1()
    vir = ctx.ehal_virial()
    err = np.abs(vir - vir_ref).max() / np.abs(vir_ref).max()
    print(f"\nehal virial {precision}: {err:.2e} of the largest component")
    assert err < (1e-10 if precision == "fp64" else 1e-5), (vir, vir_ref)
    np.testing.assert_allclose(vir, vir.T, rtol=0, atol=0)
