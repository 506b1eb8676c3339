"""Polarization gradient (epolar1c) of the CUDA path against the CPU oracle.

The oracle's gradient is itself pinned by central finite differences of its
energy (tests/test_oracle.py).  Both sides here use the same induced dipoles
(the GPU's converged ones), so the comparison isolates the gradient kernels:
FP64 form within 1e-9 of the largest gradient component; mixed form (FP32 pair
and grid arithmetic, 64-bit fixed-point accumulation) reports its force RMS
error against the FP64 oracle at the oracle's own dipoles, within 5e-5 of the
force RMS.
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
    orc = O.Oracle(ws, poleps=1e-8)
    assert orc.mlistcell()[0] == 0
    return ws, orc


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_gradient_fp64_matches_oracle(lib, case):
    ws, orc = case
    ctx = lib.Context(ws, poleps=1e-8)
    res = ctx.solve()
    ep, dep = ctx.gradient()
    uind, uinp = ctx.dipoles()
    ep_ref, dep_ref = orc.epolar1(uind, uinp)
    assert res["converged"]
    assert abs(ep - ep_ref) < 1e-10 * abs(ep_ref), (ep, ep_ref)
    assert rel(dep, dep_ref) < 1e-9, rel(dep, dep_ref)


def test_gradient_mixed_error_vs_fp64(lib, case):
    ws, orc = case
    ref = orc.solve()
    _, dep_ref = orc.epolar1(ref["uind"], ref["uinp"])
    ctx = lib.Context(ws, precision=lib.MIXED, poleps=1e-6)
    assert ctx.solve()["converged"]
    _, dep = ctx.gradient()
    err = np.sqrt(np.mean(np.sum((dep - dep_ref) ** 2, axis=1)))
    scale = np.sqrt(np.mean(np.sum(dep_ref ** 2, axis=1)))
    print(f"mixed force RMS error {err:.3e} kcal/mol/A of RMS {scale:.3e} ({err / scale:.2e})")
    # 0.8 - 1.4e-5 of the force RMS: the CG tolerance (1e-6 here against the
    # oracle's 1e-8) and FP32 pair arithmetic
    assert err < 5e-5 * scale, (err, scale)


def test_gradient_matches_finite_difference_of_solved_energy(lib, thp):
    # central differences of the GPU's own converged energy, FP64, tight CG
    ws = thp.water.make_water_box(216, cfg=0)
    ctx = lib.Context(ws, poleps=1e-11)
    ctx.solve()
    _, dep = ctx.gradient()
    h = 1e-4
    x0, y0, z0 = ws.x.copy(), ws.y.copy(), ws.z.copy()
    for atom in (0, 1, 2, 301):
        for d, arr in enumerate((x0, y0, z0)):
            e = []
            for sgn in (1.0, -1.0):
                xyz = [x0.copy(), y0.copy(), z0.copy()]
                xyz[d][atom] += sgn * h
                ctx.set_positions(*xyz)
                e.append(ctx.solve()["epol"])
            fd = (e[0] - e[1]) / (2 * h)
            assert abs(fd - dep[atom, d]) < 1e-5 * np.abs(dep).max() + 1e-6, (atom, d, fd, dep[atom, d])
    ctx.set_positions(x0, y0, z0)


def test_gradient_state_errors(lib, case):
    ws, orc = case
    ctx = lib.Context(ws)
    with pytest.raises(lib.ThpError) as e:  # no solve yet
        ctx.gradient()
    assert e.value.status == lib.THP_E_STATE
    ctx.solve()
    ctx.set_positions(ws.x + 0.01, ws.y, ws.z)
    with pytest.raises(lib.ThpError) as e:  # positions moved since the solve
        ctx.gradient()
    assert e.value.status == lib.THP_E_STATE
    bare = lib.Context(ws, frames=False, rpole=orc.rpole)
    bare.solve()
    with pytest.raises(lib.ThpError) as e:  # no frame atoms for the torques
        bare.gradient()
    assert e.value.status == lib.THP_E_STATE


def test_epolar1_dropin(lib, case):
    ws, orc = case
    L = lib.load()
    ctx = lib.Context(ws, poleps=1e-8)  # frames set: the torques have their axes
    n = ws.n
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    x, y, z = (np.ascontiguousarray(a) for a in (ws.x, ws.y, ws.z))
    rp = np.ascontiguousarray(orc.rpole)
    uind, uinp = np.zeros((n, 3)), np.zeros((n, 3))
    dep = np.full((n, 3), 7.0)  # overwritten, as epolar1c zeroes dep first
    ep = np.zeros(1)
    assert L.thp_bind_state(ctx.h, P(x), P(y), P(z), P(rp), P(uind), P(uinp), None, None, 0, P(ep)) == 0
    assert L.thp_bind_gradient(ctx.h, P(dep)) == 0
    L.epolar1_()
    assert L.thp_last_error() == 0
    ep_ref, dep_ref = orc.epolar1(uind, uinp)
    assert abs(ep[0] - ep_ref) < 1e-10 * abs(ep_ref)
    assert rel(dep, dep_ref) < 1e-9


def test_mixed_gradient_close_contact(lib, thp):
    # Two waters at a hydrogen-bond contact much closer than in the boxes
    # (O...H 1.2 A): the mixed pair terms (FP32 rsqrt and products) against
    # the FP64 form on the same dipoles, at the two close atoms.
    ws = thp.water.make_water_box(216, cfg=0)
    pos = ws.positions().copy()
    L = ws.box[0]
    o_a, o_b = 3 * 20, 3 * 120
    h_b = o_b + 1
    # move water b rigidly so its first H sits 1.2 A from O of water a
    d = pos[o_a] + np.array([1.2, 0.0, 0.0]) - pos[h_b]
    pos[o_b:o_b + 3] += d
    pos -= L * np.floor(pos / L + 0.5)
    ws2 = ws.with_positions(pos)
    f64 = lib.Context(ws2, precision=lib.FP64, poleps=1e-10)
    assert f64.solve()["converged"]
    _, g64 = f64.gradient()
    mx = lib.Context(ws2, precision=lib.MIXED, poleps=1e-10)
    assert mx.solve()["converged"]
    _, g32 = mx.gradient()
    for atom in (o_a, h_b):
        err = np.linalg.norm(g32[atom] - g64[atom]) / np.linalg.norm(g64[atom])
        # the close pair's force is large; FP32 pair arithmetic keeps it to ~1e-5
        assert err < 1e-4, (atom, err, g64[atom], g32[atom])
