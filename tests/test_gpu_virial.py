"""Internal virial of the polarization energy (epolar1c) on the device against
the CPU oracle, at the same (device-solved) induced dipoles.

The oracle's virial is itself pinned to the strain derivative of its energy
(tests/test_oracle.py::test_epolar1_virial_matches_strain_derivative).  FP64
form: both forms of thp_get_virial (the reference's accumulation, and with
the reciprocal and self torques' frame-atom terms) within 1e-9 of the
largest component.  Mixed form (FP32 pair and grid arithmetic): within 2e-6
of the largest component (0.6-2.4e-7 reached), against the oracle at the
oracle's own dipoles.
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


def test_virial_fp64_matches_oracle(lib, case):
    ws, orc = case
    ctx = lib.Context(ws, poleps=1e-8)
    ctx.set_virial(True)
    assert ctx.solve()["converged"]
    _, dep = ctx.gradient()
    v0, v1 = ctx.virial(0), ctx.virial(1)
    uind, uinp = ctx.dipoles()
    _, dep_ref, vir_ref, vfr_ref = orc.epolar1(uind, uinp, virial=True)
    scale = np.abs(vir_ref).max()
    assert np.abs(v0 - vir_ref).max() < 1e-9 * scale, (v0, vir_ref)
    assert np.abs(v1 - (vir_ref + vfr_ref)).max() < 1e-9 * scale, (v1, vir_ref + vfr_ref)
    np.testing.assert_allclose(v0, v0.T, rtol=0, atol=0)
    # the gradient is the same with the virial on
    assert np.abs(dep - dep_ref).max() < 1e-9 * np.abs(dep_ref).max()


def test_virial_mixed_against_oracle(lib, case):
    ws, orc = case
    ref = orc.solve()
    _, _, vir_ref, vfr_ref = orc.epolar1(ref["uind"], ref["uinp"], virial=True)
    ctx = lib.Context(ws, precision=lib.MIXED, poleps=1e-8)
    ctx.set_virial(True)
    assert ctx.solve()["converged"]
    ctx.gradient()
    scale = np.abs(vir_ref).max()
    err0 = np.abs(ctx.virial(0) - vir_ref).max() / scale
    err1 = np.abs(ctx.virial(1) - (vir_ref + vfr_ref)).max() / scale
    print(f"\nmixed virial error {err0:.2e} / {err1:.2e} of the largest component")
    assert err0 < 2e-6 and err1 < 2e-6, (err0, err1)


def test_virial_state_and_dropin(lib, case):
    ws, orc = case
    ctx = lib.Context(ws, poleps=1e-8)
    ctx.solve()
    ctx.gradient()
    with pytest.raises(lib.ThpError) as e:  # virial not requested
        ctx.virial()
    assert e.value.status == lib.THP_E_STATE
    # the Fortran drop-in adds the virial into the bound vir(3,3)
    L = lib.load()
    n = ws.n
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    x, y, z = (np.ascontiguousarray(a) for a in (ws.x, ws.y, ws.z))
    rp = np.ascontiguousarray(orc.rpole)
    uind, uinp = np.zeros((n, 3)), np.zeros((n, 3))
    dep = np.zeros((n, 3))
    ep = np.zeros(1)
    vir = np.full((3, 3), 2.0)
    assert L.thp_bind_state(ctx.h, P(x), P(y), P(z), P(rp), P(uind), P(uinp), None, None, 0, P(ep)) == 0
    assert L.thp_bind_gradient(ctx.h, P(dep)) == 0
    assert L.thp_bind_virial(ctx.h, P(vir)) == 0
    L.epolar1_()
    assert L.thp_last_error() == 0
    _, _, vir_ref, _ = orc.epolar1(uind, uinp, virial=True)
    assert np.abs((vir - 2.0) - vir_ref).max() < 1e-9 * np.abs(vir_ref).max()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_empole_virial_matches_oracle(lib, case, precision):
    # empole1c's virial (emrecip1's site terms and scalar sum, emreal1c's pair
    # and torque frame terms) and the reciprocal torques' frame-atom terms,
    # against the oracle's, which the strain derivative of its energy pins
    # (tests/test_oracle.py::test_empole1_virial_matches_strain_derivative).
    # Bounds relative to the sum of the energy parts' magnitudes (the virial
    # is a small difference of real and reciprocal terms of that size):
    # 1e-10 FP64, 1e-6 mixed (FP32 pair and grid arithmetic).
    ws, orc = case
    _, _, parts, vir_ref, vfr_ref = orc.empole1(virial=True)
    scale = sum(abs(p) for p in parts)
    prec = lib.FP64 if precision == "fp64" else lib.MIXED
    ctx = lib.Context(ws, precision=prec)
    ctx.set_virial(True)
    _, dem = ctx.empole1()
    v0, v1 = ctx.empole_virial(0), ctx.empole_virial(1)
    e0 = np.abs(v0 - vir_ref).max() / scale
    e1 = np.abs(v1 - (vir_ref + vfr_ref)).max() / scale
    print(f"\nempole virial {precision}: {e0:.2e} / {e1:.2e} of the parts ({scale:.3e} kcal/mol)")
    tol = 1e-10 if prec == lib.FP64 else 1e-6
    assert e0 < tol and e1 < tol, (v0, vir_ref, v1, vir_ref + vfr_ref)
    np.testing.assert_allclose(v0, v0.T, rtol=0, atol=0)
    # the energy gradient is the same with the virial off (FP64: to rounding;
    # mixed: the two kernel variants round their FP32 pair terms differently)
    ctx.set_virial(False)
    _, dem2 = ctx.empole1()
    assert np.abs(dem2 - dem).max() < (1e-12 if prec == lib.FP64 else 1e-6) * np.abs(dem).max()
