"""Velocity-Verlet dynamics on the device (thp_md_verlet) against the oracle's
restatement of verlet.f driven by its own epolar1 gradient.

Both integrate the polarization gradient alone (the only force in scope).
The device warm-starts each solve from the previous step's dipoles while the
oracle starts from the direct guess, so both solve to 1e-8 D and trajectories
agree to 1e-7 A over the steps compared here.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib(thp):
    from tinker_hp_b200 import lib as L
    L.load()
    return L


def test_md_matches_oracle_verlet(lib, thp):
    ws = thp.water.make_water_box(216, cfg=0)
    mass = thp.water.masses(ws)
    vel = thp.water.maxwell_velocities(mass, 300.0, seed=3001)
    dt, nsteps = 0.001, 5
    pos_ref, vel_ref, en_ref, _ = O.verlet(ws, vel, mass, dt, nsteps, poleps=1e-8)
    ctx = lib.Context(ws, poleps=1e-8)
    v, en, it = ctx.md_verlet(nsteps, dt, mass, vel)
    pos = ctx.positions()
    assert np.abs(pos - pos_ref).max() < 1e-7, np.abs(pos - pos_ref).max()
    assert np.abs(v - vel_ref).max() < 1e-5 * np.abs(vel_ref).max()
    np.testing.assert_allclose(en, en_ref, rtol=1e-7)


def test_md_warm_start_and_energy_drift(lib, thp):
    # 20 steps of 1 fs: later solves start from the previous dipoles.  The
    # polarization energy alone is attractive (no repulsive term is in scope),
    # so unbonded water collapses after some 60 fs at 300 K; 20 fs stays well
    # inside the window where the trajectory is physical.
    ws = thp.water.make_water_box(648, cfg=1)
    mass = thp.water.masses(ws)
    vel = thp.water.maxwell_velocities(mass, 300.0, seed=3001)
    ctx = lib.Context(ws, poleps=1e-8)
    cold = lib.Context(ws, poleps=1e-8).solve()["niter"]
    _, en, it = ctx.md_verlet(20, 0.001, mass, vel)
    # the trajectory heats up as it collapses, so the gain shrinks later on
    assert it[1] < cold and np.mean(it[1:6]) < cold, (it, cold)
    drift = abs(en[-1, 2] - en[0, 2])
    print(f"total-energy drift over 20 fs: {drift:.3e} kcal/mol (epol {en[0, 0]:.3f}, ekin {en[0, 1]:.3f})")
    assert drift < 1e-3 * abs(en[0, 1])


def test_md_rejects_bad_input(lib, thp):
    ws = thp.water.make_water_box(216, cfg=0)
    ctx = lib.Context(ws)
    mass = thp.water.masses(ws)
    with pytest.raises(lib.ThpError) as e:
        ctx.md_verlet(1, 0.001, np.zeros_like(mass), np.zeros((ws.n, 3)))
    assert e.value.status == lib.THP_E_INVALID
    with pytest.raises(lib.ThpError) as e:
        ctx.md_verlet(1, -0.001, mass, np.zeros((ws.n, 3)))
    assert e.value.status == lib.THP_E_INVALID


@pytest.mark.parametrize("mode", ["ASPC", "GEAR", "LSQR"])
def test_md_predictor_matches_oracle(lib, thp, mode):
    # 12 steps: the predictor takes over from step 7 (seven stored solutions)
    ws = thp.water.make_water_box(216, cfg=0)
    mass = thp.water.masses(ws)
    vel = thp.water.maxwell_velocities(mass, 300.0, seed=3001)
    nsteps = 12
    pos_ref, _, en_ref, it_ref = O.verlet(ws, vel, mass, 0.001, nsteps, poleps=1e-8, predictor=mode)
    ctx = lib.Context(ws, poleps=1e-8)
    ctx.set_predictor(getattr(lib, f"PRED_{mode}"))
    _, en, it = ctx.md_verlet(nsteps, 0.001, mass, vel)
    assert np.abs(ctx.positions() - pos_ref).max() < 1e-7
    np.testing.assert_allclose(en, en_ref, rtol=1e-7)
    # same guesses, same CG: iteration counts agree (a count can move by one
    # when a residual lands next to the threshold)
    assert np.abs(it - it_ref).max() <= 1, (it, it_ref)
    plain = lib.Context(ws, poleps=1e-8)
    _, _, it_prev = plain.md_verlet(nsteps, 0.001, mass, vel)
    print(mode, "iterations", it.tolist(), "previous-dipole guess", it_prev.tolist())
    if mode == "ASPC":
        assert it[7:].mean() < it_prev[7:].mean()
