"""Pins the CPU FP64 oracle (oracle/) against independent arithmetic.

The reference ships no golden vectors for this path and cannot be built here,
so the oracle is checked against: numpy's FFT, libm's erfc, a brute-force
minimum-image pair search, classical Ewald k-space sums (tests/ewald_ref.py),
a dense linear solve, and exact invariances.
"""
import dataclasses
import math

import numpy as np
import pytest
from scipy.special import erfc as sp_erfc

from oracle import oracle as O
from tests import ewald_ref

ELECTRIC = 332.063714


@pytest.fixture(scope="module")
def box216(thp):
    return thp.water.make_water_box(216, cfg=0)


def test_fft_matches_numpy():
    rng = np.random.default_rng(0)
    for shape in [(8, 6, 10), (16, 16, 16), (24, 20, 18), (5, 7, 9)]:
        g = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        fwd = O.fft3d(g, -1)
        np.testing.assert_allclose(fwd, np.fft.fftn(g), rtol=0, atol=1e-10 * np.abs(fwd).max())
        back = O.fft3d(g, +1)
        np.testing.assert_allclose(back, np.fft.ifftn(g) * g.size, rtol=0, atol=1e-10 * np.abs(back).max())


def test_erfc_matches_libm():
    for x in np.concatenate([np.linspace(0, 6, 601), [0.3, 0.46875, 0.47, 3.9999, 4.0, 4.0001, 26.0]]):
        ref = math.erfc(x)
        got = O.lib().or_erfc(float(x))
        assert abs(got - ref) <= 1e-14 * max(ref, 1e-300) + 1e-300, (x, got, ref)


def test_ewaldcof_default():
    # kewald.f:575 with the 7 A cutoff gives the 0.5446 of the workload definition
    a = O.lib().or_ewaldcof(7.0)
    assert abs(a - 0.5446) < 5e-5


def _bruteforce_pairs(ws, cut):
    pos = ws.positions()
    L = np.asarray(ws.box)
    out = []
    for i in range(ws.n - 1):
        d = pos[i] - pos[i + 1:]
        # image.f orthogonal branch, |d| < L here so a single shift suffices
        d = np.where(np.abs(d) > 0.5 * L, d - np.copysign(L, d), d)
        r2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        ks = np.nonzero(r2 <= cut * cut)[0] + i + 1
        out += [(i, k) for k in ks]
    p = np.array(out)
    return p[np.lexsort((p[:, 1], p[:, 0]))]


def test_pair_set_matches_bruteforce(box216):
    orc = O.Oracle(box216)
    st, nelst, _ = orc.mlistcell()
    assert st == 0
    ref = _bruteforce_pairs(box216, box216.ewaldcut + box216.lbuffer)
    np.testing.assert_array_equal(orc.pairs(), ref)


def test_list_overflow_and_small_box(thp, box216):
    orc = O.Oracle(box216)
    st, _, _ = orc.mlistcell(maxelst=20)
    assert st == 2  # list overflow (nblist.f:232 fatal in the reference)
    small = thp.water.make_water_box(64, cfg=0)  # 12.4 A box: half edge < 7.5 A
    assert O.Oracle(small).mlistcell()[0] == 8


def _with_grid(ws, k):
    return dataclasses.replace(ws, nfft=(k, k, k))


def test_pme_dipole_field_converges_to_ewald(box216):
    rng = np.random.default_rng(1)
    mu = rng.standard_normal((box216.n, 2, 3)) * 0.05
    ref = ewald_ref.recip_field(box216.positions(), box216.box, box216.aewald, d=mu[:, 0, :])
    errs = []
    for k in (16, 32, 64):
        orc = O.Oracle(_with_grid(box216, k))
        dip = orc.tmatxbrecip(mu)  # = grad(phi) = -E_rec
        errs.append(np.abs(-dip[:, 0, :] - ref).max() / np.abs(ref).max())
    # order-5 B-splines: the error falls at least like h^4 towards classical Ewald
    assert errs[0] < 3e-2 and errs[1] < errs[0] / 16 and errs[2] < errs[1] / 16 and errs[2] < 5e-5, errs


def test_pme_multipole_field_converges_to_ewald(box216):
    orc0 = O.Oracle(box216)
    rp = orc0.rpole
    ref = ewald_ref.recip_field(box216.positions(), box216.box, box216.aewald, q=rp[:, 0], d=rp[:, 1:4],
                                Q=rp[:, 4:13].reshape(-1, 3, 3))
    errs = []
    for k in (16, 32, 64):
        cphi = O.Oracle(_with_grid(box216, k)).efld0_recip()
        errs.append(np.abs(-cphi[:, 1:4] - ref).max() / np.abs(ref).max())
    # quadrupoles use second spline derivatives: at least h^3 convergence
    assert errs[0] < 3e-2 and errs[1] < errs[0] / 8 and errs[2] < errs[1] / 8 and errs[2] < 5e-5, errs


def _dense_operator(ws, rp, kgrid):
    """A = alpha^-1 - T built from independent real-space sums and a classical
    Ewald k-space matrix (64-water box, 16 A edge)."""
    n = ws.n
    pos = ws.positions()
    L = np.asarray(ws.box)
    a = ws.aewald
    T = np.zeros((3 * n, 3 * n))
    for i in range(n):
        for k in range(n):
            if i == k:
                continue
            r = pos[k] - pos[i]
            r -= L * np.round(r / L)
            r2 = r @ r
            if r2 > ws.ewaldcut ** 2:
                continue
            rr = math.sqrt(r2)
            b0 = sp_erfc(a * rr) / rr
            ex = math.exp(-a * a * r2)
            b1 = (b0 + 2 * a / math.sqrt(math.pi) * ex) / r2
            b2 = (3 * b1 + 4 * a ** 3 / math.sqrt(math.pi) * ex) / r2
            damp = min(ws.thole[i], ws.thole[k]) * (rr / (ws.pdamp[i] * ws.pdamp[k])) ** 3
            e = math.exp(-damp)
            l3, l5 = 1 - e, 1 - e * (1 + damp)
            dmp3 = b1 - (1 - l3) / rr ** 3
            dmp5 = b2 - 3 * (1 - l5) / rr ** 5
            T[3 * i:3 * i + 3, 3 * k:3 * k + 3] = dmp5 * np.outer(r, r) - dmp3 * np.eye(3)
    k, k2 = ewald_ref.kvectors(ws.box, a, tol=1e-16)
    V = float(np.prod(L))
    f = (4 * np.pi / V) * np.exp(-k2 / (4 * a * a)) / k2
    C, S = np.cos(pos @ k.T), np.sin(pos @ k.T)
    for p in range(3):
        for q in range(3):
            w = f * k[:, p] * k[:, q]
            T[p::3, q::3] -= (C * w) @ C.T + (S * w) @ S.T
    term = 4.0 / 3.0 * a ** 3 / math.sqrt(math.pi)
    A = -T
    A[np.diag_indices(3 * n)] += np.repeat(1.0 / ws.polarity, 3) - term
    return A


def test_pcg_matches_dense_ewald_solve(thp):
    ws = thp.water.make_water_box(64, cfg=3, edge=16.0)
    ws = _with_grid(ws, 64)  # 0.25 A spacing: PME within ~2e-6 of classical Ewald
    orc = O.Oracle(ws, poleps=1e-11)
    assert orc.mlistcell()[0] == 0
    res = orc.solve()
    assert res["converged"]
    A = _dense_operator(ws, orc.rpole, 64)
    for rhs, key in ((0, "uind"), (1, "uinp")):
        x = np.linalg.solve(A, res["ef"][:, rhs, :].reshape(-1))
        err = np.abs(x.reshape(-1, 3) - res[key]).max() / np.abs(x).max()
        assert err < 3e-6, (key, err)


def test_converged_residual_and_energy_identity(box216):
    orc = O.Oracle(box216, poleps=1e-8)
    assert orc.mlistcell()[0] == 0
    res = orc.solve()
    assert res["converged"] and res["niter"] > 3
    mu = np.stack([res["uind"], res["uinp"]], axis=1)
    term = 4.0 / 3.0 * box216.aewald ** 3 / math.sqrt(math.pi)
    h = orc.tmatxb(mu) + orc.tmatxbrecip(mu) - term * mu
    r = res["ef"] - h
    rms = np.sqrt(np.sum(r * r * box216.polarity[:, None, None]) / (3 * box216.n) / 2)
    assert rms < 1e-8
    e, parts = orc.epolar(res["uind"])
    ident = -0.5 * ELECTRIC * np.sum(res["uind"] * res["ef"][:, 1, :])
    assert abs(e - ident) < 1e-10 * abs(e)
    assert abs(sum(parts.values()) - e) < 1e-12 * abs(e)


def test_grid_translation_invariance(box216):
    # a shift by whole grid spacings leaves PME and real space unchanged
    k = box216.nfft[0]
    h = box216.box[0] / k
    shift = np.array([3 * h, -2 * h, 5 * h])
    ws2 = box216.with_positions(box216.positions() + shift)
    e = []
    for ws in (box216, ws2):
        orc = O.Oracle(ws)
        orc.mlistcell()
        res = orc.solve()
        e.append(orc.epolar(res["uind"])[0])
    assert abs(e[0] - e[1]) < 1e-9 * abs(e[0])


def test_threads_agree(box216):
    r = []
    for nt in (1, 4):
        orc = O.Oracle(box216, nthreads=nt)
        orc.mlistcell()
        r.append(orc.solve()["uind"])
    np.testing.assert_allclose(r[0], r[1], rtol=0, atol=1e-12)


def _energy(ws, poleps=1e-10):
    orc = O.Oracle(ws, poleps=poleps)
    assert orc.mlistcell()[0] == 0
    res = orc.solve()
    return orc.epolar(res["uind"])[0], orc, res


def test_epolar1_energy_matches_epolar0(box216):
    e0, orc, res = _energy(box216)
    e1, dep = orc.epolar1(res["uind"], res["uinp"])
    assert abs(e1 - e0) < 1e-10 * abs(e0)


def test_epolar1_gradient_matches_finite_differences(box216):
    _, orc, res = _energy(box216)
    _, dep = orc.epolar1(res["uind"], res["uinp"])
    pos0 = box216.positions()
    h = 1e-4
    for atom in (0, 1, 2, 301, 646):
        for d in range(3):
            e = []
            for sgn in (1, -1):
                p = pos0.copy()
                p[atom, d] += sgn * h
                e.append(_energy(box216.with_positions(p))[0])
            fd = (e[0] - e[1]) / (2 * h)
            assert abs(fd - dep[atom, d]) < 1e-5 * np.abs(dep).max() + 1e-6, (atom, d, fd, dep[atom, d])


def test_epolar1_virial_matches_strain_derivative(box216):
    # Scaling every x coordinate and the box edge along x by (1 + eps), the
    # frames rotating with the atoms and the dipoles solved again: the
    # central difference of the energy is vir(1,1) + the frame-atom virial
    # of the reciprocal and self torques (the reference's virial leaves the
    # latter out); likewise along y and z.  The tensor is symmetric.
    _, orc, res = _energy(box216)
    _, _, vir, vfr = orc.epolar1(res["uind"], res["uinp"], virial=True)
    np.testing.assert_allclose(vir, vir.T, rtol=0, atol=1e-12 * np.abs(vir).max())
    eps = 1e-5
    pos0 = box216.positions()
    for a in range(3):
        e = []
        for sgn in (1, -1):
            p = pos0.copy()
            p[:, a] *= 1.0 + sgn * eps
            box = list(box216.box)
            box[a] *= 1.0 + sgn * eps
            e.append(_energy(dataclasses.replace(box216.with_positions(p), box=tuple(box)))[0])
        fd = (e[0] - e[1]) / (2 * eps)
        assert abs(fd - (vir[a, a] + vfr[a, a])) < 2e-6 * abs(fd), (a, fd, vir[a, a], vfr[a, a])
        # the terms the reference leaves out are small but not negligible
        assert abs(vfr[a, a]) < 1e-2 * abs(fd)


def test_energy_independent_of_ewald_alpha(thp):
    # Epol is a physical quantity: at a converged real-space cutoff (9 A) and
    # grid (0.45 A spacing) the Ewald split alpha must not change it.  The
    # measured spread over alpha in {0.45, 0.5446, 0.65} is 1.1e-6 relative.
    es = []
    for a in (0.45, 0.5446, 0.65):
        ws = thp.water.make_water_box(216, cfg=0, edge=22.0, ewaldcut=9.0, grid_spacing=0.45, aewald=a)
        orc = O.Oracle(ws, poleps=1e-10)
        assert orc.mlistcell(maxelst=4000)[0] == 0
        res = orc.solve()
        es.append(orc.epolar(res["uind"])[0])
    es = np.array(es)
    assert (es.max() - es.min()) < 3e-6 * abs(es.mean()), es


def test_two_waters_reach_the_isolated_limit(thp):
    # Two waters at a hydrogen-bond distance in growing periodic boxes: the
    # Ewald/PME energy differs from the vacuum energy (direct summation, no
    # images, tests/ewald_ref.py) by the dipolar image term ~ 1/L^3; the two
    # boxes' extrapolation reproduces the vacuum value.  Measured: 2.6e-3 and
    # 1.1e-3 relative at L = 30, 40 A (ratio 2.35 for (40/30)^3 = 2.37), 1.8e-5
    # after the extrapolation.
    W = thp.water
    R, th = W.R_OH, math.radians(W.THETA_HOH) / 2
    h1 = np.array([R * math.sin(th), 0, R * math.cos(th)])
    h2 = np.array([-R * math.sin(th), 0, R * math.cos(th)])

    def rot(a, b):
        ca, sa, cb, sb = math.cos(a), math.sin(a), math.cos(b), math.sin(b)
        return np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1]]) @ np.array([[1, 0, 0], [0, cb, -sb], [0, sb, cb]])

    o1 = np.array([0.3, -0.2, 0.1])
    o2 = o1 + np.array([2.85, 0.4, -0.3])
    xyz = np.array([o1, o1 + rot(0.3, 1.1) @ h1, o1 + rot(0.3, 1.1) @ h2,
                    o2, o2 + rot(2.0, -0.7) @ h1, o2 + rot(2.0, -0.7) @ h2])
    es = {}
    for L in (30.0, 40.0):
        ws = W._assemble(2, L, xyz, 0.5, 7.0, 0.5, None)
        orc = O.Oracle(ws, poleps=1e-12)
        assert orc.mlistcell()[0] == 0
        res = orc.solve()
        es[L] = orc.epolar(res["uind"])[0]
        if L == 30.0:
            eiso = ewald_ref.isolated_epol(ws, orc.rpole)
    ratio = (es[30.0] - eiso) / (es[40.0] - eiso)
    assert abs(ratio / (40.0 / 30.0) ** 3 - 1.0) < 0.03, ratio
    einf = (es[40.0] * 40.0 ** 3 - es[30.0] * 30.0 ** 3) / (40.0 ** 3 - 30.0 ** 3)
    assert abs(einf - eiso) < 5e-5 * abs(eiso), (einf, eiso)


# ---- permanent-multipole energy and gradient (empole1c) --------------------

def _empole(ws, virial=False):
    orc = O.Oracle(ws)
    assert orc.mlistcell(maxelst=4000)[0] == 0
    return orc.empole1(virial=virial)


def test_empole1_gradient_matches_finite_differences(box216):
    # the positions move the frames too (rotpole), so the torque terms are
    # checked with the pair and grid forces
    _, dem, _ = _empole(box216)
    pos0 = box216.positions()
    h = 1e-5
    for atom in (0, 1, 2, 301, 646):
        for d in range(3):
            e = []
            for sgn in (1, -1):
                p = pos0.copy()
                p[atom, d] += sgn * h
                e.append(_empole(box216.with_positions(p))[0])
            fd = (e[0] - e[1]) / (2 * h)
            assert abs(fd - dem[atom, d]) < 1e-6 * np.abs(dem).max() + 1e-6, (atom, d, fd, dem[atom, d])


def test_empole1_virial_matches_strain_derivative(thp):
    # Scaling the coordinates and the box edge along x, y or z by (1 + eps),
    # the frames (and so the multipoles) following the atoms: the central
    # difference of the energy is vir(a,a) + the frame-atom virial of the
    # reciprocal torques, which the reference's virial leaves out.  The
    # real-space energy jumps where a pair crosses the cutoff (a charge pair
    # there is worth ~1e-7 kcal/mol), so the strain is kept small (1e-7, a
    # few pairs within reach of the cutoff) and the difference is bounded
    # against the size of the real and reciprocal parts, which cancel to a
    # total a hundred times smaller.
    box = thp.water.make_water_box(216, cfg=0)
    _, _, _, vir, vfr = _empole(box, virial=True)
    np.testing.assert_allclose(vir, vir.T, rtol=0, atol=1e-12 * np.abs(vir).max())
    eps = 1e-7
    pos0 = box.positions()
    for a in range(3):
        e, parts = [], []
        for sgn in (1, -1):
            p = pos0.copy()
            p[:, a] *= 1.0 + sgn * eps
            edge = list(box.box)
            edge[a] *= 1.0 + sgn * eps
            em, _, pt = _empole(dataclasses.replace(box.with_positions(p), box=tuple(edge)))
            e.append(em)
            parts.append(pt)
        fd = (e[0] - e[1]) / (2 * eps)
        scale = sum(abs(parts[0][q] - parts[1][q]) / (2 * eps) for q in (0, 1))
        assert abs(fd - (vir[a, a] + vfr[a, a])) < 5e-6 * scale, (a, fd, vir[a, a], vfr[a, a], scale)


def test_empole_recip_converges_to_classical_ewald(box216):
    orc0 = O.Oracle(box216)
    rp = orc0.rpole
    ref = ewald_ref.recip_energy(box216.positions(), box216.box, box216.aewald, rp[:, 0], rp[:, 1:4],
                                 rp[:, 4:13].reshape(-1, 3, 3))
    errs = []
    for k in (16, 32, 64):
        _, _, (_, erec, _) = _empole(_with_grid(box216, k))
        errs.append(abs(erec - ref) / abs(ref))
    assert errs[0] < 1e-2 and errs[1] < errs[0] / 8 and errs[2] < errs[1] / 8 and errs[2] < 1e-6, errs


def test_empole_energy_independent_of_ewald_alpha(thp):
    # The real, reciprocal and self parts each move by hundreds of kcal/mol
    # between these alphas; with the reciprocal part summed classically
    # (tests/ewald_ref.py) their total must not.  Measured: 1e-10 relative to
    # that spread (the PME reciprocal part itself is pinned by the
    # convergence test above; at 0.45 A spacing it moves by 6e-3 kcal/mol).
    es, reals = [], []
    for a in (0.5, 0.5446, 0.65):
        ws = thp.water.make_water_box(216, cfg=0, edge=22.0, ewaldcut=9.0, grid_spacing=0.45, aewald=a)
        orc = O.Oracle(ws)
        assert orc.mlistcell(maxelst=4000)[0] == 0
        _, _, (ereal, _, eself) = orc.empole1()
        rp = orc.rpole
        erec = ewald_ref.recip_energy(ws.positions(), ws.box, a, rp[:, 0], rp[:, 1:4], rp[:, 4:13].reshape(-1, 3, 3))
        es.append(ereal + erec + eself)
        reals.append(ereal)
    spread = np.ptp(reals)
    assert spread > 100.0, reals
    assert np.ptp(es) < 1e-9 * spread, (es, reals)


def test_empole_two_waters_reach_the_isolated_limit(thp):
    # The Ewald energy of two waters in growing periodic boxes approaches the
    # vacuum direct sum (tests/ewald_ref.py) through image terms in 1/L^3 and
    # 1/L^5 (the molecules carry dipoles and quadrupoles); a fit over three
    # boxes recovers the vacuum value (measured: 4e-8 relative).  The
    # reciprocal part is summed classically here: for six atoms the PME
    # self-interaction error is position dependent, about 1e-4 kcal/mol at
    # 0.5 A spacing, next to image terms of 1e-2.
    W = thp.water
    R, th = W.R_OH, math.radians(W.THETA_HOH) / 2
    h1 = np.array([R * math.sin(th), 0, R * math.cos(th)])
    h2 = np.array([-R * math.sin(th), 0, R * math.cos(th)])

    def rot(a, b):
        ca, sa, cb, sb = math.cos(a), math.sin(a), math.cos(b), math.sin(b)
        return np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1]]) @ np.array([[1, 0, 0], [0, cb, -sb], [0, sb, cb]])

    o1 = np.array([0.3, -0.2, 0.1])
    o2 = o1 + np.array([2.85, 0.4, -0.3])
    xyz = np.array([o1, o1 + rot(0.3, 1.1) @ h1, o1 + rot(0.3, 1.1) @ h2,
                    o2, o2 + rot(2.0, -0.7) @ h1, o2 + rot(2.0, -0.7) @ h2])
    es = {}
    for L in (30.0, 40.0, 60.0):
        ws = W._assemble(2, L, xyz, 0.5, 7.0, 0.5, None)
        orc = O.Oracle(ws)
        assert orc.mlistcell()[0] == 0
        _, _, (ereal, _, eself) = orc.empole1()
        rp = orc.rpole
        erec = ewald_ref.recip_energy(ws.positions(), ws.box, ws.aewald, rp[:, 0], rp[:, 1:4],
                                      rp[:, 4:13].reshape(-1, 3, 3))
        es[L] = ereal + erec + eself
        if L == 30.0:
            eiso = ewald_ref.isolated_empole(ws, rp)
    Ls = np.array(sorted(es))
    fit = np.linalg.solve(np.stack([np.ones(3), Ls ** -3, Ls ** -5], axis=1), np.array([es[L] for L in Ls]))
    assert abs(es[30.0] - eiso) > 1e-3 * abs(eiso), (es, eiso)  # the image term is visible
    assert abs(fit[0] - eiso) < 1e-6 * abs(eiso), (fit, eiso)


# ---- van der Waals (ehal1c) -------------------------------------------------

def test_ehal1_energy_matches_textbook_form(thp):
    # the reference's taper is the smoothstep expanded in powers of r, whose
    # coefficients reach 1e5 for a 0.9 A window: the two forms differ by
    # rounding at 1e-11 relative (measured 1.8e-11)
    ws = thp.water.make_water_box(216, cfg=0, edge=20.0)
    ev, _ = O.Oracle(ws).ehal1()
    ref = ewald_ref.buffered_14_7_energy(ws, ws.vdw)
    assert abs(ev - ref) < 1e-9 * abs(ref), (ev, ref)


def test_ehal1_gradient_matches_finite_differences(thp):
    # the hydrogens' reduced sites move with their oxygens, so the
    # reduction chain rule is checked too
    ws = thp.water.make_water_box(216, cfg=0, edge=20.0)
    _, dev = O.Oracle(ws).ehal1()
    pos0 = ws.positions()
    h = 1e-5
    for atom in (0, 1, 2, 300, 646):
        for d in range(3):
            e = []
            for sgn in (1, -1):
                p = pos0.copy()
                p[atom, d] += sgn * h
                e.append(O.Oracle(ws.with_positions(p)).ehal1()[0])
            fd = (e[0] - e[1]) / (2 * h)
            assert abs(fd - dev[atom, d]) < 1e-6 * np.abs(dev).max() + 1e-7, (atom, d, fd, dev[atom, d])


def test_ehal1_virial_matches_strain_derivative(thp):
    # scaling the coordinates and the box edge along x, y or z: the reduced
    # sites scale with them, and the taper makes the energy smooth at the
    # cutoff, so the central difference equals vir(a,a) (ehal1.f:431-446)
    ws = thp.water.make_water_box(216, cfg=0, edge=20.0)
    _, _, vir = O.Oracle(ws).ehal1(virial=True)
    np.testing.assert_allclose(vir, vir.T, rtol=0, atol=1e-12 * np.abs(vir).max())
    eps = 1e-5
    pos0 = ws.positions()
    for a in range(3):
        e = []
        for sgn in (1, -1):
            p = pos0.copy()
            p[:, a] *= 1.0 + sgn * eps
            edge = list(ws.box)
            edge[a] *= 1.0 + sgn * eps
            e.append(O.Oracle(dataclasses.replace(ws.with_positions(p), box=tuple(edge))).ehal1()[0])
        fd = (e[0] - e[1]) / (2 * eps)
        assert abs(fd - vir[a, a]) < 1e-6 * np.abs(vir).max(), (a, fd, vir[a, a])


def test_ehal1_refuses_a_small_box(thp):
    ws = thp.water.make_water_box(64, cfg=0, edge=16.0)  # 9 + 0.5 A exceeds half of 16 A
    with pytest.raises(RuntimeError, match="status 8"):
        O.Oracle(ws).ehal1()
