"""Independent numpy Ewald sums used to pin the oracle's PME (test helper).

Classical Ewald k-space sums over explicit reciprocal vectors for point
multipoles with the potential convention of the reference's pair kernels,
phi(R) = q/R + d.R/R^3 + 3 R.Q.R/R^5 (Q = stored traceless quadrupole), so
the structure factor is S(k) = sum_j (q_j - i d_j.k - k.Q_j.k) exp(-i k.r_j).
"""
import numpy as np


def kvectors(box, alpha, tol=1e-17):
    kmax = 2.0 * alpha * np.sqrt(-np.log(tol))
    m = [int(np.ceil(kmax * L / (2 * np.pi))) for L in box]
    r = [np.arange(-mi, mi + 1) for mi in m]
    g = np.stack(np.meshgrid(*r, indexing="ij"), axis=-1).reshape(-1, 3)
    g = g[np.any(g != 0, axis=1)]
    k = 2 * np.pi * g / np.asarray(box)
    k2 = np.einsum("ij,ij->i", k, k)
    keep = k2 <= kmax * kmax
    return k[keep], k2[keep]


def recip_field(pos, box, alpha, q=None, d=None, Q=None, chunk=4096):
    """Reciprocal-space field E_rec(r_i) = -grad phi_rec at every site."""
    n = len(pos)
    k, k2 = kvectors(box, alpha)
    V = float(np.prod(box))
    f = (4 * np.pi / V) * np.exp(-k2 / (4 * alpha * alpha)) / k2
    E = np.zeros((n, 3))
    for s in range(0, len(k), chunk):
        kk, ff = k[s:s + chunk], f[s:s + chunk]
        ph = np.exp(-1j * pos @ kk.T)  # [n, nk]
        amp = np.zeros((n, len(kk)), dtype=complex)
        if q is not None:
            amp += q[:, None]
        if d is not None:
            amp += -1j * (d @ kk.T)
        if Q is not None:
            amp += -np.einsum("ka,nab,kb->nk", kk, Q, kk)
        S = np.sum(amp * ph, axis=0)  # [nk]
        # phi(r) = sum_k f Re[S e^{ik.r}], E = -grad phi = -sum_k f Re[i k S e^{ik.r}]
        w = ff * S  # [nk]
        t = np.conj(ph) * w[None, :]  # e^{ik.r_i} * f * S
        E += -np.real(1j * t) @ kk
    return E


def _thole(pdi, pdk, ti, tk, r):
    """dampthole factors l3, l5, l7 (damping.f:74-124, AMOEBA branch)."""
    damp = pdi * pdk
    pg = min(ti, tk)
    if pg == 0.0:
        pg = max(ti, tk)
    if damp == 0.0 or pg == 0.0:
        return 1.0, 1.0, 1.0
    a = pg * (r / damp) ** 3
    if a >= 50.0:
        return 1.0, 1.0, 1.0
    e = np.exp(-a)
    return 1.0 - e, 1.0 - (1.0 + a) * e, 1.0 - (1.0 + a + 0.6 * a * a) * e


def pair_scales(ws):
    """d, p and u scale of every pair [n,n], assigned as efld0_direct /
    tmatxb_pme do (newinduce_pme.f:1062-1136, 1495-1518): p from the 1-2..1-5
    lists (the intra-group value when the partner is in ip11), d and u from
    the polarization-group lists ip11..ip14."""
    n = ws.n
    d = np.ones((n, n))
    p = np.ones((n, n))
    u = np.ones((n, n))

    def partners(name, i):
        off, idx = ws.conn[name]
        return idx[off[i]:off[i + 1]]

    for i in range(n):
        ip11 = set(partners("ip11", i).tolist())
        for b, name in enumerate(("i12", "i13", "i14", "i15")):
            for k in partners(name, i):
                p[i, k] = ws.scales["pi_scale"][b] if k in ip11 else ws.scales["p_scale"][b]
        for b, name in enumerate(("ip11", "ip12", "ip13", "ip14")):
            for k in partners(name, i):
                d[i, k] = ws.scales["d_scale"][b]
                u[i, k] = ws.scales["u_scale"][b]
    return d, p, u


def isolated_epol(ws, rpole, electric=332.063714):
    """Polarization energy of the same molecules in vacuum (no periodic
    images, no cutoff): the permanent field of charges, dipoles and
    quadrupoles with Thole damping and the pair scales, a dense solve of
    (1/alpha - T) mu = E for the d and p dipoles, and Epol = -1/2 electric
    sum mu_d . E_p."""
    n = ws.n
    pos = ws.positions()
    q = rpole[:, 0]
    dp = rpole[:, 1:4]
    Q = rpole[:, 4:13].reshape(n, 3, 3)
    ds, ps, us = pair_scales(ws)
    E = np.zeros((2, n, 3))
    T = np.zeros((3 * n, 3 * n))
    for i in range(n):
        for k in range(n):
            if i == k:
                continue
            x = pos[k] - pos[i]
            r2 = x @ x
            r = np.sqrt(r2)
            rr3 = 1.0 / (r * r2)
            rr5 = 3.0 * rr3 / r2
            rr7 = 5.0 * rr5 / r2
            l3, l5, l7 = _thole(ws.pdamp[i], ws.pdamp[k], ws.thole[i], ws.thole[k], r)
            dkr = dp[k] @ x
            qk = Q[k] @ x
            qkr = x @ qk
            for t, s in enumerate((ds[i, k], ps[i, k])):
                d3, d5, d7 = s * l3 * rr3, s * l5 * rr5, s * l7 * rr7
                rad = d3 * q[k] - d5 * dkr + d7 * qkr
                E[t, i] += -x * rad - d3 * dp[k] + 2.0 * d5 * qk
            s = us[i, k]
            T[3 * i:3 * i + 3, 3 * k:3 * k + 3] = s * l5 * rr5 * np.outer(x, x) - s * l3 * rr3 * np.eye(3)
    A = np.diag(np.repeat(1.0 / ws.polarity, 3)) - T
    mu_d = np.linalg.solve(A, E[0].ravel()).reshape(n, 3)
    return -0.5 * electric * np.sum(mu_d * E[1])


def recip_energy(pos, box, alpha, q, d, Q, electric=332.063714, chunk=4096):
    """Classical Ewald reciprocal energy of point multipoles,
    (electric/2) sum_k f(k) |S(k)|^2 with f = 4 pi exp(-k^2/4a^2) / (V k^2)."""
    k, k2 = kvectors(box, alpha)
    V = float(np.prod(box))
    f = (4 * np.pi / V) * np.exp(-k2 / (4 * alpha * alpha)) / k2
    e = 0.0
    for s in range(0, len(k), chunk):
        kk, ff = k[s:s + chunk], f[s:s + chunk]
        ph = np.exp(-1j * pos @ kk.T)
        amp = q[:, None] - 1j * (d @ kk.T) - np.einsum("ka,nab,kb->nk", kk, Q, kk)
        S = np.sum(amp * ph, axis=0)
        e += np.sum(ff * np.abs(S) ** 2)
    return 0.5 * electric * e


def isolated_empole(ws, rpole, electric=332.063714):
    """Permanent-multipole energy of the same molecules in vacuum (no images,
    no cutoff) by direct summation over pairs of sites, with the 1-2..1-5
    mpole scales: per pair q_i phi_k + d_i.grad phi_k + Q_i : grad grad phi_k
    from the Cartesian derivatives of 1/R, where site k's potential is
    phi_k(R) = q_k/R - d_k.grad(1/R) + Q_k : grad grad (1/R) (R = r - r_k)."""
    n = ws.n
    pos = ws.positions()
    q = rpole[:, 0]
    dp = rpole[:, 1:4]
    Q = rpole[:, 4:13].reshape(n, 3, 3)
    ms = np.ones((n, n))
    for b, name in enumerate(("i12", "i13", "i14", "i15")):
        off, idx = ws.conn[name]
        for i in range(n):
            for k in idx[off[i]:off[i + 1]]:
                ms[i, k] = ws.scales["m_scale"][b]
    I = np.eye(3)
    e = 0.0
    for i in range(n):
        for k in range(i + 1, n):
            if ms[i, k] == 0.0:
                continue
            R = pos[i] - pos[k]
            r = np.sqrt(R @ R)
            # derivatives of 1/r up to fourth order (rank-n tensors)
            t0 = 1.0 / r
            t1 = -R / r ** 3
            t2 = 3 * np.outer(R, R) / r ** 5 - I / r ** 3
            t3 = (-15 * np.einsum("a,b,c->abc", R, R, R) / r ** 7
                  + 3 * (np.einsum("a,bc->abc", R, I) + np.einsum("b,ac->abc", R, I)
                         + np.einsum("c,ab->abc", R, I)) / r ** 5)
            RRRR = np.einsum("a,b,c,d->abcd", R, R, R, R)
            RRI = (np.einsum("a,b,cd->abcd", R, R, I) + np.einsum("a,c,bd->abcd", R, R, I)
                   + np.einsum("a,d,bc->abcd", R, R, I) + np.einsum("b,c,ad->abcd", R, R, I)
                   + np.einsum("b,d,ac->abcd", R, R, I) + np.einsum("c,d,ab->abcd", R, R, I))
            II = np.einsum("ab,cd->abcd", I, I) + np.einsum("ac,bd->abcd", I, I) + np.einsum("ad,bc->abcd", I, I)
            t4 = 105 * RRRR / r ** 9 - 15 * RRI / r ** 7 + 3 * II / r ** 5
            # potential of k and its derivatives at i: phi = q T0 - d.T1 + Q:T2
            phi = q[k] * t0 - dp[k] @ t1 + np.einsum("ab,ab", Q[k], t2)
            g1 = q[k] * t1 - np.einsum("b,ab->a", dp[k], t2) + np.einsum("bc,abc->a", Q[k], t3)
            g2 = q[k] * t2 - np.einsum("c,abc->ab", dp[k], t3) + np.einsum("cd,abcd->ab", Q[k], t4)
            e += ms[i, k] * (q[i] * phi + dp[i] @ g1 + np.einsum("ab,ab", Q[i], g2))
    return electric * e


def buffered_14_7_energy(ws, vdw):
    """van der Waals energy by direct summation over all pairs within the
    cutoff, in the textbook form of the buffered 14-7 potential,
    E = eps ((1+d)/(rho+d))^7 ((1+g)/(rho^7+g) - 2), rho = r/Rmin, on the
    reduced (H-shifted) sites, times the smoothstep S(t) = 1 - 10t^3 + 15t^4
    - 6t^5 between the taper start and the cutoff, with the 1-2..1-5 scales."""
    n = ws.n
    pos = ws.positions()
    par = pos[vdw["ired"]]
    red = vdw["kred"][:, None] * (pos - par) + par
    L = np.asarray(ws.box)
    cls = vdw["cls"]
    scale = np.ones((n, n))
    is14 = np.zeros((n, n), dtype=bool)
    for b, name in enumerate(("i12", "i13", "i14", "i15")):
        off, idx = ws.conn[name]
        for i in range(n):
            for k in idx[off[i]:off[i + 1]]:
                scale[i, k] = vdw["v_scale"][b]
                if b == 2:
                    is14[i, k] = True
    e = 0.0
    d, g = vdw["dhal"], vdw["ghal"]
    cut, off = vdw["vdwtaper"], vdw["vdwcut"]
    for i in range(n - 1):
        x = red[i] - red[i + 1:]
        x -= L * np.round(x / L)
        r = np.sqrt(np.einsum("ij,ij->i", x, x))
        k = np.arange(i + 1, n)
        m = r <= off
        r, k = r[m], k[m]
        rv = np.where(is14[i, k], vdw["radmin4"][cls[k], cls[i]], vdw["radmin"][cls[k], cls[i]])
        ep = np.where(is14[i, k], vdw["eps4"][cls[k], cls[i]], vdw["eps"][cls[k], cls[i]]) * scale[i, k]
        rho = r / rv
        ee = ep * ((1 + d) / (rho + d)) ** 7 * ((1 + g) / (rho ** 7 + g) - 2)
        t = np.clip((r - cut) / (off - cut), 0.0, 1.0)
        e += np.sum(ee * (1 - 10 * t ** 3 + 15 * t ** 4 - 6 * t ** 5))
    return e
