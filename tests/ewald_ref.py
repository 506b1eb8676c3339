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
