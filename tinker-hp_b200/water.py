"""Seeded synthetic AMOEBA water boxes (the workload of the polarization path).

Construction: rigid waters (O-H 0.9572 A, H-O-H 104.52 deg); oxygens on a
jittered cubic lattice (n_side = ceil(Nw^(1/3)), a seeded subset of sites,
jitter rejection-sampled so that the minimum O-O distance is >= 2.5 A) at
0.997 g/cm^3 (0.033328 waters/A^3) in a cubic box of edge (Nw/rho)^(1/3)
centred on the origin (widened, at lower density, when Nw lies just above a
perfect cube and the lattice spacing would fall below 2.75 A); uniform random orientations (one seeded unit
quaternion per molecule).  Atom order is O, H1, H2 per molecule, as in
Tinker water .xyz files.

Parameters follow AMOEBA-WATER-2003 (params.py); polarization groups and
connectivity follow Tinker's water definition: each molecule is one
polarization group (ip11 = {O, H1, H2}), O-H are 1-2 and H-H 1-3 neighbours.
"""

import dataclasses
import math

import numpy as np

from . import params as P

RHO_WATER = 0.033328  # waters per A^3 at 0.997 g/cm^3 (M = 18.015 g/mol)
R_OH = 0.9572
THETA_HOH = 104.52
MIN_OO = 2.5
MIN_SPACING = 2.75  # smallest oxygen lattice spacing the jitter sampling accepts


@dataclasses.dataclass
class WaterSystem:
    n: int
    nw: int
    box: tuple
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    pole: np.ndarray       # [n, 13] local frame
    zaxis: np.ndarray      # [n] int32, 0-based
    xaxis: np.ndarray      # [n] int32, 0-based
    axt: np.ndarray        # [n] int32 frame code
    polarity: np.ndarray
    thole: np.ndarray
    pdamp: np.ndarray
    mol: np.ndarray        # [n] molecule index
    conn: dict             # name -> (offsets[n+1] int32, idx int32)
    aewald: float
    ewaldcut: float
    lbuffer: float
    nfft: tuple
    bsorder: int = P.BSORDER
    scales: dict = dataclasses.field(default_factory=lambda: dict(P.SCALES))
    vdw: dict = None       # van der Waals description (water_vdw), or None

    def positions(self):
        return np.stack([self.x, self.y, self.z], axis=1)

    def with_positions(self, pos):
        pos = np.asarray(pos, dtype=np.float64)
        return dataclasses.replace(self, x=np.ascontiguousarray(pos[:, 0]),
                                   y=np.ascontiguousarray(pos[:, 1]),
                                   z=np.ascontiguousarray(pos[:, 2]))


def box_edge(nw):
    return (nw / RHO_WATER) ** (1.0 / 3.0)


def _random_rotations(rng, m):
    """Uniform random rotation matrices from uniform unit quaternions
    (K. Shoemake, Graphics Gems III, 1992)."""
    u1, u2, u3 = rng.random(m), rng.random(m), rng.random(m)
    a = np.sqrt(1.0 - u1)
    b = np.sqrt(u1)
    qx = a * np.sin(2 * np.pi * u2)
    qy = a * np.cos(2 * np.pi * u2)
    qz = b * np.sin(2 * np.pi * u3)
    qw = b * np.cos(2 * np.pi * u3)
    r = np.empty((m, 3, 3))
    r[:, 0, 0] = 1 - 2 * (qy * qy + qz * qz)
    r[:, 0, 1] = 2 * (qx * qy - qz * qw)
    r[:, 0, 2] = 2 * (qx * qz + qy * qw)
    r[:, 1, 0] = 2 * (qx * qy + qz * qw)
    r[:, 1, 1] = 1 - 2 * (qx * qx + qz * qz)
    r[:, 1, 2] = 2 * (qy * qz - qx * qw)
    r[:, 2, 0] = 2 * (qx * qz - qy * qw)
    r[:, 2, 1] = 2 * (qy * qz + qx * qw)
    r[:, 2, 2] = 1 - 2 * (qx * qx + qy * qy)
    return r


def _close_pairs(pos, occ_idx, nside, edge, cut):
    """Flag oxygens with a periodic neighbour closer than `cut`.

    The jitter (<= 0.45 A per axis) is small against the lattice spacing
    (>= 2.9 A), so only the 26 neighbouring lattice sites can come closer than
    `cut`; they are checked with whole-lattice array shifts."""
    lat = np.full((nside, nside, nside, 3), np.nan)
    flat = lat.reshape(-1, 3)
    flat[occ_idx] = pos
    bad = np.zeros((nside, nside, nside), dtype=bool)
    for sx in (-1, 0, 1):
        for sy in (-1, 0, 1):
            for sz in (-1, 0, 1):
                if (sx, sy, sz) <= (0, 0, 0):
                    continue
                other = np.roll(lat, shift=(-sx, -sy, -sz), axis=(0, 1, 2))
                d = other - lat
                d -= edge * np.round(d / edge)
                r2 = np.einsum("...i,...i->...", d, d)
                close = np.nan_to_num(r2, nan=np.inf) < cut * cut
                bad |= close
                bad |= np.roll(close, shift=(sx, sy, sz), axis=(0, 1, 2))
    return bad.reshape(-1)[occ_idx]


def make_water_box(nw, cfg=0, edge=None, grid_spacing=1.2, ewaldcut=P.EWALD_CUTOFF,
                   lbuffer=P.LIST_BUFFER, aewald=None, jitter=0.45, seed_lattice=None,
                   seed_orient=None):
    """Build a seeded water box of `nw` molecules (seeds 1000+cfg, 2000+cfg)."""
    edge = box_edge(nw) if edge is None else float(edge)
    nside = int(math.ceil(nw ** (1.0 / 3.0) - 1e-9))
    edge = max(edge, MIN_SPACING * nside)
    rng_l = np.random.default_rng(1000 + cfg if seed_lattice is None else seed_lattice)
    rng_o = np.random.default_rng(2000 + cfg if seed_orient is None else seed_orient)
    a = edge / nside
    sites = np.sort(rng_l.choice(nside ** 3, size=nw, replace=False))
    ijk = np.stack([sites // (nside * nside), (sites // nside) % nside, sites % nside], axis=1)
    base = (ijk + 0.5) * a - 0.5 * edge
    jit = rng_l.uniform(-jitter, jitter, size=(nw, 3))
    for _ in range(1000):
        pos = base + jit
        bad = _close_pairs(pos, sites, nside, edge, MIN_OO)
        if not bad.any():
            break
        jit[bad] = rng_l.uniform(-jitter, jitter, size=(int(bad.sum()), 3))
    else:
        raise RuntimeError("could not place oxygens with min O-O >= 2.5 A")
    rot = _random_rotations(rng_o, nw)
    half = math.radians(THETA_HOH) / 2.0
    h1 = np.array([R_OH * math.sin(half), 0.0, R_OH * math.cos(half)])
    h2 = np.array([-R_OH * math.sin(half), 0.0, R_OH * math.cos(half)])
    n = 3 * nw
    xyz = np.empty((n, 3))
    xyz[0::3] = pos
    xyz[1::3] = pos + rot @ h1
    xyz[2::3] = pos + rot @ h2
    return _assemble(nw, edge, xyz, grid_spacing, ewaldcut, lbuffer, aewald)


def _assemble(nw, edge, xyz, grid_spacing, ewaldcut, lbuffer, aewald):
    n = 3 * nw
    o = np.arange(nw) * 3
    pole = np.empty((n, 13))
    pole[0::3] = P.local_pole("O")
    pole[1::3] = P.local_pole("H")
    pole[2::3] = P.local_pole("H")
    zaxis = np.empty(n, np.int32)
    xaxis = np.empty(n, np.int32)
    axt = np.empty(n, np.int32)
    zaxis[0::3], xaxis[0::3], axt[0::3] = o + 1, o + 2, P.AXT_BISECTOR
    zaxis[1::3], xaxis[1::3], axt[1::3] = o, o + 2, P.AXT_Z_THEN_X
    zaxis[2::3], xaxis[2::3], axt[2::3] = o, o + 1, P.AXT_Z_THEN_X
    polarity = np.empty(n)
    polarity[0::3] = P.WATER_POLARITY["O"]
    polarity[1::3] = P.WATER_POLARITY["H"]
    polarity[2::3] = P.WATER_POLARITY["H"]
    thole = np.full(n, P.WATER_THOLE["O"])
    pdamp = polarity ** (1.0 / 6.0)
    mol = np.repeat(np.arange(nw, dtype=np.int32), 3)
    conn = water_connectivity_fast(nw)
    k = pme_k = P.pme_grid_size(edge, grid_spacing)
    if aewald is None:
        aewald = _ewaldcof_cached(ewaldcut)
    return WaterSystem(n=n, nw=nw, box=(edge, edge, edge), x=np.ascontiguousarray(xyz[:, 0]),
                       y=np.ascontiguousarray(xyz[:, 1]), z=np.ascontiguousarray(xyz[:, 2]),
                       pole=pole, zaxis=zaxis, xaxis=xaxis, axt=axt, polarity=polarity, thole=thole,
                       pdamp=pdamp, mol=mol, conn=conn, aewald=aewald, ewaldcut=ewaldcut,
                       lbuffer=lbuffer, nfft=(k, pme_k, k), vdw=water_vdw(n))


_EWALD_CACHE = {}


def _ewaldcof_cached(cut):
    if cut not in _EWALD_CACHE:
        _EWALD_CACHE[cut] = P.ewaldcof(cut)
    return _EWALD_CACHE[cut]


def water_vdw(n, vdwcut=P.VDW_CUTOFF_DEFAULT):
    """van der Waals description of n/3 waters ordered O, H, H: classes
    (O 0, H 1), pair tables by the water rules, reduction of each H towards
    its oxygen (kvdw.f:490-503), the vdw-12..15 scales, cutoff and taper."""
    nw = n // 3
    rad = [P.WATER_VDW["O"][0], P.WATER_VDW["H"][0]]
    eps = [P.WATER_VDW["O"][1], P.WATER_VDW["H"][1]]
    radmin, epsm, radmin4, eps4 = P.vdw_pair_tables(rad, eps)
    cls = np.tile(np.array([0, 1, 1], np.int32), nw)
    o = np.repeat(np.arange(nw, dtype=np.int32) * 3, 3)
    ired = np.where(cls == 0, np.arange(n, dtype=np.int32), o).astype(np.int32)
    kred = np.where(cls == 0, P.WATER_VDW["O"][2], P.WATER_VDW["H"][2]).astype(np.float64)
    return {"nclass": 2, "cls": cls, "ired": ired, "kred": kred,
            "radmin": np.array(radmin), "eps": np.array(epsm), "radmin4": np.array(radmin4),
            "eps4": np.array(eps4), "v_scale": P.VDW_SCALE, "vdwcut": vdwcut,
            "vdwtaper": P.VDW_TAPER * vdwcut, "ghal": P.GHAL, "dhal": P.DHAL}


def water_connectivity(nw):
    """CSR lists i12, i13, ip11 (others empty) for nw waters ordered O,H,H."""
    n = 3 * nw
    o = np.arange(nw, dtype=np.int32) * 3

    def csr(rows):
        off = np.zeros(n + 1, np.int32)
        off[1:] = np.cumsum([len(r) for r in rows])
        idx = np.array([v for r in rows for v in r], dtype=np.int32)
        return off, idx

    rows12, rows13, rows11 = [], [], []
    for m in range(nw):
        O, H1, H2 = 3 * m, 3 * m + 1, 3 * m + 2
        rows12 += [[H1, H2], [O], [O]]
        rows13 += [[], [H2], [H1]]
        rows11 += [[O, H1, H2]] * 3
    empty = (np.zeros(n + 1, np.int32), np.zeros(0, np.int32))
    return {"i12": csr(rows12), "i13": csr(rows13), "i14": empty, "i15": empty,
            "ip11": csr(rows11), "ip12": empty, "ip13": empty, "ip14": empty}


def water_connectivity_fast(nw):
    """Vectorised water_connectivity for large boxes (same result)."""
    n = 3 * nw
    base = np.arange(nw, dtype=np.int32) * 3
    # i12: O -> (H1,H2); H -> (O)
    off12 = np.zeros(n + 1, np.int32)
    cnt12 = np.tile(np.array([2, 1, 1], np.int32), nw)
    off12[1:] = np.cumsum(cnt12)
    idx12 = np.stack([base + 1, base + 2, base, base], axis=1).reshape(-1).astype(np.int32)
    off13 = np.zeros(n + 1, np.int32)
    cnt13 = np.tile(np.array([0, 1, 1], np.int32), nw)
    off13[1:] = np.cumsum(cnt13)
    idx13 = np.stack([base + 2, base + 1], axis=1).reshape(-1).astype(np.int32)
    off11 = np.arange(n + 1, dtype=np.int32) * 3
    grp = np.stack([base, base + 1, base + 2], axis=1)
    idx11 = np.repeat(grp, 3, axis=0).reshape(-1).astype(np.int32)
    empty = (np.zeros(n + 1, np.int32), np.zeros(0, np.int32))
    return {"i12": (off12, idx12), "i13": (off13, idx13), "i14": empty, "i15": empty,
            "ip11": (off11, idx11), "ip12": empty, "ip13": empty, "ip14": empty}


def masses(ws):
    """Atom masses [n] g/mol (water03.prm:80-81); atoms are O, H, H per molecule."""
    m = np.full(ws.n, P.WATER_MASS["H"])
    m[0::3] = P.WATER_MASS["O"]
    return m


def maxwell_velocities(mass, kelvin=300.0, seed=3001):
    """Velocities [n,3] A/ps from the Maxwell-Boltzmann distribution at
    `kelvin` (mdinit.f:550-560, maxwell.f:23-52: each Cartesian component is
    normal with variance kB T / m)."""
    rng = np.random.default_rng(seed)
    sigma = np.sqrt(P.BOLTZMANN * kelvin / np.asarray(mass, dtype=np.float64))
    return rng.standard_normal((len(mass), 3)) * sigma[:, None]


def min_box_edge(ewaldcut=P.EWALD_CUTOFF, lbuffer=P.LIST_BUFFER, margin=0.2):
    """Smallest cubic edge with the list cutoff inside half a box
    (the reference's minimum-image check, nblist.f:147-156)."""
    return 2.0 * (ewaldcut + lbuffer) + margin


def batch_sizes(count=64, nmin=300, nmax=6000, seed=4003):
    """Atom counts drawn log-uniform in [nmin, nmax], rounded to whole waters."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(nmin), np.log(nmax), size=count))
    return [max(1, int(round(v / 3.0))) for v in n]


def make_batch(count=64, nmin=300, nmax=6000, seed=4003):
    """Independent boxes of uneven size, each built like the single box at its
    own edge; edges below min_box_edge() are widened to it (lower density)
    because the 7.0 + 0.5 A list must fit in half a box."""
    out = []
    for q, nw in enumerate(batch_sizes(count, nmin, nmax, seed)):
        edge = max(box_edge(nw), min_box_edge())
        out.append(make_water_box(nw, edge=edge, seed_lattice=seed * 100 + 2 * q,
                                  seed_orient=seed * 100 + 2 * q + 1))
    return out
