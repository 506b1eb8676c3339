"""AMOEBA water parameters and Tinker-HP defaults used by the polarization path.

Values are force-field data from Tinker-HP's AMOEBA-WATER-2003 parameter file
(v1.2/params/water03.prm:30-50 scale factors, :135-156 multipoles and
polarizabilities) and program defaults from v1.2/source (initprm.f:413-470,
cutoffs.f:40-80, kewald.f:67-91, MOD_units.f:77-82).
"""

import math

# MOD_units.f:77-82
BOHR = 0.52917721092
ELECTRIC = 332.063714
DEBYE = 4.80321

# water03.prm:135-145, local-frame multipoles in atomic units:
# charge; dipole (x, y, z); quadrupole rows xx / xy yy / xz yz zz
WATER_MULTIPOLES = {
    "O": {
        "charge": -0.51966,
        "dipole": (0.00000, 0.00000, 0.14279),
        "quad": ((0.37928, 0.0, 0.0), (0.0, -0.41809, 0.0), (0.0, 0.0, 0.03881)),
    },
    "H": {
        "charge": 0.25983,
        "dipole": (-0.03859, 0.00000, -0.05818),
        "quad": ((-0.03673, 0.0, -0.00203), (0.0, -0.10739, 0.0), (-0.00203, 0.0, 0.14412)),
    },
}

# water03.prm:80-81 (atom masses, g/mol)
WATER_MASS = {"O": 15.995, "H": 1.008}

# units.f:71,76: Boltzmann constant in g A^2/ps^2/mol/K and kcal/mol -> g A^2/ps^2
BOLTZMANN = 0.831446215
CONVERT = 418.4

# water03.prm:155-156 (polarize: alpha A^3, thole)
WATER_POLARITY = {"O": 0.837, "H": 0.496}
WATER_THOLE = {"O": 0.390, "H": 0.390}

# water03.prm:30-50 and initprm.f:417-470 defaults for the unset ones
SCALES = {
    "p_scale": (0.0, 0.0, 1.0, 1.0),   # polar-12..15-scale
    "pi_scale": (0.0, 0.0, 0.5, 1.0),  # polar-12..15-intra (p2i, p3i default 0; 14-intra 0.5)
    "d_scale": (0.0, 1.0, 1.0, 1.0),   # direct-11..14-scale
    "u_scale": (1.0, 1.0, 1.0, 1.0),   # mutual-11..14-scale
    "m_scale": (0.0, 0.0, 0.4, 0.8),   # mpole-12..15-scale (water03.prm:34-37)
}

# water03.prm:91-92 (vdw: Rmin as a diameter, epsilon, reduction factor),
# :23-27 (buffered 14-7, CUBIC-MEAN radii, HHG well depths), :30-33 (scales)
WATER_VDW = {"O": (3.4050, 0.1100, 0.0), "H": (2.6550, 0.0135, 0.910)}
VDW_RULES = {"radius": "CUBIC-MEAN", "epsilon": "HHG", "radiustype": "R-MIN", "radiussize": "DIAMETER"}
VDW_SCALE = (0.0, 0.0, 1.0, 1.0)   # vdw-12..15-scale
VDW_CUTOFF_DEFAULT = 9.0            # cutoffs.f: vdwcut
VDW_TAPER = 0.90                    # cutoffs.f: vdwtaper (fraction of the cutoff)
GHAL, DHAL = 0.12, 0.07             # initprm.f:383-384 (buffered 14-7 constants)


def vdw_pair_tables(rad, eps, rad4=None, eps4=None, rules=None):
    """Pair Rmin and epsilon tables [nc][nc] from per-class values
    (kvdw.f:318-410 for the SIGMA/DIAMETER conversions and the ARITHMETIC,
    GEOMETRIC, CUBIC-MEAN radius and ARITHMETIC, GEOMETRIC, HARMONIC, HHG
    well-depth rules)."""
    rules = dict(VDW_RULES if rules is None else rules)
    twosix = 2.0 ** (1.0 / 6.0)

    def conv(r):
        r = list(r)
        if rules.get("radiustype", "R-MIN") == "SIGMA":
            r = [twosix * v for v in r]
        if rules.get("radiussize", "RADIUS") == "DIAMETER":
            r = [0.5 * v for v in r]
        return r

    rad4 = [r4 if r4 else r for r, r4 in zip(rad, rad4 or rad)]
    eps4 = [e4 if e4 else e for e, e4 in zip(eps, eps4 or eps)]
    out = []
    for rr, ee in ((conv(rad), [abs(e) for e in eps]), (conv(rad4), [abs(e) for e in eps4])):
        nc = len(rr)
        R = [[0.0] * nc for _ in range(nc)]
        E = [[0.0] * nc for _ in range(nc)]
        for i in range(nc):
            for k in range(i, nc):
                ri, rk = rr[i], rr[k]
                if ri == 0.0 and rk == 0.0:
                    rd = 0.0
                elif rules["radius"] == "ARITHMETIC":
                    rd = ri + rk
                elif rules["radius"] == "GEOMETRIC":
                    rd = 2.0 * (math.sqrt(ri) * math.sqrt(rk))
                elif rules["radius"] == "CUBIC-MEAN":
                    rd = 2.0 * (ri ** 3 + rk ** 3) / (ri ** 2 + rk ** 2)
                else:
                    rd = ri + rk
                ei, ek = ee[i], ee[k]
                si, sk = math.sqrt(ei), math.sqrt(ek)
                if ei == 0.0 and ek == 0.0:
                    ep = 0.0
                elif rules["epsilon"] == "ARITHMETIC":
                    ep = 0.5 * (ei + ek)
                elif rules["epsilon"] == "GEOMETRIC":
                    ep = si * sk
                elif rules["epsilon"] == "HARMONIC":
                    ep = 2.0 * (ei * ek) / (ei + ek)
                elif rules["epsilon"] == "HHG":
                    ep = 4.0 * (ei * ek) / (si + sk) ** 2
                else:
                    ep = si * sk
                R[i][k] = R[k][i] = rd
                E[i][k] = E[k][i] = ep
        out += [R, E]
    return out  # radmin, eps, radmin4, eps4


# frame codes shared with the C-ABI: 1 = Z-then-X, 2 = Bisector
AXT_Z_THEN_X = 1
AXT_BISECTOR = 2

# kewald.f:67-73 FFT-friendly grid sizes
MULTI = (2, 4, 6, 8, 10, 12, 16, 18, 20, 24, 30, 32, 36, 40, 48, 50, 54, 60, 64, 72, 80, 90, 96, 100,
         108, 120, 128, 144, 150, 160, 162, 180, 192, 200, 216, 240, 250, 256, 270, 288, 300, 320, 324,
         360, 384, 400, 432, 450, 480, 486, 500, 512, 540, 576, 600, 640, 648, 720, 750, 768, 800, 810,
         864)
MINFFT = 16

# defaults of the workload (cutoffs.f:58 ewald-cutoff, list buffer per the configs)
EWALD_CUTOFF = 7.0
LIST_BUFFER = 0.5
VDW_CUTOFF = 9.0
BSORDER = 5
POLITER = 500


def pme_grid_size(box_edge, spacing=1.2):
    """Grid points along one edge: kewald.f:144-146 density rule with
    density = 1/spacing, rounded up to the MULTI list, floor MINFFT (kewald.f:213-226)."""
    dens = 1.0 / spacing
    ie = int(box_edge * dens - 1.0e-8) + 1
    n = MULTI[-1]
    for k in reversed(MULTI):
        if k >= ie:
            n = k
    return max(n, MINFFT)


def local_pole(kind):
    """13-component local-frame multipole in e, e*A, e*A^2 (kmpole.f:530-537:
    dipoles times bohr, quadrupoles times bohr^2/3)."""
    m = WATER_MULTIPOLES[kind]
    p = [m["charge"]]
    p += [d * BOHR for d in m["dipole"]]
    for row in m["quad"]:
        p += [q * BOHR * BOHR / 3.0 for q in row]
    return p


def ewaldcof(cutoff, erfc=math.erfc):
    """Ewald coefficient with erfc(a*cutoff)/cutoff < 1e-8 (kewald.f:575-620)."""
    eps = 1.0e-8
    ratio = eps + 1.0
    x = 0.5
    i = 0
    while ratio >= eps:
        i += 1
        x = 2.0 * x
        ratio = erfc(x * cutoff) / cutoff
    xlo, xhi = 0.0, x
    for _ in range(i + 60):
        x = (xlo + xhi) / 2.0
        ratio = erfc(x * cutoff) / cutoff
        if ratio >= eps:
            xlo = x
        else:
            xhi = x
    return x
