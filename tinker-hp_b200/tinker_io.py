"""Tinker input files for the polarization path: .xyz coordinates, .key
keywords and .prm force-field parameters, read into the system description
the library takes (the same fields as water.WaterSystem), and written back.

Each step restates the reference routine that does it at start-up:
  * readxyz.f:17-280 -- atom count and title, an optional periodic-box line,
    one line per atom (number, name, x, y, z, type, bonded atoms); atom
    numbers that are not 1..n in order are renumbered;
  * getkey.f / prmkey.f -- keyword lines; the parameter file named by
    `parameters`; the scale factors (mpole-1x-scale, polar-1x-scale,
    polar-1x-intra, direct-1x-scale, mutual-1x-scale) from either file;
  * readprm.f:1231-1314 (`multipole`, five lines per entry) and :1315-1360
    (`polarize`: type, polarizability, optional Thole and direct damping,
    polarization-group atom types);
  * unitcell.f:55-100 (a/b/c-axis), cutoffs.f:100-200 (ewald-cutoff,
    list-buffer), kewald.f:60-215 (ewald-alpha/pewald-alpha, pme-grid,
    pme-order; default grid from 1.2 points per A), prmkey.f:452-456
    (polar-iter, polar-eps);
  * attach.f:17-140 -- 1-3, 1-4 and 1-5 lists from the bonds;
  * kmpole.f:17-540 -- multipole frames by the four assignment passes
    (1-2 atoms only, 1-2 and 1-3 atoms, a z atom only, none), key-file
    entries ahead of the parameter file's, atom-specific entries (negative
    atom number in the key file) last; dipoles times bohr, quadrupoles times
    bohr^2/3;
  * kpolar.f:225-300 and polargrp (kpolar.f:598-800) -- polarizability,
    Thole factor, pdamp = polarity^(1/6) and the polarization groups
    ip11..ip14;
  * readprm.f:199-258 (`atom`, `vdw`, `vdw14`) and kvdw.f:318-503 -- the
    van der Waals classes, pair tables by the radius/epsilon rules and the
    reduction parents and factors.

The device path rotates Z-then-X and Bisector frames (the AMOEBA water
frames); a system with other frame types is refused with a message naming the
atom and frame.
"""

import dataclasses
import math
import os

import numpy as np

from . import params as P
from . import water as W

# frame names of kmpole.f and the device's frame codes
FRAME_CODES = {"Z-then-X": P.AXT_Z_THEN_X, "Bisector": P.AXT_BISECTOR}


class TinkerFormatError(ValueError):
    pass


# ---------------------------------------------------------------------------
# .xyz (readxyz.f)

@dataclasses.dataclass
class XyzFile:
    n: int
    title: str
    names: list
    xyz: np.ndarray          # [n, 3]
    types: np.ndarray        # [n] atom types
    i12: list                # bonded atoms per atom, 0-based, sorted
    box: tuple = None        # (a, b, c, alpha, beta, gamma) from the second line


def _is_word(tok):
    """getword: a token that starts with a letter is a name, not a number."""
    return tok[:1].isalpha() and not tok.lower().startswith(("nan", "inf"))


def read_xyz(path):
    with open(path) as f:
        lines = [ln.rstrip("\n") for ln in f]
    p = 0
    while p < len(lines) and not lines[p].strip():
        p += 1
    if p == len(lines):
        raise TinkerFormatError(f"{path}: no atom count")
    head = lines[p].split(None, 1)
    try:
        n = int(head[0])
    except ValueError as e:
        raise TinkerFormatError(f"{path}: bad atom count {head[0]!r}") from e
    if n <= 0:
        raise TinkerFormatError(f"{path}: the coordinate file contains no atoms")
    title = head[1].strip() if len(head) > 1 else ""
    p += 1
    box = None
    tags, names, xyz, types, bonds = [], [], [], [], []
    while len(tags) < n:
        if p >= len(lines):
            raise TinkerFormatError(f"{path}: error at atom {len(tags) + 1}: file ends")
        tok = lines[p].split()
        p += 1
        if not tok:
            continue
        if not tags and box is None and not any(_is_word(t) for t in tok):
            # the optional periodic-box line before the first atom: a line
            # with no atom name (readxyz.f:150-170, getword finds none)
            try:
                box = tuple(float(t.replace("d", "e").replace("D", "e")) for t in tok[:6])
            except ValueError as e:
                raise TinkerFormatError(f"{path}: bad periodic box line {' '.join(tok)!r}") from e
            if len(box) < 6:
                raise TinkerFormatError(f"{path}: the periodic box line needs a, b, c, alpha, beta, gamma")
            continue
        try:
            tags.append(int(tok[0]))
            names.append(tok[1])
            xyz.append([float(tok[2]), float(tok[3]), float(tok[4])])
            types.append(int(tok[5]))
            bonds.append([int(t) for t in tok[6:]])
        except (ValueError, IndexError) as e:
            raise TinkerFormatError(f"{path}: error at atom {len(tags) + 1}: {' '.join(tok)!r}") from e
    # renumber when the atom numbers are not 1..n in order (readxyz.f:227-246)
    pos = {t: i for i, t in enumerate(tags)}
    if len(pos) != n:
        raise TinkerFormatError(f"{path}: repeated atom numbers")
    i12 = []
    for i, b in enumerate(bonds):
        try:
            i12.append(sorted(pos[t] for t in b if t != 0))
        except KeyError as e:
            raise TinkerFormatError(f"{path}: atom {tags[i]} is bonded to unknown atom {e.args[0]}") from e
    for i, row in enumerate(i12):  # readxyz.f:250-262
        for k in row:
            if i not in i12[k]:
                raise TinkerFormatError(f"{path}: check connection of atom {tags[k]} to atom {tags[i]}")
    return XyzFile(n=n, title=title, names=names, xyz=np.asarray(xyz, dtype=np.float64),
                   types=np.asarray(types, dtype=np.int32), i12=i12, box=box)


def write_xyz(path, ws, types=None, names=None, title="", box_line=False, digits=12):
    """Tinker .xyz of a system (positions, types, bonds from conn['i12'])."""
    n = ws.n
    if types is None or names is None:
        # water atoms, O then two H (water03.prm:80-81: types 1 and 2)
        t = np.tile(np.array([1, 2, 2], np.int32), n // 3)
        nm = ["O", "H", "H"] * (n // 3)
        types = t if types is None else types
        names = nm if names is None else names
    off, idx = ws.conn["i12"]
    with open(path, "w") as f:
        f.write(f"{n:8d}  {title}\n")
        if box_line:
            b = ws.box
            f.write(f"{b[0]:.{digits}f} {b[1]:.{digits}f} {b[2]:.{digits}f} 90.0 90.0 90.0\n")
        for i in range(n):
            bonded = " ".join(f"{k + 1:7d}" for k in idx[off[i]:off[i + 1]])
            f.write(f"{i + 1:7d}  {names[i]:<3s} {ws.x[i]:.{digits}f} {ws.y[i]:.{digits}f} "
                    f"{ws.z[i]:.{digits}f} {types[i]:5d} {bonded}\n")


# ---------------------------------------------------------------------------
# keyword and parameter files (getkey.f, readprm.f, prmkey.f)

def _records(path):
    """Non-empty lines with comments removed: (KEYWORD, rest, raw)."""
    out = []
    with open(path) as f:
        for raw in f:
            line = raw.split("#", 1)[0].rstrip("\n")
            s = line.strip()
            if not s:
                out.append(None)  # keep line positions for multi-line records
                continue
            parts = s.split(None, 1)
            out.append((parts[0].upper(), parts[1] if len(parts) > 1 else "", line))
    return out


@dataclasses.dataclass
class MultipoleEntry:
    k: int          # atom type (or -atom number for an atom-specific entry)
    kz: int
    kx: int
    ky: int
    frame: str      # kmpole.f frame name
    values: list    # 13 components in atomic units, Tinker order


def _parse_multipole(recs, q, where):
    """One multipole record at recs[q] and its four continuation lines
    (readprm.f:1231-1314, kmpole.f:181-230)."""
    _, rest, _ = recs[q]
    tok = rest.split()
    ints = []
    for t in tok:
        try:
            ints.append(int(t))
        except ValueError:
            break
    nint = len(ints)
    if nint == len(tok):  # the charge is written without a decimal point
        nint -= 1
        ints = ints[:nint]
    if nint < 1:
        raise TinkerFormatError(f"{where}: bad multipole record {rest!r}")
    try:
        charge = float(tok[nint])
    except (ValueError, IndexError) as e:
        raise TinkerFormatError(f"{where}: bad multipole charge in {rest!r}") from e
    k = ints[0]
    kz = ints[1] if nint > 1 else 0
    kx = ints[2] if nint > 2 else 0
    ky = ints[3] if nint > 3 else 0
    frame = "Z-then-X"
    if kz == 0:
        frame = "None"
    if kz != 0 and kx == 0:
        frame = "Z-Only"
    if kz < 0 or kx < 0:
        frame = "Bisector"
    if kx < 0 and ky < 0:
        frame = "Z-Bisect"
    if max(kz, kx, ky) < 0:
        frame = "3-Fold"
    cont = []
    r = q + 1
    while len(cont) < 4:
        if r >= len(recs):
            raise TinkerFormatError(f"{where}: multipole record for type {k} is incomplete")
        if recs[r] is not None:
            cont.append(recs[r][2].split())
        r += 1
    try:
        d = [float(v) for v in cont[0][:3]]
        qxx = float(cont[1][0])
        qyx, qyy = (float(v) for v in cont[2][:2])
        qzx, qzy, qzz = (float(v) for v in cont[3][:3])
    except (ValueError, IndexError) as e:
        raise TinkerFormatError(f"{where}: bad multipole moments for type {k}") from e
    values = [charge, d[0], d[1], d[2], qxx, qyx, qzx, qyx, qyy, qzy, qzx, qzy, qzz]
    return MultipoleEntry(k, abs(kz), abs(kx), abs(ky), frame, values), r


def _getnumb(tok):
    """getnumb: an integer token, else 0."""
    try:
        return int(tok)
    except ValueError:
        return 0


@dataclasses.dataclass
class ParamSet:
    multipoles: list = dataclasses.field(default_factory=list)      # parameter-file entries
    key_multipoles: list = dataclasses.field(default_factory=list)  # key-file entries by type
    atom_multipoles: list = dataclasses.field(default_factory=list)  # key-file entries by atom
    polarize: dict = dataclasses.field(default_factory=dict)        # type -> (pol, thole, thd, group types)
    scales: dict = dataclasses.field(default_factory=lambda: {
        # initprm.f:413-470 defaults
        "m_scale": [0.0, 0.0, 1.0, 1.0], "p_scale": [0.0, 0.0, 1.0, 1.0],
        "pi_scale": [0.0, 0.0, 0.5, 1.0], "d_scale": [0.0, 1.0, 1.0, 1.0],
        "u_scale": [1.0, 1.0, 1.0, 1.0]})
    keywords: dict = dataclasses.field(default_factory=dict)        # KEYWORD -> last value text
    vdw: dict = dataclasses.field(default_factory=dict)             # class -> (Rmin, eps, reduction)
    vdw14: dict = dataclasses.field(default_factory=dict)           # class -> (Rmin, eps)
    atom_class: dict = dataclasses.field(default_factory=dict)      # type -> class (`atom` records)
    v_scale: list = dataclasses.field(default_factory=lambda: [0.0, 0.0, 1.0, 1.0])  # initprm.f:385-388


_SCALE_KEYS = {}
for _b, _s in enumerate(("12", "13", "14", "15")):
    _SCALE_KEYS[f"MPOLE-{_s}-SCALE"] = ("m_scale", _b)
    _SCALE_KEYS[f"POLAR-{_s}-SCALE"] = ("p_scale", _b)
    _SCALE_KEYS[f"POLAR-{_s}-INTRA"] = ("pi_scale", _b)
for _b, _s in enumerate(("11", "12", "13", "14")):
    _SCALE_KEYS[f"DIRECT-{_s}-SCALE"] = ("d_scale", _b)
    _SCALE_KEYS[f"MUTUAL-{_s}-SCALE"] = ("u_scale", _b)
_VDW_SCALE_KEYS = {f"VDW-{s_}-SCALE": b for b, s_ in enumerate(("12", "13", "14", "15"))}


def _read_records(path, ps, from_key):
    recs = _records(path)
    q = 0
    while q < len(recs):
        rec = recs[q]
        if rec is None:
            q += 1
            continue
        kw, rest, _ = rec
        where = f"{os.path.basename(path)} line {q + 1}"
        if kw == "MULTIPOLE":
            ent, q = _parse_multipole(recs, q, where)
            if not from_key:
                ps.multipoles.append(ent)
            elif ent.k < 0:
                ps.atom_multipoles.append(ent)
            else:
                ps.key_multipoles.append(ent)
            continue
        if kw == "POLARIZE":
            tok = rest.split()
            try:
                t = int(tok[0])
                pol = float(tok[1])
            except (ValueError, IndexError) as e:
                raise TinkerFormatError(f"{where}: bad polarize record {rest!r}") from e
            thl = thd = 0.0
            rest_tok = tok[2:]
            # readprm.f:1323-1345: reals before the first integer are thole,
            # then the direct damping
            if rest_tok and _getnumb(rest_tok[0]) == 0:
                thl = float(rest_tok[0])
                rest_tok = rest_tok[1:]
                if rest_tok and _getnumb(rest_tok[0]) == 0:
                    thd = float(rest_tok[0])
                    rest_tok = rest_tok[1:]
            grp = [int(v) for v in rest_tok if int(v) != 0]
            ps.polarize[t] = (pol, thl, thd, grp)
        elif kw == "VDW":  # readprm.f:233-245
            tok = rest.split()
            try:
                cl = int(tok[0])
                vals = [float(v) for v in tok[1:4]] + [0.0] * (4 - len(tok[1:4]) - 1)
            except (ValueError, IndexError) as e:
                raise TinkerFormatError(f"{where}: bad vdw record {rest!r}") from e
            ps.vdw[cl] = (vals[0], vals[1], vals[2] if len(vals) > 2 else 0.0)
        elif kw == "VDW14":  # readprm.f:249-258
            tok = rest.split()
            try:
                ps.vdw14[int(tok[0])] = (float(tok[1]), float(tok[2]))
            except (ValueError, IndexError) as e:
                raise TinkerFormatError(f"{where}: bad vdw14 record {rest!r}") from e
        elif kw == "ATOM":  # readprm.f:199: type, class, symbol, ...
            tok = rest.split()
            try:
                ps.atom_class[int(tok[0])] = int(tok[1])
            except (ValueError, IndexError) as e:
                raise TinkerFormatError(f"{where}: bad atom record {rest!r}") from e
        elif kw in _VDW_SCALE_KEYS:
            try:
                ps.v_scale[_VDW_SCALE_KEYS[kw]] = float(rest.split()[0])
            except (ValueError, IndexError) as e:
                raise TinkerFormatError(f"{where}: bad value for {kw}") from e
        elif kw in _SCALE_KEYS:
            name, b = _SCALE_KEYS[kw]
            try:
                ps.scales[name][b] = float(rest.split()[0])
            except (ValueError, IndexError) as e:
                raise TinkerFormatError(f"{where}: bad value for {kw}") from e
        else:
            ps.keywords[kw] = rest.strip()
        q += 1


def read_params(key_path=None, prm_path=None):
    """Parameter set of a key file and the parameter file it names (or
    prm_path).  Key-file keywords override the parameter file's."""
    ps = ParamSet()
    keyfile = ParamSet()
    if key_path is not None:
        _read_records(key_path, keyfile, from_key=True)
        if prm_path is None and "PARAMETERS" in keyfile.keywords:
            name = keyfile.keywords["PARAMETERS"].split()[0].strip('"')
            if not os.path.isabs(name):
                name = os.path.join(os.path.dirname(os.path.abspath(key_path)), name)
            if not os.path.exists(name) and os.path.exists(name + ".prm"):
                name += ".prm"
            prm_path = name
    if prm_path is None:
        raise TinkerFormatError("no parameter file (keyword 'parameters')")
    _read_records(prm_path, ps, from_key=False)
    if key_path is not None:
        _read_records(key_path, ps, from_key=True)  # scale keywords and overrides from the key file
    return ps


def write_water_params(path):
    """A parameter file with the AMOEBA water model used here (water03.prm
    values: atom types 1 and 2, multipoles, polarizabilities, scale factors)."""
    s = P.SCALES
    lines = ["# AMOEBA water parameters (AMOEBA-WATER-2003 values)", ""]
    for b, tag in enumerate(("12", "13", "14", "15")):
        lines.append(f"mpole-{tag}-scale   {s['m_scale'][b]:.4f}")
        lines.append(f"polar-{tag}-scale   {s['p_scale'][b]:.4f}")
        lines.append(f"polar-{tag}-intra   {s['pi_scale'][b]:.4f}")
    for b, tag in enumerate(("11", "12", "13", "14")):
        lines.append(f"direct-{tag}-scale  {s['d_scale'][b]:.4f}")
        lines.append(f"mutual-{tag}-scale  {s['u_scale'][b]:.4f}")
    for b, tag in enumerate(("12", "13", "14", "15")):
        lines.append(f"vdw-{tag}-scale     {P.VDW_SCALE[b]:.4f}")
    lines += [f"vdwtype           BUFFERED-14-7", f"radiusrule        {P.VDW_RULES['radius']}",
              f"radiustype        {P.VDW_RULES['radiustype']}", f"radiussize        {P.VDW_RULES['radiussize']}",
              f"epsilonrule       {P.VDW_RULES['epsilon']}"]
    lines += ["", 'atom          1    1    O     "AMOEBA Water O"    8   15.995    2',
              'atom          2    2    H     "AMOEBA Water H"    1    1.008    1', ""]
    ro, eo, _ = P.WATER_VDW["O"]
    rh, eh, fh = P.WATER_VDW["H"]
    lines += [f"vdw           1               {ro:.4f}     {eo:.4f}",
              f"vdw           2               {rh:.4f}     {eh:.4f}      {fh:.3f}", ""]
    for t, kind, frame in ((1, "O", "-2   -2"), (2, "H", " 1    2")):
        m = P.WATER_MULTIPOLES[kind]
        d = m["dipole"]
        qq = m["quad"]
        lines += [f"multipole     {t}   {frame}        {m['charge']:.5f}",
                  f"                              {d[0]:.5f}    {d[1]:.5f}    {d[2]:.5f}",
                  f"                              {qq[0][0]:.5f}",
                  f"                              {qq[1][0]:.5f}    {qq[1][1]:.5f}",
                  f"                              {qq[2][0]:.5f}    {qq[2][1]:.5f}    {qq[2][2]:.5f}"]
    lines.append("")
    lines.append(f"polarize      1     {P.WATER_POLARITY['O']:.3f}   {P.WATER_THOLE['O']:.3f}     2")
    lines.append(f"polarize      2     {P.WATER_POLARITY['H']:.3f}   {P.WATER_THOLE['H']:.3f}     1")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_key(path, ws, prm_name, poleps=None):
    """Key file for a system: the parameter file, the box, the Ewald and list
    settings and the PME grid of `ws`."""
    lines = [f"parameters        {prm_name}",
             f"a-axis            {ws.box[0]:.12f}", f"b-axis            {ws.box[1]:.12f}",
             f"c-axis            {ws.box[2]:.12f}",
             "ewald", f"ewald-cutoff      {ws.ewaldcut}", f"ewald-alpha       {ws.aewald!r}",
             f"list-buffer       {ws.lbuffer}",
             *([f"vdw-cutoff        {ws.vdw['vdwcut']}",
                f"vdw-taper         {ws.vdw['vdwtaper']}"] if getattr(ws, "vdw", None) else []),
             f"pme-grid          {ws.nfft[0]} {ws.nfft[1]} {ws.nfft[2]}", f"pme-order         {ws.bsorder}",
             "polarization      mutual"]
    if poleps is not None:
        lines.append(f"polar-eps         {poleps}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


# ---------------------------------------------------------------------------
# connectivity (attach.f, polargrp) and parameter assignment (kmpole, kpolar)

def attach(i12):
    """1-3, 1-4 and 1-5 lists from the bond lists (attach.f:17-140)."""
    n = len(i12)
    i13, i14, i15 = [], [], []
    for i in range(n):
        row = []
        for jj in i12[i]:
            for kk in i12[jj]:
                if kk == i or kk in i12[i]:
                    continue
                row.append(kk)
        i13.append(sorted(row))
    for i in range(n):
        row = []
        for jj in i13[i]:
            for kk in i12[jj]:
                if kk == i or kk in i12[i] or kk in i13[i]:
                    continue
                row.append(kk)
        i14.append(sorted(row))
    for i in range(n):
        row = []
        for jj in i14[i]:
            for kk in i12[jj]:
                if kk == i or kk in i12[i] or kk in i13[i] or kk in i14[i]:
                    continue
                row.append(kk)
        i15.append(sorted(row))
    return i13, i14, i15


def polargrp(types, i12, pgrp):
    """Polarization groups ip11 and the group lists ip12..ip14
    (kpolar.f:598-800): ip11 grows from each atom over bonds to atoms whose
    type is in its group list; ip12 is every member of the groups bonded to
    the atom's group, ip13 of the groups bonded to those (not already in
    ip11/ip12), ip14 one step further."""
    n = len(types)
    ip11 = []
    for i in range(n):
        row = [i]
        g = pgrp.get(int(types[i]), [])
        for jj in i12[i]:
            if int(types[jj]) in g:
                row.append(jj)
        ip11.append(row)
    # closure over the directly connected members (kpolar.f:661-708)
    for i in range(n):
        if any(jj < i for jj in ip11[i]):
            jj = min(j for j in ip11[i] if j < i)
            ip11[i] = list(ip11[jj])
            continue
        seen = set(ip11[i])
        start = 0
        while start < len(ip11[i]):
            stop = len(ip11[i])
            for j in range(start, stop):
                for kk in ip11[ip11[i][j]]:
                    if kk not in seen:
                        seen.add(kk)
                        ip11[i].append(kk)
            start = stop
        ip11[i] = sorted(ip11[i])

    def next_level(prev_levels, cur):
        out = []
        for i in range(n):
            mask = set()
            for lv in prev_levels:
                mask.update(lv[i])
            keep = []
            for jj in cur[i]:
                for kk in i12[jj]:
                    if kk not in mask and kk not in cur[i]:
                        keep.append(kk)
            lst = set()
            for jj in keep:
                lst.update(ip11[jj])
            out.append(sorted(x for x in lst if x not in mask and x not in cur[i]))
        return out

    ip12 = []
    for i in range(n):
        mask = set(ip11[i])
        keep = [kk for jj in ip11[i] for kk in i12[jj] if kk not in mask]
        lst = set()
        for jj in keep:
            lst.update(ip11[jj])
        ip12.append(sorted(lst))
    ip13 = next_level([ip11], ip12)
    ip14 = next_level([ip11, ip12], ip13)
    return ip11, ip12, ip13, ip14


def kmpole(types, i12, i13, ps):
    """Local-frame multipoles and frames per atom (kmpole.f:17-540).
    Returns pole [n,13] (dipoles in e*A, quadrupoles in e*A^2 / 3), zaxis,
    xaxis, yaxis (0-based, -1 when unused) and frame names."""
    n = len(types)
    entries = ps.key_multipoles + ps.multipoles  # key-file entries first (kmpole.f:160-230)
    pole = np.zeros((n, 13))
    zaxis = np.full(n, -1, np.int64)
    xaxis = np.full(n, -1, np.int64)
    yaxis = np.full(n, -1, np.int64)
    frame = [""] * n

    def take(i, e, z=-1, x=-1, y=-1):
        zaxis[i], xaxis[i], yaxis[i] = z, x, y
        frame[i] = e.frame
        pole[i] = e.values

    bonded = [set(r) for r in i12]
    for i in range(n):
        it = int(types[i])
        done = False
        # 1-2 atoms only
        for e in entries:
            if done or e.k != it:
                continue
            for ji in i12[i]:
                if done or int(types[ji]) != e.kz:
                    continue
                for ki in i12[i]:
                    if done or int(types[ki]) != e.kx or ki == ji:
                        continue
                    if e.ky == 0:
                        take(i, e, ji, ki)
                        done = True
                        break
                    for li in i12[i]:
                        if int(types[li]) == e.ky and li != ji and li != ki:
                            take(i, e, ji, ki, li)
                            done = True
                            break
        # 1-2 and 1-3 atoms
        for e in entries:
            if done or e.k != it:
                continue
            for ji in i12[i]:
                if done or int(types[ji]) != e.kz:
                    continue
                for ki in i13[i]:
                    if done or int(types[ki]) != e.kx or ji not in bonded[ki]:
                        continue
                    if e.ky == 0:
                        take(i, e, ji, ki)
                        done = True
                        break
                    for li in i13[i]:
                        if int(types[li]) == e.ky and li != ki and ji in bonded[li]:
                            take(i, e, ji, ki, li)
                            done = True
                            break
        # a z atom only
        for e in entries:
            if done or e.k != it:
                continue
            for ji in i12[i]:
                if int(types[ji]) == e.kz and e.kx == 0:
                    take(i, e, ji)
                    done = True
                    break
        # no connected atoms
        for e in entries:
            if done or e.k != it:
                continue
            if e.kz == 0:
                take(i, e)
                done = True
    # atom-specific key-file entries (kmpole.f:450-520): frame atoms by number
    for e in ps.atom_multipoles:
        i = -e.k - 1
        if not 0 <= i < n:
            continue
        zaxis[i] = e.kz - 1 if e.kz else -1
        xaxis[i] = e.kx - 1 if e.kx else -1
        yaxis[i] = e.ky - 1 if e.ky else -1
        frame[i] = e.frame
        pole[i] = e.values
    bohr = P.BOHR
    pole[:, 1:4] = pole[:, 1:4] * bohr  # kmpole.f:534-537
    pole[:, 4:13] = pole[:, 4:13] * bohr ** 2 / 3.0
    return pole, zaxis, xaxis, yaxis, frame


# ---------------------------------------------------------------------------
# the system

def _csr(rows):
    n = len(rows)
    off = np.zeros(n + 1, np.int32)
    off[1:] = np.cumsum([len(r) for r in rows])
    idx = np.array([v for r in rows for v in r], dtype=np.int32)
    return off, idx


def _molecules(i12):
    n = len(i12)
    mol = np.full(n, -1, np.int32)
    m = 0
    for s in range(n):
        if mol[s] >= 0:
            continue
        stack = [s]
        mol[s] = m
        while stack:
            a = stack.pop()
            for b in i12[a]:
                if mol[b] < 0:
                    mol[b] = m
                    stack.append(b)
        m += 1
    return mol, m


def _kw_float(kw, name, default):
    if name not in kw:
        return default
    try:
        return float(kw[name].split()[0].replace("d", "e").replace("D", "e"))
    except (ValueError, IndexError) as e:
        raise TinkerFormatError(f"bad value for {name}: {kw[name]!r}") from e


def _vdw_description(xf, ps, kw):
    """van der Waals description of the atoms (kvdw.f): classes from the
    `atom` records, per-class Rmin/eps/reduction, pair tables by the rules
    keywords, reduction parents (kvdw.f:490-503), vdw-1x-scale, vdw-cutoff
    and vdw-taper (cutoffs.f:74,143,178,241).  None without vdw records."""
    if not ps.vdw:
        return None
    if kw.get("VDWTYPE", "BUFFERED-14-7").split()[0].upper() != "BUFFERED-14-7":
        raise TinkerFormatError(f"vdwtype {kw['VDWTYPE']!r}: only BUFFERED-14-7 (AMOEBA) is supported")
    n = xf.n
    acls = [ps.atom_class.get(int(t), int(t)) for t in xf.types]
    used = sorted(set(acls))
    index = {c: q for q, c in enumerate(used)}
    for c in used:
        if c not in ps.vdw:
            raise TinkerFormatError(f"no vdw parameters for class {c}")
    rad = [ps.vdw[c][0] for c in used]
    eps = [ps.vdw[c][1] for c in used]
    rad4 = [ps.vdw14.get(c, (0.0, 0.0))[0] for c in used]
    eps4 = [ps.vdw14.get(c, (0.0, 0.0))[1] for c in used]
    rules = {"radius": kw.get("RADIUSRULE", "ARITHMETIC").split()[0].upper(),
             "epsilon": kw.get("EPSILONRULE", "GEOMETRIC").split()[0].upper(),
             "radiustype": kw.get("RADIUSTYPE", "R-MIN").split()[0].upper(),
             "radiussize": kw.get("RADIUSSIZE", "RADIUS").split()[0].upper()}
    radmin, epsm, radmin4, eps4t = P.vdw_pair_tables(rad, eps, rad4, eps4, rules)
    cls = np.array([index[c] for c in acls], np.int32)
    kred = np.array([ps.vdw[c][2] for c in acls], np.float64)
    ired = np.array([xf.i12[i][0] if (len(xf.i12[i]) == 1 and kred[i] != 0.0) else i for i in range(n)], np.int32)
    vdwcut = _kw_float(kw, "VDW-CUTOFF", P.VDW_CUTOFF_DEFAULT)
    taper = _kw_float(kw, "VDW-TAPER", P.VDW_TAPER)
    if taper < 1.0:
        taper = taper * vdwcut
    return {"nclass": len(used), "cls": cls, "ired": ired, "kred": kred, "radmin": np.array(radmin),
            "eps": np.array(epsm), "radmin4": np.array(radmin4), "eps4": np.array(eps4t),
            "v_scale": tuple(ps.v_scale), "vdwcut": vdwcut, "vdwtaper": taper, "ghal": P.GHAL, "dhal": P.DHAL}


def load_system(xyz_path, key_path=None, prm_path=None):
    """A system description (water.WaterSystem fields) from Tinker input
    files.  key_path defaults to the .key beside the .xyz; the parameter file
    is the key file's `parameters` unless prm_path is given."""
    if key_path is None:
        cand = os.path.splitext(xyz_path)[0] + ".key"
        key_path = cand if os.path.exists(cand) else None
    xf = read_xyz(xyz_path)
    ps = read_params(key_path, prm_path)
    kw = ps.keywords
    n = xf.n
    # box: the key file's axes, else the .xyz box line (unitcell.f:55-110)
    box = [0.0, 0.0, 0.0]
    if xf.box is not None:
        box = list(xf.box[:3])
    for d, names in enumerate((("A-AXIS", "X-AXIS"), ("B-AXIS", "Y-AXIS"), ("C-AXIS", "Z-AXIS"))):
        for nm in names:
            if nm in kw:
                box[d] = _kw_float(kw, nm, box[d])
    bmax = max(box)
    if bmax <= 0.0:
        raise TinkerFormatError("no periodic box (a-axis or an .xyz box line): the PME path needs one")
    box = [b if b > 0.0 else bmax for b in box]
    for ang in ("ALPHA", "BETA", "GAMMA"):
        if ang in kw and abs(_kw_float(kw, ang, 90.0) - 90.0) > 1e-12:
            raise TinkerFormatError("only orthogonal boxes are supported")
    if xf.box is not None and any(abs(a - 90.0) > 1e-12 for a in xf.box[3:6]):
        raise TinkerFormatError("only orthogonal boxes are supported")
    ewaldcut = _kw_float(kw, "EWALD-CUTOFF", _kw_float(kw, "CUTOFF", 7.0))  # cutoffs.f:58,135-139
    lbuffer = _kw_float(kw, "LIST-BUFFER", 2.0)         # cutoffs.f:80,191
    aewald = _kw_float(kw, "PEWALD-ALPHA", _kw_float(kw, "EWALD-ALPHA", P.ewaldcof(ewaldcut)))
    bsorder = int(_kw_float(kw, "PME-ORDER", 5))
    if "PME-GRID" in kw:
        g = [int(v) for v in kw["PME-GRID"].split()[:3]]
        g += [g[-1]] * (3 - len(g))
        nfft = tuple(g)
    else:  # kewald.f:82-91, 1.2 grid points per A
        nfft = tuple(P.pme_grid_size(b, spacing=1.0 / 1.2) for b in box)
    i13, i14, i15 = attach(xf.i12)
    pole, zaxis, xaxis, yaxis, frame = kmpole(xf.types, xf.i12, i13, ps)
    axt = np.zeros(n, np.int32)
    for i in range(n):
        if frame[i] not in FRAME_CODES:
            what = frame[i] or "no multipole parameters"
            raise TinkerFormatError(f"atom {i + 1} (type {xf.types[i]}): frame {what!r} is not supported "
                                    "(the device path rotates Z-then-X and Bisector frames)")
        axt[i] = FRAME_CODES[frame[i]]
    polarity = np.zeros(n)
    thole = np.zeros(n)
    pgrp = {}
    for t, (pol, thl, _thd, grp) in ps.polarize.items():
        pgrp[t] = grp
    for i in range(n):
        t = int(xf.types[i])
        if t not in ps.polarize:
            raise TinkerFormatError(f"atom {i + 1}: no polarize parameters for type {t}")
        polarity[i], thole[i] = ps.polarize[t][0], ps.polarize[t][1]
    pdamp = polarity ** (1.0 / 6.0)  # kpolar.f:226-238
    ip11, ip12, ip13, ip14 = polargrp(xf.types, xf.i12, pgrp)
    conn = {"i12": _csr(xf.i12), "i13": _csr(i13), "i14": _csr(i14), "i15": _csr(i15),
            "ip11": _csr(ip11), "ip12": _csr(ip12), "ip13": _csr(ip13), "ip14": _csr(ip14)}
    mol, nmol = _molecules(xf.i12)
    scales = {k: tuple(v) for k, v in ps.scales.items()}
    vdw = _vdw_description(xf, ps, kw)
    return W.WaterSystem(n=n, nw=nmol, box=tuple(box), x=np.ascontiguousarray(xf.xyz[:, 0]),
                         y=np.ascontiguousarray(xf.xyz[:, 1]), z=np.ascontiguousarray(xf.xyz[:, 2]),
                         pole=pole, zaxis=zaxis.astype(np.int32), xaxis=xaxis.astype(np.int32), axt=axt,
                         polarity=polarity, thole=thole, pdamp=pdamp, mol=mol, conn=conn, aewald=aewald,
                         ewaldcut=ewaldcut, lbuffer=lbuffer, nfft=nfft, bsorder=bsorder, scales=scales, vdw=vdw)


def save_system(directory, name, ws, poleps=None):
    """Writes name.xyz, name.key and water.prm for a water system, so the
    reference (or this reader) can run the same box."""
    os.makedirs(directory, exist_ok=True)
    write_water_params(os.path.join(directory, "water.prm"))
    write_key(os.path.join(directory, name + ".key"), ws, "water.prm", poleps=poleps)
    write_xyz(os.path.join(directory, name + ".xyz"), ws, title=f"{ws.nw} AMOEBA waters")
    return os.path.join(directory, name + ".xyz")
