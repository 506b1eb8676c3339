"""The built-in water parameters and the benchmark workload against the
reference's own input files.

tests/golden/reference_inputs.json holds what tinker_io.read_params parses
from the reference's AMOEBA water parameter files (v1.2/params/water03.prm,
water.prm) and from the key files of its 288,000-atom water benchmark "pond"
(v1.2/example/pond.key, v1.1v/example/pond/pond.key); the script beside it
wrote the file.  These tests check that:
  * params.py (the table every water box is built from) equals the parameter
    files entry by entry: local-frame multipoles, frames, polarizabilities,
    Thole factors, polarization groups and the scale factors of the path;
  * the benchmark workload uses pond's settings: real-space cutoff 7.0 A,
    the Ewald coefficient ewaldcof(7.0) (kewald.f), van der Waals cutoff
    9.0 A, a box edge within 0.02 A of pond's 142.27 A, the CG test on
    Tinker's internal units;
  * the oracle solve of a box loaded through the reference's own water03.prm
    equals the solve of the same box built from params.py;
  * where the reference tree is present, the fixture still equals a fresh
    parse of its files.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "reference_inputs.json")
REF_ROOT = "/root/reference"


@pytest.fixture(scope="module")
def ref():
    with open(FIXTURE) as f:
        return json.load(f)


def _local_multipole(P, name):
    m = P.WATER_MULTIPOLES[name]
    q = m["quad"]
    # file order: charge; dipole x y z; quadrupole xx / yx yy / zx zy zz
    return [m["charge"], *m["dipole"], q[0][0], q[1][0], q[1][1], q[2][0], q[2][1], q[2][2]]


def _file_multipole(values):
    v = values  # 13 values: q, d(3), Q(3x3) row-major
    return [v[0], v[1], v[2], v[3], v[4], v[7], v[8], v[10], v[11], v[12]]


@pytest.mark.parametrize("which", ["water03", "water", "pond_v12", "pond_v11"])
def test_params_table_equals_reference_files(thp, ref, which):
    P = thp.params
    ps = ref[which]
    by_type = {m["type"]: m for m in ps["multipoles"]}
    # type 1 = water O (Bisector frame on the two H), type 2 = water H (Z-then-X: O, then the other H)
    assert by_type[1]["frame"] == "Bisector" and (by_type[1]["kz"], by_type[1]["kx"]) == (2, 2)
    assert by_type[2]["frame"] == "Z-then-X" and (by_type[2]["kz"], by_type[2]["kx"]) == (1, 2)
    assert _file_multipole(by_type[1]["values"]) == _local_multipole(P, "O")
    assert _file_multipole(by_type[2]["values"]) == _local_multipole(P, "H")
    pol = ps["polarize"]
    assert (pol["1"]["polarity"], pol["1"]["thole"]) == (P.WATER_POLARITY["O"], P.WATER_THOLE["O"])
    assert (pol["2"]["polarity"], pol["2"]["thole"]) == (P.WATER_POLARITY["H"], P.WATER_THOLE["H"])
    # each water is one polarization group (O lists H, H lists O)
    assert pol["1"]["group"] == [2] and pol["2"]["group"] == [1]
    for key in ("p_scale", "pi_scale", "d_scale", "u_scale"):
        assert tuple(ps["scales"][key]) == tuple(P.SCALES[key]), key
    assert ps["keywords"]["POLARIZATION"] == "MUTUAL"
    # van der Waals classes (Rmin diameter, epsilon, reduction) and scales
    assert tuple(ps["vdw"]["1"]) == P.WATER_VDW["O"] and tuple(ps["vdw"]["2"]) == P.WATER_VDW["H"]
    assert tuple(ps["vdw_scale"]) == P.VDW_SCALE


def test_mpole_scales_of_water03(thp, ref):
    # water03.prm sets the 1-4 / 1-5 multipole scales; water.prm leaves the
    # initprm defaults, which no water pair reaches (water has 1-2 and 1-3
    # pairs only)
    assert tuple(ref["water03"]["scales"]["m_scale"]) == thp.params.SCALES["m_scale"]


@pytest.mark.parametrize("which", ["pond_v12", "pond_v11"])
def test_benchmark_workload_uses_pond_settings(thp, ref, which):
    P = thp.params
    kw = ref[which]["keywords"]
    assert "EWALD" in kw
    assert float(kw["EWALD-CUTOFF"]) == P.EWALD_CUTOFF == 7.0
    assert float(kw["VDW-CUTOFF"]) == P.VDW_CUTOFF_DEFAULT
    # Ewald coefficient of the 7.0 A cutoff (kewald.f ewaldcof, eps 1e-8)
    assert abs(P.ewaldcof(float(kw["EWALD-CUTOFF"])) - 0.5446) < 5e-5


def test_benchmark_box_is_pond(thp, ref):
    kw = ref["pond_v11"]["keywords"]
    edge = thp.water.box_edge(96000)
    # the 96,000-water box at 0.997 g/cm^3 is pond's cubic box of 142.27 A
    assert abs(edge - float(kw["X-AXIS"])) < 0.02, edge
    # pond solves with PCG (polar-alg 1) to polar-eps 1e-5 in Tinker's
    # internal units: the same stop test the CG here restates
    assert kw["POLAR-ALG"] == "1" and float(kw["POLAR-EPS"]) == 1e-5


def test_box_from_reference_parameter_file_solves_identically(thp, tmp_path):
    # a 216-water box written as a Tinker .xyz and loaded with the reference's
    # own water03.prm gives the same oracle solve as the box built from
    # params.py (the reader assigns multipoles, frames and groups itself)
    prm = os.path.join(REF_ROOT, "v1.2", "params", "water03.prm")
    if not os.path.exists(prm):
        pytest.skip("reference tree not present")
    from tinker_hp_b200 import tinker_io as T
    ws = thp.water.make_water_box(216, cfg=0)
    T.write_xyz(str(tmp_path / "w.xyz"), ws)
    with open(tmp_path / "w.key", "w") as f:
        f.write(f"parameters {prm}\newald\newald-cutoff 7.0\n")
        f.write(f"a-axis {ws.box[0]!r}\npme-grid {ws.nfft[0]} {ws.nfft[1]} {ws.nfft[2]}\n")
    wl = T.load_system(str(tmp_path / "w.xyz"), str(tmp_path / "w.key"))
    oa, ob = O.Oracle(ws, poleps=1e-8), O.Oracle(wl, poleps=1e-8)
    assert oa.mlistcell()[0] == 0 and ob.mlistcell()[0] == 0
    # the .xyz holds 12 decimals, so frames agree to rounding of the positions
    np.testing.assert_allclose(ob.rpole, oa.rpole, rtol=0, atol=1e-12)
    a, b = oa.solve(), ob.solve()
    assert a["niter"] == b["niter"]
    np.testing.assert_allclose(b["uind"], a["uind"], rtol=0, atol=1e-10)
    np.testing.assert_allclose(b["uinp"], a["uinp"], rtol=0, atol=1e-10)


def test_fixture_matches_reference_tree():
    if not os.path.isdir(REF_ROOT):
        pytest.skip("reference tree not present")
    import importlib.util
    spec = importlib.util.spec_from_file_location("mri", os.path.join(HERE, "golden", "make_reference_inputs.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    fresh = json.loads(json.dumps(m.parsed(REF_ROOT), sort_keys=True))
    with open(FIXTURE) as f:
        assert json.load(f) == fresh
