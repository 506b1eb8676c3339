"""Tinker input files (tinker_hp_b200/tinker_io.py): readers for .xyz, .key
and .prm, the frame assignment of kmpole, attach's 1-3..1-5 lists and the
polarization groups of polargrp, checked against the systems the package
builds directly and against the oracle."""
import dataclasses

import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def tio(thp):
    import importlib
    return importlib.import_module(thp.__name__ + ".tinker_io")


def _same_system(a, b, pos_tol=1e-10):
    assert a.n == b.n
    np.testing.assert_allclose(a.positions(), b.positions(), rtol=0, atol=pos_tol)
    np.testing.assert_allclose(a.box, b.box, rtol=0, atol=1e-10)
    np.testing.assert_allclose(a.pole, b.pole, rtol=1e-14, atol=1e-16)
    for f in ("zaxis", "xaxis", "axt"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f), err_msg=f)
    for f in ("polarity", "thole", "pdamp"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f), err_msg=f)
    for name in b.conn:
        for q in (0, 1):
            np.testing.assert_array_equal(a.conn[name][q], b.conn[name][q], err_msg=name)
    for k in b.scales:
        assert tuple(a.scales[k]) == tuple(b.scales[k]), k
    assert a.nfft == b.nfft and a.bsorder == b.bsorder
    if b.vdw is not None:
        for k in ("cls", "ired"):
            np.testing.assert_array_equal(a.vdw[k], b.vdw[k], err_msg=k)
        for k in ("kred", "radmin", "eps", "radmin4", "eps4"):
            np.testing.assert_allclose(a.vdw[k], b.vdw[k], rtol=1e-15, atol=0, err_msg=k)
        for k in ("nclass", "v_scale", "vdwcut", "vdwtaper", "ghal", "dhal"):
            assert np.allclose(a.vdw[k], b.vdw[k], rtol=1e-15, atol=0), k
    assert a.ewaldcut == b.ewaldcut and a.lbuffer == b.lbuffer and a.aewald == b.aewald


def test_water_box_round_trip(tio, thp, tmp_path):
    ws = thp.water.make_water_box(216, cfg=0)
    path = tio.save_system(str(tmp_path), "box216", ws)
    back = tio.load_system(path)
    _same_system(back, ws)
    assert back.nw == 216 and np.array_equal(back.mol, ws.mol)


def test_loaded_box_solves_like_the_built_one(tio, thp, tmp_path):
    ws = thp.water.make_water_box(216, cfg=0)
    back = tio.load_system(tio.save_system(str(tmp_path), "b", ws))
    a, b = O.Oracle(ws, poleps=1e-8), O.Oracle(back, poleps=1e-8)
    assert a.mlistcell()[0] == 0 and b.mlistcell()[0] == 0
    ra, rb = a.solve(), b.solve()
    assert ra["niter"] == rb["niter"]
    np.testing.assert_allclose(rb["uind"], ra["uind"], rtol=0, atol=1e-12)
    ea, eb = a.empole1()[0], b.empole1()[0]
    assert abs(ea - eb) < 1e-9


def test_box_line_renumbering_and_defaults(tio, thp, tmp_path):
    # a box line in the .xyz instead of axis keywords, atom numbers offset by
    # 100 (renumbered as readxyz does), and no grid, alpha, cutoff or buffer
    # keywords: Tinker's defaults apply
    ws = thp.water.make_water_box(64, cfg=0, edge=16.0)
    tio.write_water_params(str(tmp_path / "water.prm"))
    (tmp_path / "w.key").write_text("parameters water.prm\newald\n")
    off, idx = ws.conn["i12"]
    lines = [f"{ws.n}  renumbered", f"{ws.box[0]:.12f} {ws.box[1]:.12f} {ws.box[2]:.12f} 90 90 90"]
    for i in range(ws.n):
        t = 1 if i % 3 == 0 else 2
        bonded = " ".join(str(k + 101) for k in idx[off[i]:off[i + 1]])
        lines.append(f"{i + 101} {'O' if t == 1 else 'H'} {ws.x[i]:.12f} {ws.y[i]:.12f} {ws.z[i]:.12f} {t} {bonded}")
    (tmp_path / "w.xyz").write_text("\n".join(lines) + "\n")
    back = tio.load_system(str(tmp_path / "w.xyz"))
    ref = dataclasses.replace(ws, lbuffer=2.0, nfft=(20, 20, 20), vdw=None)  # 1.2 points per A over 16 A -> 20
    _same_system(back, ref)


def test_key_overrides_and_atom_multipoles(tio, thp, tmp_path):
    ws = thp.water.make_water_box(64, cfg=0, edge=16.0)
    path = tio.save_system(str(tmp_path), "w", ws)
    # scale keywords and an atom-specific multipole for atom 4 (the second
    # oxygen) in the key file
    with open(tmp_path / "w.key", "a") as f:
        f.write("mpole-14-scale 0.5\npolar-13-scale 0.25\n")
        f.write("multipole -4 -5 -6 -0.6\n 0.0 0.0 0.2\n 0.3\n 0.0 -0.4\n 0.0 0.0 0.1\n")
    back = tio.load_system(path)
    assert back.scales["m_scale"][2] == 0.5 and back.scales["p_scale"][1] == 0.25
    b = 0.52917721092
    q = b ** 2 / 3.0
    want = [-0.6, 0.0, 0.0, 0.2 * b, 0.3 * q, 0.0, 0.0, 0.0, -0.4 * q, 0.0, 0.0, 0.0, 0.1 * q]
    np.testing.assert_allclose(back.pole[3], want, rtol=1e-15, atol=0)
    assert back.zaxis[3] == 4 and back.xaxis[3] == 5 and back.axt[3] == 2
    np.testing.assert_allclose(back.pole[6], ws.pole[6], rtol=1e-14, atol=1e-16)  # other oxygens: the type's


def test_attach_and_polarization_groups_of_a_chain(tio):
    # a five-atom chain with two polarization groups {0,1} and {2,3,4}
    # (types 1-1 and 2-2-2; the group of type 1 lists type 1, of type 2 type 2)
    i12 = [[1], [0, 2], [1, 3], [2, 4], [3]]
    i13, i14, i15 = tio.attach(i12)
    assert i13 == [[2], [3], [0, 4], [1], [2]]
    assert i14 == [[3], [4], [], [0], [1]]
    assert i15 == [[4], [], [], [], [0]]
    types = np.array([1, 1, 2, 2, 2])
    ip11, ip12, ip13, ip14 = tio.polargrp(types, i12, {1: [1], 2: [2]})
    assert ip11 == [[0, 1], [0, 1], [2, 3, 4], [2, 3, 4], [2, 3, 4]]
    assert ip12 == [[2, 3, 4], [2, 3, 4], [0, 1], [0, 1], [0, 1]]
    assert ip13 == [[]] * 5 and ip14 == [[]] * 5


def test_polarize_record_forms(tio, tmp_path):
    prm = tmp_path / "p.prm"
    prm.write_text("polarize 1 0.837 0.390 2\npolarize 2 0.496 1\npolarize 3 1.0 0.39 0.7 4 5\n")
    ps = tio.read_params(prm_path=str(prm))
    assert ps.polarize[1] == (0.837, 0.39, 0.0, [2])
    assert ps.polarize[2] == (0.496, 0.0, 0.0, [1])
    assert ps.polarize[3] == (1.0, 0.39, 0.7, [4, 5])


def test_unsupported_frame_is_refused(tio, thp, tmp_path):
    ws = thp.water.make_water_box(64, cfg=0, edge=16.0)
    path = tio.save_system(str(tmp_path), "w", ws)
    # an atom-specific Z-Only frame for atom 2 (a type entry with a z atom
    # only would not win: kmpole tries the Z-then-X entry's 1-3 pass first)
    with open(tmp_path / "w.key", "a") as f:
        f.write("multipole -2 1 0.25983\n 0.0 0.0 0.1\n 0.0\n 0.0 0.0\n 0.0 0.0 0.0\n")
    with pytest.raises(tio.TinkerFormatError, match="Z-Only"):
        tio.load_system(path)


def test_bad_connection_is_refused(tio, tmp_path):
    (tmp_path / "p.prm").write_text("polarize 1 1.0 0.39\n")
    (tmp_path / "b.key").write_text("parameters p.prm\na-axis 20\n")
    (tmp_path / "b.xyz").write_text("2\n1 O 0 0 0 1 2\n2 O 1 0 0 1\n")
    with pytest.raises(tio.TinkerFormatError, match="check connection"):
        tio.load_system(str(tmp_path / "b.xyz"))


def test_pass_order_beats_entry_order(tio, thp, tmp_path):
    # kmpole tries every entry in one pass before the next pass: a key-file
    # type entry with a z atom only (pass 3) does not displace the parameter
    # file's Z-then-X entry that matches in the 1-3 pass
    ws = thp.water.make_water_box(64, cfg=0, edge=16.0)
    path = tio.save_system(str(tmp_path), "w", ws)
    with open(tmp_path / "w.key", "a") as f:
        f.write("multipole 2 1 0.25983\n 0.0 0.0 0.1\n 0.0\n 0.0 0.0\n 0.0 0.0 0.0\n")
    back = tio.load_system(path)
    np.testing.assert_array_equal(back.axt, ws.axt)
    np.testing.assert_allclose(back.pole, ws.pole, rtol=1e-14, atol=1e-16)


def test_loaded_box_vdw_matches_the_built_one(tio, thp, tmp_path):
    ws = thp.water.make_water_box(216, cfg=0, edge=20.0)
    back = tio.load_system(tio.save_system(str(tmp_path), "v", ws))
    ea, da = O.Oracle(ws).ehal1()
    eb, db = O.Oracle(back).ehal1()
    assert abs(ea - eb) < 1e-10 * abs(ea)
    np.testing.assert_allclose(db, da, rtol=0, atol=1e-9 * np.abs(da).max())


def test_group_lists_of_single_atom_groups(tio):
    # each atom its own polarization group (no group types): ip12..ip14 are
    # the atoms one, two and three bonds away along the chain 0-1-2-3-4-5
    i12 = [[1], [0, 2], [1, 3], [2, 4], [3, 5], [4]]
    ip11, ip12, ip13, ip14 = tio.polargrp(np.arange(6) + 1, i12, {})
    assert ip11 == [[i] for i in range(6)]
    assert ip12 == i12
    assert ip13 == [[2], [3], [0, 4], [1, 5], [2], [3]]
    assert ip14 == [[3], [4], [5], [0], [1], [2]]
