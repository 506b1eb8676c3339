"""CPU-side checks of the C-ABI library: it builds, loads without a GPU and
exports every function declared in include/thp.h."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "thp.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*([a-z_0-9]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_reference_dropins():
    names = declared_functions()
    for f in ("newinduce_pme2_", "inducepcg_pme2_", "tmatxb_pme_", "efld0_direct_", "efld0_recip_",
              "tmatxbrecip_", "mlistcell_", "vlistcell_", "epolar_", "epolar1_", "empole1_", "ehal1_",
              "thp_solve", "thp_ctx_create", "thp_empole1", "thp_ehal1", "thp_set_vdw", "thp_get_vlist"):
        assert f in names, f


def test_library_exports_every_declared_symbol(thp):
    from tinker_hp_b200 import lib as L
    L.load()
    lib = C.CDLL(L.LIB_PATH)
    missing = [f for f in declared_functions() if not hasattr(lib, f)]
    assert not missing, missing


def test_no_device_is_reported_not_crashed(thp):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from tinker_hp_b200 import lib as L
    ws = thp.water.make_water_box(216)
    with pytest.raises(L.ThpError) as e:
        L.Context(ws)
    assert e.value.status == L.THP_E_NO_DEVICE


def test_footprint_scales_with_size(thp):
    from tinker_hp_b200 import lib as L
    a = L.footprint(thp.water.make_water_box(216))
    b = L.footprint(thp.water.make_water_box(1000))
    assert 0 < a < b


def test_fortran_shim_binds_declared_noncolliding_symbols():
    # The shim reaches the library only through names that no Tinker-HP
    # object defines (thp_*), each declared in include/thp.h; the
    # reference-named drop-ins are for builds that drop those objects.
    src = open(os.path.join(ROOT, "tinker-hp_b200", "fortran", "thp_shim.f90")).read()
    names = re.findall(r'bind\(C,\s*name="([^"]+)"\)', src)
    assert len(names) >= 15
    declared = set(declared_functions())
    for n in names:
        assert n.startswith("thp_"), n
        assert n in declared, n
    # module variables (no TARGET attribute in Tinker-HP) never go through c_loc
    code = "\n".join(l.split("!")[0] for l in src.splitlines())
    for var in ("x", "y", "z", "rpole", "uind", "uinp", "nelst", "elst", "ep", "em", "ev", "dep", "dem", "dev",
                "polarity", "thole", "pdamp"):
        assert not re.search(r"c_loc\(\s*%s\s*\)" % var, code), var
    # maxelst comes from module sizes, lbuffer from module neigh (v1.2 modules)
    assert re.search(r"use sizes, only: maxelst", code)
    assert re.search(r"use neigh, only: lbuffer", code)
