"""Allocation-free energy entry point (thp_epolar_noalloc), checked through
the C-ABI against the energy of the regular solve entry point.

Callers such as a Fortran host whose GPU memory is pooled by OpenACC, or a
loop that must not stall on the device synchronisation cudaMalloc/cudaFree
imply, cannot allocate device memory; this entry point uses only a fixed
scratch array compiled into the library.
The file sorts last so that a run stopping at the first failure has already
run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_epolar_noalloc_matches_solve(thp):
    import torch
    from tinker_hp_b200 import lib as L
    lib = L.load()
    ws = thp.water.make_water_box(216, cfg=0)
    ctx = L.Context(ws, poleps=1e-6)
    res = ctx.solve()
    uind, _ = ctx.dipoles()
    ef = ctx.field()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    d_uind = torch.tensor(uind, dtype=torch.float64, device=dev).contiguous()
    d_ef = torch.tensor(ef, dtype=torch.float64, device=dev).contiguous()
    d_out = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # two calls in a row share (and must reset) the scratch
        d_out.fill_(float("nan"))
        st = lib.thp_epolar_noalloc(ws.n, C.c_void_p(d_uind.data_ptr()), C.c_void_p(d_ef.data_ptr()),
                                    C.c_void_p(d_out.data_ptr()), C.c_void_p(stream))
        assert st == L.THP_OK
        torch.cuda.synchronize()
        e = float(d_out.item())
        assert np.isfinite(e)
        assert abs(e - res["epol"]) < 1e-12 * abs(res["epol"]), (e, res["epol"])


def test_epolar_noalloc_rejects_oversize():
    from tinker_hp_b200 import lib as L
    lib = L.load()
    one = C.c_void_p(1)
    st = lib.thp_epolar_noalloc(L.NOALLOC_MAX_ATOMS + 1, one, one, one, None)
    assert st == L.THP_E_INVALID
