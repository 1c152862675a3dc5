"""gjx_hypJacL2_noalloc: the entry point for callers that cannot allocate device
memory (their device memory belongs to a caching allocator or pool, or was
reserved at start-up, or their hot path forbids cudaMalloc/cudaFree, which
synchronise the device).  Its working memory is a static device array of the
library, so it must give exactly what gjx_hypJacL2_dev gives -- bit for bit,
the tolerance of every parity test here -- on consecutive calls that share
that array, and it must refuse tables that do not fit the array.

This file is collected last on purpose: a failure here leaves every other
test already run.  It passes alone in a fresh process and after the others.
"""

import ctypes

import numpy as np
import pytest

from tests.golden.make_golden import case, make_input


def _dev_call(fn, alg, G, nplus):
    """Run fn (one of the two device entry points) on fresh device copies."""
    import torch
    m, n = G.shape
    dG = torch.tensor(np.ascontiguousarray(G.T), dtype=torch.float64, device="cuda")
    dV = torch.empty((n, n), dtype=torch.float64, device="cuda")
    dD = torch.empty(n, dtype=torch.float64, device="cuda")
    swp, s, b = ctypes.c_uint(), ctypes.c_ulonglong(), ctypes.c_ulonglong()
    full = bool(alg & 2)
    torch.cuda.synchronize()
    ret = fn(alg, m, n, nplus, dG.data_ptr(), m, dV.data_ptr() if full else None, n if full else 0, dD.data_ptr(),
             None, ctypes.byref(swp), ctypes.byref(s), ctypes.byref(b))
    torch.cuda.synchronize()
    return ret, swp.value, s.value, b.value, dG.cpu().numpy(), (dV.cpu().numpy() if full else None), dD.cpu().numpy()


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))


@pytest.mark.gpu
def test_noalloc_equals_device_entry_point_on_consecutive_calls(built):
    import gpujachx_b200 as g
    L = g.lib()
    cases = [case("na_a", 1024, 512, 512, 11, seed=501),
             case("na_b", 512, 256, 100, 3, seed=502, snp0="rowcyc", snp1="colcyc"),
             case("na_a_again", 1024, 512, 512, 11, seed=501)]
    for c in cases:  # consecutive calls: the static array keeps the previous call's contents
        G = make_input(c)
        g.init_strats(None, c["snp0"], 32, c["snp1"], c["n"] // 16)
        ref = _dev_call(L.gjx_hypJacL2_dev, c["alg"], G, c["nplus"])
        got = _dev_call(L.gjx_hypJacL2_noalloc, c["alg"], G, c["nplus"])
        assert ref[0] == 0 and got[0] == 0, g.last_error()
        assert got[1:4] == ref[1:4], c["name"]
        for x, y in zip(got[4:], ref[4:]):
            if y is not None:
                assert _same(x, y), c["name"]


@pytest.mark.gpu
def test_noalloc_twice_in_a_row_same_input(built):
    import gpujachx_b200 as g
    L = g.lib()
    c = case("na_twice", 2048, 1024, 400, 9, gen="graded", seed=503)
    G = make_input(c)
    g.init_strats(None, "cycwor", 32, "cycwor", c["n"] // 16)
    ref = _dev_call(L.gjx_hypJacL2_dev, c["alg"], G, c["nplus"])
    one = _dev_call(L.gjx_hypJacL2_noalloc, c["alg"], G, c["nplus"])
    two = _dev_call(L.gjx_hypJacL2_noalloc, c["alg"], G, c["nplus"])
    for got in (one, two):
        assert got[0] == 0 and got[1:4] == ref[1:4]
        assert _same(got[4], ref[4]) and _same(got[6], ref[6])


def test_noalloc_refuses_tables_beyond_its_scratch(built):
    """n1 = 896 (ncol 14336) needs 1.6 MB of table: refused before any CUDA call."""
    import gpujachx_b200 as g
    L = g.lib()
    g.init_strats(None, "cycwor", 32, "cycwor", 896)
    fake = ctypes.c_void_p(256)  # aligned, never dereferenced: the size check comes first
    swp, s, b = ctypes.c_uint(), ctypes.c_ulonglong(), ctypes.c_ulonglong()
    ret = L.gjx_hypJacL2_noalloc(0, 14336, 14336, 14336, fake, 14336, None, 0, fake, None, ctypes.byref(swp),
                                 ctypes.byref(s), ctypes.byref(b))
    assert ret == g.ERR_SCRATCH
    assert "static scratch" in g.last_error()
    # argument errors keep the reference's codes
    assert L.gjx_hypJacL2_noalloc(16, 64, 32, 32, fake, 64, None, 0, fake, None, ctypes.byref(swp), ctypes.byref(s),
                                  ctypes.byref(b)) == -1


@pytest.mark.gpu
def test_noalloc_second_call_takes_no_device_memory(built):
    """Once the first call on a device has set up the static array, a call
    changes the device's free memory by nothing: every cudaMalloc (the
    library's or a caching allocator's) would take at least one 2 MiB page."""
    import torch
    import gpujachx_b200 as g
    L = g.lib()
    c = case("na_mem", 1024, 512, 512, 11, seed=504)
    G = make_input(c)
    g.init_strats(None, "cycwor", 32, "cycwor", c["n"] // 16)
    m, n = G.shape
    dG = torch.tensor(np.ascontiguousarray(G.T), dtype=torch.float64, device="cuda")
    dG0 = dG.clone()
    dV = torch.empty((n, n), dtype=torch.float64, device="cuda")
    dD = torch.empty(n, dtype=torch.float64, device="cuda")
    swp, s, b = ctypes.c_uint(), ctypes.c_ulonglong(), ctypes.c_ulonglong()

    def call():
        dG.copy_(dG0)
        torch.cuda.synchronize()
        return L.gjx_hypJacL2_noalloc(11, m, n, 512, dG.data_ptr(), m, dV.data_ptr(), n, dD.data_ptr(), None,
                                      ctypes.byref(swp), ctypes.byref(s), ctypes.byref(b))

    assert call() == 0, g.last_error()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    assert call() == 0, g.last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
