"""Failure detection without a GPU fault: every wait in the kernels is
bounded (mbarriers, block-completion flags) and gives up with an error
status instead of hanging.  Here CTAs wait on an mbarrier that nobody
arrives at, with a short limit: all of them give up after about that many
cycles, the host reads the status, and the context stays usable for a
decomposition right after."""

import ctypes

import numpy as np
import pytest

from gpujachx_b200 import synth


@pytest.mark.gpu
def test_bounded_wait_gives_up_and_context_survives(built):
    import gpujachx_b200 as g
    L = g.lib()
    to, cy = ctypes.c_int(), ctypes.c_longlong()
    limit = 2_000_000  # about a millisecond
    assert L.gjx_wait_selftest(limit, 148, ctypes.byref(to), ctypes.byref(cy)) == 0
    assert to.value == 148
    assert limit < cy.value < 50 * limit
    G = synth.gaussian(256, 128, 3)
    g.init_strats(None, "cycwor", 32, "cycwor", 8)
    r = g.hypJacL2(11, G, 128)
    assert r.ret == 0 and r.sweeps > 0 and np.isfinite(r.D).all()


def test_selftest_checks_its_arguments(built):
    import gpujachx_b200 as g
    to, cy = ctypes.c_int(), ctypes.c_longlong()
    assert g.lib().gjx_wait_selftest(0, 1, ctypes.byref(to), ctypes.byref(cy)) == -1
    assert g.lib().gjx_wait_selftest(1000, 0, ctypes.byref(to), ctypes.byref(cy)) == -1
