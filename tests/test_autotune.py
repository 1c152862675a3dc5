"""The autotuner (gjx_autotune): argument and state errors on the CPU; on
the GPU it picks a configuration for the shape, and the decompositions that
use it are bit-identical to the untuned ones."""

import numpy as np
import pytest

from gpujachx_b200 import synth


def test_autotune_refuses_bad_arguments(built):
    import gpujachx_b200 as g
    with pytest.raises(g.GjxError):
        g.autotune(11, 100, 64, 64)          # nrow not a multiple of 64: code -2
    g.init_strats(None, "cycwor", 32, "cycwor", 8)
    with pytest.raises(g.GjxError) as e:
        g.autotune(11, 1024, 512, 512)       # tables of n1 = 8, shape of n1 = 32
    assert e.value.code == g.ERR_STRAT_ORDER


@pytest.mark.gpu
def test_autotune_keeps_the_bits(built):
    import gpujachx_b200 as g
    m, n, p, alg = 2048, 1024, 512, 11
    G = synth.make("graded", m, n, 79)
    g.init_strats(None, "cycwor", 32, "cycwor", n // 16)
    g.lib().gjx_autotune_clear()
    a = g.hypJacL2(alg, G, p)
    pick = g.autotune(alg, m, n, p, sweeps=1)
    assert pick["split"] in (1, 2, 4) and pick["mode"] in (0, 1)
    b = g.hypJacL2(alg, G, p)
    g.lib().gjx_autotune_clear()
    assert (a.sweeps, a.rot_s, a.rot_b) == (b.sweeps, b.rot_s, b.rot_b)
    for x, y in ((a.U, b.U), (a.V, b.V), (a.D, b.D)):
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64))
