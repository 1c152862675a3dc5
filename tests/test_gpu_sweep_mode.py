"""One launch per sweep (the default where every cluster of a step fits on
the GPU) against one launch per outer step: the same bits, sweeps and
counts, for cluster (2 CTAs per pair) and single-CTA pairs, trigonometric,
hyperbolic and sorted variants."""

import numpy as np
import pytest

from gpujachx_b200 import synth


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,p,alg,gen", [(256, 256, 256, 9, "svd_synth"), (1024, 512, 200, 11, "graded"),
                                           (2048, 1024, 512, 3, "graded"), (4096, 2048, 2048, 11, "gaussian"),
                                           (640, 640, 640, 1, "gaussian")])
def test_one_launch_per_sweep_equals_per_step(built, m, n, p, alg, gen):
    import gpujachx_b200 as g
    kw = {"smin": 1e-8} if gen == "svd_synth" else {}
    G = synth.make(gen, m, n, 77, **kw)
    g.init_strats(None, "cycwor", 32, "cycwor", n // 16)
    out = []
    for mode in (0, 1):
        g.lib().gjx_set_sweep_mode(mode)
        g.profile(True)
        r = g.hypJacL2(alg, G, p)
        prof = g.profile_read()
        g.profile(False)
        out.append((r, prof))
    g.lib().gjx_set_sweep_mode(1)
    (a, pa), (b, pb) = out
    assert (a.sweeps, a.rot_s, a.rot_b) == (b.sweeps, b.rot_s, b.rot_b)
    for x, y in ((a.U, b.U), (a.D, b.D)) + (((a.V, b.V),) if alg & 2 else ()):
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64))
    # per step: one launch per outer step; per sweep: fewer launches (one per sweep when it fits)
    assert pb["launches"] <= pa["launches"]


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,p,alg", [(256, 256, 256, 9), (1024, 512, 200, 11), (2048, 1024, 512, 11),
                                       (512, 256, 0, 3)])
def test_cluster_sizes_give_the_same_bits(built, m, n, p, alg):
    """1, 2 or 4 CTAs per block pair, one launch per sweep or per step."""
    import gpujachx_b200 as g
    G = synth.make("graded", m, n, 78)
    g.init_strats(None, "cycwor", 32, "cycwor", n // 16)
    runs = []
    for split in (1, 2, 4):
        for mode in (0, 1):
            g.lib().gjx_set_split(split)
            g.lib().gjx_set_sweep_mode(mode)
            runs.append(g.hypJacL2(alg, G, p))
    g.lib().gjx_set_split(0)
    g.lib().gjx_set_sweep_mode(1)
    a = runs[0]
    for b in runs[1:]:
        assert (a.sweeps, a.rot_s, a.rot_b) == (b.sweeps, b.rot_s, b.rot_b)
        for x, y in ((a.U, b.U), (a.D, b.D)) + (((a.V, b.V),) if alg & 2 else ()):
            assert np.array_equal(x.view(np.uint64), y.view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,p,alg,gen", [(256, 256, 256, 9, "svd_synth"), (1024, 480, 200, 11, "graded"),
                                           (2048, 1024, 512, 3, "graded"), (640, 640, 640, 1, "gaussian"),
                                           (512, 256, 0, 11, "gaussian")])
def test_two_pairs_per_cta_give_the_same_bits(built, m, n, p, alg, gen):
    """One CTA per block pair, per-step launches: two pairs per CTA (the form
    used when a step has more pairs than SMs; 480 columns: 15 pairs per step,
    the last one alone) against one."""
    import gpujachx_b200 as g
    kw = {"smin": 1e-8} if gen == "svd_synth" else {}
    G = synth.make(gen, m, n, 79, **kw)
    g.init_strats(None, "cycwor", 32, "cycwor", n // 16)
    g.lib().gjx_set_split(1)
    g.lib().gjx_set_sweep_mode(0)
    runs = []
    for w in (1, 2):
        g.lib().gjx_set_pairs_per_cta(w)
        runs.append(g.hypJacL2(alg, G, p))
    g.lib().gjx_set_pairs_per_cta(0)
    g.lib().gjx_set_split(0)
    g.lib().gjx_set_sweep_mode(-1)
    a, b = runs
    assert (a.sweeps, a.rot_s, a.rot_b) == (b.sweeps, b.rot_s, b.rot_b)
    for x, y in ((a.U, b.U), (a.D, b.D)) + (((a.V, b.V),) if alg & 2 else ()):
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64))
