"""The batched form (gjx_hypJacL2_batched): every matrix of a batch gets
exactly what the single-matrix device call gives it -- U, V, D bit for bit,
sweeps and rotation counts -- for mixed sizes (64..512 columns, square and
tall), mixed signatures (J = I, J = -I, mixed), all four kernel variants
(ALG 3, 9, 11, 1), one and two block pairs per CTA of 8 warps and of 4 warps (two CTAs per SM), and a
matrix with invalid arguments that is reported and left alone while the others run."""

import numpy as np
import pytest

from gpujachx_b200 import synth


def _dev(G, full):
    import torch
    m, n = G.shape
    dG = torch.tensor(np.ascontiguousarray(G.T), dtype=torch.float64, device="cuda")
    dV = torch.zeros((n, n), dtype=torch.float64, device="cuda") if full else None
    dD = torch.zeros(n, dtype=torch.float64, device="cuda")
    return dG, dV, dD


def _bits(t):
    return t.cpu().numpy().view(np.uint64)


CASES = [(64, 64, 64), (128, 128, 64), (192, 192, 0), (256, 256, 256), (320, 320, 160), (384, 384, 384),
         (448, 448, 224), (512, 512, 512), (256, 128, 128), (512, 256, 100), (128, 64, 32), (640, 320, 320)]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("width", [2, 1, 3, 4])
@pytest.mark.parametrize("alg", [11, 9, 3, 1])
def test_batched_equals_single(built, alg, width, mode):
    import torch
    import gpujachx_b200 as g
    g.lib().gjx_set_pairs_per_cta(width)   # 2 (4): two block pairs per CTA (of 4 warps), from different matrices too
    g.lib().gjx_set_batch_mode(mode)       # 0: one launch per step index, 1: one launch per sweep
    g.init_strats(None, "cycwor", 32, "cycwor", 4)   # the family; each matrix takes its own n1 table
    full = bool(alg & 2)
    mats = []
    for k, (m, n, p) in enumerate(CASES):
        gen = "svd_synth" if m == n else "graded"
        G = synth.make(gen, m, n, 5000 + k, **({"smin": 1e-6} if gen == "svd_synth" else {}))
        mats.append((G, p))
    batch = [_dev(G, full) for G, _ in mats]
    res = g.hypJacL2_batched(alg, [b[0] for b in batch], [p for _, p in mats], Vs=[b[1] for b in batch] if full else None,
                             Ds=[b[2] for b in batch])
    g.lib().gjx_set_pairs_per_cta(0)
    g.lib().gjx_set_batch_mode(-1)
    assert res.info == [0] * len(mats)
    for k, (G, p) in enumerate(mats):
        n = G.shape[1]
        g.init_strats(None, "cycwor", 32, "cycwor", n // 16)
        dG, dV, dD = _dev(G, full)
        ret, sw, rs, rb = g.hypJacL2_dev(alg, dG, p, dV, dD)
        torch.cuda.synchronize()
        assert (res.sweeps[k], res.rot_s[k], res.rot_b[k]) == (sw, rs, rb), (k, CASES[k])
        assert np.array_equal(_bits(batch[k][0]), _bits(dG)), k
        assert np.array_equal(_bits(batch[k][2]), _bits(dD)), k
        if full:
            assert np.array_equal(_bits(batch[k][1]), _bits(dV)), k


@pytest.mark.gpu
def test_batched_bad_matrix_is_reported(built):
    import torch
    import gpujachx_b200 as g
    g.init_strats(None, "cycwor", 32, "cycwor", 4)
    G1 = synth.gaussian(128, 64, 1)
    good = _dev(G1, True)
    bad = _dev(synth.gaussian(96, 48, 2), True)          # 96 rows: not a multiple of 64
    keep = bad[0].clone()
    res = g.hypJacL2_batched(11, [good[0], bad[0]], [64, 48], Vs=[good[1], bad[1]], Ds=[good[2], bad[2]])
    assert res.info[0] == 0 and res.info[1] == -2
    assert res.sweeps[1] == 0 and torch.equal(bad[0], keep)
    g.init_strats(None, "cycwor", 32, "cycwor", 4)
    ref = _dev(G1, True)
    r = g.hypJacL2_dev(11, ref[0], 64, ref[1], ref[2])
    assert res.sweeps[0] == r[1] and np.array_equal(_bits(good[0]), _bits(ref[0]))


@pytest.mark.gpu
def test_batch_autotuner_picks_and_keeps_bits(built):
    """gjx_autotune_batched times (pairs per CTA) x (per-step / per-sweep
    launches) on random matrices of the batch's shapes; the batch run after it
    (with the tuned choice) still gives every matrix the single call's bits."""
    import torch
    import gpujachx_b200 as g
    shapes = [(128, 128, 128), (256, 256, 128), (192, 192, 0), (320, 320, 320), (128, 64, 64)]
    g.init_strats(None, "cycwor", 32, "cycwor", 4)
    pick = g.autotune_batched(11, [m for m, _, _ in shapes], [n for _, n, _ in shapes], [p for _, _, p in shapes])
    assert pick["pairs_per_cta"] in (1, 2, 3, 4) and pick["mode"] in (0, 1)
    mats = [synth.make("svd_synth", m, n, 7000 + k, smin=1e-6) if m == n else synth.make("graded", m, n, 7000 + k)
            for k, (m, n, _) in enumerate(shapes)]
    batch = [_dev(G, True) for G in mats]
    res = g.hypJacL2_batched(11, [b[0] for b in batch], [p for _, _, p in shapes], Vs=[b[1] for b in batch],
                             Ds=[b[2] for b in batch])
    g.lib().gjx_autotune_clear()
    for k, (G, (m, n, p)) in enumerate(zip(mats, shapes)):
        g.init_strats(None, "cycwor", 32, "cycwor", n // 16)
        dG, dV, dD = _dev(G, True)
        ret, sw, rs, rb = g.hypJacL2_dev(11, dG, p, dV, dD)
        torch.cuda.synchronize()
        assert (res.sweeps[k], res.rot_s[k], res.rot_b[k]) == (sw, rs, rb)
        assert np.array_equal(_bits(batch[k][0]), _bits(dG)) and np.array_equal(_bits(batch[k][1]), _bits(dV))
