"""The split-precision form (gjx_hypJacL2_split): the Gram matrices and the
updates of G and V as exact int8 slice products on the tensor cores,
everything else FP64.  It is not bound to the plain form's bits (blocks of
32 columns and pairs of 64 instead of 16 and 32), so its results are checked
for accuracy, with the bounds written here:

* D against an FP64 reference -- numpy's SVD (LAPACK) for an SVD, the plain
  form (bit-identical to the reference, itself checked against LAPACK) for a
  hyperbolic SVD: |D - D_ref| <= 64 n eps max|D_ref| everywhere (absolute
  accuracy), and relative error <= 1e-12 on the well-conditioned inputs;
* ||U^T U - I||_max <= n eps, ||V^T J V - J||_max <= 2 n eps;
* the residual ||G V - U diag(sqrt|D|)||_max / ||G||_max <= n eps;
* sweeps within 2 of the plain form's.
"""

import numpy as np
import pytest

from gpujachx_b200 import synth

pytestmark = pytest.mark.gpu
EPS = 2.0 ** -53

CASES = [  # m, n, nplus, alg, generator, well-conditioned
    (256, 128, 128, 11, "gaussian", True),
    (512, 256, 100, 11, "graded", True),
    (1024, 512, 512, 3, "gaussian", True),
    (256, 256, 256, 9, "svd_synth", False),
    (384, 192, 192, 11, "gaussian", True),
    (512, 256, 0, 11, "gaussian", True),
    (448, 192, 64, 1, "graded", True),
    (2048, 1024, 512, 11, "graded", True),
]


def _run(fn, alg, G, nplus):
    import torch
    m, n = G.shape
    dG = torch.tensor(np.ascontiguousarray(G.T), dtype=torch.float64, device="cuda")
    dV = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    dD = torch.zeros(n, dtype=torch.float64, device="cuda")
    ret, sw, rs, rb = fn(alg, dG, nplus, dV, dD)
    return sw, dG.cpu().numpy().T, dV.cpu().numpy().T, dD.cpu().numpy()


@pytest.mark.parametrize("m,n,nplus,alg,gen,wellcond", CASES, ids=[f"{c[0]}x{c[1]}_np{c[2]}_alg{c[3]}" for c in CASES])
def test_split_accuracy(built, m, n, nplus, alg, gen, wellcond):
    import gpujachx_b200 as g
    G = synth.make(gen, m, n, 7, **({"smin": 1e-8} if gen == "svd_synth" else {}))
    g.init_strats(None, "cycwor", 32, "cycwor", n // 16)
    sw_p, _, _, D_p = _run(g.hypJacL2_dev, alg, G, nplus)
    sw, U, V, D = _run(g.hypJacL2_split, alg, G, nplus)
    assert abs(sw - sw_p) <= 2, (sw, sw_p)
    if nplus == n:
        ref = np.sort(np.linalg.svd(G, compute_uv=False) ** 2)
    elif nplus == 0:
        ref = np.sort(-np.linalg.svd(G, compute_uv=False) ** 2)
    else:
        ref = np.sort(D_p)
    got = np.sort(D)
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 64 * n * EPS * scale
    if wellcond:
        assert (np.abs(got - ref) / np.abs(ref)).max() <= 1e-12
    assert np.abs(U.T @ U - np.eye(n)).max() <= n * EPS
    if alg & 2:
        J = np.r_[np.ones(nplus), -np.ones(n - nplus)]
        assert np.abs((V.T * J) @ V - np.diag(J)).max() <= 2 * n * EPS
        res = np.abs(G @ V - U * np.sqrt(np.abs(D))).max() / np.abs(G).max()
        assert res <= n * EPS


def test_split_refuses_shapes_it_does_not_take(built):
    import torch
    import gpujachx_b200 as g
    g.init_strats(None, "cycwor", 32, "cycwor", 6)
    G = torch.zeros((96, 128), dtype=torch.float64, device="cuda")  # ncol 96: not a multiple of 64
    D = torch.zeros(96, dtype=torch.float64, device="cuda")
    ret, *_ = g.hypJacL2_split(9, G, 96, None, D, check=False)
    assert ret == -3
