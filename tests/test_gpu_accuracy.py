"""Accuracy of the CUDA path against FP64 LAPACK (and an eigen-oracle for the
hyperbolic case), on the benchmark configurations or scaled-down versions.

Bounds (stated per config, as asked of the plain FP64 form):
* SVD, well conditioned (config 2, i.i.d. Gaussian): max_i |D_i - s_i^2| / s_i^2
  <= 8 N eps against DGESVJ's s_i;
* SVD, ill conditioned (config 1, s_i from 1 to 1e-8, columns not graded):
  |D_i - s_i^2| / s_i^2 <= 8 N eps * s_1 / s_i (each sigma_i is accurate to
  about eps * sigma_1, so D_i to 2 eps sigma_1 sigma_i);
* HSVD: |D_i - lambda_i| <= 64 N eps ||R||^2 against the eigenvalues of
  R J R^T (G = QR; symmetric eigensolver, absolute accuracy only);
* ||U^T U - I||_max <= 4 N eps; ||V^T J V - J||_max <= 4 N eps * kappa, where
  kappa = max |D| / min |D| enters for the non-orthogonal hyperbolic V.
"""

import numpy as np
import pytest

from gpujachx_b200 import synth
from oracle import lapack

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps


def _svd(alg, G, n1, snp="cycwor"):
    import gpujachx_b200 as g
    g.init_strats(None, snp, 32, snp, n1)
    return g.hypJacL2(alg, G, G.shape[1])


@pytest.mark.parametrize("alg", [9, 11, 3])
def test_c1_svd_256(built, alg):
    G = synth.svd_synth(256, 256, 1000, smin=1e-8)
    r = _svd(alg, G, 16)
    N = 256
    s, _, _, info, _ = lapack.dgesvj(G)
    assert info == 0
    D = np.sort(r.D)[::-1]
    assert np.all(np.abs(D - s ** 2) / s ** 2 <= 8 * N * EPS * s[0] / s)
    assert np.max(np.abs(D[:16] - s[:16] ** 2) / s[:16] ** 2) <= 8 * N * EPS
    assert np.max(np.abs(r.U.T @ r.U - np.eye(N))) <= 4 * N * EPS
    if alg & 2:
        assert np.max(np.abs(r.V.T @ r.V - np.eye(N))) <= 4 * N * EPS
        # G V = U diag(sqrt(D))
        assert np.max(np.abs(G @ r.V - r.U * np.sqrt(r.D))) <= 4 * N * EPS


def test_c2_svd_scaled(built):
    G = synth.gaussian(1024, 512, 1001)
    r = _svd(11, G, 32)
    N = 512
    s, _, _, info, _ = lapack.dgesvj(G, threads=8)
    D = np.sort(r.D)[::-1]
    assert np.max(np.abs(D - s ** 2) / s ** 2) <= 8 * N * EPS
    assert np.max(np.abs(r.U.T @ r.U - np.eye(N))) <= 4 * N * EPS
    assert np.max(np.abs(r.V.T @ r.V - np.eye(N))) <= 4 * N * EPS


@pytest.mark.parametrize("alg", [11, 9])
def test_c3_hsvd_scaled(built, alg):
    import gpujachx_b200 as g
    m, n, npl = 1024, 512, 256
    G = synth.graded(m, n, 1002)
    g.init_strats(None, "cycwor", 32, "cycwor", n // 16)
    r = g.hypJacL2(alg, G, npl)
    J = np.r_[np.ones(npl), -np.ones(n - npl)]
    R = np.linalg.qr(G, mode="r")
    lam = np.linalg.eigvalsh((R * J) @ R.T)
    D = np.sort(r.D)
    nrm = np.linalg.norm(R, 2) ** 2
    assert np.max(np.abs(D - lam)) <= 64 * n * EPS * nrm
    assert np.sum(r.D > 0) == npl and np.all(r.D[:npl] > 0) and np.all(r.D[npl:] < 0)
    assert np.max(np.abs(r.U.T @ r.U - np.eye(n))) <= 4 * n * EPS
    if alg & 2:
        kappa = np.max(np.abs(r.D)) / np.min(np.abs(r.D))
        VJV = (r.V.T * J) @ r.V
        assert np.max(np.abs(VJV - np.diag(J))) <= 4 * n * EPS * np.sqrt(kappa)
        assert np.max(np.abs(G @ r.V - r.U * np.sqrt(np.abs(r.D)))) <= 64 * n * EPS * np.sqrt(nrm)
