"""The accuracy post-processor (gpujachx_b200.accuracy, csrc/gjx_pp80.c):
each figure against a plain extended-precision restatement of the reference
tool's loops (var/pp80.f90), bit for bit on small inputs, and on real
decompositions from the oracle.  CPU only."""

import numpy as np
import pytest

from gpujachx_b200 import accuracy

L = np.longdouble


def _jorth_loops(X, trans, psum, pres):
    X = np.asarray(X, dtype=np.float64)
    if trans:
        X = X.T
    nk, nr = X.shape
    MM = np.zeros((nr, nr), dtype=L)
    for j in range(nr):
        s = L(-1) if j < pres else L(1)
        for k in range(psum):
            s = s + L(X[k, j]) * L(X[k, j])
        for k in range(psum, nk):
            s = s - L(X[k, j]) * L(X[k, j])
        MM[j, j] = abs(s)
        for i in range(j + 1, nr):
            t = L(0)
            for k in range(psum):
                t = t + L(X[k, j]) * L(X[k, i])
            for k in range(psum, nk):
                t = t - L(X[k, j]) * L(X[k, i])
            MM[i, j] = abs(t)
    qmax = L(0)
    for j in range(nr):
        for i in range(j, nr):
            if MM[i, j] > qmax:
                qmax = MM[i, j]
    diag, off = L(0), L(0)
    for j in range(nr):
        diag = diag + MM[j, j] * MM[j, j]
        for i in range(j + 1, nr):
            off = off + MM[i, j] * MM[i, j]
    return float(qmax), float(np.sqrt(L(2) * off + diag))


@pytest.mark.parametrize("trans", [False, True])
@pytest.mark.parametrize("signs", [None, 5])
def test_jorth_matches_loops_bitwise(built, trans, signs):
    rng = np.random.default_rng(7)
    X = rng.standard_normal((12, 8))
    X = np.linalg.qr(X)[0] + 1e-9 * rng.standard_normal((12, 8))
    if signs is None:
        nk, nr = (8, 12) if trans else (12, 8)
        ps, pr = nk, nr
    else:
        X = X[:8, :8]
        ps = pr = signs
    got = accuracy.jorth(X, trans=trans, psum=ps, pres=pr)
    ref = _jorth_loops(X, trans, ps, pr)
    assert got == ref


def test_jorth_of_orthogonal_and_j_orthogonal(built):
    rng = np.random.default_rng(1)
    Q = np.linalg.qr(rng.standard_normal((64, 64)))[0]
    mx, fro = accuracy.jorth(Q)
    assert mx < 1e-14 and fro < 1e-13
    # a J-orthogonal matrix: product of hyperbolic rotations mixing + and - rows
    p, n = 3, 6
    V = np.eye(n)
    for (a, b, th) in [(0, 4, 0.7), (2, 5, -1.3), (1, 3, 0.2)]:
        H = np.eye(n)
        H[a, a] = H[b, b] = np.cosh(th)
        H[a, b] = H[b, a] = np.sinh(th)
        V = V @ H
    mx, fro = accuracy.jorth(V, psum=p, pres=p)
    assert mx < 1e-14
    mx_t, _ = accuracy.jorth(V, trans=True, psum=p, pres=p)
    assert mx_t < 1e-14
    # and it is not orthogonal
    assert accuracy.jorth(V)[0] > 0.1


def test_resid_matches_loops_and_permutation(built):
    rng = np.random.default_rng(3)
    m, n = 7, 4
    A = rng.standard_normal((m, m))
    U = rng.standard_normal((m, n))
    D = rng.standard_normal(n)
    ipiv = np.array([3, 2, 7, 4], dtype=np.int32)
    got = accuracy.resid(A, U, D, ipiv)
    Uq = U.astype(L)
    for k in range(n - 1, -1, -1):
        kp = abs(int(ipiv[k])) - 1
        if kp != k:
            Uq[[k, kp], :] = Uq[[kp, k], :]
    R = np.zeros((m, n), dtype=L)
    for j in range(n):
        for i in range(m):
            v = Uq[i, j] * L(D[j])
            for k in range(m):
                v = v - L(A[i, k]) * Uq[k, j]
            R[i, j] = abs(v)
    mx = float(R.max())
    ss = L(0)
    for j in range(n):
        for i in range(m):
            ss = ss + R[i, j] * R[i, j]
    Rr = R.copy()
    for j in range(n):
        qj = np.sqrt(abs(L(D[j])))
        for i in range(n):
            Rr[i, j] = Rr[i, j] / (np.sqrt(abs(L(D[i]))) * qj)
    assert got == (mx, float(np.sqrt(ss)), float(Rr.max()))


def test_derr_sorted_and_signed(built):
    D = np.array([1.0, 4.0, 2.0, 3.0])
    lam = np.array([4.0 + 1e-12, 3.0, 2.0 - 4e-12, 1.0])
    ab, rel = accuracy.derr(D, lam)
    np.testing.assert_array_equal(ab[:4], np.array([4.0 + 1e-12, 3.0, 2.0 - 4e-12, 1.0]) - [4.0, 3.0, 2.0, 1.0])
    assert ab[4] == ab[2] < 0  # the extreme entry keeps its sign
    assert rel[4] == rel[2]


def test_pp80_on_oracle_decomposition(built):
    """A full SVD and an HSVD from the oracle: every figure at roundoff level."""
    from oracle import oracle
    from gpujachx_b200 import build, synth
    s0 = oracle.load_strat(build.STRAT, "cycwor", 32)
    s1 = oracle.load_strat(build.STRAT, "cycwor", 8)
    G = synth.make("svd_synth", 128, 128, 1000, smin=1e-6)
    r = oracle.hypjac_l2(11, G, 128, s0, s1)
    assert r["ret"] == 0
    sv = np.linalg.svd(G, compute_uv=False)
    A = G @ G.T
    out = accuracy.pp80(r["G"], r["D"], V=r["V"], nplus=128, A=A, lam=sv ** 2)
    nr = out["nrms"]
    assert max(nr[0], nr[2], nr[4], nr[6]) < 1e-13
    assert out["max_rel_err"] != 0 and abs(out["max_rel_err"]) < 1e-9
    # A = G G^T is formed in FP64, so its residual is at eps ||A|| absolutely;
    # relative to sqrt(D_i D_j) it grows as D_i shrinks (pp80's _R figure)
    assert nr[8] < 1e-13 * np.abs(A).max() and np.isfinite(nr[10])
    Gh = synth.make("graded", 256, 128, 1002)
    rh = oracle.hypjac_l2(11, Gh, 64, s0, s1)
    assert rh["ret"] == 0
    outh = accuracy.pp80(rh["G"], rh["D"], V=rh["V"], nplus=64, uut=False)
    assert outh["nrms"][0] < 1e-13
    # V^T J V - J at a scale set by the hyperbolic condition; finite and small
    assert outh["nrms"][4] < 1e-6
    assert "U^T U" in accuracy.report(outh)
