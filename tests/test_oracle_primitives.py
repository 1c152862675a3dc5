"""CPU checks of the oracle's primitives against exact arithmetic.

The oracle must reproduce the reference's arithmetic bit for bit; these tests
pin the pieces whose result is defined mathematically: the correctly rounded
1/sqrt (share/device_code_common.hpp:89-133 is correctly rounded; so must be
ours), the constants of share/HypJacL.hpp:21-59, the butterfly order of
share/device_code_common_Kepler.hpp:26-74 and the rotation formulas of
share/device_code_common_rotate.hpp:16-64.
"""

import math
import struct
from fractions import Fraction

import numpy as np
import pytest


def _next(x, d):
    return np.nextafter(x, d)


def _is_rn_rsqrt(a: float, r: float) -> bool:
    """r is the double nearest to 1/sqrt(a) (exact rational test of both midpoints)."""
    A = Fraction(a)
    lo = Fraction(r) - (Fraction(r) - Fraction(_next(r, 0.0))) / 2
    hi = Fraction(r) + (Fraction(_next(r, math.inf)) - Fraction(r)) / 2
    # lo < 1/sqrt(A) < hi  <=>  lo^2 A < 1 < hi^2 A   (all positive)
    return lo * lo * A < 1 < hi * hi * A


def test_rsqrt_correctly_rounded(oracle):
    rng = np.random.default_rng(7)
    xs = list(rng.uniform(1.0, 4.0, 3000)) + list(np.exp(rng.uniform(-700, 700, 3000)))
    xs += [1.0, 2.0, 4.0, 0.25, 3.0, 1 + 2 ** -52, 4 - 2 ** -50, 2 - 2 ** -52, 5e-324, 2.2250738585072014e-308,
           1.7976931348623157e308, 1e-300, 7.0, 1e10]
    xs += [float(t) * float(t) for t in rng.uniform(0.5, 2.0, 500)]       # near-exact squares
    xs += [1.0 + float(t) * 2 ** -40 for t in rng.integers(1, 2 ** 12, 500)]  # just above 1
    bad = [x for x in xs if not _is_rn_rsqrt(x, oracle.rsqrt_rn(x))]
    assert not bad, bad[:5]


def test_rsqrt_specials(oracle):
    assert oracle.rsqrt_rn(0.0) == math.inf
    assert oracle.rsqrt_rn(-0.0) == -math.inf
    assert math.isnan(oracle.rsqrt_rn(-1.0))
    assert oracle.rsqrt_rn(math.inf) == 0.0
    assert math.isnan(oracle.rsqrt_rn(math.nan))
    assert oracle.rsqrt_rn(4.0) == 0.5 and oracle.rsqrt_rn(0.25) == 2.0


def test_constants_match_reference_literals():
    # share/HypJacL.hpp:21-59: SQRT_HEPS, SQRT_2_HEPS, HYPJAC_MYTOL, HYPJAC_COSHI_FIX
    ref = {"SQRT_HEPS": 1.05367121277235087E-08, "SQRT_2_HEPS": 1.34217728000000000E+08,
           "MYTOL": 6.28036983473510067E-16, "COSHI": 1.15470053837925146}
    ours = {"SQRT_HEPS": float.fromhex("0x1.6a09e667f3bcdp-27"), "SQRT_2_HEPS": float.fromhex("0x1.0p+27"),
            "MYTOL": float.fromhex("0x1.6a09e667f3bcdp-51"), "COSHI": float.fromhex("0x1.279a74590331cp+0")}
    for k in ref:
        assert struct.pack("<d", ref[k]) == struct.pack("<d", ours[k]), k
    assert ours["SQRT_HEPS"] == math.sqrt(2.0 ** -53)
    assert ours["MYTOL"] == math.sqrt(32.0) * 2.0 ** -53


def test_sum32_butterfly_order(oracle):
    rng = np.random.default_rng(3)
    for _ in range(200):
        v = rng.standard_normal(32) * 10.0 ** rng.uniform(-8, 8, 32)
        t = list(v)
        for k in (16, 8, 4, 2, 1):
            for i in range(k):
                t[i] = t[i] + t[i + k]
        assert oracle.sum32(v) == t[0]


def test_rotations(oracle):
    rng = np.random.default_rng(5)
    for _ in range(2000):
        dp, dq = rng.uniform(0.1, 10, 2)
        apq = rng.uniform(-1, 1) * math.sqrt(dp * dq) * 0.9
        big, c, t = oracle.rotT(apq, dp, dq)
        # [c, -c t; c t, c] zeroes the off-diagonal of [[dp, apq], [apq, dq]] (to rounding)
        s = c * t
        off = (c * c - s * s) * apq + c * s * (dp - dq)
        assert abs(off) < 1e-12 * (dp + dq)
        assert big == (c < 1.0)
    # hyperbolic: |tanh| < 1, cosh >= 1
    for _ in range(2000):
        dp, dq = rng.uniform(0.1, 10, 2)
        apq = rng.uniform(-1, 1) * 0.99 * (dp + dq) / 2
        big, c, t = oracle.rotH(apq, dp, dq)
        assert abs(t) < 1.0 and c >= 1.0
