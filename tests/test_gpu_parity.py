"""Parity of the CUDA path (through the C ABI) with the reference and the oracle.

* golden: the reference's own outputs (tests/golden/ref_golden_base.json) must
  be reproduced bit for bit by hypJacL2 -- U, V, D, sweeps, rotation counts;
* oracle: further seeded cases, compared bit for bit with the CPU oracle;
* device API: gjx_hypJacL2_dev on torch tensors equals hypJacL2;
* primitives: the device rsqrt_rn equals the oracle's on many inputs.
"""

import ctypes

import numpy as np
import pytest

from conftest import load_golden
from gpujachx_b200 import synth
from tests.golden.make_golden import make_input, case

pytestmark = pytest.mark.gpu

GOLD = load_golden("base")
CASES = GOLD["cases"] if GOLD else []


def _run(g, c, G):
    g.init_strats(None, c["snp0"], 32, c["snp1"], c["n"] // 16)
    return g.hypJacL2(c["alg"], G, c["nplus"])


@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
def test_cuda_equals_reference(c, built):
    import gpujachx_b200 as g
    G = make_input(c)
    assert synth.digest(G) == c["input_sha"]
    r = _run(g, c, G)
    o = c["out"]
    assert (r.sweeps, r.rot_s, r.rot_b) == (o["sweeps"], o["rot_s"], o["rot_b"])
    assert [float(x).hex() for x in r.D] == o["D"]
    assert synth.digest(r.U) == o["U_sha"]
    if c["alg"] & 2:
        assert synth.digest(r.V) == o["V_sha"]


EXTRA = [
    case("x_2048x256_alg11", 2048, 256, 256, 11, seed=101),
    case("x_2048x256_np77_alg3", 2048, 256, 77, 3, seed=102),
    case("x_640x320_alg8", 640, 320, 320, 8, seed=103, snp0="rowcyc", snp1="colcyc"),
    case("x_576x288_alg2", 576, 288, 288, 2, seed=104),
    case("x_4096x64_alg11", 4096, 64, 64, 11, gen="graded", seed=105),
    case("x_320x320_alg1_neg", 320, 320, 0, 1, seed=106),
    case("x_1024x1024_alg11", 1024, 1024, 1024, 11, gen="svd_synth", seed=107, smin=1e-10),
]


@pytest.mark.parametrize("c", EXTRA, ids=[c["name"] for c in EXTRA])
def test_cuda_equals_oracle(c, built, oracle, strat_path):
    import gpujachx_b200 as g
    G = make_input(c)
    r = _run(g, c, G)
    s0 = oracle.load_strat(strat_path, c["snp0"], 32)
    s1 = oracle.load_strat(strat_path, c["snp1"], c["n"] // 16)
    o = oracle.hypjac_l2(c["alg"], G, c["nplus"], s0, s1)
    assert (r.sweeps, r.rot_s, r.rot_b) == (o["sweeps"], o["rot_s"], o["rot_b"])
    assert np.array_equal(r.D.view(np.uint64), o["D"].view(np.uint64))
    assert np.array_equal(r.U.view(np.uint64), o["G"].view(np.uint64))
    if c["alg"] & 2:
        assert np.array_equal(r.V.view(np.uint64), o["V"].view(np.uint64))


def test_device_api_equals_host_api(built):
    import torch
    import gpujachx_b200 as g
    c = case("dev_1024x512", 1024, 512, 512, 11, seed=201)
    G = make_input(c)
    r = _run(g, c, G)
    dG = torch.tensor(np.ascontiguousarray(G.T), dtype=torch.float64, device="cuda")
    dV = torch.empty((512, 512), dtype=torch.float64, device="cuda")
    dD = torch.empty(512, dtype=torch.float64, device="cuda")
    ret, swp, s, b = g.hypJacL2_dev(11, dG, 512, dV, dD)
    assert ret == 0 and (swp, s, b) == (r.sweeps, r.rot_s, r.rot_b)
    assert np.array_equal(dG.cpu().numpy().T.view(np.uint64), r.U.view(np.uint64))
    assert np.array_equal(dV.cpu().numpy().T.view(np.uint64), r.V.view(np.uint64))
    assert np.array_equal(dD.cpu().numpy().view(np.uint64), r.D.view(np.uint64))
    # padded leading dimension (lddG = nrow + 64), on a side stream
    dG2 = torch.zeros((512, 1024 + 64), dtype=torch.float64, device="cuda")
    dG2[:, :1024] = torch.tensor(np.ascontiguousarray(G.T), device="cuda")
    st = torch.cuda.Stream()
    ret, swp2, _, _ = g.hypJacL2_dev(11, dG2, 512, dV, dD, stream=st, nrow=1024)
    assert ret == 0 and swp2 == r.sweeps
    assert np.array_equal(dG2[:, :1024].cpu().numpy().T.view(np.uint64), r.U.view(np.uint64))
    assert torch.count_nonzero(dG2[:, 1024:]).item() == 0


def test_rsqrt_device_equals_oracle(built, oracle):
    import torch
    import gpujachx_b200 as g
    rng = np.random.default_rng(9)
    xs = np.concatenate([rng.uniform(1, 4, 20000), np.exp(rng.uniform(-740, 709, 20000)),
                         np.array([1.0, 2.0, 4.0, 5e-324, 1e-310, 2.2250738585072014e-308, 1.7976931348623157e308,
                                   1 + 2 ** -52, 4 - 2 ** -50])])
    din = torch.tensor(xs, dtype=torch.float64, device="cuda")
    dout = torch.empty_like(din)
    assert g.lib().gjx_rsqrt_rn_dev(din.data_ptr(), dout.data_ptr(), len(xs)) == 0
    got = dout.cpu().numpy()
    want = np.array([oracle.rsqrt_rn(float(x)) for x in xs])
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
    sp = torch.tensor([0.0, -0.0, -1.0, float("inf")], dtype=torch.float64, device="cuda")
    so = torch.empty_like(sp)
    assert g.lib().gjx_rsqrt_rn_dev(sp.data_ptr(), so.data_ptr(), 4) == 0
    v = so.cpu().numpy()
    assert v[0] == np.inf and v[1] == -np.inf and np.isnan(v[2]) and v[3] == 0.0


def test_rsqrt_device_bit_patterns(built, oracle):
    """400 K inputs from raw bit patterns: every exponent of the normal range
    with random mantissas, the powers of 2 and 4 with their neighbours (the
    powers of 4 are the fast path's hand-off case), random subnormals; all
    correctly rounded, equal to the oracle's."""
    import torch
    import gpujachx_b200 as g
    rng = np.random.default_rng(10)
    expo = rng.integers(1, 2047, 300000, dtype=np.uint64)
    mant = rng.integers(0, 2 ** 52, 300000, dtype=np.uint64)
    normal = ((expo << np.uint64(52)) | mant).view(np.float64)
    p2 = np.ldexp(1.0, np.arange(-1022, 1024))
    near = np.concatenate([np.nextafter(p2, 0), p2, np.nextafter(p2, np.inf)])
    sub = (rng.integers(1, 2 ** 52, 50000, dtype=np.uint64)).view(np.float64)
    xs = np.concatenate([normal, near, sub])
    xs = xs[np.isfinite(xs) & (xs > 0)]
    din = torch.tensor(xs, dtype=torch.float64, device="cuda")
    dout = torch.empty_like(din)
    assert g.lib().gjx_rsqrt_rn_dev(din.data_ptr(), dout.data_ptr(), len(xs)) == 0
    got = dout.cpu().numpy()
    want = np.array([oracle.rsqrt_rn(float(x)) for x in xs])
    bad = np.nonzero(got.view(np.uint64) != want.view(np.uint64))[0]
    assert bad.size == 0, (xs[bad[:5]], got[bad[:5]], want[bad[:5]])


def test_second_call_reuses_cache(built):
    import gpujachx_b200 as g
    c = case("cache", 256, 128, 128, 9, seed=301)
    G = make_input(c)
    a = _run(g, c, G)
    b = _run(g, c, G)
    assert np.array_equal(a.U.view(np.uint64), b.U.view(np.uint64)) and a.sweeps == b.sweeps
    assert g.lib().gjx_release_cache() == 0
    c2 = _run(g, c, G)
    assert np.array_equal(a.D.view(np.uint64), c2.D.view(np.uint64))
