"""The reference's alternative builds on the GPU: with gjx_set_variant(1) the
pivot-block factor is the -DUSE_QR build's (Householder QR of 32-row chunks
merged by Givens rotations), with 2 the -DUSE_DRMAC build's (that factor and
Drmac's scaled-norm sweep in the definite sorting kernels).  Every recorded
output of those builds (tests/golden/ref_golden_qr.json, ref_golden_drmac.json:
the same 54 inputs as the default build's fixture) must be reproduced bit for
bit through hypJacL2, and the device and allocation-free entry points must
agree with it.  The oracle's restatement of both builds is checked against
the same fixtures on the CPU (tests/test_oracle_golden.py)."""

import numpy as np
import pytest

from conftest import load_golden
from gpujachx_b200 import synth
from tests.golden.make_golden import make_input

pytestmark = pytest.mark.gpu

CASES = [(v, c) for v in ("qr", "drmac") for c in (load_golden(v) or {"cases": []})["cases"]]


@pytest.fixture
def variant():
    import gpujachx_b200 as g
    yield g.set_variant
    g.set_variant("base")


@pytest.mark.parametrize("v,c", CASES, ids=[f"{v}-{c['name']}" for v, c in CASES])
def test_variant_build_equals_reference(v, c, built, variant):
    import gpujachx_b200 as g
    variant(v)
    G = make_input(c)
    assert synth.digest(G) == c["input_sha"]
    g.init_strats(None, c["snp0"], 32, c["snp1"], c["n"] // 16)
    r = g.hypJacL2(c["alg"], G, c["nplus"])
    o = c["out"]
    assert (r.sweeps, r.rot_s, r.rot_b) == (o["sweeps"], o["rot_s"], o["rot_b"])
    assert [float(x).hex() for x in r.D] == o["D"]
    assert synth.digest(r.U) == o["U_sha"]
    if c["alg"] & 2:
        assert synth.digest(r.V) == o["V_sha"]


def test_variant_device_entry_point_and_batched_refusal(built, variant):
    import torch
    import gpujachx_b200 as g
    c = next(c for v, c in CASES if v == "drmac" and c["alg"] == 11 and c["n"] >= 256)
    variant("drmac")
    G = make_input(c)
    g.init_strats(None, c["snp0"], 32, c["snp1"], c["n"] // 16)
    r = g.hypJacL2(c["alg"], G, c["nplus"])
    m, n = G.shape
    dG = torch.tensor(np.ascontiguousarray(G.T), dtype=torch.float64, device="cuda")
    dV = torch.empty((n, n), dtype=torch.float64, device="cuda")
    dD = torch.empty(n, dtype=torch.float64, device="cuda")
    ret, sw, s, b = g.hypJacL2_dev(c["alg"], dG, c["nplus"], dV, dD)
    assert (sw, s, b) == (r.sweeps, r.rot_s, r.rot_b)
    assert np.array_equal(dG.cpu().numpy().T.view(np.uint64), r.U.view(np.uint64))
    with pytest.raises(g.GjxError):
        g.hypJacL2_batched(c["alg"], [dG], [c["nplus"]], Vs=[dV], Ds=[dD])
