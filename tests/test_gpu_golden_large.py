"""Bit-for-bit parity with the reference at the benchmark sizes.

tests/golden/ref_golden_large.json holds what the reference's own hypJacL2
(built for sm_100a, oracle/_ref/ref_harness) gave on a B200 for:
the 8192 x 8192 configuration (G = Q1 diag(s) Q2^T, s from 1 to 1e-12, ALG 11;
it stops at the 30-sweep cap), the 4096 x 2048 and 2048 x 1024 (hyperbolic)
configurations, the 256 x 256 one with a mixed signature, and one SVD
(NPLUS = n) and one HSVD (NPLUS = n/2) matrix of every batch size
n = 64 ... 512 -- digests of U, V and D, the sweep and rotation counts.
Each input is regenerated and checked against its recorded digest first.
The batch-size matrices are also run together through the batched form.
"""

import json
import os

import numpy as np
import pytest

from gpujachx_b200 import synth
from tests.golden.make_golden import make_input

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "ref_golden_large.json")) as _f:
    LARGE = json.load(_f)["cases"]
SINGLE = [c for c in LARGE if not c["name"].startswith("c5_")]
BATCH = [c for c in LARGE if c["name"].startswith("c5_")]


def _check(c, U, V, D, sweeps, rot_s, rot_b):
    o = c["out"]
    assert (sweeps, rot_s, rot_b) == (o["sweeps"], o["rot_s"], o["rot_b"]), c["name"]
    assert synth.digest(D) == o["D_sha"], c["name"]
    assert synth.digest(U) == o["U_sha"], c["name"]
    if c["alg"] & 2:
        assert synth.digest(V) == o["V_sha"], c["name"]


@pytest.mark.parametrize("c", SINGLE, ids=[c["name"] for c in SINGLE])
def test_single_matrix_equals_reference_record(c, built):
    import gpujachx_b200 as g
    G = make_input(c)
    assert synth.digest(G) == c["input_sha"], "input generator changed"
    g.init_strats(None, c["snp0"], 32, c["snp1"], c["n"] // 16)
    r = g.hypJacL2(c["alg"], G, c["nplus"])
    _check(c, r.U, r.V, r.D, r.sweeps, r.rot_s, r.rot_b)


def test_batch_sizes_equal_reference_record_single_and_batched(built):
    import torch
    import gpujachx_b200 as g
    Gs = []
    for c in BATCH:
        G = make_input(c)
        assert synth.digest(G) == c["input_sha"], c["name"]
        Gs.append(G)
    # one at a time through the host entry point
    for c, G in zip(BATCH, Gs):
        g.init_strats(None, "cycwor", 32, "cycwor", c["n"] // 16)
        r = g.hypJacL2(c["alg"], G, c["nplus"])
        _check(c, r.U, r.V, r.D, r.sweeps, r.rot_s, r.rot_b)
    # all together through the batched form (both widths of its CTAs)
    for width in (2, 1):
        g.lib().gjx_set_pairs_per_cta(width)
        g.init_strats(None, "cycwor", 32, "cycwor", 4)
        dG = [torch.tensor(np.ascontiguousarray(G.T), dtype=torch.float64, device="cuda") for G in Gs]
        dV = [torch.zeros((c["n"], c["n"]), dtype=torch.float64, device="cuda") for c in BATCH]
        dD = [torch.zeros(c["n"], dtype=torch.float64, device="cuda") for c in BATCH]
        res = g.hypJacL2_batched(11, dG, [c["nplus"] for c in BATCH], Vs=dV, Ds=dD)
        g.lib().gjx_set_pairs_per_cta(0)
        assert res.info == [0] * len(BATCH)
        for k, c in enumerate(BATCH):
            _check(c, dG[k].cpu().numpy().T, dV[k].cpu().numpy().T, dD[k].cpu().numpy(), res.sweeps[k],
                   res.rot_s[k], res.rot_b[k])
