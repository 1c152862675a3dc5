"""The oracle against the reference itself (CPU).

tests/golden/ref_golden_base.json holds the outputs of the reference's own
hypJacL2 (its sources built for sm_100a, run on a B200 by
tests/golden/make_golden.py) on seeded inputs; ref_golden_qr.json and
ref_golden_drmac.json those of its -DUSE_QR and -DUSE_DRMAC builds on the
same inputs.  The oracle (in the matching variant) must reproduce every one
bit for bit: U, V, D, the sweep count and both rotation counts.
"""

import numpy as np
import pytest

from conftest import load_golden
from gpujachx_b200 import synth
from tests.golden.make_golden import make_input

GOLD = load_golden("base")
CASES = GOLD["cases"] if GOLD else []
VARIANT_CASES = [(v, c) for v in ("qr", "drmac") for c in (load_golden(v) or {"cases": []})["cases"]]


def test_golden_present():
    assert GOLD is not None, "tests/golden/ref_golden_base.json missing"
    assert len(CASES) >= 40


@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
def test_oracle_equals_reference(c, oracle, strat_path):
    oracle.set_variant("base")
    _check(c, oracle, strat_path)


def test_variant_goldens_present():
    assert len(VARIANT_CASES) == 2 * len(CASES)


@pytest.mark.parametrize("v,c", VARIANT_CASES, ids=[f"{v}-{c['name']}" for v, c in VARIANT_CASES])
def test_oracle_equals_reference_variant_builds(v, c, oracle, strat_path):
    oracle.set_variant(v)
    try:
        _check(c, oracle, strat_path)
    finally:
        oracle.set_variant("base")


def _check(c, oracle, strat_path):
    G = make_input(c)
    assert synth.digest(G) == c["input_sha"], "input generator drifted"
    s0 = oracle.load_strat(strat_path, c["snp0"], 32)
    s1 = oracle.load_strat(strat_path, c["snp1"], c["n"] // 16)
    r = oracle.hypjac_l2(c["alg"], G, c["nplus"], s0, s1)
    o = c["out"]
    assert r["ret"] == o["ret"] == 0
    assert (r["sweeps"], r["rot_s"], r["rot_b"]) == (o["sweeps"], o["rot_s"], o["rot_b"])
    assert [float(x).hex() for x in r["D"]] == o["D"]
    assert synth.digest(r["D"]) == o["D_sha"]
    assert synth.digest(r["G"]) == o["U_sha"]
    if c["alg"] & 2:
        assert synth.digest(r["V"]) == o["V_sha"]
