"""Shared fixtures.  Tests marked ``gpu`` need a B200; the rest run on CPU.

The CPU oracle (oracle/) is the checker here and only here (plus smoke() and
bench.py's CPU baseline); the product path never routes through it.
"""

import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def built():
    """libgjx.so, strat.so and the oracle, built if missing (nvcc cross-compiles)."""
    from gpujachx_b200 import build as B
    from oracle import oracle as O
    B.build_lib(verbose=False)
    B.build_strat(verbose=False)
    O.build()
    return dict(lib=B.LIB, strat=B.STRAT)


@pytest.fixture(scope="session")
def strat_path(built):
    return built["strat"]


@pytest.fixture(scope="session")
def oracle(built):
    from oracle import oracle as O
    return O


def load_golden(variant="base"):
    p = os.path.join(GOLDEN, f"ref_golden_{variant}.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)
