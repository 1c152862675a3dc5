"""The outer tables beyond the reference's largest order: rowcyc and colcyc of
orders 960 and 1024 (N = 15360 and 16384 columns), built by the reference's
doubling construction (strat/n2n/n2n.sh.cpp) from its tables of orders 480
and 512 (gpujachx_b200/strat_gen.py).

The construction is pinned on the reference's own tables: every shipped table
of order 2n <= 896 whose half the reference also ships is the doubling of that
half, entry for entry.  The added tables are that doubling too, load through
init_strats and pass the loader's validator.
"""

import numpy as np
import pytest

from gpujachx_b200 import strat_gen


def _load(oracle, strat_path, fam, n):
    return oracle.load_strat(strat_path, fam, n).astype(np.int64)


@pytest.mark.parametrize("fam", strat_gen.FAMILIES)
def test_doubling_reproduces_every_shipped_table(fam, oracle, strat_path):
    matched = 0
    for n in range(2, 449, 2):
        try:
            half, full = _load(oracle, strat_path, fam, n), _load(oracle, strat_path, fam, 2 * n)
        except Exception:
            continue  # an order the reference does not ship
        assert np.array_equal(strat_gen.double_table(half, fam), full), (fam, n)
        matched += 1
    assert matched >= 50  # rowcyc 58, colcyc 54 pairs of orders


@pytest.mark.parametrize("fam", strat_gen.FAMILIES)
@pytest.mark.parametrize("n", strat_gen.ORDERS)
def test_added_tables_are_the_doubling(fam, n, oracle, strat_path):
    got = _load(oracle, strat_path, fam, n)
    assert got.shape == (n - 1, n // 2, 2)
    assert np.array_equal(got, strat_gen.double_table(_load(oracle, strat_path, fam, n // 2), fam))


@pytest.mark.parametrize("fam", strat_gen.FAMILIES)
@pytest.mark.parametrize("n", strat_gen.ORDERS)
def test_added_tables_load_and_validate(fam, n, built):
    import gpujachx_b200 as g
    g.init_strats(None, "cycwor", 32, fam, n)
    info = g.strat_info()
    assert (info["steps1"], info["pairs1"]) == (n - 1, n // 2)
    v = g.validate_loaded()
    assert v["code"] == 0 and v["strat1"]["missing"] == 0 and v["strat1"]["repeats"] == 0
    t = g.strat1_table().astype(np.int64)
    pairs = set(map(tuple, t.reshape(-1, 2).tolist()))
    assert len(pairs) == n * (n - 1) // 2


def test_c_source_round_trip():
    t = strat_gen.double_table(strat_gen.double_table(np.array([[[0, 1]]]), "rowcyc"), "colcyc")
    src = strat_gen.c_source("colcyc", 8, t)
    assert src.count("{") == 1 + t.shape[0] + t.shape[0] * t.shape[1]
    back = strat_gen.parse_header(src, 8)
    assert np.array_equal(back, t)
