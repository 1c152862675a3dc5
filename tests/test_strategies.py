"""CPU checks of the strategy tables and of the loader (share/HypJacL.cu:11-121).

Every table of strat.so must be a valid parallel ordering (disjoint pairs in
each step, p < q, complete coverage); the product loader (gjx_init_strats)
must read exactly what the oracle's restatement of the reference loader reads.
"""

import ctypes
import itertools

import numpy as np
import pytest

FAMILIES = ("mmstep", "BrentL", "colcyc", "cycloc", "rowcyc", "cycwor")


def _orders(strat_path):
    lib = ctypes.CDLL(strat_path)
    out = []
    for fam in FAMILIES:
        for n in range(2, 1025, 2):
            try:
                getattr(lib, "%s%05d" % (fam, n))
            except AttributeError:
                continue
            out.append((fam, n))
    return out


def test_table_count(strat_path):
    o = _orders(strat_path)
    # every shipped header (orders up to 896), and the rowcyc / colcyc tables
    # of orders 960 and 1024 that the build adds by the doubling construction
    assert len(o) == 325 + 4
    assert max(n for _, n in o) == 1024
    assert sorted(x for x in o if x[1] > 896) == [("colcyc", 960), ("colcyc", 1024), ("rowcyc", 960),
                                                  ("rowcyc", 1024)]


def test_every_table_is_a_parallel_ordering(strat_path, oracle):
    for fam, n in _orders(strat_path):
        t = oracle.load_strat(strat_path, fam, n).astype(np.int64)
        steps = t.shape[0]
        assert steps == (n if fam == "mmstep" else n - 1), (fam, n)
        assert np.all(t[..., 0] < t[..., 1]), (fam, n)
        assert t.max() < n
        for s in range(steps):
            flat = t[s].ravel()
            assert len(np.unique(flat)) == n, (fam, n, s)  # disjoint, all indices
        pairs = set(map(tuple, t.reshape(-1, 2).tolist()))
        assert len(pairs) == n * (n - 1) // 2, (fam, n)  # every pair at least once


def test_product_loader_matches_oracle(built, oracle):
    import gpujachx_b200 as g
    for fam, n1 in [("cycwor", 16), ("cycwor", 512), ("rowcyc", 24), ("colcyc", 896), ("BrentL", 64),
                    ("cycloc", 256), ("mmstep", 288)]:
        g.init_strats(built["strat"], "cycwor", 32, fam, n1)
        ours = g.strat1_table()
        ref = oracle.load_strat(built["strat"], fam, n1)
        assert ours.dtype == np.uint16 and np.array_equal(ours, ref), (fam, n1)
        info = g.strat_info()
        assert info["steps1"] == ref.shape[0] and info["pairs1"] == n1 // 2
        assert info["strat0"] == 6 and info["steps0"] == 31


def test_strategy_ids(built):
    import gpujachx_b200 as g
    ids = {"mmstep": 1, "BrentL": 2, "colcyc": 3, "cycloc": 4, "rowcyc": 5, "cycwor": 6}
    for fam, i in ids.items():
        g.init_strats(built["strat"], fam, 32, fam, 16)
        info = g.strat_info()
        assert info["strat0"] == i and info["strat1"] == i
        assert info["steps0"] == (32 if fam == "mmstep" else 31)


def test_validator_accepts_every_shipped_table(built):
    """gjx_validate_pairs on all tables (up to n1 = 1024): perfect matchings,
    full coverage; repeats only in mmstep (n/2 pairs twice, n steps)."""
    import re
    import subprocess
    import gpujachx_b200 as g
    from oracle import oracle
    syms = subprocess.run(["nm", "-D", "--defined-only", built["strat"]], capture_output=True, text=True).stdout.split()
    names = sorted({s for s in syms if re.fullmatch(r"[A-Za-z]+\d{5}", s)})
    assert len(names) == 325 + 4  # and the added rowcyc / colcyc of orders 960, 1024
    for nm in names:
        fam, n = nm[:-5], int(nm[-5:])
        t = oracle.load_strat(built["strat"], fam, n)
        r = g.validate_pairs(t)
        assert r["code"] == 0 and r["missing"] == 0, nm
        assert r["repeats"] == (n // 2 if fam == "mmstep" else 0), nm
    g.init_strats(None, "BrentL", 32, "mmstep", 64)
    v = g.validate_loaded()
    assert v["code"] == 0 and v["strat1"]["repeats"] == 32


def test_validator_rejects_broken_tables(built):
    import gpujachx_b200 as g
    from oracle import oracle
    t = oracle.load_strat(built["strat"], "cycwor", 16).copy()
    bad = t.copy()
    bad[3, 2, 1] = bad[3, 2, 0]          # p == q
    assert g.validate_pairs(bad)["code"] == 1
    bad = t.copy()
    bad[5, 1, 0] = bad[5, 0, 0]          # an index twice in step 5
    r = g.validate_pairs(bad)
    assert r["code"] == 2 and r["bad_step"] == 5
    r = g.validate_pairs(t[:-1])         # drop the last step: its 8 pairs are missing
    assert r["code"] == 3 and r["missing"] == 8
    bad = t.copy()
    bad[0, 0, 0] = 16                    # out of range
    assert g.validate_pairs(bad)["code"] == 1
