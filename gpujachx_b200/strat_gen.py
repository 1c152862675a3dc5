"""Outer strategy tables beyond the reference's largest order (896 blocks,
N = 14336 columns): the rowcyc and colcyc tables of orders 960 and 1024
(N = 15360 and 16384), built by the reference's own doubling construction
(strat/n2n/n2n.sh.cpp:41-129) from its tables of orders 480 and 512.

The construction, for an order-n table T of n-1 parallel steps of n/2
disjoint pairs, gives the order-2n table:
  * step 0: the pairs (2k, 2k+1), k < n;
  * each step s of T becomes steps 2s+1 and 2s+2; its a-th pair (i, j) gives
    pairs 2a and 2a+1 of them: (2i, 2j), (2i+1, 2j+1) in the first;
    (2i, 2j+1), (2i+1, 2j) (rowcyc) or (2i+1, 2j), (2i, 2j+1) (colcyc) in
    the second.
Every pair of blocks meets once per sweep and each step is a perfect
matching, as in T.  The reference's tables of every order 2n <= 896 whose
half it also ships are this doubling of it (all 112 of them;
tests/test_strat_doubling.py checks it against the tables in strat.so).

Used by build.build_strat; the generated tables get the reference's symbol
names (rowcyc00960, ...) and element type (unsigned short above 256).
"""

from __future__ import annotations

import re

import numpy as np

FAMILIES = ("rowcyc", "colcyc")
ORDERS = (960, 1024)


def parse_header(text: str, n: int) -> np.ndarray:
    """The table of a reference header (``... name[S][n/2][2] = {{{i, j}, ...}, ...};``)."""
    body = text[text.index("=") + 1:]
    v = np.array([int(x) for x in re.findall(r"\d+", body)], dtype=np.int64)
    if v.size % n:
        raise ValueError(f"table of order {n}: {v.size} entries")
    return v.reshape(v.size // n, n // 2, 2)


def double_table(t: np.ndarray, family: str) -> np.ndarray:
    """The order-2n table of the doubling construction from the order-n table t."""
    if family not in FAMILIES:
        raise ValueError(f"no doubling rule for {family}")
    steps, half, _ = t.shape
    n = 2 * half
    out = np.zeros((2 * steps + 1, n, 2), dtype=np.int64)
    out[0, :, 0] = 2 * np.arange(n)
    out[0, :, 1] = 2 * np.arange(n) + 1
    i, j = t[:, :, 0], t[:, :, 1]
    first, second = out[1::2], out[2::2]
    first[:, 0::2, 0], first[:, 0::2, 1] = 2 * i, 2 * j
    first[:, 1::2, 0], first[:, 1::2, 1] = 2 * i + 1, 2 * j + 1
    if family == "rowcyc":
        second[:, 0::2, 0], second[:, 0::2, 1] = 2 * i, 2 * j + 1
        second[:, 1::2, 0], second[:, 1::2, 1] = 2 * i + 1, 2 * j
    else:
        second[:, 0::2, 0], second[:, 0::2, 1] = 2 * i + 1, 2 * j
        second[:, 1::2, 0], second[:, 1::2, 1] = 2 * i, 2 * j + 1
    return out


def c_source(family: str, n: int, t: np.ndarray) -> str:
    """A C definition of the table with the reference's symbol name and type."""
    typ = "unsigned char" if n <= 256 else "unsigned short"
    rows = []
    for step in t:
        rows.append("{" + ",".join("{%d,%d}" % (int(a), int(b)) for a, b in step) + "}")
    return ('__attribute__((visibility("default"))) %s %s%05u[%u][%u][2] = {\n%s\n};\n'
            % (typ, family, n, t.shape[0], t.shape[1], ",\n".join(rows)))


def extension_sources(strat_dir: str) -> dict[str, str]:
    """{file name: C source} of the tables to add to strat.so: each family's
    orders in ORDERS that strat_dir lacks and whose half it has."""
    import os
    out = {}
    for fam in FAMILIES:
        for n in ORDERS:
            full = os.path.join(strat_dir, fam, "%05u.h" % n)
            half = os.path.join(strat_dir, fam, "%05u.h" % (n // 2))
            if os.path.exists(full) or not os.path.exists(half):
                continue
            with open(half) as f:
                t = parse_header(f.read(), n // 2)
            out["%s%05u.c" % (fam, n)] = c_source(fam, n, double_table(t, fam))
    return out
