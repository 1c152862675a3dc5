"""The largest orders: the outer tables of 960 and 1024 blocks (N = 15360 and
16384 columns) that the build adds by the reference's doubling construction
(gpujachx_b200/strat_gen.py) load onto the GPU and drive every step of a
sweep.  The input has orthogonal columns (G = diag(s), 2 GB), so the first
sweep rotates nothing and the decomposition ends after it: D = s^2 exactly
(each column's squared norm is the square of its one nonzero) and U = I to
an ulp."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fam,n", [("rowcyc", 16384), ("colcyc", 15360)])
def test_orthogonal_input_at_the_largest_orders(built, fam, n):
    import torch
    import gpujachx_b200 as g
    g.init_strats(None, "cycwor", 32, fam, n // 16)
    s = torch.logspace(0, -6, n, dtype=torch.float64, device="cuda")
    G = torch.diag(s)  # column-major view of diag(s) is diag(s)
    D = torch.empty(n, dtype=torch.float64, device="cuda")
    ret, sweeps, rot_s, rot_b = g.hypJacL2_dev(9, G, n, None, D)
    assert ret == 0 and sweeps == 1 and rot_b == 0
    assert torch.equal(D, s * s)
    assert torch.allclose(G, torch.eye(n, dtype=torch.float64, device="cuda"), rtol=0.0, atol=4e-16)
    del G
    torch.cuda.empty_cache()
