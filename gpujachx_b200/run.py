"""One decomposition of a seeded synthetic matrix, from the command line.

    python -m gpujachx_b200.run [--m M] [--n N] [--nplus P] [--alg A]
                                [--gen gaussian|svd_synth|graded] [--seed S]
                                [--form plain|split] [--variant base|qr|drmac]

Runs gjx_hypJacL2_dev (plain form) or gjx_hypJacL2_split on cuda:0 with the
cycwor tables of the shape and prints the sweeps, rotation counts and the
wall time of the call: the command the profiles of single decompositions use.
"""

from __future__ import annotations

import argparse
import time

import numpy as np


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--m", type=int, default=4096)
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--nplus", type=int, default=-1, help="default: n (an SVD)")
    ap.add_argument("--alg", type=int, default=11)
    ap.add_argument("--gen", default="gaussian", choices=["gaussian", "svd_synth", "graded"])
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--form", default="plain", choices=["plain", "split"])
    ap.add_argument("--variant", default="base", choices=["base", "qr", "drmac"])
    a = ap.parse_args()
    import torch
    import gpujachx_b200 as g
    from gpujachx_b200 import synth
    nplus = a.n if a.nplus < 0 else a.nplus
    G = synth.make(a.gen, a.m, a.n, a.seed)
    g.init_strats(None, "cycwor", 32, "cycwor", a.n // 16)
    g.set_variant(a.variant)
    dG = torch.tensor(np.ascontiguousarray(G.T), dtype=torch.float64, device="cuda")
    dV = torch.zeros((a.n, a.n), dtype=torch.float64, device="cuda")
    dD = torch.zeros(a.n, dtype=torch.float64, device="cuda")
    fn = g.hypJacL2_split if a.form == "split" else g.hypJacL2_dev
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ret, sweeps, rot_s, rot_b = fn(a.alg, dG, nplus, dV, dD)
    torch.cuda.synchronize()
    print(f"{a.form} {a.m}x{a.n} nplus={nplus} ALG {a.alg}: ret {ret}, {sweeps} sweeps, rotations {rot_s} / "
          f"{rot_b} big, {time.perf_counter() - t0:.3f} s")
    return ret


if __name__ == "__main__":
    raise SystemExit(main())
