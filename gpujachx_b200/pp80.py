"""pp80: the accuracy report of an x1 result file, after the reference's
var/pp80.f90.

    python -m gpujachx_b200.pp80 FH5 GH5 RH5

RH5/GH5 holds x1's output (IDADIM, G = U, V, D); FH5/GH5 the generator's
file: the exact eigenvalues LAMBDA and, for the residual figures, A = G J G^T
(M x M) with the pivots IPIV, each optional here (the reference requires
them).  Prints the figures and writes NRMS (11 values, NaN where not
computed), LAMBDA, ABSERR and RELERR (N + 1 each) into RH5/GH5.
"""

from __future__ import annotations

import math
import os
import sys

import numpy as np

from . import GjxError, accuracy, h5


def _maybe(file, path, as_float=True):
    try:
        return h5.read(file, path, as_float=as_float)
    except GjxError:
        return None


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 3:
        print("pp80 FH5 GH5 RH5", file=sys.stderr)
        return 1
    fh5, gh5, rh5 = argv
    if not os.path.exists(fh5):
        print("FH5 nonexistent!", file=sys.stderr)
        return 1
    if not os.path.exists(rh5):
        print("RH5 nonexistent!", file=sys.stderr)
        return 1
    ida = h5.read(rh5, f"{gh5}/IDADIM", as_float=False).ravel()
    lda, m, n, p = (int(x) for x in ida[:4])
    for bad, msg in ((lda < m, "LDA < M"), (m < n, "M < N"), (n < p, "N < P"), (n % 2, "N ODD")):
        if bad:
            print(msg, file=sys.stderr)
            return 1
    D = h5.read(rh5, f"{gh5}/D").ravel()[:n]
    U = h5.read(rh5, f"{gh5}/G").T[:m, :n]                    # N x LDA in C order
    Vt = _maybe(rh5, f"{gh5}/V")
    V = None if Vt is None else Vt.T[:n, :n]
    A = _maybe(fh5, f"{gh5}/A")
    ipiv = _maybe(fh5, f"{gh5}/IPIV", as_float=False)
    lam = _maybe(fh5, f"{gh5}/LAMBDA")
    r = accuracy.pp80(U, D, V=V, nplus=p, A=None if A is None else A.T, ipiv=None if ipiv is None else ipiv.ravel(),
                      lam=None if lam is None else lam.ravel()[:n])
    print(accuracy.report(r, nplus_is_n=(p == n)))
    out = {"NRMS": np.array(r["nrms"], dtype=np.float64)}
    if lam is not None:
        out.update(LAMBDA=lam.ravel()[:n].astype(np.float64), ABSERR=r["abserr"], RELERR=r["relerr"])
    h5.write(rh5, gh5, out, mode=2)
    return 0 if all(math.isfinite(x) or math.isnan(x) for x in r["nrms"]) else 1


if __name__ == "__main__":
    sys.exit(main())
