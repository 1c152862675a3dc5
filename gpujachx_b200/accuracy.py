"""Accuracy post-processor of (H)SVD results: the quantities of the reference's
var/pp80.f90 (non-MAGMA build), computed in x87 extended precision by
lib/libgjx_pp.so (csrc/gjx_pp80.c).

    from gpujachx_b200 import accuracy
    r = accuracy.pp80(U, D, V=V, nplus=p, lam=exact_D)
    r["nrms"]          # the 11 norms, pp80's NRMS(1..11) (NaN where not computed)
    r["relerr"][-1]    # max relative error of D (sign kept)

NRMS layout (pp80.f90:187-760):
  1, 2   || U^T U - I ||_M, _F
  3, 4   || U U^T - I ||_M, _F          (O(M^2 N); skipped with uut=False)
  5, 6   || V^T J V - J ||_M, _F        (J = diag(+I_p, -I_{N-p}); V^T V - I if p = N)
  7, 8   || V J V^T - J ||_M, _F
  9..11  || A U - U D ||_M, _F, _R      (needs A = G J G^T of the input, M x M)
"""

from __future__ import annotations

import ctypes
import math
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
PP_PATH = os.path.join(PKG, "lib", "libgjx_pp.so")

LABELS = ["|| U^T U - I ||_M", "|| U^T U - I ||_F", "|| U U^T - I ||_M", "|| U U^T - I ||_F",
          "|| V^T J V - J ||_M", "|| V^T J V - J ||_F", "|| V J V^T - J ||_M", "|| V J V^T - J ||_F",
          "|| A U - U D ||_M", "|| A U - U D ||_F", "|| A U - U D ||_R"]

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(PP_PATH):
            raise RuntimeError(f"{PP_PATH} is missing: run `python -m gpujachx_b200.build`")
        L = ctypes.CDLL(PP_PATH)
        u, i, pd = ctypes.c_uint, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
        L.gjx_pp80_jorth.argtypes = [u, u, pd, u, i, u, u, pd]
        L.gjx_pp80_jorth.restype = i
        L.gjx_pp80_resid.argtypes = [u, u, pd, u, pd, u, pd, ctypes.POINTER(ctypes.c_int), pd]
        L.gjx_pp80_resid.restype = i
        L.gjx_pp80_derr.argtypes = [u, pd, pd, pd, pd]
        L.gjx_pp80_derr.restype = i
        _lib = L
    return _lib


def _f(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def _pd(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def jorth(X, trans: bool = False, psum: int | None = None, pres: int | None = None):
    """(max, Frobenius) norm of X^T Js X - Jr (trans: X Js X^T - Jr), with
    Js = diag(+1 x psum, -1 ...) over the summed index and Jr likewise (pres)
    over the result's; defaults: all +1."""
    Xf = _f(X)
    rows, cols = Xf.shape
    nk, nr = (cols, rows) if trans else (rows, cols)
    psum = nk if psum is None else psum
    pres = nr if pres is None else pres
    out = np.zeros(2)
    r = lib().gjx_pp80_jorth(rows, cols, _pd(Xf), max(1, rows), int(bool(trans)), psum, pres, _pd(out))
    if r:
        raise ValueError(f"gjx_pp80_jorth: bad arguments ({r})")
    return float(out[0]), float(out[1])


def resid(A, U, D, ipiv=None):
    """(max, Frobenius, relative) norm of U diag(D) - A U, rows of U
    back-permuted by the 1-based interchanges ipiv first."""
    Af, Uf = _f(A), _f(U)
    m, n = Uf.shape
    Dv = np.ascontiguousarray(D, dtype=np.float64)
    piv = None if ipiv is None else np.ascontiguousarray(ipiv, dtype=np.int32)
    out = np.zeros(3)
    r = lib().gjx_pp80_resid(m, n, _pd(Af), max(1, Af.shape[0]), _pd(Uf), max(1, m), _pd(Dv),
                             None if piv is None else piv.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _pd(out))
    if r:
        raise ValueError(f"gjx_pp80_resid: bad arguments ({r})")
    return float(out[0]), float(out[1]), float(out[2])


def derr(D, lam):
    """ABSERR and RELERR (n + 1 entries each; the last is the extreme one)."""
    Dv = np.ascontiguousarray(D, dtype=np.float64)
    lv = np.ascontiguousarray(lam, dtype=np.float64)
    n = Dv.size
    if lv.size != n:
        raise ValueError("D and LAMBDA differ in length")
    ab, rel = np.zeros(n + 1), np.zeros(n + 1)
    if lib().gjx_pp80_derr(n, _pd(Dv), _pd(lv), _pd(ab), _pd(rel)):
        raise ValueError("gjx_pp80_derr failed")
    return ab, rel


def pp80(U, D, V=None, nplus: int | None = None, A=None, ipiv=None, lam=None, uut: bool = True) -> dict:
    """All of pp80's figures that the given inputs allow."""
    U = _f(U)
    m, n = U.shape
    p = n if nplus is None else int(nplus)
    nrms = [math.nan] * 11
    nrms[0:2] = jorth(U)
    if uut:
        nrms[2:4] = jorth(U, trans=True)
    if V is not None:
        Vf = _f(V)[:n, :n]
        nrms[4:6] = jorth(Vf, psum=p, pres=p)
        nrms[6:8] = jorth(Vf, trans=True, psum=p, pres=p)
    if A is not None:
        nrms[8:11] = resid(A, U, D, ipiv)
    out = {"nrms": nrms, "labels": LABELS}
    if lam is not None:
        ab, rel = derr(D, lam)
        out.update(abserr=ab, relerr=rel, max_abs_err=float(ab[-1]), max_rel_err=float(rel[-1]))
    return out


def es25(v: float) -> str:
    """Fortran ES25.17E3: 17 decimals, a 3-digit signed exponent, width 25."""
    if math.isnan(v) or math.isinf(v):
        return f"{v:>25}"
    m, e = f"{v:.17E}".split("E")
    return f"{m}E{int(e):+04d}".rjust(25)


def report(r: dict, nplus_is_n: bool = False) -> str:
    """pp80-style text (FORMAT(A,' = ',ES25.17E3)): one line per figure
    computed; the V lines read V^T V - I when J = I, as the reference's."""
    lines = []
    for lab, v in zip(r["labels"], r["nrms"]):
        if nplus_is_n:
            lab = lab.replace("V^T J V - J", "V^T V - I").replace("V J V^T - J", "V V^T - I")
        if not math.isnan(v):
            lines.append(f"{lab} = {es25(v)}")
    if "max_abs_err" in r:
        lines.append(f"max abs err = {es25(r['max_abs_err'])}")
        lines.append(f"max rel err = {es25(r['max_rel_err'])}")
    return "\n".join(lines)
