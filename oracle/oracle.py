"""ctypes front end of the CPU oracle (oracle/gjx_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by the CPU-baseline / reference arm of bench.py, as the checker or the timed
CPU baseline.  The product package never imports this module.

The oracle restates the reference arithmetic bit for bit (reference files
cited in gjx_oracle.c); its parity with the reference is pinned by the golden
fixtures in tests/golden/.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libgjx_oracle.so")

_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle (gcc, OpenMP, no fp contraction) into oracle/_build."""
    src = os.path.join(HERE, "gjx_oracle.c")
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(src):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
           "-o", LIB, src, "-lm", "-ldl"]
    subprocess.check_call(cmd)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        d, u, i = ctypes.c_double, ctypes.c_uint, ctypes.c_int
        pd = ctypes.POINTER(ctypes.c_double)
        pu = ctypes.POINTER(ctypes.c_uint)
        pull = ctypes.POINTER(ctypes.c_ulonglong)
        pu8 = ctypes.POINTER(ctypes.c_ubyte)
        pu16 = ctypes.POINTER(ctypes.c_ushort)
        L.gjxo_rsqrt_rn.argtypes = [d]
        L.gjxo_rsqrt_rn.restype = d
        L.gjxo_sum32.argtypes = [pd]
        L.gjxo_sum32.restype = d
        L.gjxo_rotT.argtypes = [d, d, d, pd, pd]
        L.gjxo_rotT.restype = i
        L.gjxo_rotH.argtypes = [d, d, d, pd, pd]
        L.gjxo_rotH.restype = i
        L.gjxo_hypJacL2.argtypes = [u, u, u, u, pd, u, pd, u, pd, pu8, u, pu16, u, u, pu, pull, pull, i]
        L.gjxo_hypJacL2.restype = i
        L.gjxo_outer_step.argtypes = [u, u, u, u, pd, u, pd, u, pu8, u, pu16, u, u, pull, pull, i]
        L.gjxo_outer_step.restype = None
        L.gjxo_load_strat.argtypes = [ctypes.c_char_p, ctypes.c_char_p, u, pu16, u]
        L.gjxo_load_strat.restype = i
        L.gjxo_set_variant.argtypes = [i]
        L.gjxo_set_variant.restype = None
        L.gjxo_nrm2_32.argtypes = [pd]
        L.gjxo_nrm2_32.restype = d
        L.gjxo_cosa.argtypes = [d, d, pd, pd]
        L.gjxo_cosa.restype = d
        _lib = L
    return _lib


def _p(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t)) if a is not None else None


VARIANTS = {"base": 0, "qr": 1, "drmac": 2}


def set_variant(name: str) -> None:
    """Which build of the reference to restate: "base" (Gram + Cholesky),
    "qr" (-DUSE_QR: Householder/Givens factor), "drmac" (-DUSE_DRMAC: the QR
    factor and Drmac's scaled-norm sweep in the definite sorting kernels)."""
    lib().gjxo_set_variant(VARIANTS[name])


def nrm2_32(v) -> float:
    a = np.ascontiguousarray(v, dtype=np.float64)
    assert a.size == 32
    return lib().gjxo_nrm2_32(_p(a))


def rsqrt_rn(x: float) -> float:
    return lib().gjxo_rsqrt_rn(float(x))


def sum32(v) -> float:
    a = np.ascontiguousarray(v, dtype=np.float64)
    assert a.size == 32
    return lib().gjxo_sum32(_p(a))


def rotT(apq, dp, dq):
    c, t = ctypes.c_double(), ctypes.c_double()
    big = lib().gjxo_rotT(apq, dp, dq, ctypes.byref(c), ctypes.byref(t))
    return big, c.value, t.value


def rotH(apq, dp, dq):
    c, t = ctypes.c_double(), ctypes.c_double()
    big = lib().gjxo_rotH(apq, dp, dq, ctypes.byref(c), ctypes.byref(t))
    return big, c.value, t.value


def load_strat(sdy: str, name: str, n: int) -> np.ndarray:
    """[steps, n/2, 2] uint16 table, read from strat.so like the reference."""
    cap = (n + 1) * (n // 2) * 2
    out = np.zeros(cap, dtype=np.uint16)
    steps = lib().gjxo_load_strat(sdy.encode(), name.encode(), n, _p(out, ctypes.c_ushort), cap)
    if steps < 0:
        raise ValueError(f"oracle: no strategy {name}{n:05d} in {sdy} (code {steps})")
    return out[: steps * (n // 2) * 2].reshape(steps, n // 2, 2).copy()


def hypjac_l2(routine: int, G: np.ndarray, nplus: int, strat0: np.ndarray, strat1: np.ndarray,
              nthreads: int = 0):
    """Run the oracle sweep driver.  G: (nrow, ncol) float64, any layout; it is
    copied into Fortran order.  strat0: [steps, 16, 2]; strat1: [steps, n1/2, 2].
    Returns dict(ret, G=U, V, D, sweeps, rot_s, rot_b)."""
    Gf = np.asfortranarray(np.array(G, dtype=np.float64, copy=True))
    nrow, ncol = Gf.shape
    full = bool(routine & 2)
    V = np.zeros((ncol, ncol), dtype=np.float64, order="F") if full else None
    D = np.zeros(ncol, dtype=np.float64)
    s0 = np.ascontiguousarray(strat0, dtype=np.uint8)
    s1 = np.ascontiguousarray(strat1, dtype=np.uint16)
    swp = ctypes.c_uint(0)
    rs, rb = ctypes.c_ulonglong(0), ctypes.c_ulonglong(0)
    ret = lib().gjxo_hypJacL2(routine, nrow, ncol, nplus, _p(Gf), nrow, _p(V), ncol, _p(D),
                              _p(s0, ctypes.c_ubyte), s0.shape[0], _p(s1, ctypes.c_ushort),
                              s1.shape[0], s1.shape[1], ctypes.byref(swp), ctypes.byref(rs),
                              ctypes.byref(rb), nthreads)
    return dict(ret=ret, G=Gf, V=V, D=D, sweeps=swp.value, rot_s=rs.value, rot_b=rb.value)


def outer_step(routine: int, Gf: np.ndarray, V, nplus: int, strat0: np.ndarray, strat1: np.ndarray,
               step: int, nthreads: int = 0):
    """One outer step in place on Fortran-ordered G (and V); returns (s, b)."""
    nrow, ncol = Gf.shape
    s0 = np.ascontiguousarray(strat0, dtype=np.uint8)
    s1 = np.ascontiguousarray(strat1, dtype=np.uint16)
    cs, cb = ctypes.c_ulonglong(0), ctypes.c_ulonglong(0)
    lib().gjxo_outer_step(routine, nrow, ncol, nplus, _p(Gf), nrow, _p(V), ncol,
                          _p(s0, ctypes.c_ubyte), s0.shape[0], _p(s1, ctypes.c_ushort), step,
                          s1.shape[1], ctypes.byref(cs), ctypes.byref(cb), nthreads)
    return cs.value, cb.value
