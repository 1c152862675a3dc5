"""gpujachx_b200 -- B200-native (sm_100a) hierarchically blocked one-sided Jacobi
SVD / hyperbolic SVD, a drop-in for the GPUJACHx path.

The computation lives in ``lib/libgjx.so`` (hand-written CUDA kernels for sm_100a
plus the C++ sweep driver) behind the C ABI of ``include/gjx.h``.  This module is
a thin ctypes mirror of that ABI with the reference's names and argument meaning:

* :func:`init_strats` -- share/HypJacL.cu:11-121 (``init_strats``), raising
  :class:`GjxError` where the reference exits;
* :func:`hypJacL2`    -- 1/HypJacL2.cu:13-202 (``hypJacL2``), on host arrays;
* :func:`hypJacL2_dev` -- the same on device-resident torch tensors.

There is no CPU fallback: without the built library every call raises.
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import NamedTuple, Optional

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libgjx.so")
STRAT_PATH = os.path.join(PKG, "lib", "strat.so")

CDSORT_1, FULL_SVD, ACCUMV_2, BLK_ORI = 1, 2, 4, 8
ERR_CUDA, ERR_NO_STRAT, ERR_STRAT_ORDER, ERR_DEVICE, ERR_ALIGN, ERR_SCRATCH = 1, 2, 3, 4, 5, 6
STRATEGIES = ("mmstep", "BrentL", "colcyc", "cycloc", "rowcyc", "cycwor")

# exported by libgjx.so, as declared in include/gjx.h
EXPORTS = ("hypJacL2", "init_strats", "gjx_init_strats", "gjx_strat_info", "gjx_get_strat1",
           "gjx_hypJacL2_dev", "gjx_release_cache", "gjx_set_verbose", "gjx_last_error",
           "gjx_version", "gjx_rsqrt_rn_dev", "gjx_profile", "gjx_profile_read", "gjx_hypJacL2_noalloc",
           "gjx_validate_pairs", "gjx_validate_strats", "gjx_configure_device", "gjx_h5_read", "gjx_h5_write",
           "gjx_hypJacL2_batched", "gjx_set_sweep_mode", "gjx_set_split", "gjx_set_pairs_per_cta", "gjx_autotune",
           "gjx_autotune_clear", "gjx_wait_selftest")


class GjxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gjx error {code}: {msg}")
        self.code = code


_lib = None


def lib() -> ctypes.CDLL:
    """Load libgjx.so (raises if it was not built: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise GjxError(-100, f"{LIB_PATH} is missing: run `python -m gpujachx_b200.build` "
                              "(or __graft_entry__.build()) first")
    L = ctypes.CDLL(LIB_PATH)
    u, i = ctypes.c_uint, ctypes.c_int
    pd, pu = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint)
    pull = ctypes.POINTER(ctypes.c_ulonglong)
    L.hypJacL2.argtypes = [u, u, u, u, pd, u, pd, u, pd, pu, pull, pull, pd]
    L.hypJacL2.restype = i
    L.init_strats.argtypes = [ctypes.c_char_p, ctypes.c_char_p, u, ctypes.c_char_p, u]
    L.init_strats.restype = None
    L.gjx_init_strats.argtypes = [ctypes.c_char_p, ctypes.c_char_p, u, ctypes.c_char_p, u]
    L.gjx_init_strats.restype = i
    L.gjx_strat_info.argtypes = [pu] * 6
    L.gjx_strat_info.restype = i
    L.gjx_get_strat1.argtypes = [ctypes.POINTER(ctypes.c_ushort), u]
    L.gjx_get_strat1.restype = i
    L.gjx_hypJacL2_dev.argtypes = [u, u, u, u, ctypes.c_void_p, u, ctypes.c_void_p, u, ctypes.c_void_p,
                                   ctypes.c_void_p, pu, pull, pull]
    L.gjx_hypJacL2_dev.restype = i
    L.gjx_hypJacL2_noalloc.argtypes = L.gjx_hypJacL2_dev.argtypes
    L.gjx_hypJacL2_noalloc.restype = i
    L.gjx_hypJacL2_split.argtypes = L.gjx_hypJacL2_dev.argtypes
    L.gjx_hypJacL2_split.restype = i
    L.gjx_split_phase_cycles.argtypes = [ctypes.POINTER(ctypes.c_longlong)]
    L.gjx_split_phase_cycles.restype = i
    L.gjx_release_cache.argtypes = []
    L.gjx_release_cache.restype = i
    L.gjx_set_verbose.argtypes = [i]
    L.gjx_set_verbose.restype = None
    L.gjx_last_error.argtypes = []
    L.gjx_last_error.restype = ctypes.c_char_p
    L.gjx_version.argtypes = []
    L.gjx_version.restype = ctypes.c_char_p
    L.gjx_rsqrt_rn_dev.argtypes = [ctypes.c_void_p, ctypes.c_void_p, u]
    L.gjx_rsqrt_rn_dev.restype = i
    L.gjx_profile.argtypes = [i]
    L.gjx_profile.restype = None
    L.gjx_profile_read.argtypes = [pull, pull, pd]
    L.gjx_profile_read.restype = None
    L.gjx_validate_pairs.argtypes = [ctypes.POINTER(ctypes.c_ushort), u, u, pull, pull, pu]
    L.gjx_validate_pairs.restype = i
    L.gjx_validate_strats.argtypes = [pull]
    L.gjx_validate_strats.restype = i
    pp = ctypes.POINTER(ctypes.c_void_p)
    L.gjx_hypJacL2_batched.argtypes = [u, u, pu, pu, pu, pp, pu, pp, pu, pp, ctypes.c_void_p, pu, pull, pull,
                                       ctypes.POINTER(ctypes.c_int)]
    L.gjx_hypJacL2_batched.restype = i
    L.gjx_autotune.argtypes = [u, u, u, u, u, pu]
    L.gjx_autotune.restype = i
    L.gjx_wait_selftest.argtypes = [ctypes.c_longlong, u, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_longlong)]
    L.gjx_wait_selftest.restype = i
    L.gjx_autotune_clear.argtypes = []
    L.gjx_autotune_clear.restype = None
    L.gjx_set_split.argtypes = [u]
    L.gjx_set_split.restype = None
    L.gjx_set_pairs_per_cta.argtypes = [u]
    L.gjx_set_pairs_per_cta.restype = None
    L.gjx_set_variant.argtypes = [u]
    L.gjx_set_variant.restype = None
    L.gjx_set_batch_mode.argtypes = [i]
    L.gjx_set_batch_mode.restype = None
    L.gjx_autotune_batched.argtypes = [u, u, pu, pu, pu, u, pu]
    L.gjx_autotune_batched.restype = i
    L.gjx_set_sweep_mode.argtypes = [i]
    L.gjx_set_sweep_mode.restype = None
    L.gjx_configure_device.argtypes = [i]
    L.gjx_configure_device.restype = i
    L.gjx_set_verbose(0)
    _lib = L
    return L


_INIT_MSG = {-1: "SDY empty", -2: "SNP0 empty", -3: "n0 not positive even", -4: "SNP1 empty",
             -5: "n1 not positive even", -6: "SNP0 unknown", -7: "SNP1 unknown", -8: "cannot open SDY",
             -9: "NO SUCH STRATEGY for SNP0 & n0", -10: "NO SUCH STRATEGY for SNP1 & n1",
             -11: "n0 must be 32", -12: "n1 > 1024"}


def init_strats(sdy: Optional[str] = None, snp0: str = "cycwor", n0: int = 32, snp1: str = "cycwor",
                n1: int = 0) -> None:
    """Load the inner (snp0, n0 = 32) and outer (snp1, n1 = N/16) strategy tables."""
    sdy = sdy or STRAT_PATH
    r = lib().gjx_init_strats(sdy.encode(), snp0.encode(), n0, snp1.encode(), n1)
    if r:
        raise GjxError(r, _INIT_MSG.get(r, "init_strats failed"))


def strat_info() -> dict:
    v = [ctypes.c_uint() for _ in range(6)]
    r = lib().gjx_strat_info(*[ctypes.byref(x) for x in v])
    if r:
        raise GjxError(r, "no strategy tables loaded")
    k = ("strat0", "steps0", "pairs0", "strat1", "steps1", "pairs1")
    return {a: b.value for a, b in zip(k, v)}


def strat1_table() -> np.ndarray:
    info = strat_info()
    n = info["steps1"] * info["pairs1"] * 2
    out = np.zeros(n, dtype=np.uint16)
    got = lib().gjx_get_strat1(out.ctypes.data_as(ctypes.POINTER(ctypes.c_ushort)), n)
    if got != n:
        raise GjxError(got, "gjx_get_strat1")
    return out.reshape(info["steps1"], info["pairs1"], 2)


def validate_pairs(table) -> dict:
    """Check a pivot-pair table [steps][n/2][2]: entries in range, p != q,
    each step a perfect matching, every pair {p, q} covered.  Returns
    dict(code, missing, repeats, bad_step); code 0 = valid."""
    t = np.ascontiguousarray(table, dtype=np.uint16)
    if t.ndim != 3 or t.shape[2] != 2:
        raise ValueError("table must be [steps][n/2][2]")
    miss, rep, bad = ctypes.c_ulonglong(), ctypes.c_ulonglong(), ctypes.c_uint()
    code = lib().gjx_validate_pairs(t.ctypes.data_as(ctypes.POINTER(ctypes.c_ushort)), t.shape[0], 2 * t.shape[1],
                                    ctypes.byref(miss), ctypes.byref(rep), ctypes.byref(bad))
    return dict(code=code, missing=miss.value, repeats=rep.value, bad_step=bad.value)


def validate_loaded() -> dict:
    """validate_pairs of both loaded tables (inner strat0, outer strat1)."""
    out = (ctypes.c_ulonglong * 6)()
    r = lib().gjx_validate_strats(out)
    if r < 0:
        raise GjxError(r, "no strategy tables loaded")
    return dict(code=r, strat0=dict(code=out[0], missing=out[1], repeats=out[2]),
                strat1=dict(code=out[3], missing=out[4], repeats=out[5]))


def profile(enable: bool) -> None:
    """Reset the launch counters; with enable, time every block-pair launch."""
    lib().gjx_profile(1 if enable else 0)


def profile_read() -> dict:
    a, b, ms = ctypes.c_ulonglong(), ctypes.c_ulonglong(), ctypes.c_double()
    lib().gjx_profile_read(ctypes.byref(a), ctypes.byref(b), ctypes.byref(ms))
    return dict(launches=a.value, l1_launches=b.value, l1_ms=ms.value)


def last_error() -> str:
    return lib().gjx_last_error().decode()


def set_verbose(level: int) -> None:
    lib().gjx_set_verbose(int(level))


@dataclass
class HypJacResult:
    ret: int
    U: np.ndarray          # nrow x ncol, unit columns (G on output)
    V: Optional[np.ndarray]  # ncol x ncol (routine & 2)
    D: np.ndarray          # ncol, +-||g_j||^2
    sweeps: int
    rot_s: int
    rot_b: int
    timing: np.ndarray     # wall, setup + H2D, compute, D2H + cleanup (s)


def _pd(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def hypJacL2(routine: int, G: np.ndarray, nplus: int, check: bool = True) -> HypJacResult:
    """Run hypJacL2 on a host matrix (copied into Fortran order; not modified).

    Arguments and return codes are those of 1/HypJacL2.hpp:6-27; with
    ``check`` a non-zero return raises :class:`GjxError`.
    """
    Gf = np.array(G, dtype=np.float64, order="F", copy=True)
    nrow, ncol = Gf.shape
    full = bool(routine & FULL_SVD)
    V = np.zeros((ncol, ncol), dtype=np.float64, order="F") if full else None
    D = np.zeros(ncol, dtype=np.float64)
    swp = ctypes.c_uint(0)
    s, b = ctypes.c_ulonglong(0), ctypes.c_ulonglong(0)
    timing = np.zeros(4, dtype=np.float64)
    ret = lib().hypJacL2(routine, nrow, ncol, nplus, _pd(Gf), nrow, _pd(V), ncol if full else 0, _pd(D),
                         ctypes.byref(swp), ctypes.byref(s), ctypes.byref(b), _pd(timing))
    if check and ret:
        raise GjxError(ret, last_error() if ret > 0 else "invalid argument")
    return HypJacResult(ret, Gf, V, D, swp.value, s.value, b.value, timing)


def hypJacL2_dev(routine: int, G, nplus: int, V=None, D=None, stream=None, nrow: Optional[int] = None,
                 check: bool = True):
    """Run on device-resident torch tensors, in place.

    ``G`` is a CUDA float64 tensor holding the matrix column by column: a
    (ncol, lddG) row-major tensor whose row j is column j (i.e. ``G_f.T`` of a
    Fortran array); nrow defaults to lddG.  ``V`` (ncol, lddV) likewise,
    ``D`` (ncol,).  Returns (ret, sweeps, rot_s, rot_b).
    """
    ncol, lddG = G.shape
    nrow = lddG if nrow is None else nrow
    full = bool(routine & FULL_SVD)
    swp = ctypes.c_uint(0)
    s, b = ctypes.c_ulonglong(0), ctypes.c_ulonglong(0)
    st = stream.cuda_stream if stream is not None else None
    ret = lib().gjx_hypJacL2_dev(routine, nrow, ncol, nplus, G.data_ptr(), lddG,
                                 V.data_ptr() if full else None, V.shape[1] if full else 0,
                                 D.data_ptr(), st, ctypes.byref(swp), ctypes.byref(s), ctypes.byref(b))
    if check and ret:
        raise GjxError(ret, last_error() if ret > 0 else "invalid argument")
    return ret, swp.value, s.value, b.value


VARIANTS = {"base": 0, "qr": 1, "drmac": 2}


def set_variant(name: str) -> None:
    """The pivot-block factor of the reference's builds to reproduce: "base"
    (Gram + Cholesky), "qr" (-DUSE_QR), "drmac" (-DUSE_DRMAC)."""
    lib().gjx_set_variant(VARIANTS[name])


def hypJacL2_split(routine: int, G, nplus: int, V=None, D=None, stream=None, nrow: Optional[int] = None,
                   check: bool = True):
    """The split-precision form on device-resident torch tensors, in place,
    with the arguments of hypJacL2_dev: the Gram matrices and the updates of
    G and V run as exact int8 slice products on the tensor cores (blocks of
    32 columns, pairs of 64; ncol a multiple of 64).  Not bit-identical to
    the plain form: its accuracy is reported against an FP64 reference.
    Returns (ret, sweeps, rot_s, rot_b)."""
    ncol, lddG = G.shape
    nrow = lddG if nrow is None else nrow
    full = bool(routine & FULL_SVD)
    swp = ctypes.c_uint(0)
    s, b = ctypes.c_ulonglong(0), ctypes.c_ulonglong(0)
    st = stream.cuda_stream if stream is not None else None
    ret = lib().gjx_hypJacL2_split(routine, nrow, ncol, nplus, G.data_ptr(), lddG,
                                   V.data_ptr() if full else None, V.shape[1] if full else 0,
                                   D.data_ptr(), st, ctypes.byref(swp), ctypes.byref(s), ctypes.byref(b))
    if check and ret:
        raise GjxError(ret, last_error() if ret > 0 else "invalid argument")
    return ret, swp.value, s.value, b.value


class BatchResult(NamedTuple):
    ret: int
    info: list
    sweeps: list
    rot_s: list
    rot_b: list


def hypJacL2_batched(routine: int, Gs, nplus, Vs=None, Ds=None, stream=None, nrows=None) -> BatchResult:
    """The batched form on device-resident torch tensors, in place: matrix b
    is Gs[b] ((ncol, lddG) row-major, row j = column j, as hypJacL2_dev),
    Vs[b] ((ncol, lddV), ALG & 2), Ds[b] ((ncol,)).  nplus: a list, or one
    value for all.  Each matrix gets exactly what hypJacL2_dev gives it."""
    n = len(Gs)
    full = bool(routine & FULL_SVD)
    npl = list(nplus) if hasattr(nplus, "__len__") else [int(nplus)] * n
    U = ctypes.c_uint * n
    P = ctypes.c_void_p * n
    ncol = U(*[g.shape[0] for g in Gs])
    ldg = U(*[g.shape[1] for g in Gs])
    nrow = U(*(nrows if nrows is not None else [g.shape[1] for g in Gs]))
    dg = P(*[g.data_ptr() for g in Gs])
    dv = P(*[v.data_ptr() for v in Vs]) if full else None
    ldv = U(*[v.shape[1] for v in Vs]) if full else None
    dd = P(*[d.data_ptr() for d in Ds])
    sw, rs, rb = U(), (ctypes.c_ulonglong * n)(), (ctypes.c_ulonglong * n)()
    info = (ctypes.c_int * n)()
    st = stream.cuda_stream if stream is not None else None
    ret = lib().gjx_hypJacL2_batched(routine, n, nrow, ncol, U(*npl), dg, ldg, dv, ldv, dd, st, sw, rs, rb, info)
    if ret:
        raise GjxError(ret, last_error())
    return BatchResult(ret, list(info), list(sw), list(rs), list(rb))


def autotune_batched(routine: int, nrows, ncols, nplus, sweeps: int = 1) -> dict:
    """Time the batched form's configurations (block pairs per CTA, launch per
    step or per sweep) on seeded random matrices of these shapes and keep the
    fastest for later batches of the same shapes (gjx_autotune_batched);
    returns {"pairs_per_cta": 1, 2, 3 (one per CTA of 4 warps, two CTAs per
    SM) or 4 (two per CTA of 4 warps), "mode": 0 per step / 1 per sweep}."""
    n = len(ncols)
    U = ctypes.c_uint * n
    out = (ctypes.c_uint * 2)()
    npl = list(nplus) if hasattr(nplus, "__len__") else [int(nplus)] * n
    r = lib().gjx_autotune_batched(routine, n, U(*nrows), U(*ncols), U(*npl), sweeps, out)
    if r:
        raise GjxError(r, last_error() if r > 0 else "invalid argument")
    return {"pairs_per_cta": out[0], "mode": out[1]}


def autotune(routine: int, nrow: int, ncol: int, nplus: int, sweeps: int = 1) -> dict:
    """Time the launch configurations of this shape and keep the fastest for
    later calls (gjx_autotune); returns {"split": CTAs per pair, "mode": 0/1}."""
    out = (ctypes.c_uint * 2)()
    r = lib().gjx_autotune(routine, nrow, ncol, nplus, sweeps, out)
    if r:
        raise GjxError(r, last_error() if r > 0 else "invalid argument")
    return {"split": out[0], "mode": out[1]}

