"""Build recipes of gpujachx_b200 (run on the build host; nvcc cross-compiles).

* ``build_lib``   -> gpujachx_b200/lib/libgjx.so   (CUDA kernels for sm_100a + host
                                                   driver + C ABI of include/gjx.h)
* ``build_strat`` -> gpujachx_b200/lib/strat.so   (the reference's pivot-pair tables,
                                                   compiled unchanged from its
                                                   strat/<family>/NNNNN.h headers,
                                                   symbols "<family>%05u")
* ``build_x1``    -> gpujachx_b200/lib/x1         (the x1 command line)
* ``build_pp``    -> gpujachx_b200/lib/libgjx_pp.so (accuracy post-processor, host
                                                   code in x87 extended precision)

The built files are not committed; they travel with the working tree.
"""

from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libgjx.so")
STRAT = os.path.join(LIBDIR, "strat.so")
X1 = os.path.join(LIBDIR, "x1")
PP = os.path.join(LIBDIR, "libgjx_pp.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]

LIB_SOURCES = ["gjx_kernels.cu", "gjx_split.cu", "gjx_host.cpp", "gjx_noalloc.cu", "gjx_h5abi.cpp", "h5mini.cpp"]
X1_SOURCES = ["x1.cpp"]

STRAT_FAMILIES = ["mmstep", "BrentL", "colcyc", "cycloc", "rowcyc", "cycwor"]


def _newer(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build_lib(force: bool = False, verbose: bool = True) -> str:
    """Each source compiled to its own object (in parallel), then linked."""
    srcs = [os.path.join(CSRC, s) for s in LIB_SOURCES]
    hdrs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + [
        os.path.join(ROOT, "include", "gjx.h")]
    if not force and not _newer(LIB, srcs + hdrs):
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)

    def one(src):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        if force or _newer(obj, [src] + hdrs):
            _run(["nvcc"] + NVCC_FLAGS + ["-c", "-o", obj + ".tmp", src], verbose)
            os.replace(obj + ".tmp", obj)
        return obj

    with ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        objs = list(ex.map(one, srcs))
    tmp = LIB + ".tmp"
    _run(["nvcc"] + ARCH + ["-shared", "-o", tmp] + objs + ["-ldl"], verbose)
    os.replace(tmp, LIB)
    return LIB


def build_x1(force: bool = False, verbose: bool = True) -> str:
    srcs = [os.path.join(CSRC, s) for s in X1_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    if len(srcs) != len(X1_SOURCES):
        return ""
    deps = srcs + [LIB] + glob.glob(os.path.join(CSRC, "*.h"))
    if not force and not _newer(X1, deps):
        return X1
    _run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-o", X1] + srcs
         + ["-L" + LIBDIR, "-lgjx", "-Wl,-rpath,$ORIGIN", "-ldl"], verbose)
    return X1


def build_pp(force: bool = False, verbose: bool = True) -> str:
    src = os.path.join(CSRC, "gjx_pp80.c")
    if not force and not _newer(PP, [src]):
        return PP
    os.makedirs(LIBDIR, exist_ok=True)
    tmp = PP + ".tmp"
    _run(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-o", tmp, src,
          "-lm"], verbose)
    os.replace(tmp, PP)
    return PP


def build_strat(ref_root: str | None = None, force: bool = False, verbose: bool = True) -> str:
    """Compile the reference's strategy-table headers, where they lie, into strat.so.

    The headers are data (``unsigned char|short <family>NNNNN[S][N/2][2] = {...}``);
    they are consumed unchanged, as the reference's own strat/proc_*-lnx.sh
    does, with the same exported symbol names.  The rowcyc and colcyc tables
    of orders 960 and 1024, which the reference does not ship, are added by
    its doubling construction (strat_gen).
    """
    ref_root = ref_root or os.environ.get("GJX_REF_ROOT", "")
    sdir = os.path.join(ref_root, "strat") if ref_root else ""
    if not force and os.path.exists(STRAT):
        return STRAT
    if not sdir or not os.path.isdir(sdir):
        if os.path.exists(STRAT):
            return STRAT
        raise FileNotFoundError(f"no strategy tables (set GJX_REF_ROOT to the reference tree) and no prebuilt {STRAT}")
    os.makedirs(LIBDIR, exist_ok=True)
    work = tempfile.mkdtemp(prefix="gjx_strat_")
    try:
        def one(fam):
            hdrs = sorted(glob.glob(os.path.join(sdir, fam, "*.h")))
            c = os.path.join(work, fam + ".c")
            with open(c, "w") as f:
                f.write("#define USE_STRAT_ARRAY_DECLARATOR\n")
                f.write('#define EXPORT_VAR __attribute__((visibility("default")))\n')
                for h in hdrs:
                    f.write("EXPORT_VAR\n#include \"%s\"\n" % h)
            o = os.path.join(work, fam + ".o")
            subprocess.check_call(["gcc", "-O0", "-fPIC", "-c", "-o", o, c])
            return o

        def ext(item):  # the tables beyond the reference's largest order (strat_gen)
            name, src = item
            c = os.path.join(work, name)
            with open(c, "w") as f:
                f.write(src)
            o = c[:-2] + ".o"
            subprocess.check_call(["gcc", "-O0", "-fPIC", "-c", "-o", o, c])
            return o

        from . import strat_gen
        with ThreadPoolExecutor(max_workers=len(STRAT_FAMILIES)) as ex:
            objs = list(ex.map(one, STRAT_FAMILIES))
            objs += list(ex.map(ext, sorted(strat_gen.extension_sources(sdir).items())))
        tmp = STRAT + ".tmp"
        _run(["gcc", "-shared", "-o", tmp] + objs, verbose)
        os.replace(tmp, STRAT)
    finally:
        shutil.rmtree(work, ignore_errors=True)
    return STRAT


def build_all(force: bool = False, verbose: bool = True):
    build_lib(force=force, verbose=verbose)
    build_strat(force=False, verbose=verbose)  # tables from $GJX_REF_ROOT/strat
    build_x1(force=force, verbose=verbose)
    build_pp(force=force, verbose=verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
