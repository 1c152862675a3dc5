"""CPU checks of the C ABI (include/gjx.h): the library loads, exports every
declared entry point, and reproduces the reference's argument handling
(1/HypJacL2.cu:39-77, share/HypJacL.cu:11-121) without touching a GPU."""

import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "gjx.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", src)) - {"defined"})


def test_exports_every_declared_symbol(built):
    lib = ctypes.CDLL(built["lib"])
    names = _declared()
    assert "hypJacL2" in names and "init_strats" in names
    for n in names:
        assert hasattr(lib, n), n
    import gpujachx_b200 as g
    assert set(g.EXPORTS) <= set(names)


def test_version(built):
    import gpujachx_b200 as g
    assert b"sm_100a" in g.lib().gjx_version()


def _call(routine, nrow, ncol, nplus, G=True, ldG=None, V=False, ldV=0, D=True, swp=True, s=True, b=True):
    import gpujachx_b200 as g
    L = g.lib()
    pd = ctypes.POINTER(ctypes.c_double)
    buf = (ctypes.c_double * 8)()
    p = ctypes.cast(buf, pd)
    sw, rs, rb = ctypes.c_uint(), ctypes.c_ulonglong(), ctypes.c_ulonglong()
    return L.hypJacL2(routine, nrow, ncol, nplus, p if G else None, nrow if ldG is None else ldG,
                      p if V else None, ldV, p if D else None, ctypes.byref(sw) if swp else None,
                      ctypes.byref(rs) if s else None, ctypes.byref(rb) if b else None, None)


def test_argument_codes(built):
    assert _call(16, 64, 32, 32) == -1
    assert _call(0, 0, 32, 32) == -2
    assert _call(0, 96, 32, 32) == -2       # nrow % 64
    assert _call(0, 64, 0, 0) == -3
    assert _call(0, 64, 128, 0) == -3       # ncol > nrow
    assert _call(0, 128, 48, 0) == -3       # ncol % 32
    assert _call(0, 64, 32, 33) == -4
    assert _call(0, 64, 32, 32, G=False) == -5
    assert _call(0, 64, 32, 32, ldG=63) == -6
    assert _call(2, 64, 32, 32, V=False, ldV=32) == -7
    assert _call(2, 64, 32, 32, V=True, ldV=31) == -8
    assert _call(0, 64, 32, 32, D=False) == -9
    assert _call(0, 64, 32, 32, swp=False) == -10
    assert _call(0, 64, 32, 32, s=False) == -11
    assert _call(0, 64, 32, 32, b=False) == -12
    # checks run in the reference's order: the first failing one wins
    assert _call(16, 0, 0, 99, G=False, D=False) == -1
    assert _call(0, 64, 32, 99, G=False) == -4


def test_init_strats_codes(built):
    import gpujachx_b200 as g
    L = g.lib()
    S = built["strat"].encode()
    f = L.gjx_init_strats
    assert f(b"", b"cycwor", 32, b"cycwor", 16) == -1
    assert f(S, b"", 32, b"cycwor", 16) == -2
    assert f(S, b"cycwor", 31, b"cycwor", 16) == -3
    assert f(S, b"cycwor", 32, b"", 16) == -4
    assert f(S, b"cycwor", 32, b"cycwor", 15) == -5
    assert f(S, b"nosuch", 32, b"cycwor", 16) == -6
    assert f(S, b"cycwor", 32, b"nosuch", 16) == -7
    assert f(b"/nonexistent/strat.so", b"cycwor", 32, b"cycwor", 16) == -8
    assert f(S, b"cycwor", 32, b"cycwor", 960) == -10  # 00960 is not shipped
    assert f(S, b"BrentL", 32, b"BrentL", 8) == -10    # BrentL starts at 16
    assert f(S, b"cycwor", 16, b"cycwor", 16) == -11
    assert f(S, b"cycwor", 32, b"cycwor", 16) == 0
    with pytest.raises(g.GjxError):
        g.init_strats(built["strat"], "cycwor", 32, "cycwor", 17)


def _fresh(code):
    return subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, timeout=120)


def test_init_strats_exits_like_the_reference(built):
    # share/HypJacL.cu: DIE("SNP1 unknown") -> "[ERROR] ..." on stderr, exit(EXIT_FAILURE)
    p = _fresh("import ctypes; L=ctypes.CDLL('%s'); L.init_strats(b'%s', b'cycwor', 32, b'nosuch', 16)"
               % (built["lib"], built["strat"]))
    assert p.returncode == 1 and "[ERROR]" in p.stderr and "SNP1 unknown" in p.stderr


def test_no_strategy_loaded_is_an_error(built):
    # a fresh process that never called init_strats: positive code, before any CUDA call
    p = _fresh("import numpy as np, gpujachx_b200 as g;"
               "r=g.hypJacL2(0, np.ones((64,32)), 32, check=False); print(r.ret)")
    assert p.returncode == 0 and p.stdout.strip() == "2", p.stderr


def test_strategy_order_mismatch(built):
    p = _fresh("import numpy as np, gpujachx_b200 as g; g.init_strats(None,'cycwor',32,'cycwor',4);"
               "r=g.hypJacL2(0, np.ones((128,96)), 96, check=False); print(r.ret)")
    assert p.returncode == 0 and p.stdout.strip() == "3", p.stderr


def test_missing_library_fails_loudly(tmp_path):
    code = ("import gpujachx_b200 as g; g.LIB_PATH='%s';\n"
            "try:\n g.lib()\nexcept g.GjxError as e:\n print('raised', e.code)" % (tmp_path / "none.so"))
    p = _fresh(code)
    assert "raised -100" in p.stdout
