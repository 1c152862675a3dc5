"""The x1 command line (csrc/x1.cpp, after the reference's 1/main.cu) and the
pp80 report (gpujachx_b200.pp80, after var/pp80.f90).

CPU: usage, argument errors, the pp80 report on an x1-shaped result file made
from the oracle.  GPU: x1 end to end on an HDF5 input -- its output file holds
exactly what the library call gives, in the reference's layout."""

import os
import subprocess

import numpy as np
import pytest

from gpujachx_b200 import build as B
from gpujachx_b200 import h5


@pytest.fixture(scope="module")
def x1(built):
    B.build_x1(verbose=False)
    B.build_pp(verbose=False)
    assert os.path.exists(B.X1)
    return B.X1


def test_usage_and_errors(x1, tmp_path):
    r = subprocess.run([x1], capture_output=True, text=True)
    assert r.returncode == 1 and "DEV SDY SNP0 SNP1 ALG H5F H5G [H5R]" in r.stderr
    r = subprocess.run([x1, "0", B.STRAT, "cycwor", "nosuch", "11", "f.h5", "64"], capture_output=True, text=True)
    assert r.returncode == 1 and "SNP1 unknown" in r.stderr        # init_strats exits first, as the reference's
    r = subprocess.run([x1, "0", str(tmp_path / "none.so"), "cycwor", "cycwor", "11", "f.h5", "64"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "cannot open SDY" in r.stderr


def test_pp80_report_on_result_file(built, tmp_path):
    from oracle import oracle
    from gpujachx_b200 import pp80, synth
    m, n, p = 192, 128, 128
    G = synth.make("svd_synth", m, n, 1000, smin=1e-6)
    s0 = oracle.load_strat(B.STRAT, "cycwor", 32)
    s1 = oracle.load_strat(B.STRAT, "cycwor", n // 16)
    o = oracle.hypjac_l2(11, G, p, s0, s1)
    rh5, fh5 = str(tmp_path / "r.h5"), str(tmp_path / "f.h5")
    V = np.zeros((m, n))
    V[:n, :n] = o["V"]
    h5.write(rh5, str(n), {"IDADIM": np.array([m, m, n, p], np.int32), "G": o["G"].T, "V": V.T, "D": o["D"]}, 0)
    lam = np.linalg.svd(G, compute_uv=False) ** 2
    h5.write(fh5, str(n), {"LAMBDA": lam}, 0)
    assert pp80.main([fh5, str(n), rh5]) == 0
    nr = h5.read(rh5, f"{n}/NRMS")
    assert nr.shape == (11,) and max(nr[0], nr[4]) < 1e-13 and np.isnan(nr[8])
    rel = h5.read(rh5, f"{n}/RELERR")
    assert rel.shape == (n + 1,) and abs(rel[-1]) < 1e-8
    assert pp80.main([fh5, str(n), rh5]) == 0                       # rewritten in place
    r = subprocess.run(["python", "-m", "gpujachx_b200.pp80", fh5, str(n), rh5], capture_output=True, text=True,
                       cwd=os.path.dirname(os.path.dirname(B.__file__)))
    assert r.returncode == 0 and "|| U^T U - I ||_M = " in r.stdout and "E-0" in r.stdout


@pytest.mark.gpu
def test_x1_end_to_end(x1, tmp_path):
    import gpujachx_b200 as g
    from gpujachx_b200 import synth
    m, n, p, alg = 512, 256, 100, 11
    G = synth.make("graded", m, n, 1002)
    fin, fout = str(tmp_path / "in.h5"), str(tmp_path / "out.h5")
    h5.write(fin, str(n), {"IDADIM": np.array([m, m, n, p], np.int32), "G": G.T}, 0)
    r = subprocess.run([x1, "0", B.STRAT, "cycwor", "rowcyc", str(alg), fin, str(n), fout], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    assert lines[0].startswith("GLB_ROT_S(") and lines[1].endswith("sweeps")
    g.init_strats(None, "cycwor", 32, "rowcyc", n // 16)
    ref = g.hypJacL2(alg, G, p)
    same = lambda a, b: np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))  # noqa: E731
    assert same(h5.read(fout, f"{n}/G").T, ref.U)
    assert same(h5.read(fout, f"{n}/V").T[:n, :n], ref.V)
    assert same(h5.read(fout, f"{n}/D"), ref.D)
    ist = h5.read(fout, f"{n}/ISTATS", as_float=False)
    info = g.strat_info()
    assert list(ist) == [ref.sweeps, info["strat0"], info["strat1"], 0]
    assert list(h5.read(fout, f"{n}/IDADIM", as_float=False)) == [m, m, n, p]
    assert h5.read(fout, f"{n}/TIMING").shape == (4,)
    assert f"{ref.rot_s:20d}" in lines[0]
    # a second group in the same result file; the group name sets n1
    fin2 = str(tmp_path / "in2.h5")
    G2 = synth.make("gaussian", 256, 128, 5)
    h5.write(fin2, "128", {"IDADIM": np.array([256, 256, 128, 128], np.int32), "G": G2.T}, 0)
    r = subprocess.run([x1, "0", B.STRAT, "cycwor", "cycwor", "9", fin2, "128", fout], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert h5.shape(fout, "128/G") == (128, 256) and h5.shape(fout, f"{n}/G") == (n, m)
