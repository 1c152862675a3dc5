"""Generate the golden fixtures from the reference itself.

Runs the reference's own hypJacL2 -- its sources under 1/ and share/ compiled
for sm_100a by oracle/Makefile into oracle/_ref/ref_harness (add _qr / _drmac
for the -DUSE_QR / -DUSE_DRMAC builds) -- on seeded synthetic inputs and
records its outputs: sha256 of U, V, D, the full D, the sweep and rotation
counts.  It needs a B200 (the reference is GPU code), so it runs on the GPU
host:

    python tests/golden/make_golden.py [OUT.json] [--variant base|qr|drmac] [--large]

--large records the benchmark-size cases (LARGE_CASES: the 8192 x 8192
configuration, one SVD and one HSVD matrix of each batch size 64..512, the
4096 x 2048 and 2048 x 1024 configurations) into ref_golden_large.json:
digests and counts only (the 8192 x 8192 input is formed on the GPU).

The committed tests/golden/ref_golden*.json came from this script; the tests
regenerate each input, check its sha256, and compare the oracle (CPU) and the
CUDA path (GPU) with the recorded outputs bit for bit.
"""

from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gpujachx_b200 import synth  # noqa: E402

HARNESS = {"base": os.path.join(ROOT, "oracle", "_ref", "ref_harness"),
           "qr": os.path.join(ROOT, "oracle", "_ref", "ref_harness_qr"),
           "drmac": os.path.join(ROOT, "oracle", "_ref", "ref_harness_drmac")}
STRAT = os.path.join(ROOT, "gpujachx_b200", "lib", "strat.so")


def case(name, m, n, nplus, alg, gen="gaussian", seed=0, snp0="cycwor", snp1="cycwor", **kw):
    return dict(name=name, m=m, n=n, nplus=nplus, alg=alg, gen=gen, seed=seed, snp0=snp0, snp1=snp1, kw=kw)


# Small cases (the CPU oracle reruns each in about a second): every ALG, the
# three signatures (J = I, J = -I, mixed), every strategy family, graded and
# ill-conditioned inputs, an already orthogonal input, N = 32 and N = M.
CASES = [
    case("g128x64_alg%d" % a, 128, 64, 64, a, seed=11) for a in range(16)
] + [
    case("hyp128x64_np40_alg%d" % a, 128, 64, 40, a, seed=12) for a in (0, 1, 2, 3, 8, 9, 10, 11)
] + [
    case("neg128x64_alg%d" % a, 128, 64, 0, a, seed=13) for a in (0, 1, 2, 3, 9, 11)
] + [
    case("hyp128x64_np16_alg11", 128, 64, 16, 11, seed=14),
    case("hyp128x64_np48_alg3", 128, 64, 48, 3, seed=15),
    case("hyp128x64_np1_alg9", 128, 64, 1, 9, seed=16),
    case("hyp128x64_np63_alg10", 128, 64, 63, 10, seed=17),
    case("n32_64x32_alg11", 64, 32, 32, 11, seed=18),
    case("n32_64x32_hyp_alg3", 64, 32, 20, 3, seed=19),
    case("sq64_alg11", 64, 64, 64, 11, gen="svd_synth", seed=20, smin=1e-6),
    case("c1_256_alg9", 256, 256, 256, 9, gen="svd_synth", seed=1000, smin=1e-8),
    case("c1_256_alg11", 256, 256, 256, 11, gen="svd_synth", seed=1000, smin=1e-8),
    case("c1_256_alg3", 256, 256, 256, 3, gen="svd_synth", seed=1000, smin=1e-8),
    case("c3s_512x256_np128_alg11", 512, 256, 128, 11, gen="graded", seed=1002),
    case("c3s_512x256_np128_alg9", 512, 256, 128, 9, gen="graded", seed=1002),
    case("c3s_512x256_np128_alg1", 512, 256, 128, 1, gen="graded", seed=1002),
    case("g384x192_alg11_rowcyc", 384, 192, 192, 11, seed=21, snp0="rowcyc", snp1="rowcyc"),
    case("g384x192_alg11_colcyc", 384, 192, 192, 11, seed=22, snp0="colcyc", snp1="colcyc"),
    case("g384x192_alg11_cycloc", 384, 192, 192, 11, seed=23, snp0="cycloc", snp1="cycloc"),
    case("g256x256_alg11_brentl", 256, 256, 256, 11, seed=24, snp0="BrentL", snp1="BrentL"),
    case("g256x256_alg11_mmstep", 256, 256, 256, 11, seed=25, snp0="mmstep", snp1="mmstep"),
    case("g256x256_alg10_mmstep_hyp", 256, 256, 100, 10, seed=26, snp0="cycwor", snp1="mmstep"),
    case("g512x320_alg11_mixed", 512, 320, 320, 11, seed=27, snp0="BrentL", snp1="cycwor"),
    case("g1024x512_alg11", 1024, 512, 512, 11, seed=28),
    case("g1024x512_np200_alg11", 1024, 512, 200, 11, seed=29),
    case("orth_256x128_alg11", 256, 128, 128, 11, gen="orth", seed=30),
    case("ill_256x128_alg11", 256, 128, 128, 11, gen="svd_synth", seed=31, smin=1e-13),
]


# Benchmark-size cases: the reference takes about a minute on the first.
LARGE_CASES = [
    case("c4_8192_alg11", 8192, 8192, 8192, 11, gen="haar_gpu", seed=1003, smin=1e-12),
    case("c2_4096x2048_alg11", 4096, 2048, 2048, 11, seed=1001),
    case("c3_2048x1024_np512_alg11", 2048, 1024, 512, 11, gen="graded", seed=1002),
    case("c1_256_alg11_np128", 256, 256, 128, 11, gen="svd_synth", seed=1000, smin=1e-8),
] + [
    case("c5_n%d_%s" % (n, "svd" if p == n else "hsvd"), n, n, p, 11, gen="svd_synth", seed=5000 + n, smin=1e-6)
    for n in range(64, 513, 64) for p in (n, n // 2)
]


def make_input(c):
    if c["gen"] == "orth":  # orthonormal columns scaled by powers of two: no rotation at all
        Q = synth.svd_synth(c["m"], c["n"], c["seed"], smin=1.0)
        return np.asfortranarray(Q * (2.0 ** np.arange(c["n"]) % 7))
    return synth.make(c["gen"], c["m"], c["n"], c["seed"], **c["kw"])


def run_ref(c, G, variant="base", dev=0, reps=1, timeout=600):
    """One process of the reference harness on G: `reps` runs of its
    hypJacL2 (the output is the last run's); "reps_timing" lists each run's
    timing[4] (wall, setup + H2D, compute, D2H + cleanup; seconds)."""
    m, n = c["m"], c["n"]
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(np.asfortranarray(G).tobytes("F"))
        cmd = [HARNESS[variant], str(dev), STRAT, c["snp0"], c["snp1"], str(c["alg"]), str(c["nplus"]),
               str(m), str(n), fin, fout] + ([str(reps)] if reps > 1 else [])
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"reference failed on {c['name']}: {p.stdout[-500:]} {p.stderr[-500:]}")
        raw = open(fout, "rb").read()
    off = 0

    def take(dt, cnt):
        nonlocal off
        a = np.frombuffer(raw, dtype=dt, count=cnt, offset=off)
        off += a.nbytes
        return a

    ret = int(take(np.int32, 1)[0])
    swp = int(take(np.uint32, 1)[0])
    rs = int(take(np.uint64, 1)[0])
    rb = int(take(np.uint64, 1)[0])
    timing = take(np.float64, 4).copy()
    U = take(np.float64, m * n).reshape(n, m).T
    V = take(np.float64, n * n).reshape(n, n).T if (c["alg"] & 2) else None
    D = take(np.float64, n).copy()
    reps_timing = [[float(x) for x in ln.split()[4:8]] for ln in p.stdout.splitlines() if ln.startswith("REP ")]
    return dict(ret=ret, sweeps=swp, rot_s=rs, rot_b=rb, timing=timing.tolist(), U=U, V=V, D=D,
                stdout=p.stdout, reps_timing=reps_timing or [timing.tolist()])


def record(c, out):
    r = dict(ret=out["ret"], sweeps=out["sweeps"], rot_s=out["rot_s"], rot_b=out["rot_b"],
             U_sha=synth.digest(out["U"]), D_sha=synth.digest(out["D"]))
    if len(out["D"]) <= 512:
        r["D"] = [float(x).hex() for x in out["D"]]
    if out["V"] is not None:
        r["V_sha"] = synth.digest(out["V"])
    return r


def main():
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    variant = "base"
    if "--variant" in sys.argv:
        variant = sys.argv[sys.argv.index("--variant") + 1]
        args = [a for a in args if a != variant]
    large = "--large" in sys.argv
    out_path = args[0] if args else os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                f"ref_golden_{'large' if large else variant}.json")
    res = []
    for c in (LARGE_CASES if large else CASES):
        G = make_input(c)
        o = run_ref(c, G, variant)
        entry = dict(c)
        entry["input_sha"] = synth.digest(G)
        entry["out"] = record(c, o)
        entry["ref_timing"] = o["timing"]
        res.append(entry)
        print(c["name"], o["ret"], o["sweeps"], o["rot_s"], o["rot_b"], flush=True)
    os.makedirs(os.path.dirname(out_path), exist_ok=True)
    with open(out_path, "w") as f:
        json.dump(dict(variant=variant, harness="oracle/_ref/ref_harness" + ("" if variant == "base" else "_" + variant),
                       cases=res), f, indent=1)
    print("wrote", out_path)


if __name__ == "__main__":
    main()
