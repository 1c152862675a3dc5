"""Benchmark of the blocked one-sided Jacobi SVD on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the headline configuration): plain FP64 SVD of a 4096 x 2048 matrix
with i.i.d. N(0,1) entries (PCG64 seed 1001), NPLUS = N, cycwor/cycwor tables,
ALG 11 (block-oriented, U, V and D, innermost sorting).  One step = one full
decomposition to convergence.  Metric: matrices per second (whole job).

* value: device-resident input (the working copy is reset from an HBM copy of
  the input inside each step), CUDA events on the library's stream around each
  step, L2 flushed (256 MiB write) between steps outside the events;
* e2e: the public hypJacL2 call on pinned host buffers: H2D of G, D2H of U, V
  and D inside the timed region;
* roofline: the block-pair kernel, algorithmic bytes per launch (768 M + 512 N
  per block pair, 64 pairs) over its mean event-timed launch duration;
* cpu_baseline: the CPU oracle port (OpenMP, all host threads) timed on the
  first outer steps of the same decomposition, scaled to a whole one; DGESVJ
  (OpenBLAS, all host threads) on the full matrix is reported beside it
  (--config c5: one SVD and one HSVD decomposition of each n by the port,
  scaled by the batch's count of each n).

N > 1: independent replicas (the single-matrix SVD is not sharded), barrier
and max-over-ranks device time; value = matrices of all ranks / that time.

--impl reference: the reference's own implementation of the path -- its
hypJacL2 sources built for sm_100a (oracle/_ref/ref_harness; the reference
is GPU code only) -- on the same input, whole decompositions timed by its own
timer (value: its compute phase; e2e: its wall time with its own allocation
and copies); the CPU oracle port of its arithmetic is reported beside it.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# the single-matrix workloads; "c2" (the default) is the headline
WORKLOADS = {
    "c1": dict(m=256, n=256, nplus=256, alg=9, seed=1000, gen="svd_synth", kw=dict(smin=1e-8),
               metric="SVD matrices/s (256x256 FP64, U and D)",
               workload="plain FP64 SVD 256x256, G = Q1 diag(s) Q2^T, Haar Q1/Q2 seed 1000, s geometric 1..1e-8, "
                        "NPLUS=N, cycwor/cycwor, ALG 9 (U, D), one step = one decomposition to convergence"),
    "c2": dict(m=4096, n=2048, nplus=2048, alg=11, seed=1001, gen="gaussian", kw={},
               metric="SVD matrices/s (4096x2048 FP64, full SVD)",
               workload="plain FP64 SVD 4096x2048, i.i.d. N(0,1) seed 1001, NPLUS=N, cycwor/cycwor, ALG 11 "
                        "(U, V, D), one step = one decomposition to convergence"),
    "c3": dict(m=2048, n=1024, nplus=512, alg=11, seed=1002, gen="graded", kw={},
               metric="HSVD matrices/s (2048x1024 FP64, J = diag(+I_512, -I_512), full)",
               workload="hyperbolic SVD 2048x1024, G = B diag(d), B i.i.d. N(0,1), d_j = 10^U(-6,0), seed 1002, "
                        "NPLUS=512, cycwor/cycwor, ALG 11 (U, V, D), one step = one decomposition to convergence"),
    "c4": dict(m=8192, n=8192, nplus=8192, alg=11, seed=1003, gen="haar_gpu", kw=dict(smin=1e-12),
               metric="SVD matrices/s (8192x8192 FP64, full SVD)",
               workload="plain FP64 SVD 8192x8192, G = Q1 diag(s) Q2^T, Haar Q1/Q2 (QR of Gaussians, torch CUDA "
                        "generator seed 1003), s geometric 1..1e-12, NPLUS=N, cycwor/cycwor, ALG 11 (U, V, D), "
                        "one step = one decomposition to convergence"),
    "c5": dict(m=0, n=0, nplus=0, alg=11, seed=5000, gen="batch", kw={}, count=4096,
               metric="(H)SVD matrices/s, batch of 4096 FP64 matrices n x n, n uniform in {64, ..., 512}",
               workload="batch of 4096 independent decompositions, n uniform in {64, 128, ..., 512} (PCG64 seed "
                        "5000), G = Q1 diag(s) Q2^T, Haar Q1/Q2 (QR of Gaussians, torch CUDA generator seed 5000), "
                        "s geometric 1..1e-6; even-indexed matrices NPLUS = n (SVD), odd NPLUS = n/2 (HSVD); "
                        "cycwor tables of each n; ALG 11; one step = the whole batch to convergence"),
}
W = 32


def _use(name: str) -> None:
    """Bind the module-level workload constants to WORKLOADS[name]."""
    global WL, M, N, NPLUS, ALG, SEED, N1, PAIRS, STEPS1, FLOP_PER_PAIR, BYTES_PER_PAIR, METRIC, CONFIG
    WL = WORKLOADS[name]
    if WL["gen"] == "batch":
        WL = dict(WORKLOADS["c2"], **{k: v for k, v in WORKLOADS[name].items() if k in ("metric", "workload")})
        WL.update(alg=WORKLOADS[name]["alg"], seed=WORKLOADS[name]["seed"])
    M, N, NPLUS, ALG, SEED = WL["m"], WL["n"], WL["nplus"], WL["alg"], WL["seed"]
    N1 = N // 16
    PAIRS = N1 // 2
    STEPS1 = N1 - 1
    full = bool(ALG & 2)
    FLOP_PER_PAIR = 4 * M * W * W + (2 * N * W * W if full else 0)   # Gram + update of G, update of V
    BYTES_PER_PAIR = 768 * M + (512 * N if full else 0)               # G read twice, written once; V read + written
    METRIC = WL["metric"]
    CONFIG = {"workload": WL["workload"], "name": name, "m": M, "n": N, "nplus": NPLUS, "alg": ALG,
              "strategies": "cycwor/cycwor",
              "l2": "flushed between steps (256 MiB write, outside the timed events)"}


def _input() -> np.ndarray:
    from gpujachx_b200 import synth
    return synth.make(WL["gen"], M, N, SEED, **WL["kw"])


_use("c2")


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


# DRAM bytes (read + write) of one block-pair launch of the c2 workload, from
# one ncu capture of it (cold L2): dram__bytes_read.sum + dram__bytes_write.sum
# of gjx::l1_step_kernel<true,true,2>, 4096 x 2048, ALG 11
RECORDED_TRAFFIC = {"c2": 142.60e6}


class Clocks:
    """nvidia-smi sampler for the timed region (SM clock and throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev, self.rows, self.p = dev, [], None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.p = None

    def _read(self):
        for line in self.p.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.t.join(timeout=2)
        rows = [r for r in self.rows if len(r) >= 9]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def replica_throughput(local_ms: float, steps: int, world: int, device=None) -> tuple:
    """Whole-job matrices/s of `world` independent replicas that each ran
    `steps` decompositions in local_ms of device time: the slowest rank's time
    counts (max over ranks, as torch.distributed MAX), every rank's matrices
    count.  Returns (value, max_ms).  Works on gloo (CPU tensors) and nccl."""
    import torch
    import torch.distributed as dist
    t = local_ms
    if world > 1:
        x = torch.tensor([local_ms], dtype=torch.float64, device=device)
        dist.all_reduce(x, op=dist.ReduceOp.MAX)
        t = float(x.item())
    return world * steps / (t / 1000.0), t


def cpu_port_sample(G0: np.ndarray, sweeps: int, min_seconds: float = 10.0):
    """Time the oracle port (all host threads) on the first outer steps of
    the decomposition; scale by steps per sweep and the sweep count."""
    from oracle import oracle as O
    O.build()
    from gpujachx_b200 import STRAT_PATH
    s0 = O.load_strat(STRAT_PATH, "cycwor", 32)
    s1 = O.load_strat(STRAT_PATH, "cycwor", N1)
    Gf = np.array(G0, order="F", copy=True)
    V = np.asfortranarray(np.eye(N))
    cores = os.cpu_count() or 1
    done, t0 = 0, time.perf_counter()
    while done < STEPS1 and (time.perf_counter() - t0) < min_seconds:
        O.outer_step(ALG, Gf, V if ALG & 2 else None, NPLUS, s0, s1, done, nthreads=cores)
        done += 1
    dt = time.perf_counter() - t0
    per_matrix = dt / done * STEPS1 * sweeps
    return {"value": 1.0 / per_matrix, "unit": "matrices/s", "cores": cores, "kind": "port",
            "sample": f"first {done} of {STEPS1} outer steps of sweep 1 ({done * PAIRS} block pairs, "
                      f"{dt:.1f} s), scaled x{STEPS1}/{done} steps x {sweeps} sweeps",
            "seconds": dt, "outer_steps": done}


def lapack_baseline(G0: np.ndarray):
    from oracle import lapack
    cores = os.cpu_count() or 1
    s, _, _, info, dt = lapack.dgesvj(G0, jobv="V", threads=cores)
    return {"value": 1.0 / dt, "unit": "matrices/s", "cores": cores, "info": info,
            "routine": "DGESVJ JOBA=G JOBU=U JOBV=V (OpenBLAS 0.3.30 via SciPy)", "seconds": dt}


def accuracy_figures(G0: np.ndarray, U: np.ndarray, V, D: np.ndarray) -> dict:
    """pp80's figures of one result: orthogonality of U, J-orthogonality of V,
    relative error of D against an FP64 reference spectrum -- LAPACK DGESVJ's
    sigma^2 for an SVD, eigenvalues of R J R^T (G = QR) for an HSVD."""
    from gpujachx_b200 import accuracy
    if WL["gen"] == "haar_gpu":
        lam = np.logspace(0.0, 2.0 * np.log10(WL["kw"]["smin"]), N)
        ref = "the constructed spectrum s^2 (G = Q1 diag(s) Q2^T formed in FP64: absolute accuracy only)"
    elif NPLUS == N:
        from oracle import lapack
        lam = lapack.dgesvj(G0, jobv="N", threads=os.cpu_count() or 1)[0] ** 2
        ref = "LAPACK DGESVJ sigma^2"
    else:
        R = np.linalg.qr(G0, mode="r")
        J = np.r_[np.ones(NPLUS), -np.ones(N - NPLUS)]
        lam = np.linalg.eigvalsh((R * J) @ R.T)
        ref = "eigenvalues of R J R^T, G = QR (absolute accuracy only)"
    if M * N * N > 2 ** 34:  # too large for extended precision on the host: FP64 products on the GPU
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        Ut = torch.tensor(U, device=dev)
        e = (Ut.T @ Ut - torch.eye(N, dtype=torch.float64, device=dev)).abs()
        out = {"|| U^T U - I ||_M (FP64 on the GPU)": float(e.max())}
        if V is not None:
            Vt = torch.tensor(V, device=dev)
            J = torch.ones(N, dtype=torch.float64, device=dev)
            J[NPLUS:] = -1.0
            e = ((Vt.T * J) @ Vt - torch.diag(J)).abs()
            out["|| V^T J V - J ||_M (FP64 on the GPU)"] = float(e.max())
        ab, rel = accuracy.derr(D, lam)
        out.update(max_rel_err_D=float(rel[-1]), max_abs_err_D=float(ab[-1]), reference_spectrum=ref)
        return out
    r = accuracy.pp80(U, D, V=V, nplus=NPLUS, lam=lam, uut=(M * M * N <= 2 ** 33))
    out = {lab: v for lab, v in zip(r["labels"], r["nrms"]) if v == v}
    out.update(max_rel_err_D=r["max_rel_err"], max_abs_err_D=r["max_abs_err"], reference_spectrum=ref)
    return out


REF_BUILD = "reference sources (1/, share/), nvcc -arch sm_100a -DUSE_RSQRT -O3, oracle/_ref/ref_harness"


def ref_gpu_runs(G0: np.ndarray, m, n, nplus, alg, steps: int, warmup: int, budget_s: float = 240.0):
    """The reference's own hypJacL2 built for sm_100a (oracle/_ref/ref_harness)
    on G0: one probe run, then warmup + timed runs in one process, as many
    timed runs as `steps` asks for while they fit in budget_s.  Returns None
    when the reference build is absent."""
    from tests.golden.make_golden import HARNESS, case, run_ref
    if not os.path.exists(HARNESS["base"]):
        return None
    c = case("bench", m, n, nplus, alg, seed=SEED)
    probe = run_ref(c, G0)
    t1 = max(probe["timing"][0], 1e-3)
    timed = max(1, min(steps, int(budget_s / t1)))
    warm = min(warmup, max(0, int(0.25 * budget_s / t1)))
    out = run_ref(c, G0, reps=warm + timed, timeout=max(600, int(4 * t1 * (warm + timed))))
    runs = out["reps_timing"][warm:]
    return {"wall_s": [r[0] for r in runs], "compute_s": [r[2] for r in runs], "sweeps": out["sweeps"],
            "rot_s": out["rot_s"], "rot_b": out["rot_b"], "warmup": warm, "steps": len(runs), "build": REF_BUILD}


def batch_cpu_sample(sizes, seed: int):
    """The oracle port (all host threads) on the batch: one SVD (NPLUS = n)
    and one HSVD (NPLUS = n/2) decomposition per n of the batch, scaled by the
    batch's count of each n."""
    from gpujachx_b200 import STRAT_PATH, synth
    from oracle import oracle as O
    O.build()
    cores = os.cpu_count() or 1
    s0 = O.load_strat(STRAT_PATH, "cycwor", 32)
    tot, cpu_by = 0.0, {}
    for n in sorted(set(int(x) for x in sizes)):
        G = synth.make("svd_synth", n, n, seed + n, smin=1e-6)
        s1 = O.load_strat(STRAT_PATH, "cycwor", n // 16)
        per = 0.0
        for npl in (n, n // 2):
            t0 = time.perf_counter()
            O.hypjac_l2(ALG, G, npl, s0, s1, nthreads=cores)
            per += 0.5 * (time.perf_counter() - t0)
        cpu_by[n] = per
        tot += per * int((sizes == n).sum())
    return {"value": len(sizes) / tot, "unit": "matrices/s", "cores": cores, "kind": "port",
            "sample": "one SVD and one HSVD (NPLUS = n/2) per n by the oracle port, scaled by the batch's count "
                      "of each n", "seconds_by_n": cpu_by}


def reference_arm_batch(args):
    """c5 on the reference path: the reference's own sm_100a build has no
    batched form, so it is looped -- per batch size n, one SVD (NPLUS = n)
    and one HSVD (NPLUS = n/2) matrix of that n, each timed over repeated runs
    in one process (its compute phase and wall time), scaled by how many
    matrices of that n the batch holds.  The CPU oracle port, one
    decomposition of each, is reported beside it (cpu_baseline)."""
    from gpujachx_b200 import synth
    from tests.golden.make_golden import HARNESS, case, run_ref
    cfg = WORKLOADS["c5"]
    sizes = batch_sizes(cfg["count"], cfg["seed"])
    ns = sorted(set(int(x) for x in sizes))
    base = {"metric": cfg["metric"], "unit": "matrices/s", "impl": "reference", "n_gpus": args.gpus,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": cfg["workload"], "name": "c5", "count": len(sizes), "alg": ALG,
                       "parallelism": "independent batches per rank" if args.gpus > 1 else "single GPU"}}
    line = None
    if os.path.exists(HARNESS["base"]):
        comp_tot = wall_tot = 0.0
        by_n = {}
        reps = max(1, min(args.steps, 5))
        for n in ns:
            cnt = int((sizes == n).sum())
            G = synth.make("svd_synth", n, n, cfg["seed"] + n, smin=1e-6)
            c_n, w_n = 0.0, 0.0
            for npl in (n, n // 2):
                out = run_ref(case("c5", n, n, npl, ALG, seed=0), G, reps=reps + 1)
                runs = out["reps_timing"][1:]
                c_n += 0.5 * statistics.median(r[2] for r in runs)
                w_n += 0.5 * statistics.median(r[0] for r in runs)
            by_n[n] = {"compute_s": c_n, "wall_s": w_n, "count": cnt}
            comp_tot += c_n * cnt
            wall_tot += w_n * cnt
        line = dict(base, value=len(sizes) / comp_tot, steps=1, steps_requested=args.steps,
                    ms_per_step=1000.0 * comp_tot,
                    e2e={"value": len(sizes) / wall_tot, "unit": "matrices/s",
                         "h2d_bytes_per_step": int((sizes.astype(np.int64) ** 2).sum() * 8),
                         "d2h_bytes_per_step": int((2 * sizes.astype(np.int64) ** 2 + sizes).sum() * 8),
                         "api": "reference hypJacL2 per matrix (host buffers; its own allocation and copies)"},
                    reference={"kind": "reference", "build": REF_BUILD, "by_n": by_n,
                               "sample": f"one SVD and one HSVD matrix per n, {reps} timed runs each after one "
                                         "warm-up run; one step = the batch, scaled from the per-n times"})
    cpu = None if args.no_cpu else batch_cpu_sample(sizes, cfg["seed"])
    if line is None:
        line = dict(base, value=cpu["value"], steps=1, steps_requested=args.steps,
                    ms_per_step=1000.0 * len(sizes) / cpu["value"],
                    e2e={"value": cpu["value"], "unit": "matrices/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0},
                    note="reference build absent: the CPU oracle port, scaled from one matrix of each n")
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


def reference_arm(args):
    """The reference's own implementation of the path on this box: its
    hypJacL2 sources built for sm_100a (oracle/_ref/ref_harness; the
    reference is GPU code and has no CPU implementation), whole
    decompositions, timed by the reference's own timer -- value from its
    compute phase (timing[2]: the device-resident part), e2e from its wall
    time (timing[0]: allocation, H2D of G, compute, D2H of U, V, D).  The CPU
    oracle port is reported beside it (cpu_baseline) on a bounded sample."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.config == "c5":
        return reference_arm_batch(args)
    _use(args.config)
    G0 = _input()
    config = dict(CONFIG, parallelism=("replicas" if args.gpus > 1 else "single GPU"))
    base = {"metric": METRIC, "unit": "matrices/s", "impl": "reference", "n_gpus": args.gpus, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config}
    ref = ref_gpu_runs(G0, M, N, NPLUS, ALG, args.steps, args.warmup)
    sweeps = (ref or {}).get("sweeps") or int(os.environ.get("GJX_BENCH_SWEEPS", "10"))
    cpu = None if args.no_cpu else cpu_port_sample(G0, sweeps, min_seconds=10.0)
    if ref is not None:
        comp = statistics.median(ref["compute_s"])
        wall = statistics.median(ref["wall_s"])
        line = dict(base, value=1.0 / comp, steps=ref["steps"], steps_requested=args.steps,
                    ms_per_step=1000.0 * comp, step_ms=[1000.0 * x for x in ref["compute_s"]],
                    sweeps=ref["sweeps"],
                    e2e={"value": 1.0 / wall, "unit": "matrices/s", "h2d_bytes_per_step": M * N * 8,
                         "d2h_bytes_per_step": M * N * 8 + (N * N * 8 if ALG & 2 else 0) + N * 8,
                         "api": "reference hypJacL2 (host buffers; its own allocation and copies)",
                         "step_ms": [1000.0 * x for x in ref["wall_s"]]},
                    reference={"kind": "reference", "build": ref["build"], "timer": "the reference's timing[4]",
                               "rot_s": ref["rot_s"], "rot_b": ref["rot_b"]})
    else:  # no reference build on this host: the oracle port, one sampled outer step per step
        per_step = cpu["seconds"] / cpu["outer_steps"]
        line = dict(base, value=cpu["value"], steps=cpu["outer_steps"], steps_requested=args.steps,
                    ms_per_step=1000.0 * per_step,
                    e2e={"value": cpu["value"], "unit": "matrices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                    note="reference build absent: the CPU oracle port, one step = one sampled outer step "
                         f"({PAIRS} block pairs); value scaled to a whole decomposition")
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# the batched workload (c5)
# ---------------------------------------------------------------------------
def batch_sizes(count: int = 4096, seed: int = 5000) -> np.ndarray:
    return 64 * np.random.default_rng(seed).integers(1, 9, size=count)


def batch_inputs(sizes, dev, seed: int = 5000):
    """One contiguous device buffer holding every G (column major, ld = n),
    generated on the GPU: Haar Q1, Q2 from QR of Gaussians (signs fixed by
    diag(R)), s geometric from 1 to 1e-6, G = Q1 diag(s) Q2^T."""
    import torch
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    offs = np.concatenate([[0], np.cumsum(sizes.astype(np.int64) ** 2)])
    buf = torch.empty(int(offs[-1]), dtype=torch.float64, device=dev)
    for n in sorted(set(int(x) for x in sizes)):
        idx = np.nonzero(sizes == n)[0]
        k = len(idx)

        def haar():
            a = torch.randn((k, n, n), dtype=torch.float64, device=dev, generator=gen)
            q, r = torch.linalg.qr(a)
            return q * torch.sign(torch.diagonal(r, dim1=-2, dim2=-1)).unsqueeze(-2)

        q1, q2 = haar(), haar()
        sv = torch.logspace(0.0, -6.0, n, dtype=torch.float64, device=dev)
        g = (q1 * sv) @ q2.transpose(-2, -1)            # (k, n, n): row-major n x n = G
        gt = g.transpose(-2, -1).contiguous()            # row j = column j of G (column major)
        for t, b in enumerate(idx):
            buf[int(offs[b]):int(offs[b + 1])].copy_(gt[t].reshape(-1))
    return buf, offs


def shard_batch(G_all, offs_all, sizes, rank: int, world: int):
    """This rank's shard of one batch (strong scaling): the matrices the
    size-balanced partition gives it (indices `mine`, ascending), their sizes,
    their offsets in the shard and the shard's buffer (their G, each column
    major with ld = n, back to back).  G_all holds the whole batch, matrix b
    at [offs_all[b], offs_all[b + 1])."""
    import torch
    from gpujachx_b200 import batch as B
    mine = B.partition(sizes, sizes, world)[rank]
    sz = sizes[mine]
    offs = np.concatenate([[0], np.cumsum(sz.astype(np.int64) ** 2)])
    G = torch.cat([G_all[int(offs_all[b]):int(offs_all[b + 1])] for b in mine])
    return mine, sz, offs, G


def batch_flops_bytes(sizes, sweeps, full=True):
    """Algorithmic FLOP and bytes of the sweeps each matrix ran (reference
    geometry, w = 32; P_sweep = n1 (n1 - 1) / 2 cyclic block pairs)."""
    f = b = 0.0
    for n, sw in zip(sizes, sweeps):
        n1 = int(n) // 16
        p = n1 * (n1 - 1) // 2 * sw
        f += p * (4 * n * W * W + (2 * n * W * W if full else 0))
        b += p * (768 * n + (512 * n if full else 0))
    return f, b


def main_batch(args):
    import torch
    import torch.distributed as dist
    import gpujachx_b200 as g
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    cfg = dict(WORKLOADS["c5"])
    if args.count:
        cfg["count"] = args.count
    sizes = batch_sizes(cfg["count"], cfg["seed"])
    if args.shard and world > 1:
        # strong scaling: one batch, split by the size-balanced partition
        G_all, offs_all = batch_inputs(sizes, dev, cfg["seed"])
        mine, sizes, offs, G0 = shard_batch(G_all, offs_all, sizes, rank, world)
        del G_all
    else:
        # weak scaling: every rank solves its own batch of the same shapes
        G0, offs = batch_inputs(sizes, dev, cfg["seed"] + rank)
    nplus = [int(n) if b % 2 == 0 else int(n) // 2 for b, n in enumerate(sizes)]
    g.init_strats(None, "cycwor", 32, "cycwor", 4)
    # the library's batched autotuner, once per batch shape, before timing:
    # block pairs per CTA and one launch per step index or per sweep
    if args.pairs_per_cta:  # a fixed form (profiling runs): per-step launches of that form, no tuning
        g.lib().gjx_set_pairs_per_cta(args.pairs_per_cta)
        g.lib().gjx_set_batch_mode(0)
        tuned = {"pairs_per_cta": args.pairs_per_cta, "mode": 0}
    else:
        tuned = g.autotune_batched(ALG, [int(n) for n in sizes], [int(n) for n in sizes], nplus)
    width = tuned["pairs_per_cta"]
    dG = torch.empty_like(G0)
    dV = torch.empty_like(G0)
    dD = torch.empty(int(sizes.sum()), dtype=torch.float64, device=dev)
    doffs = np.concatenate([[0], np.cumsum(sizes)])
    Gs = [dG[int(offs[b]):int(offs[b + 1])].view(int(n), int(n)) for b, n in enumerate(sizes)]
    Vs = [dV[int(offs[b]):int(offs[b + 1])].view(int(n), int(n)) for b, n in enumerate(sizes)]
    Ds = [dD[int(doffs[b]):int(doffs[b + 1])] for b in range(len(sizes))]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        dG.copy_(G0)
        return g.hypJacL2_batched(ALG, Gs, nplus, Vs=Vs, Ds=Ds, stream=stream)

    for _ in range(args.warmup):
        res = step()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    g.profile(False)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    prof = g.profile_read()
    clk = clocks.stop()
    nmat = len(sizes)
    value, total_ms = replica_throughput(sum(times), args.steps * nmat, world, dev)
    if args.shard and world > 1:  # every rank's shard counts once: the whole batch per step
        value = args.steps * cfg["count"] / (total_ms / 1000.0)
    assert all(i == 0 for i in res.info)
    flops, nbytes = batch_flops_bytes(sizes, res.sweeps)
    pair_steps = sum(int(sw) * (int(n) // 16 - 1) * (int(n) // 32) for n, sw in zip(sizes, res.sweeps))
    t_s = statistics.median(times) / 1000.0
    hbm, peak_kind = _peaks()
    roof = {"bound": "hbm", "achieved": nbytes / t_s / 1e9, "peak": hbm, "unit": "GB/s",
            "frac": nbytes / t_s / 1e9 / hbm, "traffic": None,
            "kernel": ("gjx::l1_batchn2_kernel<true,true>" if width == 4 else
                       "gjx::l1_batchn_kernel<true,true>" if width == 3 else
                       ("gjx::l1_batch_flow_kernel<true,true,%d>" if tuned["mode"] else
                        "gjx::l1_batch_kernel<true,true,%d>") % width),
            "peak_kind": f"{peak_kind} HBM copy bandwidth",
            "note": "algorithmic bytes of all sweeps run, over the device time of the whole batched call",
            "fp64_tflops": flops / t_s / 1e12, "launches_per_step": prof["launches"] // max(1, args.steps)}

    # e2e: pinned host inputs, H2D + the batched call + D2H of U, V and D, per step
    hin = torch.empty(G0.numel(), dtype=torch.float64, pin_memory=True)
    hin.copy_(G0)
    hU = torch.empty_like(hin, pin_memory=True)
    hV = torch.empty_like(hin, pin_memory=True)
    hD = torch.empty(dD.numel(), dtype=torch.float64, pin_memory=True)
    e2e_t = []
    for k in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dG.copy_(hin, non_blocking=True)
        g.hypJacL2_batched(ALG, Gs, nplus, Vs=Vs, Ds=Ds, stream=stream)
        hU.copy_(dG, non_blocking=True)
        hV.copy_(dV, non_blocking=True)
        hD.copy_(dD, non_blocking=True)
        torch.cuda.synchronize()
        if k >= args.warmup:
            e2e_t.append(time.perf_counter() - t0)
    e2e_v, _ = replica_throughput(sum(e2e_t) * 1000.0, args.steps * nmat, world, dev)
    e2e = {"value": e2e_v, "unit": "matrices/s", "h2d_bytes_per_step": G0.numel() * 8,
           "d2h_bytes_per_step": 2 * G0.numel() * 8 + dD.numel() * 8, "api": "gjx_hypJacL2_batched"}

    line = {"metric": cfg["metric"], "value": value, "unit": "matrices/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "strong" if (args.shard and world > 1) else "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": cfg["workload"], "name": "c5", "count": nmat, "alg": ALG,
                       "block_pairs_per_cta": width,
                       "launches": "one per sweep" if tuned["mode"] else "one per outer step index",
                       "parallelism": ("one batch partitioned over ranks (size-balanced)" if (args.shard and world > 1)
                                       else "independent batches per rank" if world > 1 else "single GPU"),
                       "l2": "flushed between steps (256 MiB write, outside the timed events); inputs 3.4 GB > L2"},
            "sweeps_max": max(res.sweeps), "sweeps_mean": float(np.mean(res.sweeps)),
            "block_pair_steps": pair_steps,
            "us_per_block_pair_step_per_sm": statistics.median(times) * 1000.0 * 148 / max(1, pair_steps),
            "e2e": e2e, "roofline": roof,
            "clocks": clk, "gpu_launches": prof["launches"] // max(1, args.steps), "step_ms": times}
    if rank == 0 and world == 1 and not args.no_cpu:
        line["plain_loop"] = plain_loop_sample(Gs, Vs, Ds, G0, offs, sizes, nplus)
        line["cpu_baseline"] = batch_cpu_sample(sizes, cfg["seed"])
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def plain_loop_sample(Gs, Vs, Ds, G0, offs, sizes, nplus, per_size: int = 8):
    """The single-matrix device call looped over a stratified sample of the
    batch (per_size matrices of each n), scaled to the whole batch."""
    import torch
    import gpujachx_b200 as g
    tot = 0.0
    by = {}
    for n in sorted(set(int(x) for x in sizes)):
        idx = np.nonzero(sizes == n)[0][:per_size]
        g.init_strats(None, "cycwor", 32, "cycwor", n // 16)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for b in idx:
            Gs[b].view(-1).copy_(G0[int(offs[b]):int(offs[b + 1])])
            g.hypJacL2_dev(ALG, Gs[b], nplus[b], Vs[b], Ds[b])
        torch.cuda.synchronize()
        per = (time.perf_counter() - t0) / len(idx)
        by[n] = per
        tot += per * int((sizes == n).sum())
    g.init_strats(None, "cycwor", 32, "cycwor", 4)
    return {"value": len(sizes) / tot, "unit": "matrices/s", "seconds_per_matrix_by_n": by,
            "sample": f"{per_size} matrices of each n through gjx_hypJacL2_dev, scaled to the batch"}


def main_split(args):
    """The split-precision form (gjx_hypJacL2_split) on a single-matrix
    workload: device-resident value, e2e with the host copies, the roofline
    of its update kernel (HBM-bound; the int8 tensor work per launch is given
    beside it), accuracy against the FP64 reference spectrum and the plain
    form's result on request (--accuracy)."""
    import torch
    import gpujachx_b200 as g
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    g.init_strats(None, "cycwor", 32, "cycwor", N1)
    G0 = _input()
    G0d = torch.tensor(np.ascontiguousarray(G0.T), dtype=torch.float64, device=dev)
    dG = torch.empty_like(G0d)
    full = bool(ALG & 2)
    dV = torch.empty((N, N), dtype=torch.float64, device=dev)
    dD = torch.empty(N, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        dG.copy_(G0d)
        return g.hypJacL2_split(ALG, dG, NPLUS, dV, dD)[1]

    for _ in range(args.warmup):
        sweeps = step()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    g.profile(True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sweeps = step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    prof = g.profile_read()
    g.profile(False)
    clk = clocks.stop()
    value, total_ms = replica_throughput(sum(times), args.steps, world, dev)
    pairs = N // 64
    tiles = (M + 127) // 128 + ((N + 127) // 128 if full else 0)
    upd_bytes = pairs * (M + (N if full else 0)) * 64 * 8 * 2       # each tile read and written once
    upd_ops = pairs * tiles * 72 * 128 * 64 * 32 * 2                  # int8 multiply-adds x 2
    upd_s = prof["l1_ms"] / max(1, prof["l1_launches"]) / 1000.0
    hbm, peak_kind = _peaks()
    steps1 = pairs * 2 - 1
    fp64_flop = steps1 * pairs * (2 * M * 64 * 64 + 2 * (M + (N if full else 0)) * 64 * 64) * sweeps
    roof = {"bound": "hbm", "achieved": upd_bytes / upd_s / 1e9, "peak": hbm, "unit": "GB/s",
            "frac": upd_bytes / upd_s / 1e9 / hbm, "traffic": None,
            "kernel": "gjx::split::sp_update_kernel<%s>" % ("true" if full else "false"),
            "peak_kind": f"{peak_kind} HBM copy bandwidth", "per": "update launch (one per outer step), event time",
            "launch_ms": upd_s * 1000.0, "launches": prof["l1_launches"],
            "algorithmic_bytes_per_launch": upd_bytes, "int8_tensor_ops_per_launch": upd_ops,
            "int8_tops": upd_ops / upd_s / 1e12,
            "fp64_equivalent_tflops_whole_call": fp64_flop / (statistics.median(times) / 1000.0) / 1e12}
    # e2e: pinned host input, H2D + the split call + D2H of U, V, D
    hin = torch.empty((N, M), dtype=torch.float64, pin_memory=True)
    hin.copy_(G0d)
    hU = torch.empty_like(hin, pin_memory=True)
    hV = torch.empty((N, N), dtype=torch.float64, pin_memory=True)
    hD = torch.empty(N, dtype=torch.float64, pin_memory=True)
    e2e_t = []
    for k in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dG.copy_(hin, non_blocking=True)
        g.hypJacL2_split(ALG, dG, NPLUS, dV, dD)
        hU.copy_(dG, non_blocking=True)
        if full:
            hV.copy_(dV, non_blocking=True)
        hD.copy_(dD, non_blocking=True)
        torch.cuda.synchronize()
        if k >= args.warmup:
            e2e_t.append(time.perf_counter() - t0)
    e2e_v, _ = replica_throughput(sum(e2e_t) * 1000.0, args.steps, world, dev)
    e2e = {"value": e2e_v, "unit": "matrices/s", "h2d_bytes_per_step": M * N * 8,
           "d2h_bytes_per_step": M * N * 8 + (N * N * 8 if full else 0) + N * 8,
           "api": "gjx_hypJacL2_split (pinned host buffers, H2D and D2H around it)"}
    line = {"metric": METRIC, "value": value, "unit": "matrices/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 (int8 slices on the tensor cores)",
            "data": "synthetic",
            "config": dict(CONFIG, form="split-precision (blocks of 32, pairs of 64, 8 int8 digits per entry)",
                           parallelism=("replicas" if world > 1 else "single GPU")),
            "sweeps": sweeps, "e2e": e2e, "roofline": roof, "clocks": clk, "gpu_launches": prof["launches"],
            "step_ms": times}
    if rank == 0 and args.accuracy:
        line["accuracy"] = accuracy_figures(G0, dG.cpu().numpy().T, dV.cpu().numpy().T if full else None,
                                            dD.cpu().numpy())
        # the plain form on the same input, for the same figures
        g.init_strats(None, "cycwor", 32, "cycwor", N1)
        dG.copy_(G0d)
        t0 = time.perf_counter()
        _, sw_p, _, _ = g.hypJacL2_dev(ALG, dG, NPLUS, dV, dD)
        torch.cuda.synchronize()
        line["plain_form"] = {"seconds": time.perf_counter() - t0, "sweeps": sw_p,
                              "accuracy": accuracy_figures(G0, dG.cpu().numpy().T,
                                                           dV.cpu().numpy().T if full else None, dD.cpu().numpy())}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baselines")
    ap.add_argument("--config", default="c2", choices=sorted(WORKLOADS), help="workload (default: the headline c2)")
    ap.add_argument("--accuracy", action="store_true", help="add pp80 figures of the last decomposition")
    ap.add_argument("--shard", action="store_true", help="c5 over N ranks: split one batch instead of N batches")
    ap.add_argument("--count", type=int, default=0, help="c5: matrices in the batch (default 4096; profiling runs)")
    ap.add_argument("--pairs-per-cta", type=int, default=0, choices=[0, 1, 2, 3, 4],
                    help="c5: fix the batched form (per-step launches) instead of the autotuner's pick")
    ap.add_argument("--alg", type=int, default=-1, help="override the workload's ALG (studies; the config says so)")
    ap.add_argument("--form", default="plain", choices=["plain", "split"],
                    help="plain FP64 (the drop-in) or the split-precision form (gjx_hypJacL2_split)")
    args = ap.parse_args()
    _use(args.config)
    if args.alg >= 0 and args.alg != ALG:
        WORKLOADS[args.config] = dict(WORKLOADS[args.config], alg=args.alg,
                                      workload=WORKLOADS[args.config]["workload"] + f"; ALG {args.alg} instead")
        _use(args.config)
    if args.impl == "reference":
        return reference_arm(args)
    if args.config == "c5":
        return main_batch(args)
    if args.form == "split":
        return main_split(args)

    import torch
    import torch.distributed as dist
    import gpujachx_b200 as g
    from gpujachx_b200 import synth

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    g.init_strats(None, "cycwor", 32, "cycwor", N1)
    if os.environ.get("GJX_SWEEP_MODE") == "0":  # one launch per outer step (profilers cannot replay the sweep launch)
        g.lib().gjx_set_sweep_mode(0)
    tuned = g.autotune(ALG, M, N, NPLUS, sweeps=1)  # the library's autotuner, once per shape, before timing
    G0 = _input()
    dev = torch.device("cuda", local)
    # device layout: row j of the (N, M) tensor = column j of G
    G0d = torch.tensor(np.ascontiguousarray(G0.T), dtype=torch.float64, device=dev)
    dG = torch.empty_like(G0d)
    dV = torch.empty((N, N), dtype=torch.float64, device=dev)
    dD = torch.empty(N, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        dG.copy_(G0d)
        ret, swp, s, b = g.hypJacL2_dev(ALG, dG, NPLUS, dV, dD, stream=None)
        return swp

    for _ in range(args.warmup):
        sweeps = step()
    torch.cuda.synchronize()

    clocks = Clocks(local)
    clocks.start()
    g.profile(True)
    barrier()
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sweeps = step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    barrier()
    prof = g.profile_read()
    g.profile(False)
    clk = clocks.stop()
    value, total_ms = replica_throughput(sum(times), args.steps, world, dev)

    # roofline of the block-pair kernel (one launch per sweep when it fits: fewer launches than steps)
    one_launch = prof["launches"] < prof["l1_launches"]
    l1_mean_s = prof["l1_ms"] / max(1, prof["l1_launches"]) / 1000.0
    hbm, peak_kind = _peaks()
    ach = BYTES_PER_PAIR * PAIRS / l1_mean_s / 1e9
    flops = FLOP_PER_PAIR * PAIRS / l1_mean_s / 1e12
    roof = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
            "traffic": RECORDED_TRAFFIC.get(args.config),
            "kernel": "gjx::%s<%s,%s,%d>" % ("l1_sweep_kernel" if one_launch else "l1_step_kernel",
                                             "true" if ALG & 1 else "false", "true" if ALG & 2 else "false",
                                             tuned["split"]),
            "peak_kind": f"{peak_kind} HBM copy bandwidth",
            "per": ("outer step: a sweep launch's event time over its outer steps" if one_launch
                    else "outer-step launch, event time"),
            "launch_ms": l1_mean_s * 1000.0, "launches": prof["l1_launches"],
            "algorithmic_bytes_per_launch": BYTES_PER_PAIR * PAIRS,
            "algorithmic_flop_per_launch": FLOP_PER_PAIR * PAIRS, "fp64_tflops": flops,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of this "
                              "workload (cold L2), recorded from one capture (bench.RECORDED_TRAFFIC)"}

    # e2e through the public host API (pinned buffers, H2D + D2H inside)
    pin = torch.empty((N, M), dtype=torch.float64, pin_memory=True).numpy().T  # Fortran view
    pinV = torch.empty((N, N), dtype=torch.float64, pin_memory=True).numpy().T
    pinD = torch.empty(N, dtype=torch.float64, pin_memory=True).numpy()
    import ctypes
    pd = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    e2e_times = []
    L = g.lib()
    for k in range(args.warmup + args.steps):
        pin[...] = G0
        sw, rs, rb = ctypes.c_uint(), ctypes.c_ulonglong(), ctypes.c_ulonglong()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ret = L.hypJacL2(ALG, M, N, NPLUS, pd(pin), M, pd(pinV) if ALG & 2 else None, N if ALG & 2 else 0, pd(pinD),
                         ctypes.byref(sw), ctypes.byref(rs), ctypes.byref(rb), None)
        dt = time.perf_counter() - t0
        assert ret == 0, g.last_error()
        if k >= args.warmup:
            e2e_times.append(dt)
    e2e_value, _ = replica_throughput(sum(e2e_times) * 1000.0, args.steps, world, dev)
    e2e = {"value": e2e_value, "unit": "matrices/s", "h2d_bytes_per_step": M * N * 8,
           "d2h_bytes_per_step": M * N * 8 + (N * N * 8 if ALG & 2 else 0) + N * 8,
           "api": "hypJacL2 (host buffers, pinned)"}

    line = {"metric": METRIC, "value": value, "unit": "matrices/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(CONFIG, parallelism=("replicas" if world > 1 else "single GPU")),
            "sweeps": sweeps, "e2e": e2e, "roofline": roof, "clocks": clk,
            "tuned": {"ctas_per_pair": tuned["split"], "one_launch_per_sweep": bool(tuned["mode"])},
            "gpu_launches": prof["launches"], "step_ms": times}
    if rank == 0 and args.accuracy:
        line["accuracy"] = accuracy_figures(G0, dG.cpu().numpy().T, dV.cpu().numpy().T if ALG & 2 else None,
                                            dD.cpu().numpy())
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_port_sample(G0, sweeps)
        if NPLUS == N and M * N > 2 ** 25:
            line["lapack_dgesvj"] = {"skipped": "DGESVJ on the host takes about an hour at this size"}
        elif NPLUS == N:
            try:
                line["lapack_dgesvj"] = lapack_baseline(G0)
            except Exception as e:  # noqa: BLE001
                line["lapack_dgesvj"] = {"error": str(e)[:200]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
