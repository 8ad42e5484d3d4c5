#!/usr/bin/env python3
"""Benchmark of the GMRES-IR hot path on the B200.

Workloads (--config), seeded synthetic KKT systems K = [[H, A^T], [A, -delta I]]
from mpir_b200.kkt / mpir_b200.stream (the reference measures only on
SuiteSparse matrices, which are not available; these stand in with the
configured shapes and value distributions):

  stream   (default) the serving stream: requests with Poisson arrivals, each
           a 2-D or 3-D system with n log-uniform in [1e3, 5e5] and m ~ n1/4,
           60% a new right-hand side on a factor used before, 30% new values
           on a pattern used before, 10% a new pattern; 150 GB admission
           budget (150e9 bytes), 4 workers; backward error <= 1e-14.  One
           step = 8 requests of the stream (--requests-per-step).  `value` = solves/s of the serving engine
           (mpir_server_*) on the stream at a saturating arrival rate;
           `drop_in` = the same requests served one at a time through the
           drop-in GmresLDLIR (Compute + Solve per request, as the
           reference's example driver does); latencies p50/p99 at the
           saturating rate and at half the served capacity.
  grid3d   one drop-in solve per step of a new value set on the analysed
           n = 138,240 3-D system (7-point Laplacian 48^3 + 1e-2 I, 27,648
           constraint rows x 6 N(0,1), delta 1e-6): float32 LDL^T
           refactorization + float64 GMRES-IR, 1 right-hand side.
  small2d  the same step on the n = 1,280 2-D system (32^2, 256 rows x 4,
           delta 1e-4); the reference arm runs its full GMRES-IR here.
  batch2d  64 instances on one 256^2 pattern (H + diag(s), s log-uniform
           in [1e-6, 1e2], 16,384 rows x 4, delta 1e-8), 16 right-hand sides
           each: one analysis, then per step a group of --group instances
           refactorized by one graph launch and their 16 right-hand sides
           each solved in lockstep.
  illcond3d the precision tier: D L3D(grid^3) D + 1e-8 I, D log-uniform in
           [1e-3, 1e3], 8 entries per constraint row, delta 1e-8.

--impl reference runs the reference's CPU code (oracle/_ref, the
reference's own headers compiled unmodified) on the host cores instead, on
the permuted matrices of oracle/fixtures (no code of this repository's
library is loaded in that arm).  Multi-GPU: independent replicas, one
workload per rank, no collective on the data path ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

T_START = time.perf_counter()

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s + p50/p99 latency @ bwd err≤1e-14: served mixed vs drop-in, 1 B200"
UNIT = "solves/s"
BE_TOL = 1e-14
FIXTURES = os.path.join(ROOT, "oracle", "fixtures")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mpir", choices=["mpir", "reference"])
    ap.add_argument("--config", default="stream",
                    choices=["stream", "grid3d", "small2d", "batch2d", "illcond3d"])
    ap.add_argument("--grid", type=int, default=None, help="grid of grid3d / illcond3d")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-budget", type=float, default=12.0,
                    help="seconds of reference factor sampling for the CPU baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--uf", default=None, choices=["f32", "bf16", "f16"],
                    help="factor precision (default f32)")
    ap.add_argument("--gmres-iter", type=int, default=None)
    ap.add_argument("--ir-iter", type=int, default=None)
    # serving stream
    ap.add_argument("--requests-per-step", type=int, default=8)
    ap.add_argument("--workers", type=int, default=4)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--no-latency-pass", action="store_true")
    ap.add_argument("--no-dropin", action="store_true")
    ap.add_argument("--group", type=int, default=8, help="batch2d: instances per graph launch")
    ap.add_argument("--update", default=None, choices=["default", "tf32x3", "bf16x3"],
                    help="trailing-update engine of float32 factors")
    return ap.parse_args()


def load_peaks():
    """HBM GB/s and dense bf16 TFLOP/s.  The updates run inside a long step,
    so the sustained bf16 figure is the one they are held against."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        bf16 = d.get("bf16_tflops_sustained", d.get("bf16_tflops", 1590.0))
        return d.get("hbm_gbs", 6650.0), bf16, "measured (bf16 sustained)"
    return 6650.0, 1590.0, "fallback"


def gemm_traffic(grid, uf):
    """DRAM bytes per launch of the tensor-core update kernel, from the ncu
    capture summarised under profiles/ (the grid3d-48 float32 workload)."""
    if grid != 48 or uf != "f32":
        return None
    path = os.path.join(ROOT, "profiles", "k_gemm_tc_grid3d48_dram.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":")[1])
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1].split()[0]))
                mx = float(f[2].split()[0])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------
# Replicas

def rank_max(pg, v, device):
    """Max of v over the ranks of process group module pg (None: one rank)."""
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def rank_sum(pg, v, device):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def aggregate_rate(world, steps, max_ms):
    """Whole-job solves/s: every rank solves `steps` systems of its own; the
    job takes the slowest rank's time."""
    return world * steps / (max_ms / 1e3)


def replica_seed(seed, rank):
    """Each rank (replica) solves its own seeded workload."""
    return seed + rank


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_dist(local):
    import torch
    rank, world, _ = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return pg, torch.device("cuda", local)


# ----------------------------------------------------------------------------
# Workloads

def system_for(args, rank=0):
    from mpir_b200 import kkt
    seed = replica_seed(args.seed, rank)
    if args.config == "small2d":
        return kkt.small2d(seed=seed), "small2d: KKT n=1280 (5-point Laplacian 32^2 + 1e-2 I, " \
            "256 constraint rows x 4 N(0,1), delta 1e-4)"
    if args.config == "illcond3d":
        g = args.grid or 64
        n1 = g ** 3
        return kkt.illcond3d(seed=seed, grid=g), (
            f"illcond3d-{g}: KKT n={n1 + n1 // 4} (D L3D({g}^3) D + 1e-8 I, D log-uniform in "
            f"[1e-3, 1e3], {n1 // 4} constraint rows x 8, delta 1e-8)")
    g = args.grid or 48
    n1 = g ** 3
    return kkt.grid3d(seed=seed, grid=g), (
        f"grid3d-{g}: KKT n={n1 + n1 // 4} (7-point Laplacian {g}^3 + 1e-2 I, {n1 // 4} "
        f"constraint rows x 6 N(0,1), delta 1e-6)")


# ----------------------------------------------------------------------------
# CPU path of the reference (oracle/_ref), bounded samples.

def fixture_perm(name):
    p = os.path.join(FIXTURES, f"perm_{name}.npy")
    return np.load(p).astype(np.int64) if os.path.exists(p) else None


def reference_cpu_estimate(s, perm, counts, budget, log=print, keep_factor=False):
    """Seconds for one drop-in solve by the reference's CPU code on P K P^T.

    * factor: QDLDL_factor<float> (the reference's code) timed on the leading
      k x k block of the scaled, permuted matrix, k chosen so the sample takes
      about `budget` seconds; the up-looking factor computes row r from rows
      < r only, so the sample is exactly the first k rows of the full factor.
      Its rate (multiply-subtract updates per second, counted row by row by
      the oracle's walk of the same tree) extrapolates to all n rows.
    * solve: the reference's QDLDL_solve on the sampled factor gives seconds
      per factor entry; one GMRES-IR solve applies it counts['applies'] times
      to nnz(L) entries, plus counts['spmv'] MatrixMultiply at full size.
    With keep_factor the sampled factor (k, Lp, Li, Lx, D) comes back too."""
    import oracle

    R = oracle.Reference()
    O = oracle.Oracle()
    Cp, Ci, Cx = oracle.permuted_scaled_upper(O, s.n, s.Ap, s.Ai, s.Ax, perm)
    n = s.n
    w = O.row_work(n, Cp, Ci)
    W = np.cumsum(w)
    total_work = float(W[-1])
    _, Lnz, _ = O.etree(n, Cp, Ci)
    nnzL = float(Lnz.sum())
    k = int(np.searchsorted(W, min(2e8, total_work)))
    k = max(min(k, n), 16)
    t0 = time.perf_counter()
    R.factor(k, Cp, Ci, Cx)
    t = time.perf_counter() - t0
    rate = max(W[k - 1], 1.0) / max(t, 1e-6)
    target = rate * budget
    k = int(np.searchsorted(W, min(target, total_work)))
    k = max(min(k, n), 16)
    t0 = time.perf_counter()
    st, Lp, Li, Lx, D, Dinv = R.factor(k, Cp, Ci, Cx)
    t_fac = time.perf_counter() - t0
    work_k = float(W[k - 1])
    rate = work_k / max(t_fac, 1e-9)
    t_factor_full = total_work / rate
    nnz_k = float(Lp[k])
    rhs = np.ones(k)
    t0 = time.perf_counter()
    reps = 0
    while True:
        R.solve(k, Lp, Li, Lx, Dinv, rhs)
        reps += 1
        if time.perf_counter() - t0 > 1.0 or reps >= 50:
            break
    t_solve_k = (time.perf_counter() - t0) / reps
    per_entry = t_solve_k / max(2 * nnz_k + k, 1.0)
    t_apply = per_entry * (2 * nnzL + n)
    x = np.ones(n)
    t0 = time.perf_counter()
    R.matmul(n, s.Ap, s.Ai, s.Ax, x)
    t_spmv = time.perf_counter() - t0
    total = t_factor_full + counts["applies"] * t_apply + counts["spmv"] * t_spmv
    log(f"cpu sample: k={k}/{n} rows, {t_fac:.2f}s for {work_k:.3e} updates "
        f"({rate:.3e}/s); full factor {t_factor_full:.1f}s; apply {t_apply:.3f}s; "
        f"spmv {t_spmv:.4f}s; solve total {total:.1f}s")
    det = {"k": k, "factor_sample_s": t_fac, "rate_updates_per_s": rate,
           "factor_full_s_extrapolated": t_factor_full, "apply_s": t_apply,
           "seconds_per_entry": per_entry, "spmv_s": t_spmv, "work_total": total_work,
           "nnzL": nnzL}
    if keep_factor:
        det["factor"] = (k, Lp, Li, Lx, D)
        # the reference's float64 factor of the same leading block: how far
        # each float32 factor is from the exact one
        st64, Lp64, Li64, Lx64, D64, _ = R.factor(k, Cp, Ci, Cx, np.float64)
        det["factor64"] = (Lx64, D64) if st64 >= 0 else None
    return total, det


def _ref_worker(payload):
    """One worker of the parallel reference sample (spawn-started process):
    the reference's QDLDL_factor<float> on the leading k rows, then its
    QDLDL_solve on that factor; returns (factor seconds, solve seconds)."""
    k, Cp, Ci, Cx, solve_reps = payload
    import oracle
    R = oracle.Reference()
    t0 = time.perf_counter()
    st, Lp, Li, Lx, D, Dinv = R.factor(k, Cp, Ci, Cx)
    t_fac = time.perf_counter() - t0
    rhs = np.ones(k)
    t0 = time.perf_counter()
    for _ in range(solve_reps):
        R.solve(k, Lp, Li, Lx, Dinv, rhs)
    return t_fac, (time.perf_counter() - t0) / solve_reps


def _ref_full_worker(payload):
    """One worker of the full reference runs (spawn-started process): the
    reference's QDLDL_etree + QDLDL_factor<float> + GmresLDLIR<float,double,
    double>::Solve preconditioned by that factor, repeated for `seconds`.
    Returns (solves, seconds of those three phases, last x): the harness
    times each phase itself, leaving out the shipped Compute it runs only for
    the diagonal scaling (its FGPILU sweep is not on this path)."""
    n, Cp, Ci, Cx, bp, seconds = payload
    import oracle
    R = oracle.Reference()
    t0 = time.perf_counter()
    count, x, busy = 0, None, 0.0
    while True:
        x, AD, info, _, _ = R.gmres_ir_with_factor(n, Cp, Ci, Cx, bp)
        busy += info["etree_s"] + info["factor_s"] + info["solve_s"]
        count += 1
        if time.perf_counter() - t0 >= seconds:
            break
    return count, busy, x


def host_cores():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


def reference_counts(seed):
    """Preconditioner applications and SpMVs per solve of the reference's
    GMRES-IR, measured with its restated driver (bit-exact with the
    reference) on a smaller system from the same generator."""
    import oracle
    from mpir_b200 import kkt
    s = kkt.grid3d(seed=seed, grid=12)
    x, st = oracle.Oracle().gmres_ir(s.n, s.Ap, s.Ai, s.Ax, s.b, form=0)
    return {"applies": st["precond_applies"], "spmv": st["spmv"],
            "ir_steps": st["ir_steps"], "sample_n": s.n}


def reference_line(args, value, cores, kind_sample, detail, workload, lat_ms=None):
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 / value if value else None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 factor / f64 solve",
        "data": "synthetic", "config": {"workload": workload},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": kind_sample, "detail": detail},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if lat_ms is not None:
        line["latency_ms"] = {"p50": float(np.percentile(lat_ms, 50)),
                              "p99": float(np.percentile(lat_ms, 99))}
    # Whether value and ms_per_step were timed in full in this run, or
    # extrapolated from timed samples (then ms_per_step is the model's, not
    # this run's wall clock, which is given beside it).
    line["measured"] = not bool(isinstance(detail, dict) and detail.get("extrapolated"))
    line["wall_seconds"] = time.perf_counter() - T_START
    return line


def ref_small2d(args):
    """The reference's full GMRES-IR (QDLDL_etree, QDLDL_factor<float>,
    GmresLDLIR::Solve) on the n = 1,280 system, measured end to end with no
    extrapolation: every host core runs solves for a bounded time."""
    import multiprocessing as mpr

    import oracle
    from mpir_b200 import kkt
    s = kkt.small2d(seed=args.seed)
    perm = fixture_perm("small2d_s0") if args.seed == 0 else None
    if perm is None:
        perm = np.arange(s.n)
    import scipy.sparse as sp
    cols = np.repeat(np.arange(s.n), np.diff(s.Ap))
    K = sp.coo_matrix((s.Ax, (s.Ai, cols)), shape=(s.n, s.n)).tocsc()
    K = (K + sp.triu(K, 1).T).tocsr()
    U = sp.triu(K[perm][:, perm], format="csc")
    U.sort_indices()
    Cp, Ci, Cx = (U.indptr.astype(np.int64), U.indices.astype(np.int64),
                  U.data.astype(np.float64))
    bp = s.b[perm]
    cores = host_cores()
    per_step = float(np.clip(120.0 / max(args.steps + args.warmup, 1), 1.0, 10.0))
    rates, lat = [], []
    with mpr.get_context("spawn").Pool(cores) as pool:
        for i in range(args.warmup + args.steps):
            res = pool.map(_ref_full_worker, [(s.n, Cp, Ci, Cx, bp, per_step)] * cores)
            if i >= args.warmup:
                # every core serves its own solves: the sum of the per-core rates
                rates.append(sum(r[0] / r[1] for r in res))
                lat += [1e3 * r[1] / r[0] for r in res]
            xr = np.empty(s.n)
            xr[perm] = res[0][2]
    be = kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, xr, s.b)
    value = float(np.mean(rates))
    line = reference_line(
        args, value, cores,
        f"every step {cores} concurrent processes each run the reference's full GMRES-IR "
        f"(QDLDL_etree + QDLDL_factor<float> + GmresLDLIR::Solve, each phase timed) on the "
        f"permuted n={s.n} system for {per_step:.1f}s; measured, no extrapolation",
        {"backward_error": be, "forward_error": kkt.forward_error(xr, s.x_true),
         "seconds_per_step": per_step}, system_for(args)[1] + "; per step f32 LDL^T "
        "factorization + f64 GMRES-IR solve, 1 RHS", lat)
    print(json.dumps(line), flush=True)


def ref_grid3d(args):
    """The reference's QDLDL_factor<float> on a leading block of the permuted
    n = 138,240 system (its factor of the full system takes hours on one
    core), extrapolated by the per-row update counts; solves and SpMV scaled
    by the measured per-entry rates.  Every host core runs the sample at once
    (the path is sequential within a solve, so cores serve independent
    solves)."""
    import multiprocessing as mpr

    import oracle
    import psutil
    from mpir_b200 import kkt
    s, workload = system_for(args)
    perm = fixture_perm("grid3d48_s0") if (args.grid or 48) == 48 and args.seed == 0 else None
    if perm is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "no permutation fixture for this grid/seed (oracle/fixtures)"}))
        return
    counts = reference_counts(args.seed)
    O = oracle.Oracle()
    Cp, Ci, Cx = oracle.permuted_scaled_upper(O, s.n, s.Ap, s.Ai, s.Ax, perm)
    n = s.n
    W = np.cumsum(O.row_work(n, Cp, Ci))
    _, Lnz, _ = O.etree(n, Cp, Ci)
    budget = float(np.clip(150.0 / max(args.steps + args.warmup, 1), 2.0, args.cpu_budget))
    k0 = max(min(int(np.searchsorted(W, min(1e8, float(W[-1])))), n), 16)
    t0 = time.perf_counter()
    oracle.Reference().factor(k0, Cp, Ci, Cx)
    rate1 = max(W[k0 - 1], 1.0) / max(time.perf_counter() - t0, 1e-6)
    k = max(min(int(np.searchsorted(W, min(rate1 * budget, float(W[-1])))), n), 16)
    per_worker = 16.0 * float(Lnz[:k].sum()) + 64.0 * k
    cores = host_cores()
    workers = max(1, min(cores or 1, int(0.5 * psutil.virtual_memory().available / per_worker)))
    rates, dets = [], []
    for i in range(args.warmup + args.steps):
        with mpr.get_context("spawn").Pool(workers) as pool:
            res = pool.map(_ref_worker, [(k, Cp, Ci, Cx, 1)] * workers)
        t_fac = float(np.mean([r[0] for r in res]))
        t_sol = float(np.mean([r[1] for r in res]))
        rate = float(W[k - 1]) / max(t_fac, 1e-9)
        nnz_k = float(Lnz[:k].sum()) + k
        t_apply = t_sol / max(2 * nnz_k + k, 1.0) * (2 * float(Lnz.sum()) + n)
        x = np.ones(n)
        t1 = time.perf_counter()
        oracle.Reference().matmul(n, s.Ap, s.Ai, s.Ax, x)
        t_spmv = time.perf_counter() - t1
        per_solve = float(W[-1]) / rate + counts["applies"] * t_apply + counts["spmv"] * t_spmv
        print(f"reference on {workers} cores: k={k}/{n}, factor sample {t_fac:.2f}s, "
              f"one solve {per_solve:.1f}s per core", file=sys.stderr)
        if i >= args.warmup:
            rates.append(workers / per_solve)
            dets.append({"k": k, "workers": workers, "factor_sample_s": t_fac,
                         "rate_updates_per_s_per_core": rate,
                         "seconds_per_solve_per_core": per_solve, "extrapolated": True})
    value = float(np.mean(rates))
    line = reference_line(
        args, value, workers,
        "extrapolated: per step, %d concurrent processes each run the reference's "
        "QDLDL_factor<float> on the leading %d of %d rows (~%.0fs) and QDLDL_solve on that "
        "factor; scaled by update and entry counts to one full GMRES-IR solve"
        % (workers, k, n, budget), dets[-1], workload + "; per step f32 LDL^T "
        "refactorization + f64 GMRES-IR solve, 1 RHS", [workers / r * 1e3 for r in rates])
    print(json.dumps(line), flush=True)


def stream_reference_model(nreq, seed, rates, applies, workers, facts_path=None):
    """Seconds the reference's CPU path needs for each request of the serving
    stream served one at a time (etree, QDLDL_factor<float> and a GMRES-IR
    solve of `applies` preconditioner applications per request; the
    reference has no cache, so every request factors), from the per-pattern
    symbolic facts of oracle/fixtures and measured per-core rates."""
    from mpir_b200 import stream as smod
    facts = json.load(open(facts_path or os.path.join(FIXTURES, "stream_facts.json")))
    by_pid = {f["pattern"]: f for f in facts["patterns"]}
    st = smod.Stream(nreq, rate=1e3, seed=seed)
    secs = []
    for r in st.requests:
        f = by_pid[r.pattern]
        t = (f["factor_updates"] / rates["updates_per_s"]
             + applies * (2 * f["nnz_L"] + f["n"]) * rates["seconds_per_entry"]
             + (applies + 3) * f["nnz_upper"] * rates["spmv_seconds_per_entry"])
        secs.append(t)
    return np.array(secs)


def ref_stream(args):
    """The reference's CPU path on the serving stream, as a model: per-core
    rates of QDLDL_factor<float>, QDLDL_solve and MatrixMultiply measured on
    a bounded sample (the leading rows of the permuted n = 138,240 system),
    applied to each request's own update and entry counts; every host core
    serves requests one at a time."""
    import oracle
    from mpir_b200 import kkt
    nreq = args.requests_per_step * args.steps
    s = kkt.grid3d(seed=0)
    perm = fixture_perm("grid3d48_s0")
    counts = reference_counts(args.seed)
    budget = float(np.clip(60.0 / max(args.steps, 1), 2.0, args.cpu_budget))
    _, det = reference_cpu_estimate(s, perm, counts, budget,
                                    log=lambda *a: print(*a, file=sys.stderr))
    R = oracle.Reference()
    x = np.ones(s.n)
    t0 = time.perf_counter()
    for _ in range(5):
        R.matmul(s.n, s.Ap, s.Ai, s.Ax, x)
    spmv_e = (time.perf_counter() - t0) / 5 / s.nnz
    rates = {"updates_per_s": det["rate_updates_per_s"],
             "seconds_per_entry": det["seconds_per_entry"], "spmv_seconds_per_entry": spmv_e}
    secs = stream_reference_model(nreq, args.seed, rates, counts["applies"], 1)
    cores = host_cores()
    value = cores * len(secs) / float(secs.sum())
    line = reference_line(
        args, value, cores,
        "extrapolated: per-core rates of the reference's QDLDL_factor<float> (leading %d rows "
        "of the permuted n=138240 system, %.1fs), QDLDL_solve and MatrixMultiply, applied to "
        "each of the %d stream requests' own update and entry counts (oracle/fixtures); "
        "%d cores serving requests one at a time" % (det["k"], det["factor_sample_s"], nreq,
                                                      cores),
        {"rates": rates, "applies_per_solve": counts["applies"],
         "seconds_total_one_core": float(secs.sum()), "extrapolated": True},
        stream_workload(args, nreq), 1e3 * secs)
    print(json.dumps(line), flush=True)


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    {"small2d": ref_small2d, "grid3d": ref_grid3d, "stream": ref_stream}.get(
        args.config, lambda a: print(json.dumps(
            {"impl": "reference", "unavailable": f"no reference arm for --config {a.config}; "
             "it runs for stream, grid3d and small2d"})))(args)


# ----------------------------------------------------------------------------
# GPU arms

def roofline_from_classes(info, kt, applies, uf, grid=None):
    hbm, bf16, peak_kind = load_peaks()
    cls_ms = {k: v[0] for k, v in kt.items()}
    dom = max(cls_ms, key=cls_ms.get)
    work = {
        "trailing_update": ("tensor", info["update_flops"] / 1e12, "TFLOP/s", bf16),
        "panel_solve": ("tensor", info["trsm_flops"] / 1e12, "TFLOP/s", bf16),
        "solve_forward": ("hbm", applies * info["panel_read_bytes"] / 1e9, "GB/s", hbm),
        "solve_backward": ("hbm", applies * info["panel_read_bytes"] / 1e9, "GB/s", hbm),
    }
    bound, amount, unit, peak = work.get(dom, ("hbm", float("nan"), "GB/s", hbm))
    dom_s = cls_ms[dom] / 1e3
    achieved = amount / dom_s if dom_s > 0 else float("nan")
    names = {"trailing_update": "k_gemm_tc (tensor-core updates) + k_split_reduce",
             "solve_forward": "k_fwd_fronts / k_fwd_small",
             "solve_backward": "k_bwd_fronts / k_bwd_chunks / k_bwd_small"}
    solve_ms = cls_ms.get("solve_forward", 0) + cls_ms.get("solve_backward", 0)
    solve_gbs = (2 * applies * info["panel_read_bytes"] / 1e9) / (solve_ms / 1e3) if solve_ms else None
    return {"bound": bound, "kernel": names.get(dom, dom), "class": dom, "achieved": achieved,
            "peak": peak, "unit": unit, "frac": achieved / peak, "peak_source": peak_kind,
            "traffic": gemm_traffic(grid, uf) if dom == "trailing_update" else None,
            "traffic_unit": "bytes per launch (DRAM read + write, one ncu capture)",
            "frac_of_tf32x3_ceiling": (achieved / (peak / 6.0)
                                       if dom == "trailing_update" and uf == "f32" else None),
            "solve_gbs": solve_gbs, "solve_frac_of_hbm": solve_gbs / hbm if solve_gbs else None,
            "class_ms": {k: round(v, 3) for k, v in cls_ms.items() if v > 0},
            "class_launches": {k: v[1] for k, v in kt.items() if v[1] > 0}}


def leading_parity(solver, det):
    """Relative difference between the GPU factor's leading k x k block and
    the reference's QDLDL_factor<float> of the leading k x k block of the same
    scaled, permuted matrix (QDLDL computes row r from rows < r only, so the
    two are the same rows of the same factor)."""
    import mpir_b200 as mp
    k, Lp_r, Li_r, Lx_r, D_r = det["factor"]
    Lp, Li, Lx, D = mp.export_factor_leading(solver, k)
    if not (np.array_equal(Lp, Lp_r[:k + 1]) and np.array_equal(Li, Li_r[:Lp_r[k]])):
        return {"rows": k, "pattern_equal": False, "L_rel": None}
    a, b = Lx.astype(np.float64), Lx_r[:Lp_r[k]].astype(np.float64)
    da, db = D.astype(np.float64), D_r[:k].astype(np.float64)

    def rel(x, y):
        return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))

    out = {"rows": k, "pattern_equal": True, "tol": 1e-5, "L_rel": rel(a, b), "D_rel": rel(da, db)}
    if det.get("factor64") is not None:
        Lx64, D64 = det["factor64"]
        out["vs_float64_factor"] = {"gpu_L": rel(a, Lx64), "gpu_D": rel(da, D64),
                                    "reference_L": rel(b, Lx64), "reference_D": rel(db, D64)}
    return out


def run_system(args):
    """grid3d / small2d / illcond3d: one refactorization + one GMRES-IR
    solve per step."""
    import torch

    import mpir_b200 as mp
    from mpir_b200 import kkt
    rank, world, local = dist_env()
    pg, dev = init_dist(local)
    uf = args.uf or "f32"

    def barrier():
        if pg is not None:
            pg.barrier()

    s, workload = system_for(args, rank)
    solver = mp.GmresLDLIR(uf=uf, device=local)
    if args.update:
        solver.set_update(args.update)
    low = uf != "f32" or args.config == "illcond3d"
    solver.SetMaxGmresIterations(args.gmres_iter or (50 if low else 10))
    solver.SetMaxIRIterations(args.ir_iter or (30 if low else 10))
    stream = torch.cuda.current_stream(dev)
    solver.set_stream(stream.cuda_stream)
    solver.analyze(s.Ap, s.Ai, s.Ax)
    info = solver.info()
    d_Ax = torch.from_numpy(s.Ax).to(dev)
    d_b = torch.from_numpy(s.b).to(dev)
    d_x = torch.empty_like(d_b)
    L = mp.lib()

    def step():
        assert solver.factor_device(d_Ax.data_ptr()) == 0
        return solver.solve_device(d_b.data_ptr(), d_x.data_ptr())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    t_all0, t_all1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = mp.launch_count()
    reps = []
    t_all0.record(stream)
    for i in range(args.steps):
        evs[i][0].record(stream)
        reps.append(step())
        evs[i][1].record(stream)
    t_all1.record(stream)
    torch.cuda.synchronize()
    launches = mp.launch_count() - launches0
    clk = clocks.stop()
    barrier()
    lat = [a.elapsed_time(b) for a, b in evs]
    total_ms = rank_max(pg, t_all0.elapsed_time(t_all1), dev)
    value = aggregate_rate(world, args.steps, total_ms)
    be = max(r["backward_error"] for r in reps)
    converged = be <= BE_TOL
    # the precision tier reports what its factor types reach; the others must
    # reach the target
    assert converged or args.config == "illcond3d", f"backward error {be} above {BE_TOL}"
    x_host = d_x.cpu().numpy()
    fe = kkt.forward_error(x_host, s.x_true)

    # end to end through the C ABI with host buffers
    h_Ax = torch.from_numpy(s.Ax).pin_memory()
    h_b = torch.from_numpy(s.b).pin_memory()
    h_x = torch.empty(s.n, dtype=torch.float64).pin_memory()
    rep = mp.Report()

    def step_e2e():
        r = L.mpir_solver_factor(solver._h, h_Ax.data_ptr())
        assert r == 0, mp.last_error()
        r = L.mpir_solver_solve(solver._h, h_b.data_ptr(), h_x.data_ptr(), mp.C.byref(rep))
        assert r == 0, mp.last_error()
        return rep.backward_error

    step_e2e()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    be_e2e = 0.0
    for _ in range(args.steps):
        be_e2e = max(be_e2e, step_e2e())
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = rank_max(pg, e0.elapsed_time(e1), dev)
    assert be_e2e <= BE_TOL or not converged
    e2e_value = aggregate_rate(world, args.steps, e2e_ms)

    mp.kernel_timer(True)
    step()
    torch.cuda.synchronize()
    kt = mp.kernel_times()
    mp.kernel_timer(False)
    rep0 = reps[-1]
    applies = rep0["precond_applies"]
    roofline = roofline_from_classes(info, kt, applies, uf, args.grid or 48)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": f"{uf} factor / f64 solve",
        "data": "synthetic (seeded KKT generator, one system per rank)",
        "config": {"workload": workload + f"; per step {uf} LDL^T refactorization + f64 "
                   "GMRES-IR solve, 1 RHS", "global_batch": world, "seq_len": None,
                   "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (factor panels %.1f GB)" % (info["panel_bytes"] / 1e9)
                   if info["panel_bytes"] > 126e6 else
                   "factor smaller than L2: steps are back to back on L2-resident data"},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "backward_error_max": be, "forward_error": fe, "converged": converged,
        "stop_reason": reps[-1]["stop_reason"],
        "iterations": {"ir": rep0["ir_iterations"], "gmres": rep0["gmres_iterations"],
                       "precond_applies": applies},
        "factor_ms": rep0["factor_ms"], "solve_ms": rep0["solve_ms"],
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": s.Ax.nbytes + s.b.nbytes,
                "d2h_bytes_per_step": s.n * 8},
        "gpu_launches": launches, "clocks": clk, "roofline": roofline,
        "info": {k: info[k] for k in ("n", "nnz_L", "supernodes", "levels", "max_front")},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.config != "illcond3d":
        try:
            counts = {"applies": applies, "spmv": rep0["spmv_count"]}
            perm = solver.symbolic()["perm"]
            t, det = reference_cpu_estimate(s, perm, counts, args.cpu_budget,
                                            log=lambda *a: print(*a, file=sys.stderr),
                                            keep_factor=True)
            line["parity"] = leading_parity(solver, det)
            det.pop("factor")
            det.pop("factor64", None)
            line["cpu_baseline"] = {
                "value": 1.0 / t, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "reference QDLDL_factor<float> on the leading %d of %d rows of the "
                          "scaled permuted matrix (%.1fs), QDLDL_solve on that factor, full "
                          "MatrixMultiply; extrapolated to one solve with %d preconditioner "
                          "applications" % (det["k"], s.n, det["factor_sample_s"], applies),
                "detail": det}
        except Exception as e:  # the baseline never blocks the GPU line
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 1,
                                    "kind": "reference", "sample": f"failed: {e}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    solver.close()
    if pg is not None:
        pg.destroy_process_group()


def stream_workload(args, nreq):
    return (f"serving stream: {nreq} requests ({args.requests_per_step} per step), Poisson "
            "arrivals, 2-D/3-D KKT systems with n log-uniform in [1e3, 5e5], m ~ n1/4, "
            "60% new RHS on a factor used before / 30% new values on a pattern used before / "
            f"10% new pattern; {args.budget_gb:.0f} GB admission budget; bwd err <= 1e-14")


def failure_summary(recs):
    """Failed requests by status and message (count, first request index)."""
    out = {}
    for r in recs:
        if r["status"] != 0:
            key = f'{r["status"]}: {r.get("message", "")[:120]}'
            c = out.setdefault(key, {"count": 0, "first": r["index"], "n": r["n"]})
            c["count"] += 1
    return out


def run_stream(args):
    """The serving stream: the engine against the one-at-a-time drop-in."""
    import torch

    import mpir_b200 as mp
    from mpir_b200 import replay
    from mpir_b200 import stream as smod
    rank, world, local = dist_env()
    pg, dev = init_dist(local)
    uf = args.uf or "f32"
    low = uf != "f32"
    ir_iter = args.ir_iter or (30 if low else 10)
    gmres_iter = args.gmres_iter or (30 if low else 10)
    nreq = args.requests_per_step * args.steps
    srv_kw = dict(uf=uf, workers=args.workers, max_batch=16, update=args.update or "default",
                  budget_bytes=int(args.budget_gb * 1e9), ir_iter=ir_iter,
                  gmres_iter=gmres_iter, tol=1e-10, device=local)
    st = smod.Stream(nreq, rate=1e4, seed=replica_seed(args.seed, rank))
    arrays = replay.materialise(st)
    # warm-up: a short stream of small systems through both paths
    warm = smod.Stream(max(args.requests_per_step * args.warmup, 8), rate=1e4,
                       seed=10_000 + rank, n_range=(1e3, 2e4))
    warm_arrays = replay.materialise(warm)
    replay.served(warm, warm_arrays, check=False, **srv_kw)
    replay.dropin(warm, warm_arrays, check=False)
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    launches0 = mp.launch_count()
    summ, recs, stats = replay.served(st, arrays, progress=30, **srv_kw)
    launches = mp.launch_count() - launches0
    clk = clocks.stop()
    seconds = rank_max(pg, summ["seconds"], dev)
    completed = rank_sum(pg, summ["completed"], dev)
    value = completed / seconds
    arrivals_span = st.requests[-1].t_arrival
    lat_pass = None
    if not args.no_latency_pass:
        rate = 0.5 * summ["solves_per_s"]
        st.retime(rate, seed=replica_seed(args.seed, rank) + 7)
        lsum, lrecs, _ = replay.served(st, arrays, check=False, progress=30, **srv_kw)
        lat_pass = {"rate_per_s": rate, "p50_ms": lsum["p50_ms"], "p99_ms": lsum["p99_ms"],
                    "solves_per_s": lsum["solves_per_s"]}
        st.retime(1e4, seed=replica_seed(args.seed, rank))
    drop = None
    if not args.no_dropin:
        dsum, drecs = replay.dropin(st, arrays, uf="f32", progress=30)
        d_seconds = rank_max(pg, dsum["seconds"], dev)
        d_completed = rank_sum(pg, dsum["completed"], dev)
        drop = {"solves_per_s": d_completed / d_seconds, "p50_ms": dsum["p50_ms"],
                "p99_ms": dsum["p99_ms"], "factor": "f32", "completed": dsum["completed"],
                "failed": dsum["failed"], "backward_error_max": dsum["backward_error_max"],
                "forward_error_max": dsum["forward_error_max"],
                "failures": failure_summary(drecs)}
        if lat_pass:
            # the same service times under the half-capacity arrivals
            t_done, lat = 0.0, []
            for r, rec in zip(st.retime(lat_pass["rate_per_s"],
                                        seed=replica_seed(args.seed, rank) + 7).requests, drecs):
                start = max(r.t_arrival, t_done)
                t_done = start + rec["service_ms"] / 1e3
                lat.append(1e3 * (t_done - r.t_arrival))
            drop["at_half_served_rate"] = {"p50_ms": float(np.percentile(lat, 50)),
                                           "p99_ms": float(np.percentile(lat, 99))}
    ok = [r for r in recs if r["status"] == 0]
    h2d = sum(arrays[i][2].nbytes + (arrays[i][1].nbytes if recs[i]["path"] else 0)
              for i in range(len(recs)))
    d2h = sum(arrays[i][0].n * 8 for i in range(len(recs)))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * seconds / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": f"{uf} factor (served) / f32 factor (drop-in) / f64 GMRES-IR",
        "data": "synthetic (seeded KKT request stream, one stream per rank)",
        "config": {"workload": stream_workload(args, nreq), "global_batch": world * nreq,
                   "seq_len": None, "parallelism": f"replicas{world}",
                   "served": {"uf": uf, "update": args.update or "default",
                              "workers": args.workers, "max_batch": 16,
                              "ir_iter": ir_iter, "gmres_iter": gmres_iter},
                   "l2": "inputs larger than L2 (factors up to tens of GB)"},
        "latency_ms": {"p50": summ["p50_ms"], "p99": summ["p99_ms"],
                       "note": "saturating arrival rate (all requests within ~"
                               f"{arrivals_span:.2f}s)"},
        "latency_half_capacity_ms": lat_pass,
        "drop_in": drop,
        "served_over_drop_in": (value / drop["solves_per_s"]) if drop else None,
        "backward_error_max": summ["backward_error_max"],
        "forward_error_max": summ["forward_error_max"],
        "requests": {"completed": summ["completed"], "failed": summ["failed"],
                     "refused_over_budget": stats["refused"],
                     "failures": failure_summary(recs),
                     "paths": {p: sum(1 for r in ok if r["path"] == p) for p in (0, 1, 2)},
                     "batched_rhs": stats["batched_rhs"], "evictions": stats["evictions"],
                     "jobs": {k: stats[k] for k in ("analyses", "factorizations", "solves",
                                                    "batched_solves")},
                     "distinct_factors": len({(r.pattern_key, r.values_key)
                                              for r in st.requests}),
                     "peak_gb": stats["peak_bytes"] / 1e9,
                     "budget_gb": args.budget_gb,
                     "plans_rebuilt_from_kept_analysis": stats["analysis_reuses"],
                     "plans_uploaded_again": stats["plan_uploads"],
                     "worker_seconds": {k: round(stats[k + "_ms"] / 1e3, 2)
                                        for k in ("analysis", "plan", "factor", "solve",
                                                  "factor_device", "solve_device",
                                                  "setup", "trim", "plan_upload")}},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": h2d / args.steps,
                "d2h_bytes_per_step": d2h / args.steps,
                "note": "the served arm is itself end to end: host arrays in through "
                        "mpir_server_submit, x back on the host"},
        "gpu_launches": launches, "clocks": clk,
    }
    if summ["backward_error_max"] > BE_TOL:
        line["warning"] = "a served solve above the backward-error target"
    # roofline: the largest admitted pattern of the stream, one profiled
    # factor + solve with per-class CUDA events
    try:
        big = max((i for i, r in enumerate(recs) if r["status"] == 0),
                  key=lambda i: arrays[i][0].nnz)
        s, Ax, b, _ = arrays[big]
        g = mp.GmresLDLIR(uf=uf, device=local)
        if args.update:
            g.set_update(args.update)
        g.SetMaxGmresIterations(gmres_iter)
        g.SetMaxIRIterations(ir_iter)
        g.Compute(s.Ap, s.Ai, Ax)
        mp.kernel_timer(True)
        g.factor(Ax)
        g.Solve(b)
        kt = mp.kernel_times()
        mp.kernel_timer(False)
        line["roofline"] = roofline_from_classes(g.info(), kt, g.last_report["precond_applies"],
                                                 uf)
        line["roofline"]["system_n"] = s.n
        g.close()
    except Exception as e:
        line["roofline"] = {"error": str(e)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from mpir_b200 import kkt
            s48 = kkt.grid3d(seed=0)
            # The GPU factor of the system the CPU sample factors: parity of
            # the leading rows against the reference's QDLDL_factor<float>.
            g48 = mp.GmresLDLIR(device=local)
            g48.Compute(s48.Ap, s48.Ai, s48.Ax)
            perm = g48.symbolic()["perm"]
            counts = {"applies": 11, "spmv": 13}
            _, det = reference_cpu_estimate(s48, perm, counts, args.cpu_budget,
                                            log=lambda *a: print(*a, file=sys.stderr),
                                            keep_factor=True)
            line["parity"] = dict(leading_parity(g48, det),
                                  system="grid3d-48, n = 138,240: the system the CPU "
                                         "baseline samples")
            g48.close()
            det.pop("factor")
            det.pop("factor64", None)
            import oracle
            R = oracle.Reference()
            x = np.ones(s48.n)
            t0 = time.perf_counter()
            R.matmul(s48.n, s48.Ap, s48.Ai, s48.Ax, x)
            spmv_e = (time.perf_counter() - t0) / s48.nnz
            rates = {"updates_per_s": det["rate_updates_per_s"],
                     "seconds_per_entry": det["seconds_per_entry"],
                     "spmv_seconds_per_entry": spmv_e}
            secs = stream_reference_model(nreq, args.seed, rates, 11, 1) if args.seed == 0 \
                else None
            line["cpu_baseline"] = {
                "value": len(secs) / float(secs.sum()) if secs is not None else None,
                "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "extrapolated: the reference's QDLDL_factor<float> on the leading "
                          f"{det['k']} rows of the permuted n=138240 system ({det['factor_sample_s']:.1f}s), "
                          "its QDLDL_solve and MatrixMultiply rates, applied to every request's "
                          "own counts (one request at a time, every request factors)",
                "detail": {"rates": rates}}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 1,
                                    "kind": "reference", "sample": f"failed: {e}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


def run_batch2d(args):
    """Config 4: same-pattern instances, 16 right-hand sides each.  One step
    = one group of --group instances: their refactorizations in one graph
    launch (mpir_group_factor), then each instance's 16 right-hand sides
    solved in lockstep (one several-vector triangular solve per
    preconditioner application).  --steps 8 with groups of 8 covers the 64
    instances; the drop-in comparison (one factor + 16 one-at-a-time solves
    per instance, through GmresLDLIR) runs on the first group."""
    import torch

    import mpir_b200 as mp
    from mpir_b200 import kkt
    rank, world, local = dist_env()
    pg, dev = init_dist(local)
    uf = args.uf or "f32"
    G = args.group
    ninst = G * max(args.steps, 1)
    insts = kkt.batch2d(instances=ninst, grid=args.grid or 256, nrhs=16,
                        seed=replica_seed(args.seed, rank))
    solver = mp.GmresLDLIR(uf=uf, device=local)
    solver.analyze(insts[0].Ap, insts[0].Ai, insts[0].Ax)
    info = solver.info()
    grp = mp.FactorGroup(solver, G)

    def step(i):
        group = insts[(i * G) % ninst:(i * G) % ninst + G]
        assert np.all(grp.factor([s.Ax for s in group]) > 0)
        be, solves = 0.0, 0
        for j, s in enumerate(group):
            X = grp.SolveBatch(j, s.b)
            solves += X.shape[0]
            be = max(be, max(r["backward_error"] for r in grp.last_reports))
        return be, solves

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    clocks = Clocks(local)
    clocks.start()
    launches0 = mp.launch_count()
    t0 = time.perf_counter()
    be, lat, solves = 0.0, [], 0
    for i in range(args.steps):
        t1 = time.perf_counter()
        b_i, s_i = step(i)
        lat.append(1e3 * (time.perf_counter() - t1))
        be, solves = max(be, b_i), solves + s_i
    seconds = rank_max(pg, time.perf_counter() - t0, dev)
    launches = mp.launch_count() - launches0
    clk = clocks.stop()
    value = rank_sum(pg, solves, dev) / seconds
    fe = None
    # the same first group one at a time through the drop-in: a factor and
    # 16 single-right-hand-side solves per instance
    t1 = time.perf_counter()
    for s in insts[:G]:
        assert solver.factor(s.Ax) == 0
        for k in range(s.b.shape[0]):
            x = solver.Solve(s.b[k])
            fe = max(fe or 0.0, kkt.forward_error(x, s.x_true[k]))
    drop = G * 16 / (time.perf_counter() - t1)
    n = insts[0].n
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * seconds / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": f"{uf} factor / f64 solve", "data": "synthetic (seeded same-pattern batch)",
        "config": {"workload": f"batch2d: {ninst} instances of n={n} on one pattern "
                               "(L2D 256^2 + diag(s), s log-uniform [1e-6, 1e2], m=16384 x 4, "
                               f"delta 1e-8), 16 RHS each; per step {G} refactorizations in one "
                               f"graph launch + {G} x 16 lockstep GMRES-IR solves (host arrays "
                               "through the C ABI)",
                   "global_batch": world * G * 16, "group": G},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "note": f"per step ({G} factors + {G * 16} solves)"},
        "backward_error_max": be, "forward_error_max_dropin": fe,
        "drop_in": {"solves_per_s": drop, "note": "first group: per instance one factor + 16 "
                    "one-at-a-time GmresLDLIR solves"},
        "e2e": {"value": value, "unit": UNIT,
                "h2d_bytes_per_step": G * (insts[0].Ax.nbytes + 16 * n * 8),
                "d2h_bytes_per_step": G * 16 * n * 8},
        "gpu_launches": launches, "clocks": clk,
        "info": {k: info[k] for k in ("n", "nnz_L", "supernodes", "levels", "max_front")},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    grp.close()
    solver.close()
    if pg is not None:
        pg.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.config == "stream":
        run_stream(args)
    elif args.config == "batch2d":
        run_batch2d(args)
    else:
        run_system(args)


if __name__ == "__main__":
    main()
