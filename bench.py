#!/usr/bin/env python3
"""Benchmark: PDHG iterations/s on the large power-law LP (one B200 per rank).

Workload ("zipf_lp_2Mx5M"): m = 2,000,000 rows, n = 5,000,000 columns, row
lengths Zipf(1.5) capped at 5000, uniform distinct columns, FP32 N(0,1) values
times log-uniform row scales in [1e-2, 1e2], feasible by construction
(seeded synthetic data; the actual nnz is reported).  One step = one PDHG
iteration of the reference algorithm (A x̄ + dual update, Aᵀ y + primal
update), inputs resident in HBM.  The CSR streams (~0.9 GB per product) are
far larger than L2, so no flush is needed between steps.

Lines printed (rank 0, one JSON line):
  value      iterations/s over all ranks (replicas: every rank solves its own copy)
  e2e        the same metric through pramaan_pdhg_solve() with pinned host
             buffers: upload, 1000 iterations (checks every 100), download
  roofline   the dominant product kernel's algorithmic bytes / CUDA-event time
  cpu_baseline  the oracle's multi-threaded FP32 iteration on the host cores
  banded_spmv   the same iteration on a banded LP of the same size (local
             gathers): per-kernel GB/s against the measured HBM bandwidth
  small_lp, rolling_horizon, learned_stream   the plain-PDHG LP, the batched
             rolling-horizon LPs and the learned warm start (see each section)

`--impl reference` times the reference algorithm's CPU restatement (the
oracle; the reference has no CPU implementation of this path) on all host
cores, for the same workload and metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "pdhg_iterations_per_s"
UNIT = "iterations/s"
WORKLOAD = "zipf_lp_2Mx5M"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="pramaan_b200", choices=["pramaan_b200", "reference"])
    p.add_argument("--m", type=int, default=2_000_000)
    p.add_argument("--n", type=int, default=5_000_000)
    p.add_argument("--cap", type=int, default=5000)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--e2e-iters", type=int, default=1000)
    p.add_argument("--e2e-calls", type=int, default=3)
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-reference-gpu", action="store_true",
                   help="reference arm: skip timing the reference's own GPU solver")
    p.add_argument("--rh-count", type=int, default=512,
                   help="LPs of the batched rolling-horizon section (the published batch: 512)")
    p.add_argument("--ladder-m", type=int, default=200_000, help="rows of the precision-ladder LP")
    p.add_argument("--ladder-n", type=int, default=500_000, help="columns of the precision-ladder LP")
    p.add_argument("--no-ladder", action="store_true", help="skip the precision-ladder section")
    p.add_argument("--solver-cap-s", type=float, default=20.0,
                   help="wall-clock cap of one reference CPU solve at full size (reported as DNF)")
    p.add_argument("--rh-plain", type=int, default=8, help="LPs of that batch also solved one by one")
    p.add_argument("--batch-iters", type=int, default=1024,
                   help="iterations of the batched-products timing (every LP active)")
    p.add_argument("--stream-count", type=int, default=32, help="streams of the learned warm-start section")
    p.add_argument("--stream-windows", type=int, default=4, help="windows per stream in that section")
    p.add_argument("--stream-T", type=int, nargs=2, default=(24, 336), help="periods of the stream windows")
    p.add_argument("--stream-P", type=int, nargs=2, default=(5, 50), help="products of the stream windows")
    p.add_argument("--weights", default=None, help="warm-start network weights (.npz; default: the committed ones)")
    p.add_argument("--learned-tail", type=int, default=4,
                   help="periods at the end of each window where the network's prediction replaces the shifted "
                        "previous solution (0: the network everywhere, the certificate choosing between "
                        "candidate starts after --probe-iters iterations)")
    p.add_argument("--probe-iters", type=int, default=64,
                   help="with --learned-tail 0: PDHG iterations from each candidate start before the certificate "
                        "chooses")
    p.add_argument("--no-rolling", action="store_true", help="skip both rolling-horizon sections")
    p.add_argument("--no-banded", action="store_true", help="skip the banded-LP bandwidth section")
    p.add_argument("--banded-iters", type=int, default=50)
    p.add_argument("--launch-blocks", type=int, default=0,
                   help="fixed blocks per SM of the products (0: autotuned); with --gather-cache 1 or -1 "
                        "the launch shape is fixed, for profiles")
    p.add_argument("--only", default=None, choices=["banded", "gnn", "small", "rolling", "stream", "ceiling", "ladder", "solvers", "batch",
                            "tail"],
                   help="run one section alone on the given sizes and print its JSON (profiling runs)")
    p.add_argument("--gnn-lps", type=int, default=64, help="rolling-horizon LPs of the network throughput section")
    p.add_argument("--gnn-reps", type=int, default=5)
    p.add_argument("--panel-split", type=int, default=0,
                   help="A x̄ product: 0 column panels for the long rows of a power-law A (automatic), "
                        "1 whenever feasible, >= 2 rows of that many entries as long rows, -1 tiled only")
    p.add_argument("--gather-cache", type=int, default=0, choices=[0, 1, -1],
                   help="0: hot gather targets in shared memory, L1-cached gathers where faster (the "
                        "default); 1: L1-cached gathers wherever there are no hot slots; -1: plain")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload_config(args, nnz):
    return {"workload": WORKLOAD, "m": args.m, "n": args.n, "nnz": int(nnz), "zipf_s": 1.5,
            "row_len_cap": args.cap, "seed": args.seed, "step": "one PDHG iteration (reference algorithm)",
            "l2": "inputs larger than L2 (CSR ~0.9 GB per product); no flush",
            "parallelism": f"replicas x{args.gpus}"}


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    """HBM copy bandwidth (GB/s) for the rooflines and where it came from:
    MEASURED_PEAKS.json when present, else the pool's earlier measurement."""
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback: 6,650 GB/s measured earlier on this pool (MEASURED_PEAKS.json absent)"


def ncu_traffic(kernel_tag: str):
    """Per-launch DRAM bytes recorded from an ncu capture in profiles/."""
    f = REPO / "profiles" / f"{kernel_tag}.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch_full_size:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def gather_ceiling(n: int, device: int) -> dict:
    """The device's random 4-byte gather rate from an n-entry vector (the
    library's ceiling kernel), L2 (ld.global.cg) and L1-cached."""
    import ctypes as C

    import torch

    from pramaan_b200 import _lib as L

    x = torch.rand(n, device=f"cuda:{device}", dtype=torch.float32)
    torch.cuda.synchronize(device)
    out = {"n": n}
    for name, cached in (("l2_gathers_per_s", 0), ("l1_cached_gathers_per_s", 1)):
        r = C.c_double(0.0)
        L.check(L.lib().pramaan_measure_gather_rate(x.data_ptr(), n, cached, 5, C.byref(r)))
        out[name] = r.value
    return out


# ---------------------------------------------------------------------------
def cpu_baseline(model, seconds: float):
    """Oracle FP32 iteration on all host threads, on a bounded number of full
    iterations of the same LP; returns (iterations/s, threads, sample text)."""
    import ctypes as C

    import oracle
    from oracle import ptr

    h = oracle.orc()
    m, n = model.numRows(), model.numVars()
    v32 = model.values.astype(np.float32)
    order = np.argsort(model.col_idx, kind="stable")
    rows = np.repeat(np.arange(m, dtype=np.int32), np.diff(model.row_ptr))
    tci = rows[order].astype(np.int32)
    tv = v32[order]
    trp = np.zeros(n + 1, np.int32)
    trp[1:] = np.cumsum(np.bincount(model.col_idx, minlength=n))
    sig, tau = oracle.step_sizes(model)
    c = model.obj_coeffs.astype(np.float32)
    lr = model.row_lower.astype(np.float32)
    ur = model.row_upper.astype(np.float32)
    lx = model.var_lower.astype(np.float32)
    ux = model.var_upper.astype(np.float32)
    x = np.maximum(lx, np.minimum(0, ux)).astype(np.float32)
    xb = x.copy()
    y = np.zeros(m, np.float32)
    args = [ptr(model.row_ptr), ptr(model.col_idx), ptr(v32), ptr(trp), ptr(tci), ptr(tv), ptr(sig),
            ptr(lr), ptr(ur), ptr(tau), ptr(c), ptr(lx), ptr(ux), ptr(x), ptr(xb), ptr(y)]
    threads = h.orc_num_threads()
    t0 = time.perf_counter()
    h.orc_pdhg_iterations_mt(m, n, *args, 1)
    one = time.perf_counter() - t0
    iters = max(1, int(seconds / max(one, 1e-6)))
    t0 = time.perf_counter()
    h.orc_pdhg_iterations_mt(m, n, *args, iters)
    dt = time.perf_counter() - t0
    return iters / dt, threads, f"{iters} full iterations of the same LP after 1 untimed ({dt:.1f} s)"


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import torch

    from pramaan_b200.generators import zipf_lp

    # the same instance as the GPU arm: torch's CPU and CUDA generators draw
    # different streams, so generate where that arm does when a GPU is present
    gen_dev = "cuda:0" if torch.cuda.is_available() else "cpu"
    model = zipf_lp(args.m, args.n, cap=args.cap, seed=args.seed, device=gen_dev)
    import oracle
    from oracle import ptr

    h = oracle.orc()
    m, n = model.numRows(), model.numVars()
    v32 = model.values.astype(np.float32)
    order = np.argsort(model.col_idx, kind="stable")
    rows = np.repeat(np.arange(m, dtype=np.int32), np.diff(model.row_ptr))
    tci = rows[order].astype(np.int32)
    tv = v32[order]
    trp = np.zeros(n + 1, np.int32)
    trp[1:] = np.cumsum(np.bincount(model.col_idx, minlength=n))
    sig, tau = oracle.step_sizes(model)
    c = model.obj_coeffs.astype(np.float32)
    lr, ur = model.row_lower.astype(np.float32), model.row_upper.astype(np.float32)
    lx, ux = model.var_lower.astype(np.float32), model.var_upper.astype(np.float32)
    x = np.maximum(lx, np.minimum(0, ux)).astype(np.float32)
    xb = x.copy()
    y = np.zeros(m, np.float32)
    a = [ptr(model.row_ptr), ptr(model.col_idx), ptr(v32), ptr(trp), ptr(tci), ptr(tv), ptr(sig),
         ptr(lr), ptr(ur), ptr(tau), ptr(c), ptr(lx), ptr(ux), ptr(x), ptr(xb), ptr(y)]
    for _ in range(args.warmup):
        h.orc_pdhg_iterations_mt(m, n, *a, 1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        h.orc_pdhg_iterations_mt(m, n, *a, 1)
    dt = time.perf_counter() - t0
    v = args.steps / dt
    threads = h.orc_num_threads()
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * dt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args, model.nnz()), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{args.steps} full iterations (the reference has no CPU PDHG; "
                                       "its algorithm restated in C, OpenMP over rows/columns)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if torch.cuda.is_available() and not args.no_reference_gpu:
        torch.cuda.empty_cache()
        line["reference_gpu"] = reference_gpu_section(args, model)
    print(json.dumps(line), flush=True)


def reference_gpu_section(args, model):
    """The reference's own GPU PDHG (src/gpu/pdhg_solver.cu, compiled for
    sm_100a into oracle/_ref), reported beside this library: iterations/s on
    the same 2 M x 5 M LP (difference of a 300- and a 100-iteration solve,
    each with its FP64 host check every 100 iterations, so setup cancels and
    the checks are counted as the reference runs them) and time to its 1e-4
    criterion on the 1000 x 3000 plain LP."""
    import oracle
    from pramaan_b200.generators import random_sparse_lp

    if oracle.ref_gpu() is None:
        return {"unavailable": "oracle/_ref/libref_gpu.so is not built"}
    out = {"source": "src/gpu/pdhg_solver.cu (PdhgSolver::solve), nvcc -gencode arch=compute_100a,code=sm_100a"}
    with ClockSampler(0) as clk:
        times = {}
        for iters in (100, 300):
            t0 = time.perf_counter()
            r = oracle.ref_solve("pdhg", model, max_iterations=iters, tolerance=0.0, check_frequency=100)
            times[iters] = time.perf_counter() - t0
        small = random_sparse_lp(1000, 3000, 4, seed=args.seed)
        oracle.ref_solve("pdhg", small, max_iterations=200, tolerance=1e-4, check_frequency=100)
        t0 = time.perf_counter()
        rs = oracle.ref_solve("pdhg", small, max_iterations=100000, tolerance=1e-4, check_frequency=100)
        t_small = time.perf_counter() - t0
    out[WORKLOAD] = {"iterations_per_s": 200.0 / (times[300] - times[100]), "solve_100_s": times[100],
                     "solve_300_s": times[300], "status_300": int(r["status"])}
    out["random_sparse_lp_1000x3000_to_1e-4"] = {"seconds": t_small, "iterations": int(rs["iterations"]),
                                                 "status": int(rs["status"]), "objective": rs["objective_value"]}
    out["clocks"] = clk.summary()
    return out


# ---------------------------------------------------------------------------
def _certified(models, results, tol, device):
    from pramaan_b200.certificate import certify_batch
    from pramaan_b200.gnn import WarmStart

    cert = certify_batch(models, [[WarmStart(r.x, r.y) for r in results]], device)[0]
    return sum(1 for c in cert if c.kkt <= tol * 1.0001)


def rolling_horizon_section(args, device, dist=None):
    """Batched rolling-horizon LPs (T ~ U{24..336}, P ~ U{5..50}) at 1e-6
    relative KKT: one packed batch against the same Halpern PDHG solving the
    LPs one by one (a sample of them).  With N ranks the batch has N x
    --rh-count LPs and every rank solves its non-zero-balanced share on its
    own GPU (no collective on the data path); the time is the maximum over
    the ranks (weak scaling)."""
    import torch

    from pramaan_b200 import PdhgOptions, PdhgSolver, SolveStatus, solve_batch
    from pramaan_b200.certificate import certify_batch
    from pramaan_b200.generators import rolling_horizon_batch
    from pramaan_b200.gnn import WarmStart
    from pramaan_b200.parallel import shard_plan, solve_batch_sharded
    from pramaan_b200.pdhg import ALGO_HALPERN

    tol = 1e-6
    world = dist.get_world_size() if dist else 1
    rank = dist.get_rank() if dist else 0
    o = PdhgOptions(tolerance=tol, max_iterations=400000, check_frequency=64, algorithm=ALGO_HALPERN,
                    device=device)
    models = rolling_horizon_batch(args.rh_count * world, seed=args.seed)
    mine = shard_plan([m.nnz() for m in models], world)[rank]
    solve_batch(models[:2], o)                       # warm-up (module load, occupancy queries)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    res = solve_batch_sharded(models, o, gather=False)
    tb = time.perf_counter() - t0
    mres = [res[i] for i in mine]
    mmod = [models[i] for i in mine]
    cert = certify_batch(mmod, [[WarmStart(r.x, r.y) for r in mres]], device)[0] if mmod else []
    counts = torch.tensor([sum(r.status == SolveStatus.kOptimal for r in mres),
                           sum(1 for c in cert if c.kkt <= tol * 1.0001)], dtype=torch.float64, device=f"cuda:{device}")
    tmax = torch.tensor([tb], dtype=torch.float64, device=f"cuda:{device}")
    if dist:
        dist.all_reduce(counts, op=dist.ReduceOp.SUM)
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    tb = float(tmax.item())
    its = [r.iterations for r in mres]
    idx = [mine[k] for k in np.linspace(0, len(mine) - 1, min(args.rh_plain, len(mine))).astype(int)]
    solver = PdhgSolver(o)
    plain_t, plain_it = [], []
    for i in idx:
        t0 = time.perf_counter()
        r = solver.solve(models[i])
        plain_t.append(time.perf_counter() - t0)
        plain_it.append(r.iterations)
    batched = len(models) / tb
    plain = world * len(idx) / sum(plain_t)
    return {"workload": f"rolling_horizon_batch {len(models)} LPs (T~U{{24..336}}, P~U{{5..50}}), "
                        f"rel KKT {tol:g}, seed {args.seed}; restarted Halpern PDHG, batched and one by one"
                        + (f"; {world} ranks, LPs sharded by non-zeros" if world > 1 else ""),
            "rows": sum(m.numRows() for m in models), "cols": sum(m.numVars() for m in models),
            "nnz": sum(m.nnz() for m in models),
            "batched_lps_per_s": batched, "batched_s": tb,
            "batched_iterations_median": float(np.median(its)) if its else None,
            "optimal": int(counts[0].item()), "certified": int(counts[1].item()),
            "plain_lps_per_s": plain, "plain_sample": int(len(idx)) * world,
            "plain_time_to_tol_median_s": float(np.median(plain_t)),
            "plain_iterations_median": float(np.median(plain_it)),
            "batched_over_plain": batched / plain}


def batch_iteration_section(args, device, models=None):
    """The batched products' own speed: the rolling-horizon batch run for a
    fixed number of iterations with every LP active (tolerance 0), timed as
    the difference of a 2K- and a K-iteration solve so that set-up cancels.
    Algorithmic bytes per iteration over the packed operand: the matrix
    streams and gathers of both products (16 nnz + 8 (m + n)) plus the
    Halpern epilogues' vectors (primal: tau, c, bounds, x, LP index read,
    x and x-bar written, 32 B per column; dual: sigma, bounds, master y,
    y, LP index read, y written, 28 B per row)."""
    import torch

    from pramaan_b200 import PdhgOptions, solve_batch
    from pramaan_b200.generators import rolling_horizon_batch
    from pramaan_b200.pdhg import ALGO_HALPERN

    if models is None:
        models = rolling_horizon_batch(args.rh_count, seed=args.seed)
    K = args.batch_iters
    times = {}
    for k in (K, 2 * K):
        o = PdhgOptions(tolerance=0.0, max_iterations=k, check_frequency=64, algorithm=ALGO_HALPERN, device=device,
                        gather_cache=args.gather_cache, launch_blocks=args.launch_blocks)
        if k == K:
            solve_batch(models, o)   # warm-up: module load, the operand's launch tuning (remembered)
        torch.cuda.nvtx.range_push("timed")
        t0 = time.perf_counter()
        solve_batch(models, o)
        times[k] = time.perf_counter() - t0
        torch.cuda.nvtx.range_pop()
    per_it = (times[2 * K] - times[K]) / K
    m = sum(md.numRows() for md in models)
    n = sum(md.numVars() for md in models)
    nnz = sum(md.nnz() for md in models)
    by = 16.0 * nnz + 8.0 * (m + n) + 32.0 * n + 28.0 * m
    hbm, kind = measured_peaks()
    return {"workload": f"rolling_horizon_batch {len(models)} LPs, every LP active (tolerance 0), {K} vs {2 * K} "
                        "iterations, checks every 64 included",
            "rows": m, "cols": n, "nnz": nnz, "us_per_iteration": per_it * 1e6,
            "algorithmic_bytes_per_iteration": by, "achieved_gbs": by / per_it / 1e9, "frac": by / per_it / 1e9 / hbm,
            "peak_gbs": hbm, "peak_kind": kind}


def batch_tail_section(args, device):
    """The batch's tail: the 128-LP rolling-horizon batch's largest LP, and
    its two largest together, iterated by the per-LP cluster kernel (the
    default once a batch is down to a few LPs) and by the packed tiled
    products, each for a fixed number of iterations (tolerance 0) and timed
    as the difference of a 4K- and a K-iteration solve, checks every 64
    iterations included."""
    import torch

    from pramaan_b200 import PdhgOptions, solve_batch
    from pramaan_b200.generators import rolling_horizon_batch
    from pramaan_b200.pdhg import ALGO_HALPERN

    batch = rolling_horizon_batch(128, seed=args.seed)
    order = sorted(range(len(batch)), key=lambda i: -batch[i].nnz())
    K = 640
    out = {"workload": f"rolling_horizon_batch 128 LPs (seed {args.seed}): its largest LP and its two largest, "
                       f"{K} vs {4 * K} iterations, median of 3"}
    for tag, idx in (("largest", order[:1]), ("two_largest", order[:2])):
        models = [batch[i] for i in idx]
        row = {"rows": sum(m.numRows() for m in models), "cols": sum(m.numVars() for m in models),
               "nnz": sum(m.nnz() for m in models)}
        for path, persistent in (("cluster_kernel", 2), ("tiled", -1)):
            def run(k):
                o = PdhgOptions(tolerance=0.0, max_iterations=k, check_frequency=64, algorithm=ALGO_HALPERN,
                                device=device, persistent=persistent)
                t0 = time.perf_counter()
                solve_batch(models, o)
                return time.perf_counter() - t0
            run(K)   # warm-up
            torch.cuda.nvtx.range_push("timed")
            a = sorted(run(K) for _ in range(3))[1]
            b = sorted(run(4 * K) for _ in range(3))[1]
            torch.cuda.nvtx.range_pop()
            row[f"{path}_us_per_iteration"] = (b - a) / (3 * K) * 1e6
        out[tag] = row
    return out


def learned_stream_section(args, device):
    """S streams of rolling-horizon windows solved step by step (window w of
    every stream is one batch), cold against the certified learned warm start
    (network refining the previous window's shifted solution) and against the
    shifted solution alone."""
    from pramaan_b200 import PdhgOptions, SolveStatus, solve_batch
    from pramaan_b200.gnn import WarmStartNet, warm_solve_batch
    from pramaan_b200.pdhg import ALGO_HALPERN
    from pramaan_b200.train_warm_start import DEFAULT_OUT, stream_windows

    wpath = Path(args.weights) if args.weights else DEFAULT_OUT
    if not wpath.exists():
        return {"unavailable": f"no trained weights at {wpath.name}"}
    rec = json.loads(str(np.load(wpath)["record"]))
    net = WarmStartNet(device=device, seed=0)
    net.load(wpath)
    tol = 1e-6
    o = PdhgOptions(tolerance=tol, max_iterations=400000, check_frequency=64, algorithm=ALGO_HALPERN,
                    device=device)
    S, W = args.stream_count, args.stream_windows
    T, P = tuple(args.stream_T), tuple(args.stream_P)
    ms, _ = stream_windows(range(700000 + args.seed, 700000 + args.seed + S), W, T, P)
    windows = [[ms[s * W + w] for s in range(S)] for w in range(W)]
    out = {"workload": f"{S} streams x {W} windows (rolling_horizon_stream, T~U{{{T[0]}..{T[1]}}}, "
                       f"P~U{{{P[0]}..{P[1]}}}, AR(1) phi 0.9 sigma 0.1; a seeded sub-sample of the "
                       f"10,000-window stream), rel KKT {tol:g}; window w of every stream is one batch",
           "trained_on": {k: rec[k] for k in ("instances_solved", "instances_trained", "epochs", "T", "P")
                          if k in rec},
           "learned_start": (f"the network's prediction on the last {args.learned_tail} periods of each window, "
                             "the shifted previous solution elsewhere" if args.learned_tail > 0 else
                             f"the certificate's choice among the network's point, the hint, their midpoint and "
                             f"cold after {args.probe_iters} probe iterations each")}
    solve_batch(windows[0][:2], o)                   # warm-up
    # the plain per-LP solver on a sample of the same windows
    from pramaan_b200 import PdhgSolver
    sample = [windows[w][s] for w in range(W) for s in range(0, S, max(1, S // 2))][:8]
    solver = PdhgSolver(o)
    t0 = time.perf_counter()
    for md in sample:
        solver.solve(md)
    out["plain"] = {"lps_per_s": len(sample) / (time.perf_counter() - t0), "sample": len(sample)}
    for mode in ("cold", "hint", "learned"):
        prev = None
        its, t, ok, cert, choices = 0, 0.0, 0, 0, {}
        phases = {"predict_s": 0.0, "certify_s": 0.0, "solve_s": 0.0, "fallback_s": 0.0, "fallbacks": 0,
                  "probe_iterations": 0}
        for w in range(W):
            batch = windows[w]
            hints = None if prev is None else _hints_for(batch, prev)
            t0 = time.perf_counter()
            if mode == "cold" or hints is None:
                res = solve_batch(batch, o)
            elif mode == "hint":
                res = solve_batch(batch, o, warm=hints)
            else:
                if args.learned_tail > 0:
                    res, info = warm_solve_batch(batch, net, o, hints=hints, select=False,
                                                 refine_masks=_tail_masks(batch, hints, args.learned_tail))
                else:
                    res, info = warm_solve_batch(batch, net, o, hints=hints, probe_iterations=args.probe_iters)
                for c in info.choices:
                    choices[c] = choices.get(c, 0) + 1
                for k in phases:
                    phases[k] += getattr(info, k)
                its += info.probe_iterations      # every candidate's probe counts
            t += time.perf_counter() - t0
            its += sum(r.iterations for r in res)
            ok += sum(r.status == SolveStatus.kOptimal for r in res)
            cert += _certified(batch, res, tol, device)
            prev = res
        out[mode] = {"lps_per_s": S * W / t, "seconds": t, "iterations": its, "optimal": ok, "certified": cert}
        if choices:
            out[mode]["starts"] = choices
            out[mode]["phases"] = phases
    for mode in ("hint", "learned"):
        out[mode]["iterations_vs_cold"] = out[mode]["iterations"] / out["cold"]["iterations"]
        out[mode]["speedup_vs_cold"] = out[mode]["lps_per_s"] / out["cold"]["lps_per_s"]
    for mode in ("cold", "hint", "learned"):
        out[mode]["speedup_vs_plain"] = out[mode]["lps_per_s"] / out["plain"]["lps_per_s"]
    return out


def small_lp_section(args, device):
    """The plain-PDHG LP (m = 1000, n = 3000, 4 non-zeros per column, N(0,1)
    values, feasible by construction): time to 1e-4 with the reference
    algorithm and criterion, and with the Halpern mode to 1e-4 / 1e-8 relative
    KKT (FP64 certificate of each answer)."""
    from pramaan_b200 import PdhgOptions, PdhgSolver
    from pramaan_b200.certificate import certify
    from pramaan_b200.generators import random_sparse_lp
    from pramaan_b200.pdhg import ALGO_HALPERN

    md = random_sparse_lp(1000, 3000, 4, seed=args.seed)
    out = {"workload": f"random_sparse_lp 1000 x 3000, 4 nnz/col, seed {args.seed}"}
    PdhgSolver(PdhgOptions(tolerance=1e-4, device=device)).solve(md)          # warm-up
    for name, o in (("reference_1e-4", PdhgOptions(tolerance=1e-4, device=device)),
                    ("halpern_1e-4", PdhgOptions(tolerance=1e-4, algorithm=ALGO_HALPERN, check_frequency=64,
                                                 device=device)),
                    ("halpern_1e-8", PdhgOptions(tolerance=1e-8, algorithm=ALGO_HALPERN, check_frequency=64,
                                                 max_iterations=400000, device=device))):
        t0 = time.perf_counter()
        r = PdhgSolver(o).solve(md)
        dt = time.perf_counter() - t0
        c = certify(md, r.x, r.y, device)
        out[name] = {"status": r.status.name, "iterations": r.iterations, "seconds": dt,
                     "rel_kkt": c.kkt, "objective": r.objective_value}
    return out


def ladder_section(args, device):
    """The precision-ladder LP (m = 200,000, n = 500,000, 8 non-zeros per
    column, row and column scales log-uniform in [1e-4, 1e4], feasible by
    construction): restarted Halpern PDHG with FP64 refinement to 1e-4, then
    to 1e-8 relative KKT, each answer certified in FP64 on the GPU."""
    from pramaan_b200 import PdhgOptions, PdhgSolver
    from pramaan_b200.certificate import certify
    from pramaan_b200.generators import ill_conditioned_lp
    from pramaan_b200.pdhg import ALGO_HALPERN

    md = ill_conditioned_lp(args.ladder_m, args.ladder_n, 8, seed=args.seed)
    out = {"workload": f"ill_conditioned_lp {args.ladder_m} x {args.ladder_n}, 8 nnz/col, scales 10^+-4, "
                       f"seed {args.seed}", "nnz": int(md.nnz())}
    PdhgSolver(PdhgOptions(tolerance=1e-2, algorithm=ALGO_HALPERN, check_frequency=64, device=device)).solve(md)
    for tol in (1e-4, 1e-8):
        o = PdhgOptions(tolerance=tol, algorithm=ALGO_HALPERN, check_frequency=64, max_iterations=1_000_000,
                        device=device)
        t0 = time.perf_counter()
        r = PdhgSolver(o).solve(md)
        dt = time.perf_counter() - t0
        c = certify(md, r.x, r.y, device)
        out[f"halpern_{tol:g}"] = {"status": r.status.name, "iterations": r.iterations, "restarts": r.restarts,
                                   "seconds": dt, "certified_rel_kkt": c.kkt, "certified": bool(c.kkt <= tol * 1.0001),
                                   "objective": r.objective_value}
    return out


def reference_solvers_section(args, device):
    """The reference's FP64 CPU solvers (its dual simplex and interior-point
    method, compiled from its sources into oracle/_ref) on the host cores:
    the Netlib fixtures and m <= 300 replicas of the plain, precision-ladder
    and rolling-horizon LPs, each also solved by this library on the GPU
    (Halpern, 1e-8) to state its error against the FP64 oracle; and one capped
    attempt at the full-size plain LP.  The reference solvers are single
    threaded."""
    import multiprocessing as mp

    import oracle
    from pramaan_b200 import PdhgOptions, PdhgSolver
    from pramaan_b200.generators import ill_conditioned_lp, random_sparse_lp, rolling_horizon_lp
    from pramaan_b200.pdhg import ALGO_HALPERN

    if oracle.ref_cpu() is None:
        return {"unavailable": "oracle/_ref is not built"}
    cases = {"cfg0_replica_100x300": random_sparse_lp(100, 300, 4, seed=args.seed),
             "cfg2_replica_100x250": ill_conditioned_lp(100, 250, 8, seed=args.seed),
             "cfg3_replica_T24_P5": rolling_horizon_lp(24, 5, seed=args.seed),
             "cfg3_replica_T48_P5": rolling_horizon_lp(48, 5, seed=args.seed + 1)}
    mps_dir = REPO / "oracle" / "_ref" / "run" / "tests" / "data"
    for name in ("afiro", "adlittle"):
        if (mps_dir / f"{name}.mps").exists():
            cases[name] = oracle.ref_load_mps(str(mps_dir / f"{name}.mps"))
    gpu = PdhgSolver(PdhgOptions(tolerance=1e-8, algorithm=ALGO_HALPERN, check_frequency=64,
                                 max_iterations=1_000_000, device=device))
    out = {"cores": 1, "host_threads": os.cpu_count(), "tolerance_gpu": 1e-8, "cases": {}}
    for name, md in cases.items():
        rec = {"rows": md.numRows(), "cols": md.numVars(), "nnz": int(md.nnz())}
        best = None
        for kind in ("dual", "ipm"):
            t0 = time.perf_counter()
            try:
                r = oracle.ref_solve(kind, md, max_iterations=200000, tolerance=1e-9)
                rec[kind] = {"status": int(r["status"]), "iterations": int(r["iterations"]),
                             "seconds": time.perf_counter() - t0, "objective": r["objective_value"]}
                if r["status"] == 0 and best is None:
                    best = r
            except Exception as e:   # a reference failure is reported, not raised
                rec[kind] = {"error": str(e)[:200], "seconds": time.perf_counter() - t0}
        t0 = time.perf_counter()
        g = gpu.solve(md)
        rec["gpu_halpern"] = {"status": g.status.name, "iterations": g.iterations,
                              "seconds": time.perf_counter() - t0, "objective": g.objective_value}
        if best is not None:
            ref_obj = best["objective_value"]
            rec["oracle_error"] = {
                "against": "dual simplex" if rec["dual"].get("status") == 0 else "ipm",
                "objective_rel": abs(g.objective_value - ref_obj) / (1.0 + abs(ref_obj)),
                "x_inf_rel": float(np.max(np.abs(g.x - best["x"])) / (1.0 + np.max(np.abs(best["x"])))),
                "note": "x of an LP need not be unique; the objective error is the oracle's measure"}
        out["cases"][name] = rec
    # the full-size plain LP under a wall-clock cap, in a child process
    full = random_sparse_lp(1000, 3000, 4, seed=args.seed)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    proc = ctx.Process(target=_ref_solve_child, args=(full, q))
    t0 = time.perf_counter()
    proc.start()
    proc.join(args.solver_cap_s)
    if proc.is_alive():
        proc.terminate()
        proc.join(10)
        out["cfg0_full_1000x3000_dual_simplex"] = {"status": "DNF", "cap_s": args.solver_cap_s}
    else:
        res = q.get() if not q.empty() else {"status": "no result"}
        res["seconds"] = time.perf_counter() - t0
        out["cfg0_full_1000x3000_dual_simplex"] = res
    return out


def _ref_solve_child(md, q):
    import oracle
    r = oracle.ref_solve("dual", md, max_iterations=10_000_000, tolerance=1e-9)
    q.put({"status": int(r["status"]), "iterations": int(r["iterations"]), "objective": r["objective_value"]})


def banded_section(args, device):
    """The same iteration on a banded LP of the headline size (2,000,000 x
    5,000,000, 54 columns per row within +-256 of i*n/m): local gathers, so the
    products can run at the HBM roofline.  Device-timed per-kernel bandwidth
    (algorithmic bytes over CUDA-event time) with the autotuner's gather mode
    and with plain L2 gathers."""
    import torch

    from pramaan_b200 import PdhgOptions
    from pramaan_b200.generators import banded_lp, model_from_tensors
    from pramaan_b200.pdhg import Session

    t = banded_lp(args.m, args.n, per_row=54, band=256, seed=args.seed, device=f"cuda:{device}", as_tensors=True)
    model = model_from_tensors(t)
    del t
    torch.cuda.empty_cache()
    hbm, kind = measured_peaks()
    out = {"workload": f"banded_lp {args.m} x {args.n}, 54 per row, band 256, seed {args.seed}",
           "nnz": int(model.nnz()), "peak_gbs": hbm, "peak_kind": kind, "iterations": args.banded_iters}
    modes = (("auto", args.gather_cache), ("l2_gathers", -1)) if args.gather_cache != -1 else (("l2_gathers", -1),)
    for name, cache in modes:
        with Session(model, PdhgOptions(device=device, use_graph=False, profile_kernels=True,
                                        gather_cache=cache, launch_blocks=args.launch_blocks)) as sess:
            for _ in range(3):
                sess.iterate(1)
            sess.synchronize()
            sess.kernel_times(reset=True)
            stream = torch.cuda.ExternalStream(sess.stream(), device=device)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.nvtx.range_push("timed")
            e0.record(stream)
            for _ in range(args.banded_iters):
                sess.iterate(1)
            e1.record(stream)
            e1.synchronize()
            torch.cuda.nvtx.range_pop()
            ms_dual, ms_primal, _ = sess.kernel_times(reset=True)
            b_dual, b_primal = sess.kernel_bytes()
            k = args.banded_iters
            res = {"iterations_per_s": k / (e0.elapsed_time(e1) / 1000.0), "gather": sess.gather_info()}
            for tag, ms, by in (("dual", ms_dual, b_dual), ("primal", ms_primal, b_primal)):
                gbs = by / (ms / 1000.0 / k) / 1e9
                res[tag] = {"avg_launch_ms": ms / k, "achieved_gbs": gbs, "frac": gbs / hbm}
            out[name] = res
    return out


def gnn_section(args, device):
    """Throughput of the warm-start network on a batch of rolling-horizon LPs
    with the batched benchmark's shapes (T ~ U{24..336}, P ~ U{5..50}): the
    forward pass (predict) and one training step (forward + backward + Adam).
    Dense-layer work per layer and side: 2 * rows * 128 * 64 FLOPs forward,
    twice that backward (input and weight gradients), and 384 bytes per row
    forward (a 256-byte BF16 input row read, a 128-byte output row written)."""
    from pramaan_b200.generators import rolling_horizon_batch
    from pramaan_b200.gnn import WarmStart, WarmStartNet

    models = rolling_horizon_batch(args.gnn_lps, seed=args.seed)
    m = sum(md.numRows() for md in models)
    n = sum(md.numVars() for md in models)
    rng = np.random.default_rng(args.seed)
    targets = [WarmStart(rng.uniform(0, 10, md.numVars()), rng.normal(0, 1, md.numRows()), 1.0) for md in models]
    net = WarmStartNet(device=device, seed=0)
    t0 = time.perf_counter()
    g = net.graph(models, targets)
    t_graph = time.perf_counter() - t0
    net.predict(g)
    net.train_step(g, 1e-4)
    t0 = time.perf_counter()
    for _ in range(args.gnn_reps):
        net.predict(g)
    t_fwd = (time.perf_counter() - t0) / args.gnn_reps
    t0 = time.perf_counter()
    for _ in range(args.gnn_reps):
        net.train_step(g, 1e-4)
    t_step = (time.perf_counter() - t0) / args.gnn_reps
    layers = 3
    fwd_flops = layers * 2 * 128 * 64 * (m + n)
    return {"workload": f"rolling_horizon_batch {args.gnn_lps} LPs, seed {args.seed}", "rows": m, "cols": n,
            "nodes": m + n, "nnz": sum(md.nnz() for md in models), "graph_build_s": t_graph,
            "forward_ms": t_fwd * 1e3, "train_step_ms": t_step * 1e3,
            "dense_forward_flops": fwd_flops, "dense_train_flops": 3 * fwd_flops,
            "dense_forward_bytes": layers * 384 * (m + n),
            "nodes_per_s_forward": (m + n) / t_fwd, "nodes_per_s_train": (m + n) / t_step}


def _tail_masks(batch, hints, k):
    """The last k periods of every window that has a hint (rolling_horizon_lp layout)."""
    from pramaan_b200.generators import rolling_horizon_tail_mask

    out = []
    for md, h in zip(batch, hints):
        PT = md.numVars() // 3
        T = md.numRows() - PT
        out.append(None if h is None else rolling_horizon_tail_mask(T, PT // T, k))
    return out


def _hints_for(batch, prev):
    """Each stream's previous window solution shifted onto its current window."""
    from pramaan_b200 import SolveStatus
    from pramaan_b200.generators import rolling_horizon_shift
    from pramaan_b200.gnn import WarmStart

    out = []
    for md, r in zip(batch, prev):
        if r.status != SolveStatus.kOptimal:
            out.append(None)
            continue
        PT = md.numVars() // 3
        T = md.numRows() - PT
        xs, ys = rolling_horizon_shift(r.x, r.y, T, PT // T)
        out.append(WarmStart(xs, ys, 0.0))
    return out


# ---------------------------------------------------------------------------
def run_gpu_arm(args):
    import torch

    t_start = time.perf_counter()

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    import pramaan_b200
    from pramaan_b200 import PdhgOptions, Session
    from pramaan_b200.generators import model_from_tensors, zipf_lp

    if args.only:
        sections = {"banded": banded_section, "gnn": gnn_section, "small": small_lp_section,
                    "stream": learned_stream_section,
                    "ceiling": lambda a, d: gather_ceiling(a.n, d),
                    "ladder": ladder_section, "solvers": reference_solvers_section,
                    "batch": batch_iteration_section, "tail": batch_tail_section,
                    "rolling": lambda a, d: rolling_horizon_section(a, d, dist)}
        out = sections[args.only](args, local)
        if rank == 0:
            print(json.dumps({"section": args.only, **out}), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    t = zipf_lp(args.m, args.n, cap=args.cap, seed=args.seed, device=f"cuda:{local}", as_tensors=True)
    model = model_from_tensors(t)
    del t
    torch.cuda.empty_cache()
    nnz = model.nnz()

    opts = PdhgOptions(device=local, use_graph=False, profile_kernels=True, gather_cache=args.gather_cache,
                       launch_blocks=args.launch_blocks, panel_split=args.panel_split)
    sess = Session(model, opts)
    gather = sess.gather_info()
    panel = sess.panel_info()
    stream = torch.cuda.ExternalStream(sess.stream(), device=local)
    for _ in range(args.warmup):
        sess.iterate(1)
    sess.synchronize()
    sess.kernel_times(reset=True)

    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("timed")
        ev0.record(stream)
        for _ in range(args.steps):
            sess.iterate(1)
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    if dist:
        tt = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    ms_dual, ms_primal, launches = sess.kernel_times(reset=True)
    b_dual, b_primal = sess.kernel_bytes()
    # The reference checks the FP64 residuals every check_frequency (100)
    # iterations; the timed steps run none.  Their cost, amortised:
    t0 = time.perf_counter()
    for _ in range(5):
        sess.residuals()
    check_ms = (time.perf_counter() - t0) / 5 * 1000.0
    sess.close()
    value = world * args.steps / (ms / 1000.0)

    # dominant kernel roofline
    hbm, peak_kind = measured_peaks()
    kinds = [("spmv_dual_fused", ms_dual, b_dual), ("spmv_primal_fused", ms_primal, b_primal)]
    tag, kms, kbytes = max(kinds, key=lambda k: k[1])
    avg_s = kms / 1000.0 / args.steps
    achieved = kbytes / avg_s / 1e9
    roofline = {"bound": "hbm", "kernel": tag, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_kind": peak_kind,
                "traffic": ncu_traffic(f"{tag}_zipf_lp_2Mx5M"),
                "algorithmic_bytes_per_launch": kbytes, "avg_launch_ms": avg_s * 1000,
                "timed_span": ("one A x̄ product: the column-panel kernel of the long rows, the short rows' "
                               "tiled product and its completion kernel, the long rows' finish kernel"
                               if tag == "spmv_dual_fused" and panel["panels"] else
                               "one Aᵀy product: the column-panel kernel of the hot rows, the tiled product of "
                               "the other entries and its completion kernel"
                               if tag == "spmv_primal_fused" and panel["primal_hot_rows"] else
                               "one product: its main kernel and its crossing-row completion kernel")}
    other = [k for k in kinds if k[0] != tag][0]
    roofline["other_kernel"] = {"kernel": other[0], "achieved": other[2] / (other[1] / 1000 / args.steps) / 1e9,
                                "frac": other[2] / (other[1] / 1000 / args.steps) / 1e9 / hbm,
                                "avg_launch_ms": other[1] / args.steps}
    if panel["panels"]:
        roofline["dual_panel_split"] = {**panel, "long_share": panel["long_nnz"] / nnz}
    # Second roofline: every non-zero is one random 4-byte gather of x̄ (A x̄)
    # or y (Aᵀ y, whose hot targets are read from shared memory instead).
    ceil = gather_ceiling(args.n, local)
    ceil["per_kernel"] = {}
    for k_tag, k_ms in (("spmv_dual_fused", ms_dual), ("spmv_primal_fused", ms_primal)):
        eps = nnz / (k_ms / 1000.0 / args.steps)
        ceil["per_kernel"][k_tag] = {"entries_per_s": eps, "frac_of_l2_gather_rate": eps / ceil["l2_gathers_per_s"]}
    roofline["gather_ceiling"] = ceil

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {**workload_config(args, nnz),
                       "gather": gather, "panel_split": panel},
            "gpu_launches": int(launches),
            "clocks": clk.summary(), "roofline": roofline,
            "residual_checks": {
                "note": "the timed steps run no FP64 residual check; the reference checks every 100 iterations",
                "check_ms": check_ms,
                "value_with_checks_every_100": world * args.steps / (ms / 1000.0 + args.steps / 100 * check_ms / 1000.0)}}

    # ---- end-to-end through the public C ABI with pinned host buffers ----
    if not args.no_e2e:
        pin = {}
        for name in ("obj_coeffs", "row_ptr", "col_idx", "values", "row_lower", "row_upper",
                     "var_lower", "var_upper"):
            a = getattr(model, name)
            tt = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
            tt.numpy()[...] = a
            pin[name] = tt
        from pramaan_b200.pdhg import ModelIR
        pm = ModelIR(*(pin[k].numpy() for k in ("obj_coeffs", "row_ptr", "col_idx", "values",
                                               "row_lower", "row_upper", "var_lower", "var_upper")),
                     model.obj_sense, model.obj_offset)
        solver = pramaan_b200.PdhgSolver(PdhgOptions(device=local, tolerance=0.0,
                                                     max_iterations=args.e2e_iters, check_frequency=100,
                                                     gather_cache=args.gather_cache,
                                                     panel_split=args.panel_split))
        solver.solve(pm)   # warm-up (module load, first-touch)
        times = []
        for _ in range(args.e2e_calls):
            t0 = time.perf_counter()
            r = solver.solve(pm)
            times.append(time.perf_counter() - t0)
        m, n = model.numRows(), model.numVars()
        # per call: the LP up (row_ptr, col_idx, values, c, bounds), x, y, the
        # row activity and the 8 FP64 check scalars of every check down
        h2d = 4 * (m + 1) + 4 * nnz + 8 * nnz + 8 * n + 16 * m + 16 * n
        d2h = 8 * n + 8 * m + 8 * m + 8 * 8 * (r.checks + 1)
        line["e2e"] = {"value": world * args.e2e_iters / statistics.median(times), "unit": UNIT,
                       "h2d_bytes_per_step": h2d / args.e2e_iters, "d2h_bytes_per_step": d2h / args.e2e_iters,
                       "h2d_bytes_per_call": h2d, "d2h_bytes_per_call": d2h,
                       "iterations_per_call": args.e2e_iters, "calls": args.e2e_calls,
                       "call_s_median": statistics.median(times),
                       "note": "pramaan_pdhg_solve from pinned host buffers, residual checks every 100 "
                               "iterations; the calls after the warm-up call reuse the library's device-memory "
                               "cache and its remembered launch shapes (repeated solves of one LP)"}

    # Sections: every rank runs the batched rolling-horizon section (its LPs
    # shard over the ranks); the single-LP sections are replicas and run on
    # one GPU only.
    single = world == 1
    wall = {"headline_and_e2e": time.perf_counter() - t_start}

    def section(key, fn, *a):
        t0 = time.perf_counter()
        line[key] = fn(*a)
        wall[key] = time.perf_counter() - t0

    if single and not args.no_banded:
        section("banded_spmv", banded_section, args, local)
    if single and not args.no_rolling:
        section("small_lp", small_lp_section, args, local)
    if single and not args.no_ladder:
        section("ladder_lp", ladder_section, args, local)
    if not args.no_rolling:
        section("rolling_horizon", rolling_horizon_section, args, local, dist)
    if single and not args.no_rolling:
        section("batched_products", batch_iteration_section, args, local)
        section("batch_tail", batch_tail_section, args, local)
    if single and not args.no_rolling:
        section("learned_stream", learned_stream_section, args, local)
        section("gnn_throughput", gnn_section, args, local)
    if rank == 0 and single and not args.no_cpu_baseline:
        t0 = time.perf_counter()
        v, threads, sample = cpu_baseline(model, args.cpu_seconds)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": sample,
                                "reference_solvers": reference_solvers_section(args, local)}
        wall["cpu_baseline"] = time.perf_counter() - t0
    line["section_wall_s"] = {k: round(v, 1) for k, v in wall.items()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_gpu_arm(args)


if __name__ == "__main__":
    main()
