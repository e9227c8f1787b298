"""Benchmark: plain FP32 CCD++ and SGD on the 100M-nonzero Zipf(1.1) tensor
(500,000 x 20,000 x 2,000, rank-16 CP values + N(0, 0.25^2) noise clipped to
[1, 5], 90/10 train/test split, R = 32).

One step = one CCD++ outer iteration (3 inner sweeps, lambda 0.1) followed by
one SGD epoch (lambda 0.01, lr 1e-3 decayed x0.95 per epoch, Hogwild), both
on HBM-resident data through libctc's device session.  metric: training
nonzeros processed per second (2 x nnz_train per step, whole job over all
ranks).  The tensor is larger than L2 (90M x 16 B per copy), so no L2 flush
is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's update rules on the host cores: the
OpenMP FP64 restatement in oracle/ (the reference ships its updates only as
CUDA kernels), on a seeded random sample of the same training tensor.
Multi-GPU runs are independent replicas (the path does not shard).
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

METRIC = "training nnz/s (CCD++ outer iteration + SGD epoch per step), 100M-nnz Zipf tensor, R=32"
UNIT = "nnz/s"
B_NZ = 16  # canonical bytes per nonzero: 3 x u32 coordinates + one FP32 value


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="zipf-100m")
    ap.add_argument("--nnz", type=int, default=0, help="override the nonzero count (smaller runs)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--sample", type=int, default=2_000_000, help="CPU baseline sample size")
    ap.add_argument("--no-extras", action="store_true", help="skip e2e / time-to-RMSE / CPU legs")
    ap.add_argument("--ccdpp-tile", type=int, default=0, help="CCD++ tile length (0 = library default)")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched 256-instance leg")
    ap.add_argument("--no-fo", action="store_true", help="skip the first-order (order-4 Adam) leg")
    ap.add_argument("--instances", type=int, default=0, help="batch workloads: a K-instance sample of the same distribution")
    ap.add_argument("--tune-cache", default="", help="autotuner cache file (default: a fresh temporary one)")
    ap.add_argument("--no-tune", action="store_true", help="library defaults instead of autotuned parameters")
    ap.add_argument("--als", action="store_true",
                    help="the ALS leg alone on --workload (zipf-400m runs it by default)")
    ap.add_argument("--sgd-atomic", type=int, default=-1,
                    help="with --no-tune: the Hogwild reduction mode of the step's SGD (1 vector atomics, 2 bulk "
                         "rows, 3 block-merged hot rows; default: the library's)")
    ap.add_argument("--mixed-step", action="store_true",
                    help="run the timed step's CCD++ in mixed precision (packed residual slots) instead of FP32 "
                         "(for profiling the mixed pass; the headline step is FP32)")
    ap.add_argument("--ref-cuda", action="store_true",
                    help="with --impl reference: time the reference's own CUDA kernels (built from its sources "
                         "for sm_100a) on this GPU instead of the CPU restatement")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


# ---------------------------------------------------------------------------
def make_workload(args, device):
    from cutc_b200 import synth
    w = synth.WORKLOADS[args.workload]
    if args.nnz:
        w = synth.scaled(w, args.nnz)
    data = synth.generate(w, seed=args.seed, device=device)
    return w, data


def sort_modes_torch(ind, vals, dims, device):
    """Stable sorts by (ind[m], ind[m+1]) for m = 0, 1, 2 on the GPU."""
    import torch
    ti = torch.from_numpy(ind.astype(np.int64)).to(device)
    out = []
    for m in range(3):
        key = ti[m] * (dims[(m + 1) % 3] + 1) + ti[(m + 1) % 3]
        _, order = torch.sort(key, stable=True)
        o = order.cpu().numpy()
        out.append((ind[:, o], vals[o]))
        del key, order
    del ti
    torch.cuda.empty_cache()
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.dev)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profile_traffic(kernel_tag):
    """DRAM bytes per launch of a kernel at the full workload, from the
    committed record of its ncu capture (profiles/<kernel_tag>.json, which
    holds the capture command and how the figure was scaled)."""
    p = os.path.join(ROOT, "profiles", f"{kernel_tag}.json")
    try:
        with open(p) as f:
            return float(json.load(f)["dram_bytes_per_launch_full"])
    except (OSError, KeyError, ValueError):
        return None


def max_over_ranks(x: float, device, world: int) -> float:
    """The slowest rank's value (all ranks take part; 1 rank: x)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
def cpu_als_small(seed):
    """The small uniform workload as configured (2,000 x 1,500 x 200, 200k
    nonzeros, 90/10 split, R 16, lambda 0.05, 10 iterations, factors
    U(0,1)/sqrt(16)) on the host cores: the OpenMP FP64 restatement of the
    reference's ALS update (the reference ships its updates only as CUDA).
    Returns seconds per iteration, nnz/s, threads and the final test RMSE."""
    from cutc_b200 import synth
    from oracle import pyoracle as po
    w = synth.WORKLOADS["small-als"]
    g = synth.generate(w, seed=seed, device="cpu")
    dims = list(w.dims)
    tr = [po.Tensor(*synth.sort_for_mode(*g["train"], m), dims=dims) for m in range(3)]
    te = po.Tensor(*g["test"], dims=dims)
    rng = np.random.default_rng(seed)
    U = [rng.uniform(0, 1, (d, w.rank)) / np.sqrt(w.rank) for d in dims]
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    for _ in range(10):
        for m in range(3):
            po.als_mode(tr[m], m, U, 0.05, None, False, nthreads=threads)
    s = (time.perf_counter() - t0) / 10
    return {"workload": w.name, "s_per_iteration": s, "nnz_per_s": tr[0].nnz / s, "cores": threads,
            "iterations": 10, "test_rmse": po.rmse(te, U, nthreads=threads), "kind": "port",
            "note": "OpenMP FP64 restatement of the reference ALS update (sgpu/als.cu:186-317, 467-491)"}


def gpu_als_small(ctc, ctx, seed):
    """The small uniform ALS workload (as cpu_als_small, same seeded tensor
    and factors) on the GPU: FP32, 10 iterations from the host tensors
    through ctc_run; device time of the update epochs per iteration and the
    whole call's wall time (staging, epochs, evaluation, factors back)."""
    from cutc_b200 import synth
    w = synth.WORKLOADS["small-als"]
    g = synth.generate(w, seed=seed, device="cpu")
    rng = np.random.default_rng(seed)
    U = [rng.uniform(0, 1, (d, w.rank)) / np.sqrt(w.rank) for d in w.dims]
    tr = ctc.Tensor.from_coo(*synth.sort_for_mode(*g["train"], 0), dims=w.dims)
    te = ctc.Tensor.from_coo(*g["test"], dims=w.dims)
    p = ctc.params("als", rank=w.rank, iters=10, early_stop=0, eval_every=0, **{"lambda": 0.05})
    res = None
    for _ in range(2):  # the first call pays one-time module loads
        m = ctc.Model(w.dims, w.rank)
        m.set_factors(U)
        t0 = time.perf_counter()
        out = ctc.run(ctx, [tr], None, te, m, p)
        wall = time.perf_counter() - t0
        res = {"workload": w.name, "s_per_iteration": out.result["total_ms"] / 1000.0 / 10,
               "nnz_per_s": tr.nnz / (out.result["total_ms"] / 1000.0 / 10), "call_s": wall,
               "test_rmse": out.epochs[-1]["rmse_te"], "precision": "f32"}
    return res


def cpu_baseline(train_sorted0, dims, R, sample, seed, steps=1):
    """The reference's update rules on the host cores (OpenMP FP64 oracle)
    on a seeded random sample: CCD++ outer iteration (3 inner, lambda 0.1)
    + Hogwild SGD epoch; returns (nnz/s, seconds per step, threads)."""
    from oracle import pyoracle as po
    ind, vals = train_sorted0
    n = ind.shape[1]
    rng = np.random.default_rng(seed + 17)
    pick = np.sort(rng.choice(n, size=min(sample, n), replace=False))
    T = po.Tensor(ind[:, pick], vals[pick], list(dims))
    threads = os.cpu_count() or 1
    U = [rng.uniform(0, 1, (d, R)) / np.sqrt(R) for d in dims]
    r = po.residual(T, U)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        po.ccdpp_outer(T, U, 0.1, 3, r, nthreads=threads)
        po.sgd_epoch_hogwild(T, U, 1e-3, 0.01, 1.0, threads)
        times.append(time.perf_counter() - t0)
    s = statistics.median(times)
    return 2 * T.nnz / s, s, threads, T.nnz


# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist

    import cutc_b200 as ctc

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    device = f"cuda:{local}"
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))

    w, data = make_workload(args, device)
    dims = w.dims
    R = w.rank
    train_ind, train_vals = data["train"]
    test_ind, test_vals = data["test"]
    del data
    sorted3 = sort_modes_torch(train_ind, train_vals, dims, device)
    del train_ind, train_vals
    torch.cuda.empty_cache()

    ctx = ctc.Context(local)
    tr = [ctc.Tensor.from_coo(i, v, dims=dims) for i, v in sorted3]
    te = ctc.Tensor.from_coo(test_ind, test_vals, dims=dims)
    n_train = sorted3[0][0].shape[1]
    n_test = test_ind.shape[1]
    base0 = sorted3[0] if (rank == 0 and not args.no_extras) else None
    del sorted3

    p_ccd = ctc.params("ccdpp", rank=R, inner=3, early_stop=0, iters=10, tile_len=args.ccdpp_tile,
                       precision=ctc.PREC_MIXED if args.mixed_step else ctc.PREC_F32, **{"lambda": 0.1})
    p_sgd = ctc.params("sgd", rank=R, lr=1e-3, lr_scale=1.0, lr_schedule=ctc.LR_EXP_DECAY, lr_decay=0.95,
                       early_stop=0, iters=20, **{"lambda": 0.01})
    if args.sgd_atomic >= 0:
        p_sgd.sgd_atomic = args.sgd_atomic
    # autotuned tile length / lanes per nonzero / column staging for this
    # shape (the library defaults are among the candidates: their epoch
    # times are reported as the plain form)
    tuned = None
    cache = None
    if not args.no_tune and not args.ccdpp_tile:
        import tempfile
        cache = args.tune_cache or os.path.join(tempfile.mkdtemp(), "tune.txt")
        t0 = time.time()
        p_ccd, tr_ccd = ctc.autotune(ctx, tr, p_ccd, cache_path=cache)
        p_sgd, tr_sgd = ctc.autotune(ctx, [tr[0]], p_sgd, cache_path=cache)
        tuned = {"search_s": time.time() - t0, "cache_hit": bool(tr_ccd and tr_ccd[0]["cached"]),
                 "ccdpp": {"tile_len": p_ccd.tile_len, "smem_budget": p_ccd.smem_budget, "trials": tr_ccd},
                 "sgd": {"tile_len": p_sgd.tile_len, "threads_per_row": p_sgd.threads_per_row,
                         "sgd_atomic": p_sgd.sgd_atomic, "threads_per_block": p_sgd.threads_per_block,
                         "trials": tr_sgd}}
    ds_ccd = ctc.Dataset(ctx, tr, None, te, p_ccd)
    ds_sgd = ctc.Dataset(ctx, [tr[0]], None, te, p_sgd)
    mdims = ds_ccd.dims()
    m_ccd = ctc.Model(mdims, R).init_uniform(args.seed + 1, 1.0 / np.sqrt(R))
    m_sgd = ctc.Model(mdims, R).init_uniform(args.seed + 1, 1.0 / np.sqrt(R))
    ds_ccd.set_model(m_ccd)
    ds_sgd.set_model(m_sgd)

    ext = torch.cuda.ExternalStream(ctx.stream(), device=device)
    lr = [1e-3]

    def step():
        ds_ccd.epochs(1)
        ds_sgd.epochs(1)
        lr[0] *= 0.95
        ds_sgd.set_lr(lr[0])

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ctx.set_profiling(True)
    ctx.reset_kernel_times()
    launches0 = ctx.launches()
    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps * 2 + 1)]
    ev[0].record(ext)
    for s in range(args.steps):
        ds_ccd.epochs(1)
        ev[2 * s + 1].record(ext)
        ds_sgd.epochs(1)
        ev[2 * s + 2].record(ext)
        lr[0] *= 0.95
        ds_sgd.set_lr(lr[0])
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    launches = ctx.launches() - launches0
    total_ms = ev[0].elapsed_time(ev[-1])
    ccd_ms = sum(ev[2 * s].elapsed_time(ev[2 * s + 1]) for s in range(args.steps)) / args.steps
    sgd_ms = sum(ev[2 * s + 1].elapsed_time(ev[2 * s + 2]) for s in range(args.steps)) / args.steps
    pass_n, pass_ms = ctx.kernel_time("k_ccdpp_pass")
    sgd_n, sgd_kms = ctx.kernel_time("k_sgd")
    ctx.set_profiling(False)
    ms_per_step = max_over_ranks(total_ms / args.steps, device, world)
    value = world * 2 * n_train / (ms_per_step / 1000.0)

    # roofline of the dominant kernel (the CCD++ column pass): algorithmic
    # bytes per launch = (B_nz + 4) * nnz_train + column traffic, the
    # canonical count (16-byte nonzero + 4-byte residual).  The kernel's own
    # layout moves fewer: 8-byte packed keys + 4-byte residual per nonzero,
    # plus a 4-byte residual write in the first sweep of each column (1 in
    # `inner` launches).
    peak, peak_src = measured_peaks()
    col_bytes = 4 * (sum(mdims) + max(mdims))
    pass_bytes = (B_NZ + 4) * n_train + col_bytes
    inner = 3
    layout_bytes = 12 * n_train + 4 * n_train / inner + col_bytes
    pass_avg_ms = pass_ms / max(pass_n, 1)
    achieved = pass_bytes / (pass_avg_ms / 1000.0) / 1e9
    layout_gbps = layout_bytes / (pass_avg_ms / 1000.0) / 1e9
    sgd_bytes = B_NZ * n_train + 2 * sum(mdims) * R * 4
    sgd_avg_ms = sgd_kms / max(sgd_n, 1)

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Zipf CP tensor)",
        "config": {"workload": w.name, "dims": list(dims), "nnz_total": w.nnz, "nnz_train": n_train,
                   "nnz_test": n_test, "rank": R, "ccdpp": {"lambda": 0.1, "inner": 3},
                   "sgd": {"lambda": 0.01, "lr": 1e-3, "decay": 0.95,
                           "order": {0: "hogwild-stores", 1: "hogwild-vector-atomics", 2: "hogwild-bulk-rows",
                                     3: "hogwild-block-merged-hot-rows"}[p_sgd.sgd_atomic],
                           "tile_len": p_sgd.tile_len, "threads_per_row": p_sgd.threads_per_row,
                           "threads_per_block": p_sgd.threads_per_block},
                   "ccdpp_precision": "mixed (packed slots)" if args.mixed_step else "f32",
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (no flush)"},
        "epoch_s": {"ccdpp_outer": ccd_ms / 1000.0, "sgd": sgd_ms / 1000.0},
        "nnz_per_s": {"ccdpp": n_train / (ccd_ms / 1000.0), "sgd": n_train / (sgd_ms / 1000.0)},
        "roofline": {"bound": "hbm", "kernel": "k_ccdpp_pass", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_src,
                     "traffic": profile_traffic("k_ccdpp_pass__zipf100m"),
                     "bytes_per_launch": pass_bytes, "launches": pass_n, "avg_launch_ms": pass_avg_ms,
                     "share_of_step": pass_ms / max(total_ms, 1e-9),
                     "layout_bytes_per_launch": layout_bytes, "layout_GBps": layout_gbps,
                     "layout_frac": layout_gbps / peak},
        "sgd_kernel": {"kernel": "k_sgd", "avg_launch_ms": sgd_avg_ms,
                       "algorithmic_GBps": sgd_bytes / (sgd_avg_ms / 1000.0) / 1e9,
                       "frac_hbm": sgd_bytes / (sgd_avg_ms / 1000.0) / 1e9 / peak},
        "gpu_launches": int(launches),
        "clocks": clk,
        "tuned": tuned,
    }

    if rank == 0 and not args.no_extras:
        # plain FP32 ALS on the same tensor (lambda 0.1), staged from the
        # mode-1 tensor alone: its copies are sorted on the device
        # ALS, plain and mixed, each with its own tuned tile length
        p_als = ctc.params("als", rank=R, early_stop=0, iters=10, **{"lambda": 0.1})
        p_als_mx = ctc.params("als", rank=R, precision=ctc.PREC_MIXED, early_stop=0, iters=10, **{"lambda": 0.1})
        if cache:
            p_als, _ = ctc.autotune(ctx, [tr[0]], p_als, cache_path=cache)
            p_als_mx, _ = ctc.autotune(ctx, [tr[0]], p_als_mx, cache_path=cache)
            tuned["als"] = {"tile_len": p_als.tile_len}
            tuned["als_mixed"] = {"tile_len": p_als_mx.tile_len}
        ds_als = ctc.Dataset(ctx, [tr[0]], None, te, p_als)
        out["time_to_rmse"] = time_to_rmse(ctc, ds_ccd, ds_sgd, mdims, R, args.seed, ds_als)
        ds_als.free()
        out["mixed_vs_plain"] = mixed_vs_plain(ctc, ctx, tr, te, mdims, R, args.seed, p_ccd, out["time_to_rmse"],
                                               p_als_mx)
        out["e2e"] = e2e(ctc, ctx, tr, te, mdims, R, n_train, n_test, args, p_ccd, p_sgd)
        out["ciss_build"] = ciss_build_times(ctc, ctx, tr[0])
        out["als_small"] = gpu_als_small(ctc, ctx, args.seed)
        v, s, threads, nsamp = cpu_baseline(base0, dims, R, args.sample, args.seed)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"{nsamp} of {n_train} training nonzeros (seeded random), one "
                                         f"CCD++ outer (3 inner) + one Hogwild SGD epoch, FP64 OpenMP, "
                                         f"{s:.2f} s per step"}
    elif not args.no_extras:
        out["e2e"] = None
    out["sse_kernel"] = sse_roofline(ctx, ds_sgd, n_train, n_test, mdims, R, peak)
    ds_ccd.free()
    ds_sgd.free()
    del tr, te
    if rank == 0 and not args.no_extras and not args.no_batch:
        out["batched"] = batch_leg(ctc, ctx, args, device)
    if rank == 0 and not args.no_extras and not args.no_fo:
        out["first_order"] = fo_leg(ctc, ctx, argparse.Namespace(**{**vars(args), "nnz": 0}), device)
    if rank == 0:
        print(json.dumps(out))
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def batch_leg(ctc, ctx, args, device):
    """Batched small instances: the 256-instance workload (dims log-U[1e3,
    5e4] per mode, nnz log-U[1e4, 5e6] per instance, uniform distinct cells,
    CP rank 8 + N(0, 0.1^2), R = 16), all instances stacked into one batch,
    10 epochs of ALS and of Hogwild SGD, each epoch one CUDA-graph launch.
    Reports total training nonzeros/s and each instance's time to reach
    1.005 x its own final test RMSE."""
    from cutc_b200 import synth
    bw = synth.BATCH_WORKLOADS["batch-256"]
    if args.instances:
        bw = synth.BatchWorkload(bw.name + f"@{args.instances}", args.instances, bw.dim_range, bw.nnz_range,
                                 bw.cp_rank, bw.rank, bw.sigma)
    R = bw.rank
    t0 = time.time()
    train, test, idims = [], [], []
    ntr = nte = 0
    for inst in synth.generate_batch(bw, seed=args.seed, device=device):
        train.append(ctc.Tensor.from_coo(*inst["train"], dims=inst["dims"]))
        test.append(ctc.Tensor.from_coo(*inst["test"], dims=inst["dims"]))
        idims.append(inst["dims"])
        ntr += int(inst["train"][1].size)
        nte += int(inst["test"][1].size)
    out = {"workload": bw.name, "instances": bw.ninst, "nnz_train": ntr, "nnz_test": nte, "rank": R,
           "epochs": 10, "generate_s": time.time() - t0,
           "params": {"als": {"lambda": 2.0}, "sgd": {"lr": 3e-2, "decay": 0.95, "lambda": 0.01}}}
    # the workload fixes neither lambda nor lr: a 32-instance sweep (ALS
    # lambda in {0.05, 0.5, 2, 5, 20}; SGD lr in {1e-3, 1e-2, 3e-2, 0.1} x
    # lambda in {0.01, 0.1}) gave the lowest median test RMSE at these
    legs = {
        "als": ctc.params("als", rank=R, iters=10, early_stop=0, eval_every=1, use_graph=1, **{"lambda": 2.0}),
        "sgd": ctc.params("sgd", rank=R, lr=3e-2, lr_scale=1.0, lr_schedule=ctc.LR_EXP_DECAY, lr_decay=0.95,
                          iters=10, early_stop=0, eval_every=1, use_graph=1, **{"lambda": 0.01}),
    }
    for name, p in legs.items():
        t1 = time.time()
        B = ctc.Batch(ctx, train, test, p)
        stage_s = time.time() - t1
        models = [ctc.Model(d, R).init_uniform(args.seed + 1 + b, 1.0 / np.sqrt(R)) for b, d in enumerate(idims)]
        l0 = ctx.launches()
        run = B.run(models, p)
        launches = ctx.launches() - l0
        ms = np.array([e[1] for e in run.epochs])          # epoch 0: evaluation only
        te = np.stack([e[3] for e in run.epochs])          # (epochs + 1) x instances
        final = te[-1]
        cum = np.cumsum(ms) / 1000.0
        reach = [float(cum[int(np.argmax(te[:, b] <= 1.005 * final[b]))]) for b in range(te.shape[1])]
        total_s = float(ms.sum()) / 1000.0
        out[name] = {
            "epoch_ms": 1000.0 * total_s / 10, "nnz_per_s": 10 * ntr / total_s, "stage_s": stage_s,
            "launches_per_epoch_incl_eval": launches / 10,
            "time_to_rmse_s": {"median": float(np.median(reach)), "p90": float(np.percentile(reach, 90)),
                               "max": float(np.max(reach))},
            "final_test_rmse": {"median": float(np.median(final)), "min": float(final.min()),
                                "max": float(final.max())},
        }
        B.free()
        for m in models:
            m.free()
    return out


def fo_leg(ctc, ctx, args, device):
    """Adjoint-driven minibatch Adam on the order-4 workload (1M x 200k x 1k
    x 24, 250M Zipf(1.2) cells, CP rank 32 + N(0, 0.1^2), R = 64, minibatch
    2^20 nonzeros, Adam lr 1e-3): epochs in FP32 and with BF16 gathers
    (FP32 masters and accumulation).  Reports epoch time, nonzeros/s, the
    adjoint kernel's share and throughput, and the test RMSE of both."""
    import torch

    from cutc_b200 import synth
    w = synth.WORKLOADS["zipf4-250m"]
    if args.nnz:
        w = synth.scaled(w, args.nnz)
    t0 = time.time()
    data = synth.generate(w, seed=args.seed, device=device)
    tr = ctc.Tensor.from_coo(*data["train"], dims=w.dims)
    te = ctc.Tensor.from_coo(*data["test"], dims=w.dims)
    ntr, nte = int(data["train"][1].size), int(data["test"][1].size)
    del data
    torch.cuda.empty_cache()
    out = {"workload": w.name, "dims": list(w.dims), "nnz_train": ntr, "nnz_test": nte, "rank": w.rank,
           "batch": 1 << 20, "lr": 1e-3, "lambda": 1e-4, "generate_s": time.time() - t0}
    epochs = 2
    for name, prec in (("fp32", ctc.PREC_F32), ("mixed_bf16", ctc.PREC_MIXED)):
        p = ctc.fo_params(rank=w.rank, precision=prec, lr=1e-3, batch=1 << 20, epochs=epochs, eval_every=0,
                          seed=args.seed + 1, **{"lambda": 1e-4})
        t1 = time.time()
        F = ctc.FirstOrder(ctx, tr, te, p)
        stage_s = time.time() - t1
        m = ctc.Model(w.dims, w.rank).init_uniform(args.seed + 1, 1.0 / np.sqrt(w.rank))
        ctx.set_profiling(True)
        ctx.reset_kernel_times()
        run = F.run(m, p)
        kn, kms = ctx.kernel_time("k_fo_grad")
        an, ams = ctx.kernel_time("k_fo_adam")
        ctx.set_profiling(False)
        ep_ms = [run.result["total_ms"] / epochs] * epochs  # device time of the update epochs
        steps = (ntr + (1 << 20) - 1) >> 20
        grad_launches = steps * epochs
        # adjoint kernel per launch: 16 B indices + 4 B value per nonzero and
        # four gathered rows (R elements each) per nonzero
        gbytes = 2 if prec == ctc.PREC_MIXED else 4
        per_nz = 20 + 4 * w.rank * gbytes
        grad_avg = kms / max(kn, 1)
        out[name] = {"epoch_s": float(np.mean(ep_ms)) / 1000.0, "nnz_per_s": ntr / (float(np.mean(ep_ms)) / 1000.0),
                     "stage_s": stage_s, "test_rmse": run.epochs[-1]["rmse_te"],
                     "train_rmse": run.epochs[-1]["rmse_tr"], "initial_test_rmse": run.epochs[0]["rmse_te"],
                     "adjoint": {"launches": kn, "avg_ms": grad_avg,
                                 "share": kms / max(sum(ep_ms), 1e-9),
                                 "gathered_GBps": (1 << 20) * per_nz / (grad_avg / 1000.0) / 1e9},
                     "adam": {"launches": an, "avg_ms": ams / max(an, 1)}}
        F.free()
        m.free()
    return out


def time_to_rmse(ctc, ds_ccd, ds_sgd, mdims, R, seed, ds_als=None, legs=None, targets=None):
    """Plain FP32 schedules (CCD++ 10 outer x 3 inner, SGD 20 epochs, ALS
    10 iterations); the target is 1.005 x the final test RMSE (or the given
    targets[name]); time = device time of the update epochs until the test
    RMSE first reaches it."""
    import torch
    res = {}
    if legs is None:
        legs = [("ccdpp", ds_ccd, 10), ("sgd", ds_sgd, 20)]
        if ds_als is not None:
            legs.append(("als", ds_als, 10))
    for name, ds, iters in legs:
        m = ctc.Model(mdims, R).init_uniform(seed + 1, 1.0 / np.sqrt(R))
        ds.set_model(m)
        ext = torch.cuda.ExternalStream(ds.ctx.stream())
        lr = 1e-3
        if name == "sgd":
            ds.set_lr(lr)
        hist = []
        t = 0.0
        for e in range(iters):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(ext)
            ds.epochs(1)
            b.record(ext)
            b.synchronize()
            t += a.elapsed_time(b) / 1000.0
            st = ds.evaluate()
            hist.append((t, st["rmse_te"], st["rmse_tr"]))
            if name == "sgd":
                lr *= 0.95
                ds.set_lr(lr)
        final = hist[-1][1]
        target = targets[name] if targets and name in targets else final * 1.005
        reach = next((h[0] for h in hist if h[1] <= target), None)
        res[name] = {"epochs": iters, "final_test_rmse": final, "final_train_rmse": hist[-1][2],
                     "target_test_rmse": target, "time_to_target_s": reach, "total_s": hist[-1][0],
                     "epoch_s": hist[-1][0] / iters}
    return res


def mixed_vs_plain(ctc, ctx, tr, te, mdims, R, seed, p_ccd, plain, p_als_mx=None):
    """The mixed-precision forms on the same tensor and schedules, against
    the plain FP32 runs of time_to_rmse (`plain`): ALS with BF16 factor
    copies into tcgen05 Gram blocks for the pieces of long rows (FP64 row
    solves), and CCD++ with packed 8-byte slots (the residual in the key
    word's low bits).  Target: 1.005 x the plain form's final test RMSE.
    Hogwild SGD has no mixed form (its epoch is bound by same-row L2
    reductions into the FP32 rows, which a narrower gather does not
    remove)."""
    legs = []
    if p_als_mx is None:
        p_als_mx = ctc.params("als", rank=R, precision=ctc.PREC_MIXED, early_stop=0, iters=10, **{"lambda": 0.1})
    ds_als = ctc.Dataset(ctx, [tr[0]], None, te, p_als_mx)
    q = ctc.params("ccdpp", rank=R, inner=3, early_stop=0, iters=10, precision=ctc.PREC_MIXED,
                   tile_len=p_ccd.tile_len, smem_budget=p_ccd.smem_budget, **{"lambda": 0.1})
    ds_ccd = ctc.Dataset(ctx, [tr[0]], None, te, q)
    legs = [("ccdpp", ds_ccd, 10), ("als", ds_als, 10)]
    targets = {k: plain[k]["final_test_rmse"] * 1.005 for k in ("ccdpp", "als")}
    mixed = time_to_rmse(ctc, None, None, mdims, R, seed, legs=legs, targets=targets)
    ds_als.free()
    ds_ccd.free()
    res = {}
    for k in ("ccdpp", "als"):
        a, b = plain[k], mixed[k]
        res[k] = {"plain_epoch_s": a["epoch_s"], "mixed_epoch_s": b["epoch_s"],
                  "epoch_speedup": a["epoch_s"] / b["epoch_s"],
                  "plain_final_test_rmse": a["final_test_rmse"], "mixed_final_test_rmse": b["final_test_rmse"],
                  "final_rmse_rel_diff": (b["final_test_rmse"] - a["final_test_rmse"]) / a["final_test_rmse"],
                  "target_test_rmse": targets[k], "plain_time_to_target_s": a["time_to_target_s"],
                  "mixed_time_to_target_s": b["time_to_target_s"],
                  "time_to_target_speedup": (a["time_to_target_s"] / b["time_to_target_s"]
                                             if a["time_to_target_s"] and b["time_to_target_s"] else None)}
    res["sgd"] = None
    return res


def sse_roofline(ctx, ds, n_train, n_test, mdims, R, peak):
    """The per-nonzero residual / squared-error kernel (k_sse) over the
    training copy and the test tensor of the SGD dataset (one evaluation):
    algorithmic bytes = 16 B per nonzero + one read of the three factors,
    per launch, over its event-timed duration."""
    ds.evaluate()  # warm
    ctx.set_profiling(True)
    ctx.reset_kernel_times()
    for _ in range(3):
        ds.evaluate()
    n, ms = ctx.kernel_time("k_sse")
    ctx.set_profiling(False)
    fac = sum(mdims) * R * 4
    nbytes = B_NZ * (n_train + n_test) + 2 * fac
    per_eval_ms = ms / 3.0
    gbps = nbytes / (per_eval_ms / 1000.0) / 1e9
    return {"kernel": "k_sse", "launches_per_eval": n // 3, "ms_per_eval": per_eval_ms,
            "algorithmic_bytes_per_eval": nbytes, "achieved_GBps": gbps, "frac_hbm": gbps / peak}


def ciss_build_times(ctc, ctx, t0):
    """The reference's CISS layout (tile length 32, mode 1) of the mode-1
    training copy, built by the host builder and by the device builder
    through the C ABI (host tensor in, host CISS object out: the device
    build includes its transfers); the export to numpy is not timed."""
    import ctypes as C
    L = ctc.lib()
    res = {}
    for name, build in (("host_s", lambda h: L.ctc_ciss_build(t0.h, 1, 32, C.byref(h))),
                        ("gpu_s", lambda h: L.ctc_ciss_build_gpu(ctx.h, t0.h, 1, 32, 0, C.byref(h)))):
        h = C.c_void_p()
        t = time.perf_counter()
        rc = build(h)
        res[name] = time.perf_counter() - t
        if rc != 0:
            raise RuntimeError(f"CISS build failed ({rc})")
        L.ctc_ciss_free(h)
    return res


def e2e(ctc, ctx, tr, te, mdims, R, n_train, n_test, args, p_ccd=None, p_sgd=None):
    """The same metric through the reference-facing call with host buffers:
    ctc_run on the mode-1 training tensor alone, as the reference's tc_ccd /
    tc_sgd take one training tensor and build their own copies (the
    records go to the device once; the other mode orders, tile plans and
    CCD++ slots are made there), then one epoch, evaluation and the factors
    copied back, for CCD++ and for SGD, with the tuned tile length, lanes,
    column staging and reduction mode when given (a tuning cache hit)."""

    def knobs(p):
        return {} if p is None else dict(tile_len=p.tile_len, threads_per_row=p.threads_per_row,
                                         smem_budget=p.smem_budget, sgd_atomic=p.sgd_atomic,
                                         threads_per_block=p.threads_per_block)
    h2d = 2 * (n_train + n_test) * 16 + 2 * sum(mdims) * R * 4
    d2h = 2 * 2 * sum(mdims) * R * 4
    times = []
    for _ in range(2):
        m1 = ctc.Model(mdims, R).init_uniform(args.seed + 1, 1.0 / np.sqrt(R))
        m2 = ctc.Model(mdims, R).init_uniform(args.seed + 1, 1.0 / np.sqrt(R))
        t0 = time.perf_counter()
        ctc.run(ctx, [tr[0]], None, te, m1, ctc.params("ccdpp", rank=R, inner=3, iters=1, early_stop=0,
                                                  eval_every=0, **knobs(p_ccd), **{"lambda": 0.1}))
        ctc.run(ctx, [tr[0]], None, te, m2, ctc.params("sgd", rank=R, lr=1e-3, lr_scale=1.0, iters=1,
                                                       lr_schedule=ctc.LR_CONSTANT, early_stop=0,
                                                       eval_every=0, **knobs(p_sgd), **{"lambda": 0.01}))
        times.append(time.perf_counter() - t0)
    s = min(times)
    return {"value": 2 * n_train / s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "s_per_step": s,
            "note": "ctc_run from the host mode-1 tensor: staging (records, device-sorted copies, tile plans, "
                    "CCD++ slots), one epoch, evaluation and the factors back, inside the timed call"}


# ---------------------------------------------------------------------------
def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    import torch
    device = f"cuda:{local}" if torch.cuda.is_available() else "cpu"
    w, data = make_workload(args, device)
    s0 = data["train"]
    n_train = s0[0].shape[1]
    del data
    vals_list = []
    for _ in range(args.warmup):
        cpu_baseline(s0, w.dims, w.rank, args.sample, args.seed)
    t = []
    for k in range(args.steps):
        v, s, threads, nsamp = cpu_baseline(s0, w.dims, w.rank, args.sample, args.seed + k)
        t.append(s)
        vals_list.append(v)
    s = statistics.median(t)
    value = 2 * nsamp / s
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": s * 1000.0, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Zipf CP tensor)", "impl": "reference",
           "config": {"workload": w.name, "dims": list(w.dims), "nnz_total": w.nnz, "nnz_train": n_train,
                      "rank": w.rank},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                            "sample": f"{nsamp} of {n_train} training nonzeros per step (seeded random); "
                                      f"CCD++ outer (3 inner) + Hogwild SGD epoch, FP64 OpenMP restatement of "
                                      f"the reference update rules (its updates ship only as CUDA)"},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    # the small uniform ALS workload, which the reference's configuration
    # defines to run on the CPU path
    out["als_small_cpu"] = cpu_als_small(args.seed)
    print(json.dumps(out))


def als_leg(ctc, ctx, args, device):
    """ALS on --workload: at rank 64 (the 400M-nonzero Zipf(1.3) tensor,
    1M x 600k x 300, CP rank 24 + N(0, 0.2^2), lambda 0.05) iterations in
    FP32 and in mixed precision (BF16 factor copies into tcgen05 Gram blocks
    for the pieces of long rows, FP64 row solves with one refinement step);
    at other ranks (the 100M-nonzero rank-32 tensor, lambda 0.1) FP32."""
    import torch

    from cutc_b200 import synth
    w = synth.WORKLOADS[args.workload]
    if args.nnz:
        w = synth.scaled(w, args.nnz)
    t0 = time.time()
    data = synth.generate(w, seed=args.seed, device=device)
    ti, tv = data["train"]
    te = ctc.Tensor.from_coo(*data["test"], dims=w.dims)
    ntr = int(tv.size)
    del data
    srt = sort_modes_torch(ti, tv, w.dims, device)
    del ti, tv
    torch.cuda.empty_cache()
    tr = [ctc.Tensor.from_coo(i, v, dims=w.dims) for i, v in srt]
    del srt
    lam = 0.05 if w.rank == 64 else 0.1
    out = {"workload": w.name, "dims": list(w.dims), "nnz_train": ntr, "rank": w.rank, "lambda": lam,
           "generate_s": time.time() - t0}
    iters = 3
    forms = [("fp32", ctc.PREC_F32)] + ([("mixed_tc", ctc.PREC_MIXED)] if w.rank in (32, 64) else [])
    for name, prec in forms:
        p = ctc.params("als", rank=w.rank, precision=prec, iters=iters, early_stop=0, eval_every=0,
                       **{"lambda": lam})
        trials = None
        if not args.no_tune:
            # tile length per form (mixed precision also tries 128, sending more
            # rows to the tensor-core Gram); the search is not timed
            p, trials = ctc.autotune(ctx, tr, p, cache_path=args.tune_cache or None)
        t1 = time.time()
        ds = ctc.Dataset(ctx, tr, None, te, p)
        stage_s = time.time() - t1
        m = ctc.Model(ds.dims(), w.rank).init_uniform(args.seed + 1, 1.0 / np.sqrt(w.rank))
        ctx.set_profiling(True)
        ctx.reset_kernel_times()
        run = ds.run(m, p)
        kt = {k: ctx.kernel_time(k) for k in ("k_als_tile", "k_als_sum_pieces", "k_als_fix", "k_als_gram_tc")}
        ctx.set_profiling(False)
        it_s = run.result["total_ms"] / 1000.0 / iters
        out[name] = {"iteration_s": it_s, "nnz_per_s": ntr / it_s, "stage_s": stage_s, "tile_len": p.tile_len,
                     "test_rmse": run.epochs[-1]["rmse_te"], "train_rmse": run.epochs[-1]["rmse_tr"],
                     "kernels": {k: {"launches": v[0], "ms_per_iter": v[1] / iters} for k, v in kt.items() if v[0]},
                     "tune_trials": trials}
        ds.free()
        m.free()
    return out


def run_als_only(args):
    """--workload zipf-400m: the rank-64 ALS leg alone, as its own JSON line."""
    import torch

    import cutc_b200 as ctc
    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    ctx = ctc.Context(local)
    a = als_leg(ctc, ctx, args, f"cuda:{local}")
    form = "mixed_tc" if "mixed_tc" in a else "fp32"
    metric = ("ALS training nnz/s (rank 64, mixed precision with tensor-core Gram blocks)" if form == "mixed_tc"
              else f"ALS training nnz/s (rank {a['rank']}, FP32)")
    print(json.dumps({"metric": metric,
                      "value": a[form]["nnz_per_s"], "unit": UNIT, "n_gpus": 1, "steps": 3, "warmup": 0,
                      "ms_per_step": 1000.0 * a[form]["iteration_s"], "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None,
                      "dtype": "bf16/f32/f64" if form == "mixed_tc" else "f32/f64",
                      "data": "synthetic (seeded Zipf CP tensor)", "config": {"workload": a["workload"]},
                      "als": a}))
    ctx.close()


def run_fo_only(args):
    """--workload zipf4-250m: the first-order leg alone, as its own JSON line."""
    import torch

    import cutc_b200 as ctc
    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    ctx = ctc.Context(local)
    f = fo_leg(ctc, ctx, args, f"cuda:{local}")
    print(json.dumps({"metric": "first-order training nnz/s (minibatch Adam epoch, BF16 gathers)",
                      "value": f["mixed_bf16"]["nnz_per_s"], "unit": UNIT, "n_gpus": 1, "steps": 2, "warmup": 0,
                      "ms_per_step": 1000.0 * f["mixed_bf16"]["epoch_s"], "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "bf16/f32",
                      "data": "synthetic (seeded order-4 Zipf CP tensor)", "config": {"workload": f["workload"]},
                      "first_order": f}))
    ctx.close()


def run_batch_only(args):
    """--workload batch-256: the batched leg alone, as its own JSON line."""
    import torch

    import cutc_b200 as ctc
    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    ctx = ctc.Context(local)
    b = batch_leg(ctc, ctx, args, f"cuda:{local}")
    ntr = b["nnz_train"]
    step_s = (b["als"]["epoch_ms"] + b["sgd"]["epoch_ms"]) / 1000.0
    print(json.dumps({"metric": "batched training nnz/s (one ALS + one SGD epoch of all instances per step)",
                      "value": 2 * ntr / step_s, "unit": UNIT, "n_gpus": 1, "steps": 10, "warmup": 0,
                      "ms_per_step": 1000.0 * step_s, "higher_is_better": True, "scaling": "weak",
                      "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uniform CP instances)",
                      "config": {"workload": b["workload"]}, "batched": b}))
    ctx.close()


def run_reference_cuda(args):
    """The reference's own CUDA kernels (sgpu/als.cu, ccd.cu, sgd.cu, built
    from its sources for sm_100a at the workload's rank by
    oracle/build_ref.sh and driven by oracle/ref_kernels_harness.cu with the
    reference drivers' launch sequences and grids), timed with CUDA events
    on this GPU on the workload's training tensor: its CISS copies come from
    the reference's own ciss_alloc (oracle/_ref/libref_host.so), its
    factors are U(0,1)/sqrt(R).  ALS: one iteration of three mode updates
    (lambda 0.1; MTTKRP + Gram kernel, batched cuSOLVER Cholesky); CCD:
    the reference's "CCD+" iteration of three modes (lambda 0.1; its grid
    reaches about 1/32 of the tiles, sgpu/ccd.cu:520); SGD: one Hogwild
    epoch with FP64 atomics (lr 1e-3, lambda 0.01).  All FP64, as the
    reference computes.  Data transfers are outside the timed region."""
    import ctypes as C

    import torch

    from oracle import pyoracle as po
    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    device = f"cuda:{local}"
    w, data = make_workload(args, device)
    R = w.rank
    suffix = "" if R == 16 else f"_r{R}"
    libs = {}
    for alg in ("als", "ccd", "sgd"):
        path = os.path.join(po.REF_DIR, f"libref_{alg}{suffix}.so")
        if not os.path.exists(path):
            print(json.dumps({"impl": "reference", "unavailable": f"{path} not built (oracle/build_ref.sh)"}))
            return
        L = C.CDLL(path)
        L.refh_rank.restype = C.c_int
        if L.refh_rank() != R:
            raise RuntimeError(f"{path} is built for rank {L.refh_rank()}, the workload needs {R}")
        libs[alg] = L
    ti, tv = data["train"]
    n = int(tv.size)
    del data
    srt = sort_modes_torch(ti, tv, w.dims, device)
    del ti, tv
    torch.cuda.empty_cache()
    dims = [int(d) for d in w.dims]
    t0 = time.time()
    ciss = []
    for m in range(3):
        T = po.Tensor(srt[m][0], srt[m][1], dims)
        ciss.append(po.ref_ciss_alloc(T, m + 1))
        del T
    del srt
    ciss_s = time.time() - t0
    _u64p, _f64p = C.POINTER(C.c_uint64), C.POINTER(C.c_double)
    rng = np.random.default_rng(args.seed + 1)
    U0 = [rng.uniform(0, 1, (d, R)) / np.sqrt(R) for d in dims]
    dims3 = np.array(dims, dtype=np.uint64)

    def arr(xs, t):
        return (C.POINTER(t) * len(xs))(*[x.ctypes.data_as(C.POINTER(t)) for x in xs])

    ent = arr([c["entries"] for c in ciss], C.c_double)
    dirs = arr([c["directory"] for c in ciss], C.c_uint64)
    size_rows = (C.c_uint64 * 3)(*[c["size_rows"] for c in ciss])
    dlen = (C.c_uint64 * 3)(*[c["dlength"] for c in ciss])
    out = {}
    ms = C.c_double()
    for alg, lam, iters in (("als", 0.1, 1), ("ccd", 0.1, 2)):
        U = [u.copy() for u in U0]
        fn = getattr(libs[alg], f"refh_{alg}_bench")
        fn.argtypes = [C.POINTER(_f64p), _u64p, C.POINTER(_u64p), _u64p, C.c_uint64, _u64p, C.POINTER(_f64p),
                       C.c_double, C.c_int, C.POINTER(C.c_double)]
        rc = fn(ent, size_rows, dirs, dlen, n, dims3.ctypes.data_as(_u64p), arr(U, C.c_double), lam, iters,
                C.byref(ms))
        out[alg] = {"rc": rc, "ms_per_iteration": ms.value if rc == 0 else None,
                    "nnz_per_s": n / (ms.value / 1000.0) if rc == 0 and ms.value > 0 else None,
                    "iterations_timed": iters}
    U = [u.copy() for u in U0]
    fn = libs["sgd"].refh_sgd_bench
    fn.argtypes = [_f64p, C.c_uint64, _u64p, _u64p, C.c_uint64, C.c_uint64, _u64p, C.POINTER(_f64p), C.c_double,
                   C.c_double, C.c_int, C.POINTER(C.c_double)]
    c0 = ciss[0]
    rc = fn(c0["entries"].ctypes.data_as(_f64p), c0["size_rows"], c0["directory"].ctypes.data_as(_u64p),
            c0["dcounter"].ctypes.data_as(_u64p), c0["dlength"], n, dims3.ctypes.data_as(_u64p),
            arr(U, C.c_double), 1e-3, 0.01, 2, C.byref(ms))
    out["sgd"] = {"rc": rc, "ms_per_epoch": ms.value if rc == 0 else None,
                  "nnz_per_s": n / (ms.value / 1000.0) if rc == 0 and ms.value > 0 else None, "epochs_timed": 2,
                  "note": "refused by the harness when nnz % 32 == 0 (the reference kernel's endless loop)"}
    print(json.dumps({"impl": "reference", "kind": "reference CUDA kernels on this GPU", "dtype": "f64",
                      "config": {"workload": w.name, "dims": dims, "nnz_train": n, "rank": R},
                      "ciss_build_s": ciss_s, "reference_cuda": out,
                      "gpu": torch.cuda.get_device_name(local)}))


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference" and a.ref_cuda:
        run_reference_cuda(a)
    elif a.impl == "reference":
        run_reference(a)
    elif a.workload.startswith("batch"):
        run_batch_only(a)
    elif a.workload.startswith("zipf4"):
        run_fo_only(a)
    elif a.workload == "zipf-400m" or a.als:
        run_als_only(a)
    else:
        run_ours(a)
