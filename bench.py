#!/usr/bin/env python3
"""Benchmark: reaction-Burgers step-truncation RK2 steps/s at d=40, n=256,
rank-max 64, tol 1e-8 (config 4 of the benchmark plan), one trajectory per
GPU (replicas; the step has no data-parallel exchange).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  `value` is steps/s over all GPUs with the state
resident in HBM (CUDA events on the library's stream, L2 flushed before every
step, flush outside the events); `e2e` is the same metric through the
reference-facing C API (pattac_rxn_burgers_midpoint_st on host cores, pinned),
host<->device copies inside the timed region; `roofline` is the dominant
kernel class (TSQR factorisation tree) timed launch by launch with events
during the timed steps; `cpu_baseline` is the reference's own C
(oracle/_ref/libparatt_ref.so) on this host, extrapolated from a bounded
per-bond sample of the same roundings.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK steps/s d=40,n=256: learned-sketch vs plain rounding, 1 B200, err≤1e-8"
CFG = dict(d=40, n=256, maxrank=64, tol=1e-8, dt=1e-3, ngauss=3, seed=3)
REF_RANK = 20  # representative state rank for the reference's extrapolation


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [t.strip() for t in l.split(",")]
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU reference: per-bond cost of paratt_truncate at the step's rank profile
# ---------------------------------------------------------------------------
def reference_step_seconds(r, n, d, reps=1):
    """Seconds for one RK2 step on the reference CPU path, extrapolated.

    The step rounds 2 formal products (interior rank r^2, attacHadamard) and
    8 sums / operator TTs (rank 2r) -- 10 paratt_truncate calls, each a
    left-to-right QR sweep and a right-to-left LQ+SVD sweep over d-1 bonds.
    Sample: paratt_truncate of 3-core trains (2 bonds) with those interior
    ranks and n=256, timed on this host, scaled by (d-1)/2 bonds."""
    from oracle import ref_lib as R  # CPU-baseline leg only

    rng = np.random.default_rng(11)

    def per_bond(rank):
        ts = []
        for _ in range(reps):
            cores = [rng.standard_normal((1, n, rank)), rng.standard_normal((rank, n, rank)),
                     rng.standard_normal((rank, n, 1))]
            t0 = time.perf_counter()
            R.ref_truncate(cores, 1e-300, [1, rank, rank, 1])
            ts.append(time.perf_counter() - t0)
        return min(ts) / 2.0

    t_prod = per_bond(r * r)
    t_sum = per_bond(2 * r)
    return (d - 1) * (2 * t_prod + 8 * t_sum), t_prod, t_sum


def cpu_threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


def run_reference(args, rank):
    if rank != 0:
        return 0
    nthr = cpu_threads()
    os.environ.setdefault("OPENBLAS_NUM_THREADS", str(nthr))
    try:
        from oracle import ref_lib as R  # noqa: F401
        if not R.available():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libparatt_ref.so not built"}))
            return 0
    except Exception as e:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": f"reference library failed to load: {e}"}))
        return 0
    d, n, r = CFG["d"], CFG["n"], REF_RANK
    for _ in range(args.warmup):
        reference_step_seconds(r, 64, 3)
    ts = []
    for _ in range(args.steps):
        t, tp, tsum = reference_step_seconds(r, n, d)
        ts.append(t)
    sec = statistics.median(ts)
    v = 1.0 / sec
    sample = (f"paratt_truncate of 3-core trains, n={n}, interior rank {r*r} (formal u.u) and {2*r} (sums), "
              f"per-bond time x (d-1) x (2 + 8 roundings per RK2 step); state rank {r}")
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "RK2 steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "config4 reaction-Burgers RK2 (extrapolated per-bond reference cost)",
                   "d": d, "n": n, "maxrank": CFG["maxrank"], "tol": CFG["tol"], "state_rank": r},
        "cpu_baseline": {"value": v, "unit": "RK2 steps/s", "cores": int(os.environ["OPENBLAS_NUM_THREADS"]),
                         "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "RK2 steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, rank, world, local_rank):
    import paratt_b200 as P
    from paratt_b200 import workloads as Wl
    from paratt_b200.capi import HostTT, capi

    dist = None
    if world > 1:
        import torch
        import torch.distributed as td
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        td.init_process_group("nccl", timeout=timedelta(seconds=600))
        dist = (torch, td)

    d, n, maxr = CFG["d"], CFG["n"], CFG["maxrank"]
    ctx = P.Context(local_rank)
    u0 = Wl.initial_condition(d, n, CFG["ngauss"], CFG["seed"] + rank)
    tol = CFG["tol"] * Wl.rms_norm(u0)
    sim = P.RxnBurgers(ctx, d, n, maxrank=maxr, dt=CFG["dt"], tol=tol, seed=7 + rank)
    cap = [1] + [2 * maxr] * (d - 1) + [1]
    U = P.TT(ctx, [n] * d, cap, u0)
    for _ in range(args.warmup):
        sim.step(U)
    ctx.sync()
    start_cores = U.get()

    def barrier():
        if dist:
            dist[1].barrier()

    # ---- device-resident timed region --------------------------------------
    ctx.time_kernels(P.TIME_TSQR)
    l0 = ctx.launches
    barrier()
    step_ms = []
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
            ctx.flush_l2()
            ctx.mark(0)
            sim.step(U)
            ctx.mark(1)
            step_ms.append(ctx.elapsed_ms(0, 1))
    ctx.sync()
    barrier()
    launches = ctx.launches - l0 - args.steps  # minus the flush kernels
    ktime_ms, klaunch = ctx.kernel_time()
    kwork = ctx.kernel_work()
    ctx.time_kernels(0)
    ranks_after = U.ranks()
    total_ms = float(sum(step_ms))
    if dist:
        t = dist[0].tensor([total_ms], device="cuda")
        dist[1].all_reduce(t, op=dist[1].ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * args.steps / (total_ms / 1e3)

    # ---- end to end through the reference-facing C API ---------------------
    L = capi()
    host = HostTT(start_cores, capacity=cap)
    host.pin()
    h2d = d2h = 0
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        h2d += host.core_bytes()
        L.pattac_rxn_burgers_midpoint_st(host.p, CFG["dt"], tol, maxr)
        d2h += host.core_bytes()
    e2e_s = time.perf_counter() - t0
    if L.paratt_last_error() != 0:
        raise RuntimeError("C API step failed")
    if dist:
        t = dist[0].tensor([e2e_s], device="cuda")
        dist[1].all_reduce(t, op=dist[1].ReduceOp.MAX)
        e2e_s = float(t.item())
    host.free()
    e2e = world * args.steps / e2e_s

    if rank != 0:
        if dist:
            dist[1].destroy_process_group()
        return 0

    hbm, src = peaks()
    achieved = (kwork / 1e9) / (ktime_ms / 1e3) if ktime_ms > 0 else 0.0  # GB/s
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "traffic": None, "kernel": "k_tsqr_factor",
            "launches": klaunch, "avg_launch_us": 1e3 * ktime_ms / max(klaunch, 1),
            "peak_source": f"{src} MEASURED_PEAKS.json hbm_gbs" if src == "measured" else "fallback 6650 GB/s"}
    out = {
        "metric": METRIC, "value": value, "unit": "RK2 steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "config4: reaction-Burgers step-truncation RK2, d=40, n=256, rank-max 64, "
                               "tol 1e-8 x ||u0||_RMS, dt 1e-3, 3-Gaussian IC (seed 3), plain FP64 rounding",
                   "method": "plain", "l2": "flushed before every step (2 x L2 write, outside the events)",
                   "ranks_after": max(ranks_after), "parallelism": f"replicas x{world}"},
        "roofline": roof,
        "e2e": {"value": e2e, "unit": "RK2 steps/s", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        nthr = cpu_threads()
        os.environ.setdefault("OPENBLAS_NUM_THREADS", str(nthr))
        r = max(ranks_after)
        try:
            sec, tp, tsum = reference_step_seconds(r, n, d)
            out["cpu_baseline"] = {"value": 1.0 / sec, "unit": "RK2 steps/s",
                                   "cores": int(os.environ["OPENBLAS_NUM_THREADS"]), "kind": "reference",
                                   "sample": f"paratt_truncate of 3-core trains n={n} at interior rank {r*r} "
                                             f"({tp:.3f} s/bond) and {2*r} ({tsum:.4f} s/bond), x (d-1) x 10 "
                                             f"roundings per step (extrapolated)"}
        except Exception as e:
            out["cpu_baseline"] = {"value": None, "unit": "RK2 steps/s", "cores": 0, "kind": "reference",
                                   "sample": f"unavailable: {e}"}
    print(json.dumps(out))
    sim.close()
    U.close()
    ctx.close()
    if dist:
        dist[1].destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference(args, rank)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
