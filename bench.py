#!/usr/bin/env python3
"""Benchmark: reaction-Burgers step-truncation RK2 steps/s at d=40, n=256,
rank-max 64, tol 1e-8 x ||u0||_RMS, dt 1e-3, 3-Gaussian initial condition
(config 4 of the benchmark plan), one trajectory per GPU (replicas; the step
has no data-parallel exchange).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  After W plain warm-up steps from the initial
condition, the same state is advanced K steps by

  * the learned-sketch method (`value`): before each step the MLP proposes
    per-bond sketch ranks from the previous step's spectra, every rounding
    goes through a Gaussian sketch of those ranks with the deterministic
    truncation as judge and fallback (paratt_b200.learned.LearnedStepper);
  * the plain method (`plain`): every rounding is the deterministic FP64
    TSQR + Jacobi-SVD truncation (ptt_rxn_burgers_rk2_step).

Both run with the state resident in HBM, timed by CUDA events on the
library's stream around each step, L2 flushed before every step (outside
the events).  `err_vs_plain` is the relative L2 difference between one
learned and one plain step from the same state; `fallback_rate` the share of
sketch roundings the judge sent back to the deterministic path.  `e2e` is the
learned method with the state on the host (page-locked): upload, step,
download every step, timed by the host clock.  `roofline` is the
factorisation class (per bond: the cluster Cholesky QR, with the Householder
TSQR for a bond it does not finish) timed launch by launch with events during
a second pass of the learned steps.  `cpu_baseline` / `--impl reference` time the reference's
own C (oracle/_ref/libparatt_ref.so: paratt_truncate, pattacHadamard,
attac_tt_axpby) composing the same RK2 step on this host's cores.
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
# CPU reference: the same RK2 step composed from the reference's own C
# ---------------------------------------------------------------------------
WORKLOAD = ("config4: reaction-Burgers step-truncation RK2, d=40, n=256, rank-max 64, tol 1e-8 x ||u0||_RMS, "
            "dt 1e-3, 3-Gaussian IC (seed 3), state after the warm-up steps")


def cpu_threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


def reference_steps(u, tol, steps):
    """Advance `u` by `steps` reference RK2 steps; returns (state, seconds)."""
    from oracle import ref_lib as R  # CPU-baseline leg only

    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        u = R.ref_rxn_burgers_rk2_step(u, CFG["dt"], tol, CFG["maxrank"])
        ts.append(time.perf_counter() - t0)
    return u, ts


def run_reference(args, rank):
    if rank != 0:
        return 0
    nthr = cpu_threads()
    os.environ.setdefault("OPENBLAS_NUM_THREADS", str(nthr))
    try:
        from oracle import ref_lib as R
        if not R.available():
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libparatt_ref.so not built"}))
            return 0
    except Exception as e:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": f"reference library failed to load: {e}"}))
        return 0
    from paratt_b200 import workloads as Wl

    d, n = CFG["d"], CFG["n"]
    u = Wl.initial_condition(d, n, CFG["ngauss"], CFG["seed"])
    tol = CFG["tol"] * Wl.rms_norm(u)
    u, _ = reference_steps(u, tol, args.warmup)
    u, ts = reference_steps(u, tol, args.steps)
    sec = sum(ts) / len(ts)
    v = 1.0 / sec
    ranks = [c.shape[2] for c in u[:-1]]
    sample = (f"{args.steps} full RK2 steps after {args.warmup} warm-up steps (state rank {max(ranks)}), "
              f"{nthr} OpenBLAS threads")
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "RK2 steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "d": d, "n": n, "maxrank": CFG["maxrank"], "tol": CFG["tol"],
                   "method": "plain (reference paratt_truncate)", "state_rank": max(ranks)},
        "cpu_baseline": {"value": v, "unit": "RK2 steps/s", "cores": int(os.environ["OPENBLAS_NUM_THREADS"]),
                         "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "RK2 steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


def autotune(ctx):
    """The context's Cholesky-QR cluster-size table (3 x 6, 0 = size rule
    kept), or the reason the tuning failed; the built-in rule stays in force
    then, so a failed tuning never stops the benchmark."""
    try:
        table = ctx.autotune().tolist()
        tm64, fill = ctx.autotune_gemm()
        return {"cq_cluster_sizes": table, "gemm_tile64_from": tm64, "gemm_splitk_tiles": fill}
    except Exception as e:  # noqa: BLE001 -- reported in the JSON line
        return f"not tuned: {e}"


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, rank, world, local_rank):
    import paratt_b200 as P
    from paratt_b200 import learned as Lr
    from paratt_b200 import workloads as Wl

    # independent replicas: NCCL only for the barrier and the max of the times
    from paratt_b200.replicas import Replicas
    rep = Replicas("nccl")
    barrier = rep.barrier
    max_over_ranks = rep.max

    d, n, maxr, dt = CFG["d"], CFG["n"], CFG["maxrank"], CFG["dt"]
    ctx = P.Context(local_rank)
    tuned = autotune(ctx) if not args.no_autotune else "not tuned (--no-autotune)"
    u0 = Wl.initial_condition(d, n, CFG["ngauss"], CFG["seed"] + rank)
    tol = CFG["tol"] * Wl.rms_norm(u0)
    cap = [1] + [2 * maxr] * (d - 1) + [1]
    plain = P.RxnBurgers(ctx, d, n, maxrank=maxr, dt=dt, tol=tol, seed=7 + rank)
    plain.log(True)
    S0 = P.TT(ctx, [n] * d, cap, u0)
    for _ in range(args.warmup):
        plain.step(S0)
    spec0 = Lr.kind_spectra(plain, d)
    plain.log(False)  # the timed plain steps read nothing back
    ctx.sync()

    def copy_of(src):
        t = P.TT(ctx, [n] * d, cap)
        t.copy_from(src)
        return t

    def timed(stepper_step, U):
        barrier()
        ms = []
        for _ in range(args.steps):
            ctx.flush_l2()
            ctx.mark(0)
            stepper_step(U)
            ctx.mark(1)
            ms.append(ctx.elapsed_ms(0, 1))
        ctx.sync()
        barrier()
        return max_over_ranks(float(sum(ms)))

    # ---- learned-sketch method (the headline) --------------------------------
    ls = Lr.LearnedStepper(ctx, d, n, maxr, dt, tol, seed=3 + rank)
    ls.seed_from(spec0)
    UL = copy_of(S0)
    l0 = ctx.launches
    with ClockSampler(local_rank) as clk:
        learned_ms = timed(ls.step, UL)
    launches = ctx.launches - l0 - args.steps  # minus the flush kernels
    calls, fallbacks = ls.counts()
    value = world * args.steps / (learned_ms / 1e3)

    # ---- the same learned steps again with every factorisation launch timed
    # by its own event pair (kept out of the headline region)
    lk = Lr.LearnedStepper(ctx, d, n, maxr, dt, tol, seed=3 + rank)
    lk.seed_from(spec0)
    UK = copy_of(S0)
    ctx.time_kernels(P.TIME_TSQR)
    timed(lk.step, UK)
    ktime_ms, klaunch = ctx.kernel_time()
    kwork = ctx.kernel_work()
    ctx.time_kernels(0)
    lk.close()
    UK.close()

    # ---- plain method from the same state ------------------------------------
    UP = copy_of(S0)
    plain_ms = timed(plain.step, UP)
    plain_value = world * args.steps / (plain_ms / 1e3)

    # ---- error of one learned step against one plain step --------------------
    A, B = copy_of(S0), copy_of(S0)
    plain.step(A)
    chk = Lr.LearnedStepper(ctx, d, n, maxr, dt, tol, seed=3 + rank)
    chk.seed_from(spec0)
    chk.step(B)
    def rel_diff(X, Y):
        # ||X - Y|| / ||Y||: the difference formed as a train and orthogonalised
        # (zero-tolerance rounding) before its norm, so nothing cancels
        D = P.TT(ctx, [n] * d, [1] * (d + 1))  # grown to the exact sum ranks
        P.axpby(1.0, X, -1.0, Y, D)
        D.round(0.0)
        v = D.norm() / Y.norm()
        D.close()
        return float(v)

    err_step = rel_diff(B, A)
    err_traj = rel_diff(UL, UP)
    chk.close()
    A.close()
    B.close()

    # ---- end to end: learned method with the state on the host --------------
    host = P.HostTrain([n] * d, cap, S0.get())
    ue = P.TT(ctx, [n] * d, cap)
    le = Lr.LearnedStepper(ctx, d, n, maxr, dt, tol, seed=3 + rank)
    le.seed_from(spec0)
    h2d = d2h = 0
    ctx.sync()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        h2d += host.nbytes()
        host.upload(ue)
        le.step(ue)
        host.download(ue)
        d2h += host.nbytes()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = world * args.steps / e2e_s
    start_cores = S0.get()
    le.close()
    ue.close()
    host.close()

    if rank != 0:
        rep.close()
        return 0

    hbm, src = peaks()
    achieved = (kwork / 1e9) / (ktime_ms / 1e3) if ktime_ms > 0 else 0.0  # GB/s
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm,
            # DRAM read + write of one k_cq_factor<16> launch of this step
            # (an ~3072 x <= 16 unfolding), from an ncu --set full capture
            "traffic": 372480.0,
            "traffic_source": "ncu: one k_cq_factor<16> launch of the learned step (m ~3072, c <= 16)",
            "kernel": "factorisation: k_cq_factor (cluster Cholesky QR), k_wfactor/k_tsqr_factor fallback",
            "launches": klaunch, "avg_launch_us": 1e3 * ktime_ms / max(klaunch, 1),
            "algorithmic_bytes_per_launch": kwork / max(klaunch, 1),
            "timing": "event pair per launch in a second pass of the same K learned steps",
            "peak_source": f"{src} MEASURED_PEAKS.json hbm_gbs" if src == "measured" else "fallback 6650 GB/s"}
    out = {
        "metric": METRIC, "value": value, "unit": "RK2 steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": learned_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "method": "learned-sketch (MLP-proposed sketch ranks, pad 4)",
                   "autotune": tuned,
                   "l2": "flushed before every step (2 x L2 write, outside the events)",
                   "state_rank": max(UL.ranks()), "parallelism": f"replicas x{world}"},
        "plain": {"value": plain_value, "unit": "RK2 steps/s", "ms_per_step": plain_ms / args.steps},
        "learned_over_plain": value / plain_value,
        "err_vs_plain": {"one_step": err_step, "after_steps": err_traj, "steps": args.steps},
        "fallback_rate": fallbacks / max(calls, 1),
        "sketch_roundings": calls,
        "roofline": roof,
        "e2e": {"value": e2e, "unit": "RK2 steps/s", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    # the rank-64 -> 32 rounding of config 1 (d=40, n=256), recorded beside
    # the step: the path that the step's low ranks never reach
    c1 = config1_rounding(P, ctx, 3, 1)
    out["round_c1"] = {k: c1[k] for k in ("ms", "ranks_out", "achieved_gbs", "frac", "fp64_tflops", "breakdown")}
    c1o = config1_rounding(P, ctx, 3, 1, ozaki=True)
    out["round_c1_ozaki"] = {k: c1o[k] for k in ("ms", "ranks_out", "rel_diff_vs_fp64", "breakdown")}
    out["round_c1_ozaki"]["gram"] = "7 BF16 digit slices per element, tcgen05.mma FP32 accumulation, FP64 recombination"
    if world == 1 and not args.no_cpu_baseline:
        nthr = cpu_threads()
        os.environ.setdefault("OPENBLAS_NUM_THREADS", str(nthr))
        try:
            ref_state, ts = reference_steps(start_cores, tol, 2)
            sec = sum(ts) / len(ts)
            out["cpu_baseline"] = {"value": 1.0 / sec, "unit": "RK2 steps/s",
                                   "cores": int(os.environ["OPENBLAS_NUM_THREADS"]), "kind": "reference",
                                   "sample": f"2 full RK2 steps of the reference routines from the warmed-up "
                                             f"state (rank {max(r.shape[2] for r in start_cores[:-1])})"}
            # parity: the same 2 plain steps on the GPU from the same state
            G = copy_of(S0)
            plain.step(G)
            plain.step(G)
            Rt = P.TT(ctx, [n] * d, cap, ref_state)
            ref_ranks = [1] + [c.shape[2] for c in ref_state]
            out["parity"] = {"ranks_equal": G.ranks() == ref_ranks, "rel_l2": rel_diff(G, Rt),
                             "steps": 2, "against": "reference C (paratt_truncate composition), plain GPU step"}
            G.close()
            Rt.close()
        except Exception as e:
            out["cpu_baseline"] = {"value": None, "unit": "RK2 steps/s", "cores": 0, "kind": "reference",
                                   "sample": f"unavailable: {e}"}
    print(json.dumps(out))
    for t in (UL, UP, S0):
        t.close()
    ls.close()
    plain.close()
    ctx.close()
    rep.close()
    return 0


# ---------------------------------------------------------------------------
# batched rounding (--workload batch): 64 independent trains
# ---------------------------------------------------------------------------
def run_batch(args, rank, world, local_rank):
    """64 trains of uneven d/n/r (workloads.batch_shapes), each rounded to
    tol 1e-8 x its RMS norm with rank cap floor(r_k/2): ptt_round_batch
    (concurrent worker streams) against the one-train-at-a-time loop, both
    from fresh copies of the same inputs every repetition; device time by
    events on the context stream (rank read-backs included).  With N ranks
    the 64 trains are split by instance, balanced by rounding cost
    (workloads.shard_by_cost), each rank rounds its share on its GPU with no
    collective on the data path; the time of a repetition is the slowest
    rank's, and rank 0 gathers every train's ranks."""
    import paratt_b200 as P
    from paratt_b200 import workloads as Wl
    from paratt_b200.replicas import Replicas

    rep = Replicas("nccl")
    ctx = P.Context(local_rank)
    tuned = autotune(ctx) if not args.no_autotune else "not tuned (--no-autotune)"
    shapes = Wl.batch_shapes(64, 4)
    costs = [Wl.rounding_cost(sh) for sh in shapes]
    shards = Wl.shard_by_cost(costs, world)
    mine = shards[rank]
    orig = Wl.batch_trains(ctx, 64, 4, only=set(mine))
    tts = [t for t, _ in orig]
    caps = [sh[3] for _, sh in orig]
    tols = [1e-8 * t.norm() for t in tts]
    work = []
    for t, (d, n, r, cap) in orig:
        w = P.TT(ctx, [n] * d, r)
        work.append(w)
    elems = sum(sum(r[k] * n * r[k + 1] for k in range(d)) for _, (d, n, r, _) in orig)

    def fresh():
        for w, t in zip(work, tts):
            w.copy_from(t)
        ctx.sync()

    def timed(fn):
        fresh()
        rep.barrier()
        ctx.mark(0)
        fn()
        ctx.mark(1)
        ctx.sync()
        return rep.max(ctx.elapsed_ms(0, 1))

    def loop():
        for w, tol, cap in zip(work, tols, caps):
            w.round(tol, cap)

    lanes = 8
    t_loop, t_batch = [], []
    ranks_loop = ranks_batch = []
    for i in range(args.warmup + args.steps):
        a = timed(loop)
        ranks_loop = [w.ranks() for w in work]
        b = timed(lambda: P.round_batch(work, tols, caps, lanes=lanes) if work else None)
        ranks_batch = [w.ranks() for w in work]
        if i >= args.warmup:
            t_loop.append(a)
            t_batch.append(b)
    results = rep.gather([(idx, rl, rb) for idx, rl, rb in zip(mine, ranks_loop, ranks_batch)])
    elems_all = rep.gather(elems)
    for t in tts + work:
        t.close()
    ctx.close()
    if rank != 0:
        rep.close()
        return 0
    per_train = sorted(x for part in results for x in part)
    same = all(rl == rb for _, rl, rb in per_train) and [x[0] for x in per_train] == list(range(64))
    tb, tl = statistics.median(t_batch), statistics.median(t_loop)
    loads = [sum(costs[i] for i in sh) for sh in shards]
    out = {
        "metric": "batched TT rounding: 64 trains (d 10-40, n 32-512, r 8-96), roundings/s", "value": 64e3 / tb,
        "unit": "roundings/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": tb,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "batched rounding of 64 independent trains (seed 4), tol 1e-8 x ||X||_RMS, "
                               "rank cap floor(r/2); left-orthonormal cores, bond spectra 2^-j",
                   "lanes": lanes, "input_gb": sum(elems_all) * 8 / 1e9,
                   "parallelism": f"instances split over {world} ranks by rounding cost" if world > 1 else "one GPU",
                   "trains_per_rank": [len(sh) for sh in shards],
                   "cost_share_per_rank": [l / sum(loads) for l in loads]},
        "loop": {"value": 64e3 / tl, "unit": "roundings/s", "ms": tl},
        "batch_over_loop": tl / tb,
        "same_ranks_as_loop": bool(same),
        "autotune": tuned,
    }
    print(json.dumps(out))
    rep.close()
    return 0


# ---------------------------------------------------------------------------
# single rounding (--workload round): x + y of two rank-32 trains -> rank 32
# ---------------------------------------------------------------------------
def config1_rounding(P, ctx, steps, warmup, ozaki=False):
    """d=40, n=256: z = x + y of two seeded random trains of interior rank
    32 (entries N(0, 1/(n r)) -- std 1/sqrt(n r)), rounded to tol 1e-10 x
    ||z||_RMS with rank cap 32, plain FP64 (ozaki: the Gram matrices of the
    factorisations by the Ozaki split on the tensor cores, the result's
    relative difference to the FP64 path reported).  Device time by events on the
    context stream, L2 flushed before each rounding (outside the events);
    roofline against the algorithmic bytes 8 sum_k (3 R_k n R_{k+1} +
    r_k n r_{k+1}); the algorithmic FP64 flops (Householder QR and Q of every
    left unfolding, R X, LQ and Q of every right unfolding, 22 c^3 per SVD,
    V_r^T Q and X U_r S_r) are reported beside it."""
    d, n, r = 40, 256, 32
    sd = 1.0 / np.sqrt(n * r)

    def rnd(seed):
        rng = np.random.default_rng(seed)
        rr = [1] + [r] * (d - 1) + [1]
        return [rng.standard_normal((rr[k], n, rr[k + 1])) * sd for k in range(d)]

    X = P.TT.from_cores(ctx, rnd(1))
    Y = P.TT.from_cores(ctx, rnd(2))
    cap = [1] + [2 * r] * (d - 1) + [1]
    Z = P.TT(ctx, [n] * d, cap)
    P.axpby(1.0, X, 1.0, Y, Z)
    tol = 1e-10 * Z.norm()
    W = P.TT(ctx, [n] * d, cap)
    ctx.ozaki(ozaki)
    ts = []
    for i in range(warmup + steps):
        W.copy_from(Z)
        ctx.flush_l2()
        ctx.mark(0)
        W.round(tol, r)
        ctx.mark(1)
        ctx.sync()
        if i >= warmup:
            ts.append(ctx.elapsed_ms(0, 1))
    rk_in, rk_out = Z.ranks(), W.ranks()
    alg = 8.0 * sum(3 * rk_in[k] * n * rk_in[k + 1] + rk_out[k] * n * rk_out[k + 1] for k in range(d))
    flops = 0.0
    for k in range(d - 1):  # orthogonalisation: QR + Q of (R_k n) x R_{k+1}, then R X_{k+1}
        m, c = rk_in[k] * n, rk_in[k + 1]
        flops += 2 * (2.0 * m * c * c - 2.0 * c ** 3 / 3) + 2.0 * c * c * n * rk_in[k + 2]
    for k in range(d - 1, 0, -1):  # truncation: LQ + Q, SVD, V_r^T Q, X_{k-1} U_r S_r
        m, c, q = n * rk_out[k + 1], rk_in[k], rk_out[k]
        flops += 2 * (2.0 * m * c * c - 2.0 * c ** 3 / 3) + 22.0 * c ** 3 + 2.0 * q * c * m
        flops += 2.0 * rk_in[k - 1] * n * c * q
    t = statistics.median(ts)
    # per kernel class: one more rounding with every launch of that class
    # timed by its own event pair (outside the timed repetitions above)
    breakdown = {}
    for name, kind in (("factorisation", P.TIME_TSQR), ("svd", P.TIME_SVD)):
        W.copy_from(Z)
        ctx.sync()
        ctx.time_kernels(kind)
        W.round(tol, r)
        kms, kl = ctx.kernel_time()
        ctx.time_kernels(0)
        breakdown[name] = {"ms": kms, "launches": kl}
    sweeps = [int(v) for v in ctx.round_stats(d)[1:, 2]]
    diff = None
    if ozaki:  # ||W_ozaki - W_fp64|| / ||W_fp64||, the difference formed as a train
        ctx.ozaki(False)
        W2 = P.TT(ctx, [n] * d, cap)
        W2.copy_from(Z)
        W2.round(tol, r)
        D = P.TT(ctx, [n] * d, [1] + [4 * r] * (d - 1) + [1])
        P.axpby(1.0, W, -1.0, W2, D)
        D.round(0.0, 4 * r)  # orthogonal gauge first: the norm of the formal difference cancels
        diff = D.norm() / W2.norm()
        D.close()
        W2.close()
    ctx.ozaki(False)
    for t_ in (X, Y, Z, W):
        t_.close()
    hbm, src = peaks()
    return {"ms": t, "rel_diff_vs_fp64": diff, "ms_all": ts, "ranks_out": max(rk_out), "algorithmic_bytes": alg, "algorithmic_flops": flops,
            "achieved_gbs": alg / (t / 1e3) / 1e9, "frac": alg / (t / 1e3) / 1e9 / hbm, "peak": hbm,
            "peak_source": src, "fp64_tflops": flops / (t / 1e3) / 1e12, "breakdown": breakdown,
            "jacobi_sweeps": sweeps}


def run_round(args, rank, world, local_rank):
    """The rank-64 -> 32 rounding of config1_rounding as its own JSON line."""
    import paratt_b200 as P

    if rank != 0:
        return 0
    ctx = P.Context(local_rank)
    if not args.no_autotune:
        autotune(ctx)  # Cholesky-QR cluster sizes, timed once per context
    c1 = config1_rounding(P, ctx, args.steps, args.warmup, ozaki=args.ozaki)
    t = c1["ms"]
    gram = "Ozaki split (BF16 slices, tcgen05)" if args.ozaki else "FP64"
    out = {
        "metric": f"TT rounding d=40, n=256, ranks 64 -> 32 (Gram: {gram}), roundings/s", "value": 1e3 / t,
        "unit": "roundings/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "round(x + y), x, y seeded rank-32 trains, N(0, 1/(n r)) entries, tol 1e-10 x "
                               "||z||_RMS, rank cap 32", "ranks_out": c1["ranks_out"], "l2": "flushed before each"},
        "roofline": {"bound": "hbm", "achieved": c1["achieved_gbs"], "peak": c1["peak"], "unit": "GB/s",
                     "frac": c1["frac"], "traffic": None, "algorithmic_bytes": c1["algorithmic_bytes"],
                     "peak_source": c1["peak_source"]},
        "fp64": {"algorithmic_flops": c1["algorithmic_flops"], "tflops": c1["fp64_tflops"]},
        "breakdown": c1["breakdown"],
        "jacobi_sweeps": c1["jacobi_sweeps"],
        "rel_diff_vs_fp64": c1["rel_diff_vs_fp64"],
    }
    print(json.dumps(out))
    ctx.close()
    return 0


# ---------------------------------------------------------------------------
# formal kernels at full rank (--workload formal)
# ---------------------------------------------------------------------------
def run_formal(args, rank, world, local_rank):
    """The HBM-bound formal kernels at the benchmark's full rank (d=40, n=256,
    r=64 trains, outputs of rank 128): axpby, the all-modes stencil operator
    (op_sum), one single-mode stencil, a Hadamard product of rank-8 trains and
    a train copy.  Device time by events, L2 flushed before each launch
    (outside the events); achieved = algorithmic bytes (reads + writes, the
    zero blocks of formal cores included) / time, against the measured HBM
    copy bandwidth.  W untimed launches of each, then the median of K."""
    import paratt_b200 as P

    if rank != 0:
        return 0
    d, n, r = args.formal_d, 256, 64
    ctx = P.Context(local_rank)
    rng = np.random.default_rng(1)
    rr = [1] + [r] * (d - 1) + [1]
    X = P.TT.from_cores(ctx, [rng.standard_normal((rr[k], n, rr[k + 1])) for k in range(d)])
    Y = P.TT.from_cores(ctx, [rng.standard_normal((rr[k], n, rr[k + 1])) for k in range(d)])
    cap2 = [1] + [2 * r] * (d - 1) + [1]
    Z, W = P.TT(ctx, [n] * d, cap2), P.TT(ctx, [n] * d, cap2)
    r8 = [1] + [8] * (d - 1) + [1]
    X8 = P.TT.from_cores(ctx, [rng.standard_normal((r8[k], n, r8[k + 1])) for k in range(d)])
    H = P.TT(ctx, [n] * d, [1] + [64] * (d - 1) + [1])
    e_in = sum(rr[k] * n * rr[k + 1] for k in range(d))
    e_out = sum(cap2[k] * n * cap2[k + 1] for k in range(d))
    e8 = sum(r8[k] * n * r8[k + 1] for k in range(d))
    sten = [0.3, -0.6, 0.3]
    cases = [
        ("k_axpby", lambda: P.axpby(1.0, X, 2.0, Y, Z), 8.0 * (2 * e_in + e_out)),
        ("k_opsum", lambda: P.op_sum(X, sten, 1.0, W), 8.0 * (e_in + e_out)),
        ("k_stencil (mode d/2)", lambda: X.stencil(d // 2, sten), 16.0 * r * n * r),
        ("k_hadamard (rank 8 x 8)", lambda: P.hadamard(X8, X8, H), 8.0 * (2 * e8 + e_in)),
        ("k_copy_tt", lambda: Z.copy_from(X), 16.0 * e_in),
    ]
    hbm, src = peaks()
    out = {}
    for name, fn, nbytes in cases:
        for _ in range(args.warmup):
            fn()
        ts = []
        for _ in range(args.steps):
            ctx.flush_l2()
            ctx.mark(0)
            fn()
            ctx.mark(1)
            ctx.sync()
            ts.append(ctx.elapsed_ms(0, 1))
        t = statistics.median(ts)
        out[name] = {"ms": t, "bytes": nbytes, "GBs": nbytes / (t / 1e3) / 1e9, "frac": nbytes / (t / 1e3) / 1e9 / hbm}
    line = {
        "metric": "formal TT kernels at full rank (d=40, n=256, r=64): HBM GB/s", "value": out["k_axpby"]["GBs"],
        "unit": "GB/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "dtype": "f64", "data": "synthetic", "peak": hbm, "peak_source": src,
        "config": {"workload": f"axpby of two rank-64 trains (rank-128 output), all-modes stencil operator, one-mode "
                               f"stencil, rank-8 Hadamard, copy; d={d}, n=256", "l2": "flushed before each launch"},
        "kernels": out,
    }
    print(json.dumps(line))
    for t_ in (X, Y, Z, W, X8, H):
        t_.close()
    ctx.close()
    return 0


# ---------------------------------------------------------------------------
# one step for profilers (--one-step plain|learned)
# ---------------------------------------------------------------------------
def run_one_step(args, local_rank):
    """W plain warm-up steps, then exactly one step of the chosen method;
    prints the number of kernel launches before that step (the value for
    `ncu -s`)."""
    import paratt_b200 as P
    from paratt_b200 import learned as Lr
    from paratt_b200 import workloads as Wl

    d, n, maxr, dt = CFG["d"], CFG["n"], CFG["maxrank"], CFG["dt"]
    ctx = P.Context(local_rank)
    tuned = autotune(ctx) if not args.no_autotune else "not tuned (--no-autotune)"
    u0 = Wl.initial_condition(d, n, CFG["ngauss"], CFG["seed"])
    tol = CFG["tol"] * Wl.rms_norm(u0)
    plain = P.RxnBurgers(ctx, d, n, maxrank=maxr, dt=dt, tol=tol, seed=7)
    plain.log(True)
    U = P.TT(ctx, [n] * d, [1] + [2 * maxr] * (d - 1) + [1], u0)
    for _ in range(args.warmup):
        plain.step(U)
    step = plain.step
    if args.one_step == "learned":
        ls = Lr.LearnedStepper(ctx, d, n, maxr, dt, tol, seed=3)
        ls.seed_from(plain)
        ls.step(U)  # first learned step: the MLP and sketch workspaces warm up
        step = ls.step
    ctx.sync()
    l0 = ctx.launches
    print(f"launches before the measured step: {l0}", flush=True)
    ctx.mark(0)
    step(U)
    ctx.mark(1)
    ctx.sync()
    print(f"launches in the step: {ctx.launches - l0}, device time {ctx.elapsed_ms(0, 1):.2f} ms", flush=True)
    ctx.close()
    return 0


# ---------------------------------------------------------------------------
# the reference's own driver program (--workload driver)
# ---------------------------------------------------------------------------
def run_driver(args, rank, world, local_rank):
    """The reference's Burgers-Hopf CDF driver program
    (mpi_pattac_rxn_burgers_rank_max_read_file.c, compiled unmodified from the
    reference tree by oracle/Makefile) on libparatt_b200.so against the same
    program on the compiled reference (host cores), from the same seeded
    initial condition: d = 20 Gaussian modes of n = 256 points, rank cap
    32, max(steps, 10) time steps of dt 1e-5 (fixed in the driver).  Times are
    the driver's own (MPI_Wtime around its time loop, from its log): value =
    the driver's steps/s on the GPU library.  The ranks it prints and the TT
    folder it writes at t = 0 are compared between the two runs."""
    import re
    import subprocess
    import tempfile

    from oracle import tt_oracle as O  # checker of the two runs' outputs

    if rank != 0:
        return 0
    here = os.path.dirname(os.path.abspath(__file__))
    bins = {k: os.path.join(here, "oracle", "_ref", f"cdf_driver_{k}") for k in ("b200", "ref")}
    if not all(os.path.exists(b) for b in bins.values()):
        print(json.dumps({"workload": "driver", "unavailable": "oracle/_ref/cdf_driver_* not built (make -C oracle)"}))
        return 0
    d, n, rmax = 20, 256, 32
    steps = max(args.steps, 10)
    T, t, count = steps * 1e-5, 0.0, 0
    while t < T:  # the driver's own loop: time_now += dt until >= t_end
        t += 1e-5
        count += 1
    x = np.linspace(-1.3, 1.3, n)
    res = {}
    with tempfile.TemporaryDirectory() as tmp:
        for k, b in bins.items():
            wd = os.path.join(tmp, k)
            os.makedirs(os.path.join(wd, "ic"))
            for m in range(d):
                v = np.exp(-(x - 0.05 * m) ** 2 / (2 * 0.3 ** 2)) / (0.3 * np.sqrt(2 * np.pi))
                with open(os.path.join(wd, "ic", f"core_{m + 1}.cr"), "w") as f:
                    f.write(f"1,{n},1\n")
                    f.writelines("%+1.16e\n" % a for a in v)
            env = dict(os.environ, PARATT_DEVICE=str(local_rank))
            out = subprocess.run([b, "ic", str(d), str(rmax), "1e-5", "0.0", repr(T), "0"], cwd=wd, env=env,
                                 capture_output=True, text=True, timeout=1800)
            if out.returncode != 0:
                raise RuntimeError(f"driver ({k}) failed: {out.stderr[-500:]}")
            log = open(os.path.join(wd, "kse_cdf_timing_nprocs=1.log")).read().split()
            folder = os.path.join(wd, "data", f"bg_rxn_d{d}_rk{rmax}_tt", "cdf_t_0.000")
            cores = []
            for m in range(d):
                with open(os.path.join(folder, f"core_{m + 1}.cr")) as f:
                    rl, nn, rr = (int(v) for v in f.readline().split(","))
                    cores.append(np.array([float(v) for v in f.read().split()]).reshape((rl, nn, rr), order="F"))
            res[k] = {"seconds": float(log[-1]), "ranks": re.findall(r"tt rank:\n([\d\t ]+)\n", out.stdout),
                      "cores": cores}
    g, r = res["b200"], res["ref"]
    out = {
        "metric": "reference CDF driver program, unmodified, on the library: time steps/s", "value": count / g["seconds"],
        "unit": "steps/s", "n_gpus": 1, "steps": count, "warmup": 0, "ms_per_step": 1e3 * g["seconds"] / count,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "mpi_pattac_rxn_burgers_rank_max_read_file.c (Burgers-Hopf CDF), d=20 Gaussian modes, "
                               "n=256, rank cap 32, dt 1e-5", "timing": "the driver's MPI_Wtime around its time loop"},
        "reference": {"value": count / r["seconds"], "unit": "steps/s", "seconds": r["seconds"], "cores": cpu_threads(),
                      "kind": "reference", "sample": f"the same program linked to the compiled reference, {count} steps"},
        "speedup_vs_reference": r["seconds"] / g["seconds"],
        "parity": {"ranks_equal": g["ranks"] == r["ranks"], "rel_tt_t0": O.rel_diff_exact(g["cores"], r["cores"])},
    }
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ozaki", action="store_true",
                    help="--workload round: Gram matrices by the Ozaki split on the tensor cores")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the built-in cluster-size and tile rules (short runs under a profiler)")
    ap.add_argument("--formal-d", type=int, default=40, help="cores of the trains of --workload formal")
    ap.add_argument("--one-step", choices=["plain", "learned"], default=None,
                    help="profiling aid: W warm-up steps, then one step; prints the launch index to skip to")
    ap.add_argument("--workload", default="rk2", choices=["rk2", "batch", "round", "formal", "driver"],
                    help="rk2: the headline reaction-Burgers steps; batch: 64 independent roundings; "
                         "round: one rank-64 -> 32 rounding; formal: the HBM-bound formal kernels at full rank; "
                         "driver: the reference's own CDF driver program on the library and on the reference")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference(args, rank)
    if args.one_step:
        return run_one_step(args, local_rank)
    if args.workload == "batch":
        return run_batch(args, rank, world, local_rank)
    if args.workload == "round":
        return run_round(args, rank, world, local_rank)
    if args.workload == "formal":
        return run_formal(args, rank, world, local_rank)
    if args.workload == "driver":
        return run_driver(args, rank, world, local_rank)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
