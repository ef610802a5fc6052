"""Learned sketch ranks for the reaction-Burgers sketch step.

A step has three kinds of roundings (KIND_*): the product u.u, the field F
(one sketch of the formal sum a + b) and the two stage roundings (u_s and
u+); their ranks differ (at the benchmark ~5, ~15 and ~7), so the sketch
rank is proposed per kind and bond.  Features of (kind, bond k) at step t:
the top-16 singular values of bond k after the last rounding of that kind in
step t-1, as log10(sigma_j / delta) clipped to [-4, 16] and scaled by 1/4
(delta = the bond's truncation threshold, so the count of values above 0 is
the deterministic rank when it is <= 16), the bond position k/d,
log10(dt) + 3 and the kind (one-hot).  Target: the largest rank bond k keeps
in the roundings of that kind in step t (logged from plain, deterministic
runs).  The proposal is ell = max(ceil(prediction), r_prev + 1) + pad,
clamped to [pad + 1, maxrank + pad], where r_prev is the rank the roundings
of that kind kept at that bond in the previous step.

Training data comes from plain runs of the config-2 shape (d=40, n=128,
rank cap 32, tol 1e-8) at seeds 10-19; under-predictions are weighted 16x
in the loss (each costs a deterministic fallback); training and inference
run on the GPU through the MLP kernels (ptt_mlp_*).

    python -m paratt_b200.learned --out paratt_b200/models/sketch_rank_mlp.npz
    python -m paratt_b200.learned --evaluate c4 --steps 1000
"""
from __future__ import annotations

import argparse
import os
import time

import numpy as np

from . import KINDS, STAT_NSIG, MLP, Context, RxnBurgers, TT, axpby
from . import workloads as W

NIN = STAT_NSIG + 2 + KINDS
MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "models", "sketch_rank_mlp.npz")


def features(sig, delta, d, dt, kind):
    """sig: (d+1, 16) bond spectra (row k = bond k); returns (d-1, NIN)."""
    s = np.maximum(np.asarray(sig[1:d], dtype=np.float64), 1e-300)
    lg = np.clip(np.log10(s / max(delta, 1e-300)), -4.0, 16.0) / 4.0
    k = (np.arange(1, d) / d)[:, None]
    t = np.full((d - 1, 1), np.log10(dt) + 3.0)
    oh = np.zeros((d - 1, KINDS))
    oh[:, kind] = 1.0
    return np.hstack([lg, k, t, oh]).astype(np.float32)


def propose(mlp, specs, d, dt, pad, maxrank, prev=None):
    """specs[kind] = (sig, delta); returns the KINDS x (d+1) sketch ranks.
    prev[kind] (optional, d+1 ints): the ranks the roundings of that kind
    kept in the previous step; a proposal never goes below prev + 1 (a rail
    against a rank that grows past what the training runs showed; each
    under-proposal costs a deterministic fallback)."""
    x = np.vstack([features(specs[t][0], specs[t][1], d, dt, t) for t in range(KINDS)])
    y = np.ceil(mlp.forward(x).reshape(KINDS, d - 1)).astype(int)
    if prev is not None:
        y = np.maximum(y, np.asarray(prev, dtype=int)[:, 1:d] + 1)
    ell = np.clip(y + pad, pad + 1, maxrank + pad)
    out = np.ones((KINDS, d + 1), dtype=int)
    out[:, 1:d] = ell
    return out


def kind_spectra(sim, d):
    """Per-kind (spectra, threshold, kept ranks) of the last step of `sim`
    (a logging RxnBurgers)."""
    out = []
    for t in range(KINDS):
        ranks, sig, delta = sim.last_step_kind(t, d)
        out.append((sig, delta, ranks))
    return out


class LearnedStepper:
    """Reaction-Burgers RK2 steps by the learned-sketch method: before every
    step the MLP proposes per-kind, per-bond sketch ranks from the previous
    step's spectra; the step rounds through Gaussian sketches of those ranks,
    with the deterministic truncation as the judge and fallback
    (ptt_rxn_burgers_rk2_step_sketch_kinds).  Without spectra (first step)
    the step is the plain deterministic one, which records them."""

    def __init__(self, ctx, d, n, maxrank, dt, tol, pad=4, model=MODEL, seed=3):
        self.d, self.dt, self.pad, self.maxrank = d, dt, pad, maxrank
        self.sim = RxnBurgers(ctx, d, n, maxrank=maxrank, dt=dt, tol=tol, seed=seed)
        self.sim.log(True)
        z = np.load(model)
        if int(z["nin"]) != NIN:
            raise ValueError(f"{model}: model has {int(z['nin'])} inputs, the features have {NIN}")
        self.mlp = MLP(ctx, int(z["nin"]), int(z["width"]))
        self.mlp.set_params(z["params"])
        self.spec = None
        self.ell = None

    def seed_from(self, src):
        """Take the per-kind spectra of the last step of another (logging)
        RxnBurgers, e.g. a plain warm-up step, or a kind_spectra() list."""
        specs = src if isinstance(src, list) else kind_spectra(src, self.d)
        self.spec = [(np.array(g, copy=True), float(dl), list(r)) for g, dl, r in specs]

    def step(self, U):
        if self.spec is None:
            self.sim.step(U)
        else:
            self.ell = propose(self.mlp, self.spec, self.d, self.dt, self.pad, self.maxrank,
                               prev=[sp[2] for sp in self.spec])
            self.sim.step_sketch_kinds(U, self.ell, pad=self.pad)
        self.spec = kind_spectra(self.sim, self.d)

    def counts(self):
        """(sketch roundings, deterministic fallbacks) so far."""
        return self.sim.sketch_counts()

    def close(self):
        self.mlp.close()
        self.sim.close()


def collect(ctx, cfg, seed, steps, warm=1):
    """Plain run with logging; returns features (previous step's spectra per
    kind) and targets (this step's largest kept rank per kind) for every
    kind, bond and step."""
    d, n = cfg["d"], cfg["n"]
    u0 = W.initial_condition(d, n, cfg["ngauss"], seed)
    tol = cfg["tol"] * W.rms_norm(u0)
    sim = RxnBurgers(ctx, d, n, maxrank=cfg["maxrank"], dt=cfg["dt"], tol=tol, seed=seed)
    sim.log(True)
    U = TT(ctx, [n] * d, [1] + [2 * cfg["maxrank"]] * (d - 1) + [1], u0)
    X, T = [], []
    prev = None
    for s in range(steps):
        sim.step(U)
        cur = []
        for t in range(KINDS):
            ranks, sig, delta = sim.last_step_kind(t, d)
            cur.append((sig.copy(), delta, ranks))
        if prev is not None and s >= warm:
            for t in range(KINDS):
                X.append(features(prev[t][0], prev[t][1], d, cfg["dt"], t))
                T.append(np.asarray(cur[t][2][1:d], dtype=np.float32))
        prev = cur
    sim.close()
    U.close()
    return np.vstack(X), np.concatenate(T)


def train(mlp, X, T, epochs=300, lr=3e-3, batch=512, seed=0):
    rng = np.random.default_rng(seed)
    losses = []
    for ep in range(epochs):
        idx = rng.permutation(len(T))
        for b in range(0, len(T), batch):
            j = idx[b:b + batch]
            losses.append(mlp.train_step(X[j], T[j], lr))
    return losses


def rel_diff(ctx, X, Y):
    """||X - Y|| / ||Y|| with the difference formed as a train and
    orthogonalised (zero-tolerance rounding) before its norm, so nothing
    cancels."""
    D = TT(ctx, X.dims, [1] * (X.d + 1))
    axpby(1.0, X, -1.0, Y, D)
    D.round(0.0)
    v = D.norm() / Y.norm()
    D.close()
    return float(v)


def evaluate(ctx, cfg, steps, every=50, pad=4, model=MODEL):
    """Learned and plain trajectories from the same initial condition, side
    by side: time per step of each, sketch roundings and fallbacks, largest
    proposed sketch rank, state rank, and the relative difference of the two
    states every `every` steps.  Returns a summary dict."""
    d, n, maxr, dt = cfg["d"], cfg["n"], cfg["maxrank"], cfg["dt"]
    u0 = W.initial_condition(d, n, cfg["ngauss"], cfg["seed"])
    tol = cfg["tol"] * W.rms_norm(u0)
    cap = [1] + [2 * maxr] * (d - 1) + [1]
    plain = RxnBurgers(ctx, d, n, maxrank=maxr, dt=dt, tol=tol, seed=7)
    ls = LearnedStepper(ctx, d, n, maxr, dt, tol, pad=pad, model=model, seed=3)
    UP = TT(ctx, [n] * d, cap, u0)
    UL = TT(ctx, [n] * d, cap, u0)
    tp = tl = 0.0
    ell_max, rank_max, diffs = 0, 0, []
    for s in range(steps):
        ctx.sync()
        t0 = time.perf_counter()
        plain.step(UP)
        ctx.sync()
        t1 = time.perf_counter()
        ls.step(UL)
        ctx.sync()
        t2 = time.perf_counter()
        tp += t1 - t0
        tl += t2 - t1
        if ls.ell is not None:
            ell_max = max(ell_max, int(np.max(ls.ell)))
        rank_max = max(rank_max, max(UL.ranks()))
        if (s + 1) % every == 0 or s == steps - 1:
            diffs.append((s + 1, rel_diff(ctx, UL, UP)))
    calls, fb = ls.counts()
    out = {"steps": steps, "plain_ms_per_step": 1e3 * tp / steps, "learned_ms_per_step": 1e3 * tl / steps,
           "learned_over_plain": tp / tl, "sketch_roundings": calls, "fallbacks": fb,
           "fallback_rate": fb / max(calls, 1), "max_sketch_rank": ell_max, "max_state_rank": rank_max,
           "rel_diff_vs_plain": diffs}
    for t in (UP, UL):
        t.close()
    ls.close()
    plain.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=MODEL)
    ap.add_argument("--seeds", type=int, nargs="*", default=list(range(10, 20)))
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--under-weight", type=float, default=16.0,
                    help="loss weight of under-predicted ranks (an under-prediction costs a fallback)")
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--evaluate", default=None, choices=["c2", "c4"],
                    help="instead of training: run the learned and plain methods side by side on a "
                         "configuration for --steps steps and print a JSON summary")
    args = ap.parse_args()
    ctx = Context(0)
    if args.evaluate:
        import json

        res = evaluate(ctx, W.CONFIGS[args.evaluate], args.steps)
        res["config"] = args.evaluate
        print(json.dumps(res), flush=True)
        ctx.close()
        return
    cfg = dict(W.CONFIGS["c2"])
    t0 = time.time()
    Xs, Ts = [], []
    for sd in args.seeds:
        X, T = collect(ctx, cfg, sd, args.steps)
        Xs.append(X)
        Ts.append(T)
        print(f"seed {sd}: {len(T)} samples, target ranks {T.min():.0f}..{T.max():.0f}", flush=True)
    X, T = np.vstack(Xs), np.concatenate(Ts)
    mlp = MLP(ctx, NIN, 64, seed=1)
    mlp.set_under_weight(args.under_weight)
    losses = train(mlp, X, T, epochs=args.epochs)
    pred = mlp.forward(X)
    under = float(np.mean(np.ceil(pred) < T))
    print(f"{len(T)} samples, final loss {losses[-1]:.4f}, under-predicted {100 * under:.1f}%, "
          f"{time.time() - t0:.0f} s", flush=True)
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    np.savez(args.out, params=mlp.params(), nin=NIN, width=64, X=X, T=T)
    mlp.close()
    ctx.close()


if __name__ == "__main__":
    main()
