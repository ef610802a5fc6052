"""Seeded synthetic inputs for the paratt_b200 benchmark and examples.

Gaussian-sum initial conditions on the periodic box [-L/2, L/2)^d with grid
x_j = -L/2 + j L/n, stored as rank-G tensor trains in the layout the
reference's attac_sum_of_product builds (paratt.c:517-568): core 0 =
[v_0 | v_1 | ...], diagonal interior cores, stacked last core.
"""
from __future__ import annotations

import numpy as np

# Reaction-Burgers configurations (d, n, rank cap, tol, dt, steps, Gaussians, seed)
CONFIGS = {
    "c0": dict(d=20, n=64, maxrank=20, tol=1e-8, dt=1e-3, steps=100, ngauss=1, seed=0),
    "c2": dict(d=40, n=128, maxrank=32, tol=1e-8, dt=1e-3, steps=500, ngauss=3, seed=3),
    "c4": dict(d=40, n=256, maxrank=64, tol=1e-8, dt=1e-3, steps=1000, ngauss=3, seed=3),
}


def grid(n, L=10.0):
    return -L / 2 + np.arange(n) * (L / n)


def gaussian_sum_tt(d, n, centres, widths, L=10.0):
    x = grid(n, L)
    G = len(widths)
    cores = []
    for k in range(d):
        vecs = [np.exp(-(x - centres[g][k]) ** 2 / (2 * widths[g] ** 2)) for g in range(G)]
        if G == 1:
            cores.append(vecs[0].reshape(1, n, 1))
        elif k == 0:
            cores.append(np.stack(vecs, axis=1).reshape(1, n, G))
        elif k == d - 1:
            cores.append(np.stack(vecs, axis=0).reshape(G, n, 1))
        else:
            c = np.zeros((G, n, G))
            for g in range(G):
                c[g, :, g] = vecs[g]
            cores.append(c)
    return cores


def initial_condition(d, n, ngauss, seed, L=10.0):
    """Sum of `ngauss` Gaussians, centres U[-2,2]^d and widths U[0.3,0.8]
    (ngauss == 1 with seed 0: the centred Gaussian of width 0.5)."""
    if ngauss == 1 and seed == 0:
        return gaussian_sum_tt(d, n, np.zeros((1, d)), np.array([0.5]), L)
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-2.0, 2.0, size=(ngauss, d))
    widths = rng.uniform(0.3, 0.8, size=ngauss)
    return gaussian_sum_tt(d, n, centres, widths, L)


def rms_norm(cores):
    """||X||_F / sqrt(prod n) by transfer matrices (host, small ranks only)."""
    a = np.ones((1, 1))
    for c in cores:
        t = np.einsum("ik,kjd->ijd", a, c)
        a = np.einsum("ijb,ijd->bd", c, t) / c.shape[1]
    return float(np.sqrt(max(a[0, 0], 0.0)))


def batch_shapes(count=64, seed=4):
    """Shapes of the batched-rounding workload: per train d ~ U{10..40},
    one mode size n ~ U{32, 64, 128, 256, 512}, interior ranks r_k ~
    U{8..96} clamped to r_{k-1} n and n r_{k+1} (a valid TT), rank cap
    floor(r_k / 2) per bond."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        d = int(rng.integers(10, 41))
        n = int(rng.choice([32, 64, 128, 256, 512]))
        r = [1] + [int(v) for v in rng.integers(8, 97, size=d - 1)] + [1]
        for k in range(1, d):  # left-to-right, then right-to-left clamp
            r[k] = min(r[k], r[k - 1] * n)
        for k in range(d - 1, 0, -1):
            r[k] = min(r[k], r[k + 1] * n)
        cap = [1] + [max(1, v // 2) for v in r[1:-1]] + [1]
        out.append((d, n, r, cap))
    return out


def rounding_cost(shape):
    """Work of one rounding of a train of this (d, n, r, cap) shape, in
    proportion to its flops: sum_k r_k n r_{k+1} max(r_k, r_{k+1}) (every
    bond's QR, and the products around it, scale with the unfolding's size
    times its column count)."""
    d, n, r, _ = shape
    return float(sum(r[k] * n * r[k + 1] * max(r[k], r[k + 1]) for k in range(d)))


def shard_by_cost(costs, world):
    """Split independent instances over `world` ranks so that the largest
    per-rank total is small: longest first, each to the least loaded rank
    (ties to the lower rank).  Deterministic, so every rank computes the same
    split without communicating.  Returns one list of indices per rank."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        w = min(range(world), key=lambda k: (load[k], k))
        out[w].append(i)
        load[w] += costs[i]
    return [sorted(o) for o in out]


def batch_trains(ctx, count=64, seed=4, only=None):
    """The batched-rounding workload as device trains: left-orthonormal
    random cores (QR of a Gaussian matrix) whose bond column j is scaled by
    2^-j, so every bond's spectrum decays as 2^-j.  Train i is generated
    from its own seed (seed * 1000 + i), so any subset (`only`: indices) is
    the same trains on any rank.  Generated on the GPU with torch (input
    preparation only).  Returns [(TT, shape)] in index order."""
    import torch

    from . import TT

    dev = torch.device("cuda", ctx.device)
    g = torch.Generator(device=dev)
    trains = []
    for idx, (d, n, r, cap) in enumerate(batch_shapes(count, seed)):
        if only is not None and idx not in only:
            continue
        g.manual_seed(seed * 1000 + idx)
        T = TT(ctx, [n] * d, r)
        cores = []
        for k in range(d):
            a = torch.randn(r[k] * n, r[k + 1], dtype=torch.float64, device=dev, generator=g)
            q, _ = torch.linalg.qr(a)
            if k < d - 1:
                q = q * torch.pow(2.0, -torch.arange(r[k + 1], dtype=torch.float64, device=dev))
            # (r_k n) x r_{k+1} column-major == the core's layout
            cores.append(q.t().contiguous().t())
        T.set_device(r, [c.data_ptr() for c in cores])
        torch.cuda.synchronize(dev)
        trains.append((T, (d, n, r, cap)))
    return trains
