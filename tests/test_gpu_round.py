"""TT rounding (ptt_round, paratt_truncate semantics) on the GPU against the
oracle on identical seeded inputs: ranks equal and the rounded tensors agree
to 1e-12 of ||X|| (gauge-free comparison through inner products of the
difference, which is formed as a TT and orthogonalised).  Inputs are built
with a spectral gap at the cutoff so LAPACK and the GPU cannot disagree on a
rank by round-off."""
import numpy as np
import pytest

import paratt_b200 as P
from oracle import tt_oracle as O

pytestmark = pytest.mark.gpu


def gapped_tt(dims, ranks, seed, keep, decay=1e-9):
    """Random TT whose bond k has `keep[k]` singular values O(1) and the rest
    ~decay: a left-orthonormal train with the first keep[k] columns scaled 1
    and the others by decay."""
    rng = np.random.default_rng(seed)
    cores = []
    for k, n in enumerate(dims):
        r, r1 = ranks[k], ranks[k + 1]
        a = rng.standard_normal((r * n, r1))
        q, _ = np.linalg.qr(a)
        s = np.ones(r1)
        if k < len(dims) - 1:
            s[keep[k + 1]:] = decay * (1 + rng.random(r1 - keep[k + 1]))
        cores.append((q[:, :r1] * s).reshape(r, n, r1, order="F"))
    return cores


CASES = [
    # dims, ranks, keep (per bond), rel tol, maxrank
    ([6, 5, 7, 4, 6], [1, 6, 8, 9, 6, 1], [1, 3, 4, 5, 2, 1], 1e-6, 64),
    ([4] * 8, [1, 4, 9, 12, 12, 12, 9, 4, 1], [1, 2, 3, 3, 4, 3, 2, 2, 1], 1e-6, 64),
    ([32, 16, 8], [1, 20, 30, 1], [1, 5, 7, 1], 1e-6, 64),
    ([10, 10, 10, 10], [1, 10, 40, 10, 1], [1, 6, 12, 6, 1], 1e-6, 8),   # rank cap binds
    ([64, 64, 64], [1, 64, 64, 1], [1, 40, 50, 1], 1e-6, 64),           # CT = 64
    ([20, 7, 20], [1, 20, 100, 1], [1, 15, 60, 1], 1e-6, 128),          # CT = 128
]


@pytest.mark.parametrize("dims,ranks,keep,rtol,maxr", CASES)
def test_round_parity(ctx, dims, ranks, keep, rtol, maxr):
    x = gapped_tt(dims, ranks, 11, keep)
    tol = rtol * O.norm(x)
    ref = O.round_tt(x, tol, maxr)
    X = P.TT.from_cores(ctx, x)
    X.round(tol, [maxr] * (len(dims) + 1))
    got = X.get()
    assert O.ranks_of(got) == O.ranks_of(ref)
    assert O.rel_diff_exact(got, ref) <= 1e-12
    # cores 1..d-1 right-orthonormal, as the reference leaves them
    for c in got[1:]:
        m = O.right_unfold(c)
        np.testing.assert_allclose(m @ m.T, np.eye(m.shape[0]), atol=1e-12)


def test_round_rank_deficient_sum(ctx):
    """x + x has exactly rank-deficient unfoldings (the case CholeskyQR cannot
    take); the result must be rank(x) with norm 2||x|| (round(a f + b f))."""
    x = gapped_tt([8, 6, 8, 5], [1, 5, 7, 4, 1], 21, [1, 5, 7, 4, 1], decay=1.0)
    z = O.axpby(1.0, x, 2.0, x)
    tol = 1e-10 * O.norm(z)
    ref = O.round_tt(z, tol, 64)
    Z = P.TT.from_cores(ctx, z)
    Z.round(tol)
    got = Z.get()
    assert O.ranks_of(got) == O.ranks_of(ref) == O.ranks_of(x)
    assert abs(O.norm(got) / O.norm(x) - 3.0) < 1e-12
    assert O.rel_diff_exact(got, ref) <= 1e-12


def test_round_small_modes(ctx):
    """Unfoldings with fewer rows than columns (q = m < c)."""
    x = O.random_tt([2, 3, 2, 3, 2], [1, 2, 6, 6, 3, 1], 31)
    tol = 1e-12 * O.norm(x)
    ref = O.round_tt(x, tol, 64)
    X = P.TT.from_cores(ctx, x)
    X.round(tol)
    got = X.get()
    assert O.ranks_of(got) == O.ranks_of(ref)
    assert O.rel_diff_exact(got, ref) <= 1e-12


def test_fixed_plans_same_result(ctx):
    """Capacity-sized plans (no rank read-back) give the same rounding."""
    x = gapped_tt([6, 5, 7, 4, 6], [1, 6, 8, 9, 6, 1], 11, [1, 3, 4, 5, 2, 1])
    tol = 1e-6 * O.norm(x)
    A = P.TT.from_cores(ctx, x, [1] + [100] * 4 + [1])
    B = P.TT.from_cores(ctx, x, [1] + [100] * 4 + [1])
    A.round(tol, 64)
    ctx.fixed_plans(True)
    try:
        B.round(tol, 64)
    finally:
        ctx.fixed_plans(False)
    a, b = A.get(), B.get()
    assert O.ranks_of(a) == O.ranks_of(b)
    assert O.rel_diff_exact(a, b) <= 1e-13


def test_graph_replay_bit_exact(ctx):
    """Roundings replayed from cached CUDA graphs equal direct launches
    bit for bit: first call (capture), repeats (replay), other ranks (a
    second graph), and a train at a new address."""
    shapes = [([6, 5, 7, 4, 6], [1, 6, 8, 9, 6, 1], [1, 3, 4, 5, 2, 1]),
              ([9, 8, 7, 6], [1, 7, 12, 5, 1], [1, 4, 6, 3, 1])]
    for dims, full, keep in shapes:
        x = gapped_tt(dims, full, 12, keep)
        tol = 1e-6 * O.norm(x)
        A = P.TT.from_cores(ctx, x)
        A.round(tol, 64)
        a = A.get()
        A.close()
        ctx.graphs(True)
        try:
            for _ in range(3):
                B = P.TT.from_cores(ctx, x)
                B.round(tol, 64)
                b = B.get()
                B.close()
                assert O.ranks_of(a) == O.ranks_of(b)
                for u, v in zip(a, b):
                    np.testing.assert_array_equal(u, v)
        finally:
            ctx.graphs(False)


@pytest.mark.parametrize("decay", [1e-3, 1e-9, 1e-14, 0.0])
def test_cholqr_matches_householder(ctx, decay):
    """The Cholesky-QR factorisation (default for <= 32 columns) and the
    Householder TSQR give the same rounding, for well separated, graded,
    near-singular and exactly rank-deficient unfoldings; the Cholesky path is
    the one that ran."""
    dims, full, keep = [9, 16, 7, 12, 8], [1, 7, 12, 10, 9, 1], [1, 4, 6, 5, 3, 1]
    x = gapped_tt(dims, full, 13, keep, decay=decay)
    if decay == 0.0:
        x = O.axpby(1.0, x, 0.5, x)  # repeated columns in every unfolding (ranks <= 24)
    tol = 1e-6 * O.norm(x)
    got = {}
    for on in (False, True):
        ctx.cholqr(on)
        before = ctx.qr_counts()
        X = P.TT.from_cores(ctx, x)
        X.round(tol, 64)
        got[on] = X.get()
        X.close()
        after = ctx.qr_counts()
        if on:
            assert after[0] > before[0]
        else:
            assert after == before
    ctx.cholqr(True)
    ref = O.round_tt(x, tol, 10**6)
    for on in (False, True):
        assert O.ranks_of(got[on]) == O.ranks_of(ref)
        assert O.rel_diff_exact(got[on], ref) <= 1e-12
    assert O.rel_diff_exact(got[True], got[False]) <= 1e-12


def test_pdl_same_bits(ctx):
    """Programmatic dependent launch changes scheduling only: the rounding is
    bit-identical with it on (default) and off."""
    x = gapped_tt([9, 16, 7, 12, 8], [1, 7, 12, 10, 9, 1], 14, [1, 4, 6, 5, 3, 1], decay=1e-10)
    tol = 1e-8 * O.norm(x)
    got = []
    for on in (True, False):
        ctx.pdl(on)
        X = P.TT.from_cores(ctx, x)
        X.round(tol, 64)
        got.append(X.get())
        X.close()
    ctx.pdl(True)
    assert O.ranks_of(got[0]) == O.ranks_of(got[1])
    for a, b in zip(*got):
        np.testing.assert_array_equal(a, b)


def test_autotune(ctx):
    """The autotuner keeps a valid cluster size (or the built-in rule) for
    every bucket, and roundings with its table agree with the untuned ones."""
    x = gapped_tt([9, 16, 7, 12, 8], [1, 7, 12, 10, 9, 1], 15, [1, 4, 6, 5, 3, 1], decay=1e-9)
    tol = 1e-8 * O.norm(x)
    X = P.TT.from_cores(ctx, x)
    X.round(tol, 64)
    before = X.get()
    X.close()
    table = ctx.autotune()
    assert table.shape == (3, 6)
    assert all(v in (0, 1, 2, 4, 8, 16) for v in table.ravel())  # 0: the row-count rule is kept
    tm64, fill = ctx.autotune_gemm()  # contraction tiles and split-K target
    assert tm64 in (48, 65) and fill in (74, 148, 296, 592)
    X = P.TT.from_cores(ctx, x)
    X.round(tol, 64)
    after = X.get()
    X.close()
    assert O.ranks_of(after) == O.ranks_of(before)
    assert O.rel_diff_exact(after, before) <= 1e-12


@pytest.mark.parametrize("decay", [1e-3, 1e-9, 1e-14, 0.0])
def test_grid_cholqr_matches_householder(ctx, decay):
    """33 to 64 columns: the grid Cholesky QR (rows spread over all SMs, one
    launch per Gram stage) against the Householder TSQR and the oracle, for
    well separated, graded, near-singular and exactly rank-deficient
    unfoldings; the Cholesky path is the one that ran."""
    dims = [9, 16, 7, 12, 8]
    if decay == 0.0:
        full, keep = [1, 7, 30, 28, 20, 1], [1, 5, 12, 10, 6, 1]
    else:
        full, keep = [1, 9, 48, 60, 40, 1], [1, 5, 20, 24, 7, 1]
    x = gapped_tt(dims, full, 23, keep, decay=decay)
    if decay == 0.0:
        x = O.axpby(1.0, x, 0.5, x)  # repeated columns: 40 to 60 per unfolding
    assert 32 < max(O.ranks_of(x)) <= 64
    tol = 1e-6 * O.norm(x)
    got = {}
    for on in (False, True):
        ctx.cholqr(on)
        before = ctx.qr_counts()
        X = P.TT.from_cores(ctx, x)
        X.round(tol, 64)
        got[on] = X.get()
        X.close()
        after = ctx.qr_counts()
        if on:
            assert after[0] > before[0]
        else:
            assert after == before
    ctx.cholqr(True)
    ref = O.round_tt(x, tol, 10**6)
    for on in (False, True):
        assert O.ranks_of(got[on]) == O.ranks_of(ref)
        assert O.rel_diff_exact(got[on], ref) <= 1e-12
    assert O.rel_diff_exact(got[True], got[False]) <= 1e-12
