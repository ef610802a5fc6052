"""Batched rounding (ptt_round_batch): independent trains of different
shapes rounded concurrently give the same ranks and tensors as the oracle's
paratt_truncate on each train, and leave the context's stream ordered after
them."""
import numpy as np
import pytest

import paratt_b200 as P
from oracle import tt_oracle as O
from test_gpu_round import CASES, gapped_tt

pytestmark = pytest.mark.gpu


def test_round_batch_parity(ctx):
    trains, tols, caps, refs = [], [], [], []
    for i, (dims, ranks, keep, rtol, maxr) in enumerate(CASES):
        x = gapped_tt(dims, ranks, 40 + i, keep)
        tol = rtol * O.norm(x)
        refs.append(O.round_tt(x, tol, maxr))
        trains.append(P.TT.from_cores(ctx, x))
        tols.append(tol)
        caps.append(maxr if i % 2 == 0 else [maxr] * (len(dims) + 1))
    P.round_batch(trains, tols, caps, lanes=4)
    for T, ref in zip(trains, refs):
        got = T.get()
        assert O.ranks_of(got) == O.ranks_of(ref)
        assert O.rel_diff_exact(got, ref) <= 1e-12
    # the context's stream follows the batch: an op on it sees rounded trains
    Z = P.TT(ctx, trains[0].dims, [1] * (trains[0].d + 1))
    P.axpby(1.0, trains[0], -1.0, trains[0], Z)
    assert O.ranks_of(Z.get()) == [1] + [2 * r for r in O.ranks_of(refs[0])[1:-1]] + [1]


def test_round_batch_matches_single(ctx):
    """The same train rounded alone and inside a batch of copies."""
    x = gapped_tt([16, 8, 16, 8], [1, 16, 30, 20, 1], 7, [1, 9, 12, 8, 1])
    tol = 1e-6 * O.norm(x)
    A = P.TT.from_cores(ctx, x)
    A.round(tol)
    copies = [P.TT.from_cores(ctx, x) for _ in range(6)]
    P.round_batch(copies, [tol] * 6, None, lanes=3)
    a = A.get()
    for T in copies:
        b = T.get()
        assert O.ranks_of(a) == O.ranks_of(b)
        assert O.rel_diff_exact(a, b) <= 1e-13


def test_round_batch_rejects_repeats(ctx):
    x = gapped_tt([6, 5, 7], [1, 6, 8, 1], 3, [1, 3, 4, 1])
    A = P.TT.from_cores(ctx, x)
    with pytest.raises(P.PttError):
        P.round_batch([A, A], [1e-6, 1e-6])
