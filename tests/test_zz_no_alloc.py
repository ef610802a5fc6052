"""ptt_dot_noalloc: the inner product for callers that must not have the
library allocate device memory (its scratch is a fixed device array instead
of the context workspace).  Checked through the C ABI against ptt_dot, the
allocating entry point, on two calls in a row (the second call finds the
first call's leftovers in the shared array), plus the size limit.

This file is collected last on purpose, so a run that stops at the first
failure has already run every other test."""
import numpy as np
import pytest

import paratt_b200 as P
from oracle import tt_oracle as O

pytestmark = pytest.mark.gpu


def test_noalloc_dot_matches_dot_twice(ctx):
    dims = [16, 9, 32, 12, 8]
    for seed in (1, 2):  # two different problems back to back
        x = O.random_tt(dims, [1, 4, 7, 6, 5, 1], 10 * seed)
        y = O.random_tt(dims, [1, 3, 5, 8, 2, 1], 10 * seed + 1)
        X, Y = P.TT.from_cores(ctx, x), P.TT.from_cores(ctx, y)
        ref = X.dot(Y)
        got = X.dot_noalloc(Y)
        assert abs(got - ref) <= 1e-13 * max(abs(ref), O.norm(x) * O.norm(y))
        assert abs(got - O.dot(x, y)) <= 1e-13 * O.norm(x) * O.norm(y)
        X.close()
        Y.close()


def test_noalloc_dot_allocates_nothing(ctx):
    """With the trains made and one call done, another call leaves the
    context's workspaces and the device's free memory as they were."""
    dims = [32, 24, 16, 40]
    x = O.random_tt(dims, [1, 9, 12, 7, 1], 5)
    y = O.random_tt(dims, [1, 6, 11, 10, 1], 6)
    X, Y = P.TT.from_cores(ctx, x), P.TT.from_cores(ctx, y)
    first = X.dot_noalloc(Y)
    ws0, (free0, _) = ctx.workspace_bytes(), ctx.mem_info()
    second = X.dot_noalloc(Y)
    ws1, (free1, _) = ctx.workspace_bytes(), ctx.mem_info()
    assert ws1 == ws0
    assert free1 == free0
    assert first == second
    assert abs(second - O.dot(x, y)) <= 1e-13 * O.norm(x) * O.norm(y)
    X.close()
    Y.close()


def test_noalloc_rejects_oversize(ctx):
    dims = [256, 256, 256]
    x = O.random_tt(dims, [1, 64, 64, 1], 3)
    X = P.TT.from_cores(ctx, x)
    with pytest.raises(P.PttError) as e:
        X.dot_noalloc(X)  # 64*256*64 + 2*64*64 doubles > 2^19
    assert e.value.code == P.PTT_ERR_CAPACITY
    assert np.isfinite(X.dot(X))
    X.close()
