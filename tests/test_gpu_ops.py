"""Parity of the formal TT operations and contractions (CUDA, through the C
ABI) against the CPU oracle on the same seeded inputs.

axpby, Hadamard, scale and diagonal multiply only copy or multiply each
element once, so they must be bit-exact; stencils and contractions sum in a
different order (fused multiply-add on the GPU) and are checked to 1e-13
relative."""
import numpy as np
import pytest

import paratt_b200 as P
from oracle import tt_oracle as O

pytestmark = pytest.mark.gpu

SHAPES = [
    ([6, 5, 7, 4, 6], [1, 3, 4, 5, 3, 1]),
    ([3, 4], [1, 2, 1]),
    ([16, 1, 9, 32], [1, 5, 5, 7, 1]),
]


def _same(a, b):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert x.shape == y.shape
        np.testing.assert_array_equal(x, y)


def _close(a, b, rtol=1e-13):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert x.shape == y.shape
        s = max(np.abs(y).max(), 1e-300)
        assert np.abs(x - y).max() <= rtol * s


@pytest.mark.parametrize("dims,ranks", SHAPES)
def test_axpby_bit_exact(ctx, dims, ranks):
    x = O.random_tt(dims, ranks, 1)
    y = O.random_tt(dims, [1] + [r + 1 for r in ranks[1:-1]] + [1], 2)
    X, Y = P.TT.from_cores(ctx, x), P.TT.from_cores(ctx, y)
    Z = P.TT(ctx, dims, [1] * (len(dims) + 1))
    P.axpby(0.75, X, -1.5, Y, Z)
    _same(Z.get(), O.axpby(0.75, x, -1.5, y))
    # output aliasing an input
    P.axpby(2.0, X, 1.0, X, X)
    _same(X.get(), O.axpby(2.0, x, 1.0, x))


@pytest.mark.parametrize("dims,ranks", SHAPES)
def test_hadamard_bit_exact(ctx, dims, ranks):
    x = O.random_tt(dims, ranks, 3)
    y = O.random_tt(dims, [1] + [2] * (len(dims) - 1) + [1], 4)
    X, Y = P.TT.from_cores(ctx, x), P.TT.from_cores(ctx, y)
    Z = P.TT(ctx, dims, [1] * (len(dims) + 1))
    P.hadamard(X, Y, Z)
    _same(Z.get(), O.hadamard(x, y))


@pytest.mark.parametrize("dims,ranks", SHAPES)
def test_square_sym(ctx, dims, ranks):
    """x (.) x at ranks r(r+1)/2 is the same tensor as the formal square."""
    x = O.random_tt(dims, ranks, 5)
    X = P.TT.from_cores(ctx, x)
    Z = P.TT(ctx, dims, [1] * (len(dims) + 1))
    P.square_sym(X, Z)
    z = Z.get()
    assert [c.shape[0] for c in z] + [1] == [r * (r + 1) // 2 for r in ranks]
    ref = O.full(O.hadamard(x, x))
    np.testing.assert_allclose(O.full(z), ref, rtol=0, atol=1e-13 * np.abs(ref).max())
    # the rounded square matches the rounded formal square
    tol = 1e-10 * O.norm(x) ** 2
    Z.round(tol)
    zr = O.round_tt(O.hadamard(x, x), tol, 10**6)
    assert [c.shape[0] for c in Z.get()] == [c.shape[0] for c in zr]
    np.testing.assert_allclose(O.full(Z.get()), O.full(zr), rtol=0, atol=1e-11 * np.abs(ref).max())


def test_scale_and_diag(ctx):
    dims, ranks = SHAPES[0]
    x = O.random_tt(dims, ranks, 5)
    X = P.TT.from_cores(ctx, x)
    X.scale(-3.25)
    _same(X.get(), O.scale(-3.25, x))
    v = np.linspace(-1, 2, dims[2])
    X.mult_diag(2, v)
    _same(X.get(), O.mult_diag(O.scale(-3.25, x), 2, v))


@pytest.mark.parametrize("sten", [[1.0, -2.0, 1.0], [-0.5, 0.0, 0.5], [1, 2, 3, 4, 5], [2.0], [1, 2, 3, 4]])
def test_stencil(ctx, sten):
    dims, ranks = [8, 12, 5, 9], [1, 3, 4, 2, 1]
    x = O.random_tt(dims, ranks, 6)
    for mode in range(len(dims)):
        X = P.TT.from_cores(ctx, x)
        X.stencil(mode, sten)
        _close(X.get(), O.periodic_stencil(x, mode, sten), 1e-14)


def test_contractions(ctx):
    dims, ranks = SHAPES[0]
    x = O.random_tt(dims, ranks, 7)
    y = O.random_tt(dims, [1, 2, 2, 3, 2, 1], 8)
    X, Y = P.TT.from_cores(ctx, x), P.TT.from_cores(ctx, y)
    assert abs(X.dot(Y) - O.dot(x, y)) <= 1e-13 * O.norm(x) * O.norm(y)
    assert abs(X.norm() - O.norm(x)) <= 1e-13 * O.norm(x)
    for idx in ([0, 0, 0, 0, 0], [5, 4, 6, 3, 5], [2, 1, 3, 0, 4]):
        assert abs(X.entry(idx) - O.entry(x, idx)) <= 1e-13 * max(1.0, abs(O.entry(x, idx)))
