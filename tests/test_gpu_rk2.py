"""Reaction-Burgers pieces on the GPU against the oracle composition
(oracle/tt_oracle.py: op_sum_apply, rxn_burgers_F, rxn_burgers_rk2_step).

* ptt_op_sum builds the structured rank-2r operator TT: same cores as the
  oracle to 1e-14 (stencil sums in a different order).
* ptt_round_hadamard (randomised sketch, product never formed) is checked
  against the deterministic rounding of the formal product: the error is a
  small multiple of the tolerance.
* one RK2 step and a few steps at small sizes where the product is formed
  formally: ranks equal and relative difference <= 1e-9 of ||u||."""
import numpy as np
import pytest

import paratt_b200 as P
from oracle import tt_oracle as O

pytestmark = pytest.mark.gpu


def _close(a, b, rtol):
    for x, y in zip(a, b):
        assert x.shape == y.shape
        assert np.abs(x - y).max() <= rtol * max(np.abs(y).max(), 1e-300)


@pytest.mark.parametrize("d", [1, 2, 5])
def test_op_sum(ctx, d):
    dims = [12] * d
    ranks = [1] + [3] * (d - 1) + [1]
    x = O.random_tt(dims, ranks, 40 + d)
    sten = [0.3, -0.6, 0.3]
    X = P.TT.from_cores(ctx, x)
    Y = P.TT(ctx, dims, [1] * (d + 1))
    P.op_sum(X, sten, 1.5, Y)
    ref = O.op_sum_apply(x, [sten] * d, 1.5)
    got = Y.get()
    _close(got, ref, 1e-14)
    # the operator TT represents sum_i S_i x + 1.5 x
    if d <= 2:
        full = O.full(x) * 1.5
        for i in range(d):
            full = full + O.full(O.periodic_stencil(x, i, sten))
        np.testing.assert_allclose(O.full(got), full, rtol=1e-12, atol=1e-12 * np.abs(full).max())


def test_round_hadamard_sketch(ctx):
    dims = [10] * 5
    x = O.config_ic(5, 10, 3, 7)
    x = O.round_tt(O.axpby(1.0, x, 0.3, O.periodic_stencil(x, 2, [1, -2, 1])), 1e-14, 64)
    y = O.round_tt(O.axpby(1.0, x, 1.0, O.random_tt(dims, [1, 2, 2, 2, 2, 1], 5, 0.1)), 1e-14, 64)
    tol = 1e-8 * O.norm(O.hadamard(x, y))
    ref = O.round_tt(O.hadamard(x, y), tol, 64)
    X, Y = P.TT.from_cores(ctx, x), P.TT.from_cores(ctx, y)
    Z = P.TT(ctx, dims, [1] * 6)
    rr = O.ranks_of(ref)
    P.round_hadamard(X, Y, Z, [1] + [r + 8 for r in rr[1:-1]] + [1], 1234, tol, 64)
    got = Z.get()
    err = O.rel_diff_exact(got, ref)
    assert err <= 5e-8, err
    assert all(a <= b + 1 for a, b in zip(O.ranks_of(got), rr))


def test_rk2_step_matches_oracle(ctx):
    d, n = 4, 16
    u0 = O.config_ic(d, n, 1, 3)
    tol = 1e-8 * O.norm(u0)
    dt = 1e-3
    sim = P.RxnBurgers(ctx, d, n, maxrank=20, dt=dt, tol=tol)
    U = P.TT.from_cores(ctx, u0, [1] + [40] * (d - 1) + [1])
    ref = u0
    for step in range(3):
        ref = O.rxn_burgers_rk2_step(ref, dt, tol, 20)
        sim.step(U)
        got = U.get()
        assert O.ranks_of(got) == O.ranks_of(ref), (step, O.ranks_of(got), O.ranks_of(ref))
        assert O.rel_diff_exact(got, ref) <= 1e-9
    f, s = sim.counts()
    assert f > 0 and s == 0  # small ranks: the product was formed formally
    sim.close()
