"""Learned sketch path: MLP kernels against the numpy oracle (forward and
gradients), training, the explicit-TT sketch rounding and its acceptance
check, and the sketch RK2 step against the plain step."""
import numpy as np
import pytest

import paratt_b200 as P
from oracle import mlp_oracle as M
from oracle import tt_oracle as O

pytestmark = pytest.mark.gpu


def test_mlp_forward_and_gradients(ctx):
    nin, w, B = 18, 64, 300
    rng = np.random.default_rng(0)
    x = rng.standard_normal((B, nin)).astype(np.float32)
    t = (rng.random(B) * 30).astype(np.float32)
    net = P.MLP(ctx, nin, w, seed=3)
    p = net.params()
    y = net.forward(x)
    yr, _ = M.forward(p, x, nin, w)
    np.testing.assert_allclose(y, yr, rtol=1e-4, atol=1e-4 * np.abs(yr).max())
    g, loss = net.grads(x, t)
    gr, lr = M.grads(p, x, t, nin, w)
    assert abs(loss - lr) <= 1e-4 * lr
    assert np.abs(g - gr).max() <= 2e-4 * np.abs(gr).max()
    net.close()


def test_mlp_training_reduces_loss(ctx):
    nin, w = 18, 64
    rng = np.random.default_rng(1)
    x = rng.standard_normal((512, nin)).astype(np.float32)
    t = (5 + 3 * x[:, 0] - 2 * x[:, 1] ** 2).astype(np.float32)
    net = P.MLP(ctx, nin, w, seed=2)
    l0 = net.grads(x, t)[1]
    for _ in range(300):
        net.train_step(x, t, 3e-3)
    l1 = net.grads(x, t)[1]
    assert l1 < 0.05 * l0
    net.close()


def test_round_sketch_explicit(ctx):
    dims = [12] * 6
    x = O.config_ic(6, 12, 3, 5)
    z = O.axpby(1.0, x, 0.01, O.periodic_stencil(x, 2, [1, -2, 1]))
    tol = 1e-8 * O.norm(z)
    ref = O.round_tt(z, tol, 64)
    Z = P.TT.from_cores(ctx, z)
    out = P.TT(ctx, dims, [1] * 7)
    rr = O.ranks_of(ref)
    ok = P.round_sketch(Z, None, out, [1] + [r + 6 for r in rr[1:-1]] + [1], 7, tol, 64, pad=2)
    got = out.get()
    assert ok
    assert O.rel_diff_exact(got, ref) <= 5e-8
    # a sketch smaller than the needed rank is rejected
    small = [1] + [max(1, r - 2) for r in rr[1:-1]] + [1]
    assert not P.round_sketch(Z, None, out, small, 7, tol, 64, pad=2)


def test_sketch_step_close_to_plain(ctx):
    d, n = 6, 16
    u0 = O.config_ic(d, n, 3, 3)
    tol = 1e-8 * O.norm(u0)
    plain = P.RxnBurgers(ctx, d, n, maxrank=20, dt=1e-3, tol=tol)
    sk = P.RxnBurgers(ctx, d, n, maxrank=20, dt=1e-3, tol=tol, seed=5)
    A = P.TT.from_cores(ctx, u0, [1] + [40] * (d - 1) + [1])
    B = P.TT.from_cores(ctx, u0, [1] + [40] * (d - 1) + [1])
    for _ in range(3):
        plain.step(A)
        sk.step_sketch(B, [1] + [24] * (d - 1) + [1], pad=4)
    a, b = A.get(), B.get()
    assert O.rel_diff_exact(b, a) <= 1e-7
    calls, fb = sk.sketch_counts()
    assert calls > 0
    plain.close()
    sk.close()
