"""GPU parity at the benchmark configurations, on identical seeded inputs.

* config 1 (d=40, n=256): x + y of two seeded rank-32 trains (entries with
  standard deviation 1/sqrt(n r)) rounded to tol 1e-10 x ||z||_RMS with rank
  cap 32 by ptt_round and by the reference's own paratt_truncate
  (paratt.c:316-342 -> pattac.c:590-675, compiled C in oracle/_ref): ranks
  equal, relative difference <= 1e-12;
* config 0 (d=20, n=64, rank cap 20, tol 1e-8 x ||u0||_RMS, dt 1e-3, centred
  Gaussian): 10 plain RK2 steps on the GPU against the oracle's composition
  (pinned to the reference's routines by test_oracle_vs_ref): ranks equal after
  every step, relative L2 difference <= 1e-9 (a tenth of the tolerance);
* one plain step from a state of rank 16, whose square exceeds 128 ranks, so
  the GPU step takes the sketched-product branch (the product is never
  formed) while the oracle forms u.u at rank 256: ranks equal, difference a
  small multiple of the tolerance.

Differences are gauge-free: the difference is formed as a train and
orthogonalised before its norm (tt_oracle.rel_diff_exact)."""
import numpy as np
import pytest

import paratt_b200 as P
from oracle import tt_oracle as O

pytestmark = pytest.mark.gpu

try:
    from oracle import ref_lib as R

    HAVE_REF = R.available()
except Exception:  # pragma: no cover
    HAVE_REF = False


def config1_inputs(d=40, n=256, r=32):
    """The two seeded trains of the rank-64 rounding workload (seeds 1, 2)."""
    sd = 1.0 / np.sqrt(n * r)
    out = []
    for seed in (1, 2):
        rng = np.random.default_rng(seed)
        rr = [1] + [r] * (d - 1) + [1]
        out.append([rng.standard_normal((rr[k], n, rr[k + 1])) * sd for k in range(d)])
    return out


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built (make -C oracle)")
def test_config1_rounding_vs_reference(ctx):
    x, y = config1_inputs()
    z = O.axpby(1.0, x, 1.0, y)
    tol = 1e-10 * O.norm(z)
    ref = R.ref_truncate(z, tol, 32)
    Z = P.TT.from_cores(ctx, z)
    Z.round(tol, 32)
    got = Z.get()
    assert O.ranks_of(got) == O.ranks_of(ref)
    assert O.ranks_of(got) == [1] + [32] * 39 + [1]
    err = O.rel_diff_exact(got, ref)
    assert err <= 1e-12, err
    Z.close()


def test_config0_trajectory_vs_oracle(ctx):
    from paratt_b200 import workloads as Wl

    cfg = Wl.CONFIGS["c0"]
    d, n, maxr, dt = cfg["d"], cfg["n"], cfg["maxrank"], cfg["dt"]
    u0 = Wl.initial_condition(d, n, cfg["ngauss"], cfg["seed"])
    tol = cfg["tol"] * O.norm(u0)
    sim = P.RxnBurgers(ctx, d, n, maxrank=maxr, dt=dt, tol=tol)
    U = P.TT.from_cores(ctx, u0, [1] + [2 * maxr] * (d - 1) + [1])
    ref = u0
    errs = []
    for step in range(10):
        ref = O.rxn_burgers_rk2_step(ref, dt, tol, maxr)
        sim.step(U)
        got = U.get()
        assert O.ranks_of(got) == O.ranks_of(ref), (step, O.ranks_of(got), O.ranks_of(ref))
        errs.append(O.rel_diff_exact(got, ref))
    assert max(errs) <= 1e-9, errs
    U.close()
    sim.close()


def test_plain_step_sketched_product_vs_oracle(ctx):
    # sum of 16 Gaussians: rank 16, so u.u has formal rank 256 and symmetric
    # rank 136 > 128; its rounding keeps ranks [13, 60, 14] at this tol, below
    # the cap 64 (the sketch ranks are 64 + 8), so both methods truncate by
    # the tolerance rather than by the cap
    d, n, G, maxr, dt = 4, 16, 16, 64, 1e-3
    u0 = O.config_ic(d, n, G, 5)
    assert max(O.ranks_of(u0)) == G and G * (G + 1) // 2 > 128
    tol = 1e-8 * O.norm(u0)
    sim = P.RxnBurgers(ctx, d, n, maxrank=maxr, dt=dt, tol=tol)
    U = P.TT.from_cores(ctx, u0, [1] + [2 * maxr] * (d - 1) + [1])
    sim.step(U)
    got = U.get()
    f, s = sim.counts()
    assert s > 0  # the product of the first F was rounded through the sketch
    ref = O.rxn_burgers_rk2_step(u0, dt, tol, maxr)
    assert O.ranks_of(got) == O.ranks_of(ref), (O.ranks_of(got), O.ranks_of(ref))
    err = O.rel_diff_exact(got, ref)
    assert err <= 1e-7, err
    U.close()
    sim.close()
