"""The oracle's restatement of the reference's CDF-problem stencils and
marginals (tt_oracle.cdf_*, marginal_*, scale_weight_sum, apply_marginal)
against the reference's own compiled C (paratt.c:772-1618, one process), on
seeded cores, every mode including the first and the last."""
import numpy as np
import pytest

from oracle import tt_oracle as O

try:
    from oracle import ref_lib as R

    HAVE_REF = R.available()
except Exception:  # pragma: no cover
    HAVE_REF = False

pytestmark = pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built (make -C oracle)")

DIMS = [9, 7, 11, 8]
RANKS = [1, 3, 4, 2, 1]


def _close(a, b, rtol=1e-13):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert x.shape == y.shape
        assert np.abs(x - y).max() <= rtol * max(np.abs(y).max(), 1e-300)


@pytest.mark.parametrize("mode", range(4))
@pytest.mark.parametrize("sten", [[1.0, -2.0, 1.0], [0.1, -0.4, 0.9, -0.4, 0.1], [0.3, 0.2, -0.7, 0.6]])
def test_cdf_stencil(mode, sten):
    x = O.random_tt(DIMS, RANKS, 1 + mode)
    _close(O.cdf_stencil(x, mode, sten), R.ref_cdf_op("cdf_stencil", x, mode, sten))


@pytest.mark.parametrize("mode", range(4))
def test_cdf_fluxes(mode):
    x = O.random_tt(DIMS, RANKS, 11 + mode)
    n = DIMS[mode]
    rng = np.random.default_rng(mode)
    w, gw, src, b = rng.standard_normal(n), rng.standard_normal(2), rng.standard_normal(n), rng.standard_normal(n + 1)
    dt, dx = 0.01, 0.2
    _close(O.cdf_lf_flux(x, mode, w, gw, src, dt, dx),
           R.ref_cdf_op("cdf_lf_flux", x, mode, w, gw, src, scalars=(dt, dx)))
    _close(O.cdf_lw_rhs(x, mode, w, gw, b, src, dt, dx),
           R.ref_cdf_op("cdf_lw_rhs", x, mode, w, gw, b, src, scalars=(dt, dx)))


@pytest.mark.parametrize("mode", range(4))
def test_marginal_scans(mode):
    x = O.random_tt(DIMS, RANKS, 21 + mode)
    n = DIMS[mode]
    rng = np.random.default_rng(30 + mode)
    w, s = rng.random(n), rng.standard_normal(n)
    _close(O.marginal_cusum(x, mode, w), R.ref_cdf_op("marginal_cusum", x, mode, w))
    _close(O.marginal_trap(x, mode, w), R.ref_cdf_op("marginal_trap", x, mode, w))
    _close(O.scale_weight_sum(x, mode, s, w), R.ref_cdf_op("scale_weight_sum", x, mode, s, w))


@pytest.mark.parametrize("mode", range(4))
def test_apply_marginal(mode):
    x = O.random_tt(DIMS, RANKS, 41 + mode)
    w = np.random.default_rng(mode).random(DIMS[mode])
    got, ref = O.apply_marginal(x, mode, w), R.ref_apply_marginal(x, mode, w)
    assert O.ranks_of(got) == O.ranks_of(ref) and O.dims_of(got) == O.dims_of(ref)
    _close(got, ref)
