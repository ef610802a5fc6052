"""The CDF-problem stencils and marginals on the GPU: the device ABI
(ptt_cdf_*, ptt_marginal_*, ptt_scale_weight_sum, ptt_apply_marginal)
against the oracle, and the reference-signature calls of libparatt_b200.so
(pattac_apply_cdf_stencil ... pattac_apply_marginal, host cores) against the
reference's own compiled C (paratt.c:772-1618, one process) on identical
inputs.  The oracle is pinned to the reference by tests/test_cdf_oracle.py."""
import ctypes as C

import numpy as np
import pytest

import paratt_b200 as P
from oracle import tt_oracle as O

pytestmark = pytest.mark.gpu

DIMS = [9, 7, 11, 8]
RANKS = [1, 3, 40, 2, 1]  # a mode with 40-row fibers (several warps per fiber group)


def _close(a, b, rtol=1e-13):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert x.shape == y.shape
        assert np.abs(x - y).max() <= rtol * max(np.abs(y).max(), 1e-300)


def _vecs(mode, seed):
    n = DIMS[mode]
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n), rng.standard_normal(2), rng.standard_normal(n), rng.standard_normal(n + 1), rng.random(n)


@pytest.mark.parametrize("mode", range(4))
def test_device_cdf_ops_vs_oracle(ctx, mode):
    x = O.random_tt(DIMS, RANKS, 5 + mode)
    w, gw, src, b, pos = _vecs(mode, mode)
    dt, dx = 0.02, 0.3
    cases = [
        (lambda T: T.cdf_stencil(mode, [0.1, -0.4, 0.9, -0.4, 0.1]), O.cdf_stencil(x, mode, [0.1, -0.4, 0.9, -0.4, 0.1])),
        (lambda T: T.cdf_stencil(mode, [1.0, -2.0, 1.0, 7.0]), O.cdf_stencil(x, mode, [1.0, -2.0, 1.0, 7.0])),
        (lambda T: T.cdf_lf_flux(mode, w, gw, src, dt, dx), O.cdf_lf_flux(x, mode, w, gw, src, dt, dx)),
        (lambda T: T.cdf_lw_rhs(mode, w, gw, b, src, dt, dx), O.cdf_lw_rhs(x, mode, w, gw, b, src, dt, dx)),
        (lambda T: T.marginal_cusum(mode, pos), O.marginal_cusum(x, mode, pos)),
        (lambda T: T.marginal_trap(mode, pos), O.marginal_trap(x, mode, pos)),
        (lambda T: T.scale_weight_sum(mode, w, pos), O.scale_weight_sum(x, mode, w, pos)),
    ]
    for op, ref in cases:
        T = P.TT.from_cores(ctx, x)
        op(T)
        _close(T.get(), ref)
        T.close()
    # marginal: a d-1 mode train
    X = P.TT.from_cores(ctx, x)
    ref = O.apply_marginal(x, mode, pos)
    Z = P.TT(ctx, O.dims_of(ref), O.ranks_of(ref))
    X.apply_marginal(mode, pos, Z)
    got = Z.get()
    assert O.ranks_of(got) == O.ranks_of(ref)
    _close(got, ref)
    X.close()
    Z.close()


try:
    from oracle import ref_lib as R

    HAVE_REF = R.available()
except Exception:  # pragma: no cover
    HAVE_REF = False


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built (make -C oracle)")
@pytest.mark.parametrize("mode", [0, 2, 3])
def test_reference_signatures_vs_reference(mode):
    from paratt_b200 import capi as A

    L = A.capi()
    Pp, dp = C.POINTER(A.Paratt), C.POINTER(C.c_double)
    L.pattac_apply_cdf_stencil.argtypes = [Pp, C.c_int, dp, C.c_int]
    L.pattac_apply_cdf_lf_flux.argtypes = [Pp, C.c_int, dp, dp, dp, C.c_double, C.c_double]
    L.pattac_apply_cdf_lw_rhs.argtypes = [Pp, C.c_int, dp, dp, dp, dp, C.c_double, C.c_double]
    L.pattac_marginal_cusum.argtypes = [Pp, C.c_int, dp]
    L.pattac_marginal_trap.argtypes = [Pp, C.c_int, dp]
    L.pattac_scale_weight_sum.argtypes = [Pp, C.c_int, dp, dp]
    L.pattac_apply_marginal.argtypes = [Pp, C.POINTER(Pp), C.c_int, dp]
    x = O.random_tt(DIMS, RANKS, 50 + mode)
    w, gw, src, b, pos = [np.ascontiguousarray(v) for v in _vecs(mode, 60 + mode)]
    sten = np.array([0.2, -1.0, 0.6])
    dt, dx = 0.01, 0.25

    def p(v):
        return v.ctypes.data_as(dp)

    runs = [
        ("cdf_stencil", lambda t: L.pattac_apply_cdf_stencil(t.p, mode, p(sten), 3), (sten,), ()),
        ("cdf_lf_flux", lambda t: L.pattac_apply_cdf_lf_flux(t.p, mode, p(w), p(gw), p(src), dt, dx),
         (w, gw, src), (dt, dx)),
        ("cdf_lw_rhs", lambda t: L.pattac_apply_cdf_lw_rhs(t.p, mode, p(w), p(gw), p(b), p(src), dt, dx),
         (w, gw, b, src), (dt, dx)),
        ("marginal_cusum", lambda t: L.pattac_marginal_cusum(t.p, mode, p(pos)), (pos,), ()),
        ("marginal_trap", lambda t: L.pattac_marginal_trap(t.p, mode, p(pos)), (pos,), ()),
        ("scale_weight_sum", lambda t: L.pattac_scale_weight_sum(t.p, mode, p(w), p(pos)), (w, pos), ()),
    ]
    for name, call, vecs, scal in runs:
        t = A.HostTT(x)
        call(t)
        _close(t.cores(), R.ref_cdf_op(name, x, mode, *vecs, scalars=scal))
        t.free()
    t = A.HostTT(x)
    out = Pp()
    L.pattac_apply_marginal(t.p, C.byref(out), mode, p(pos))
    m = A.HostTT(ptr=out)
    ref = R.ref_apply_marginal(x, mode, pos)
    got = m.cores()
    assert O.ranks_of(got) == O.ranks_of(ref)
    _close(got, ref)
    m.free()
    t.free()
