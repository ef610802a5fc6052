"""Ozaki split-precision Gram matrices on the fifth-generation tensor cores.

* ptt_gram (method 1: seven BF16 digit slices per element, tcgen05.mma with
  FP32 accumulation in tensor memory, recombined in FP64; method 0: FP64 mma)
  against the Gram matrix computed in extended precision (numpy longdouble,
  64-bit significand) on the host: max_ij |G_ij - G*_ij| / (||a_i|| ||a_j||)
  <= 1e-14 for both methods, on Gaussian columns, on columns scaled by powers
  of two from 2^-300 to 2^300, with a zero column, a single row, and the
  config-1 unfolding shape 16384 x 64.  The measured errors are printed.
* Bit-for-bit repeatability of the Ozaki Gram (fixed summation order).
* The config-1 rounding (d=40, n=256, ranks 64 -> 32, tol 1e-10 x ||z||) with
  the Gram stages of the grid Cholesky QR on the Ozaki path
  (ptt_ctx_ozaki): ranks equal to the reference's paratt_truncate
  (pattac.c:590-675, compiled in oracle/_ref), relative difference <= 1e-12,
  and the same against the FP64 path of this library.  With ptt_ctx_ozaki the
  R X products of the left sweep (R x core_{k+1}, K = the bond rank <= 64)
  are Ozaki products too.
* Roundings of gapped trains with 33-64-column unfoldings on the Ozaki path
  against the oracle (ranks equal, <= 1e-12, right-orthonormal cores)."""
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


def _gram_dev(ctx, a, method):
    import torch

    m, c = a.shape
    A = torch.from_numpy(np.asfortranarray(a).T.copy()).cuda()  # (c, m) rows = columns of a
    G = torch.zeros((c, c), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.gram(A.data_ptr(), m, c, m, G.data_ptr(), method)
    return G.cpu().numpy().T  # column-major c x c


def _gram_err(a, g):
    al = a.astype(np.longdouble)
    ref = al.T @ al
    nrm = np.sqrt(np.maximum(np.diag(ref), np.longdouble(1e-300)))
    scale = np.outer(nrm, nrm)
    return float(np.max(np.abs(g.astype(np.longdouble) - ref) / scale))


def _cases():
    rng = np.random.default_rng(7)
    yield "gauss 16384x64", rng.standard_normal((16384, 64))
    yield "gauss 1000x33", rng.standard_normal((1000, 33))
    a = rng.standard_normal((5000, 48))
    a *= np.ldexp(1.0, rng.integers(-300, 300, size=48))[None, :]
    yield "scaled 2^+-300", a
    a = rng.standard_normal((700, 40))
    a[:, 5] = 0.0
    yield "zero column", a
    yield "one row", rng.standard_normal((1, 17))
    yield "q of an unfolding", np.linalg.qr(rng.standard_normal((16384, 64)))[0]


@pytest.mark.parametrize("name,a", list(_cases()), ids=lambda v: v if isinstance(v, str) else "")
def test_gram_methods_vs_extended(ctx, name, a):
    e_fp = _gram_err(a, _gram_dev(ctx, a, 0))
    e_oz = _gram_err(a, _gram_dev(ctx, a, 1))
    print(f"{name}: FP64 mma {e_fp:.2e}, Ozaki {e_oz:.2e}")
    assert e_fp <= 1e-14, e_fp
    assert e_oz <= 1e-14, e_oz


def test_gram_ozaki_repeatable(ctx):
    a = np.random.default_rng(3).standard_normal((16384, 64))
    g1 = _gram_dev(ctx, a, 1)
    g2 = _gram_dev(ctx, a, 1)
    assert np.array_equal(g1, g2)
    assert np.array_equal(g1, g1.T)


def test_gram_bad_arguments(ctx):
    with pytest.raises(P.PttError):
        ctx.gram(0, 10, 65, 10, 0, 1)


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built (make -C oracle)")
def test_config1_rounding_ozaki_vs_reference(ctx):
    from test_gpu_configs import config1_inputs

    x, y = config1_inputs()
    z = O.axpby(1.0, x, 1.0, y)
    tol = 1e-10 * O.norm(z)
    ref = R.ref_truncate(z, tol, 32)
    outs = {}
    for oz in (True, False):
        ctx.ozaki(oz)
        Z = P.TT.from_cores(ctx, z)
        Z.round(tol, 32)
        outs[oz] = Z.get()
        Z.close()
    ctx.ozaki(False)
    got = outs[True]
    assert O.ranks_of(got) == O.ranks_of(ref) == [1] + [32] * 39 + [1]
    err = O.rel_diff_exact(got, ref)
    err_fp = O.rel_diff_exact(got, outs[False])
    print(f"config-1 rounding, Ozaki Gram: vs reference {err:.2e}, vs FP64 path {err_fp:.2e}")
    assert err <= 1e-12, err
    assert err_fp <= 1e-12, err_fp


OZ_CASES = [
    # dims, ranks, keep (per bond), maxrank: 33-64-column unfoldings, where the
    # Gram stages and the R X products take the Ozaki path
    ([64, 64, 64], [1, 64, 64, 1], [1, 40, 50, 1], 64),
    ([16, 40, 24, 16], [1, 16, 60, 48, 1], [1, 12, 35, 20, 1], 64),
    ([48, 48, 48, 48], [1, 48, 64, 48, 1], [1, 33, 45, 30, 1], 40),  # rank cap binds
]


@pytest.mark.parametrize("dims,ranks,keep,maxr", OZ_CASES)
def test_round_parity_ozaki(ctx, dims, ranks, keep, maxr):
    """Rounding with the Ozaki Gram matrices and R X products against the
    oracle on gapped trains: ranks equal, difference <= 1e-12 of ||X||, and
    cores 1..d-1 right-orthonormal."""
    from test_gpu_round import gapped_tt

    x = gapped_tt(dims, ranks, 13, keep)
    tol = 1e-6 * O.norm(x)
    ref = O.round_tt(x, tol, maxr)
    ctx.ozaki(True)
    try:
        X = P.TT.from_cores(ctx, x)
        X.round(tol, [maxr] * (len(dims) + 1))
        got = X.get()
        X.close()
    finally:
        ctx.ozaki(False)
    assert O.ranks_of(got) == O.ranks_of(ref)
    assert O.rel_diff_exact(got, ref) <= 1e-12
    for c in got[1:]:
        m = O.right_unfold(c)
        np.testing.assert_allclose(m @ m.T, np.eye(m.shape[0]), atol=1e-12)
