"""Pins the numpy oracle (oracle/tt_oracle.py) to the reference itself:
golden fixtures produced by the reference's compiled C (always run), and
live comparisons against oracle/_ref/libparatt_ref.so when it is built."""
import os

import numpy as np
import pytest

from oracle import tt_oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def unpack(z, prefix):
    r, n = z[f"{prefix}_ranks"], z[f"{prefix}_dims"]
    return [z[f"{prefix}_{k}"].reshape((r[k], n[k], r[k + 1]), order="F") for k in range(len(n))]


def same(a, b, rtol=0.0):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert x.shape == y.shape
        if rtol == 0.0:
            np.testing.assert_array_equal(x, y)
        else:
            assert np.abs(x - y).max() <= rtol * max(np.abs(y).max(), 1e-300)


@pytest.mark.parametrize("i", range(4))
def test_round_golden(i):
    z = np.load(os.path.join(GOLD, f"round_{i}.npz"))
    x, ref = unpack(z, "in"), unpack(z, "out")
    got = O.round_tt(x, float(z["tol"]), int(z["maxrank"]))
    assert O.ranks_of(got) == O.ranks_of(ref)
    assert O.rel_diff_exact(got, ref) < 1e-12


def test_ops_golden():
    z = np.load(os.path.join(GOLD, "ops.npz"))
    x, y = unpack(z, "x"), unpack(z, "y")
    same(O.axpby(0.75, x, -1.5, y), unpack(z, "axpby"))
    same(O.hadamard(x, y), unpack(z, "had"))
    for m in range(4):
        same(O.periodic_stencil(x, m, [1.0, -2.0, 1.0]), unpack(z, f"sten{m}"), 1e-14)
    assert abs(O.norm(x) - float(z["norm"])) < 1e-13 * float(z["norm"])
    assert abs(O.dot(x, y) - float(z["dot"])) < 1e-13 * O.norm(x) * O.norm(y)
    assert abs(O.entry(x, list(z["entry_idx"])) - float(z["entry"])) < 1e-12


def test_ic_fixture_is_the_gaussian_pdf():
    """The reference's initial-condition cores (gaussian_dim_*/core_k.cr) are
    the N(0, 0.25^2) pdf sampled on linspace(-1.3, 1.3, 64)."""
    z = np.load(os.path.join(GOLD, "ic_core.npz"))
    assert list(z["header"]) == [1, 64, 1]
    x = np.linspace(-1.3, 1.3, 64)
    pdf = np.exp(-x**2 / (2 * 0.25**2)) / (0.25 * np.sqrt(2 * np.pi))
    assert np.abs(z["values"] - pdf).max() <= 1e-13 * pdf.max()


def test_round_known_answer():
    """round(a f + b f) has rank(f) and norm |a + b| ||f|| (a known-answer
    case: the reference's truncation of the formal sum must drop the
    duplicated half exactly)."""
    f = O.random_tt([7, 6, 5, 8], [1, 3, 4, 2, 1], 5)
    z = O.axpby(1.0, f, 2.0, f)
    g = O.round_tt(z, 1e-12 * O.norm(z), 64)
    assert O.ranks_of(g) == O.ranks_of(O.round_tt(f, 1e-12 * O.norm(f), 64))
    assert abs(O.norm(g) / O.norm(f) - 3.0) < 1e-12


def test_stencil_known_answer():
    """[1,-2,1] on a sampled sine along one mode multiplies it by the
    eigenvalue 2 cos(2 pi k / n) - 2 (a known-answer case of the periodic
    stencil)."""
    n, k = 32, 3
    v = np.sin(2 * np.pi * k * np.arange(n) / n)
    f = [v.reshape(1, n, 1), np.ones((1, 5, 1))]
    g = O.periodic_stencil(f, 0, [1.0, -2.0, 1.0])
    lam = 2 * np.cos(2 * np.pi * k / n) - 2
    np.testing.assert_allclose(g[0].ravel(), lam * v, atol=1e-13)


# ---------------------------------------------------------------------------
# live comparisons with the compiled reference
# ---------------------------------------------------------------------------
try:
    from oracle import ref_lib as R

    HAVE_REF = R.available()
except Exception:  # pragma: no cover
    HAVE_REF = False

needs_ref = pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built (make -C oracle)")


@needs_ref
@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("rtol,mr", [(1e-1, 64), (1e-4, 64), (1e-9, 64), (1e-9, 3)])
def test_round_vs_reference(seed, rtol, mr):
    dims, ranks = [6, 5, 7, 4, 6], [1, 3, 4, 5, 3, 1]
    x = O.random_tt(dims, ranks, seed)
    z = O.axpby(1.0, x, 0.5, O.random_tt(dims, ranks, seed + 50))
    tol = rtol * O.norm(z)
    got = O.round_tt(z, tol, mr)
    ref = R.ref_truncate(z, tol, mr)
    assert O.ranks_of(got) == O.ranks_of(ref)
    assert O.rel_diff_exact(got, ref) < 1e-12


@needs_ref
def test_round_rank_deficient_vs_reference():
    x = O.random_tt([6, 5, 7, 4], [1, 3, 4, 2, 1], 9)
    z = O.axpby(1.0, x, 1.0, x)
    tol = 1e-10 * O.norm(z)
    got, ref = O.round_tt(z, tol, 64), R.ref_truncate(z, tol, 64)
    assert O.ranks_of(got) == O.ranks_of(ref)
    assert O.rel_diff_exact(got, ref) < 1e-12


@needs_ref
def test_round_zero_and_repeated_columns_vs_reference():
    """Exact zero columns inside every core (a left-orthonormal train with
    bond spectra cut to zero) plus the repeated blocks of x + x/2: the case
    in which the GPU Jacobi once ran to its sweep limit on noise columns."""
    rng = np.random.default_rng(13)
    dims, full, keep = [9, 16, 7, 12, 8], [1, 7, 12, 10, 9, 1], [1, 4, 6, 5, 3, 1]
    x = []
    for k, n in enumerate(dims):
        q, _ = np.linalg.qr(rng.standard_normal((full[k] * n, full[k + 1])))
        if k < len(dims) - 1:
            q[:, keep[k + 1]:] = 0.0
        x.append(q.reshape(full[k], n, full[k + 1], order="F"))
    z = O.axpby(1.0, x, 0.5, x)
    for rtol in (0.0, 1e-6):
        tol = rtol * O.norm(z)
        got, ref = O.round_tt(z, tol, 64), R.ref_truncate(z, tol, 64)
        assert O.ranks_of(got) == O.ranks_of(ref)
        assert O.rel_diff_exact(got, ref) < 1e-12


@needs_ref
def test_ops_vs_reference():
    x = O.random_tt([6, 5, 7, 4, 6], [1, 3, 4, 5, 3, 1], 1)
    y = O.random_tt([6, 5, 7, 4, 6], [1, 2, 3, 3, 2, 1], 2)
    same(O.axpby(1.0, x, 0.5, y), R.ref_axpby(1.0, x, 0.5, y))
    same(O.hadamard(x, y), R.ref_hadamard(x, y))
    for m in range(5):
        same(O.periodic_stencil(x, m, [1, -2, 1]), R.ref_stencil(x, m, [1, -2, 1]), 1e-15)
    assert abs(O.norm(x) - R.ref_norm(x)) < 1e-13 * O.norm(x)
    assert abs(O.dot(x, y) - R.ref_dot(x, y)) < 1e-13 * O.norm(x) * O.norm(y)
    assert abs(O.entry(x, [1, 2, 3, 1, 0]) - R.ref_entry(x, [1, 2, 3, 1, 0])) < 1e-12


@needs_ref
def test_five_point_stencil_reference_branches():
    """The oracle is periodic for every stencil length, as the reference's
    serial attac_apply_periodic_stencil; its P=1 pattac branch differs for 5
    taps at 0 < a < h (documented deviation)."""
    import ctypes as C

    x = O.random_tt([6, 5, 7, 4, 6], [1, 3, 4, 5, 3, 1], 1)
    s5 = np.array([1.0, 2.0, 3.0, 4.0, 5.0])
    t = R.RefTT(x)
    R.lib().attac_apply_periodic_stencil(t.p.contents.x, 2, s5.ctypes.data_as(C.POINTER(C.c_double)), 5)
    same(O.periodic_stencil(x, 2, s5), t.cores(), 1e-15)
    t.free()
    p = R.ref_stencil(x, 2, s5)
    assert np.abs(p[2] - O.periodic_stencil(x, 2, s5)[2]).max() > 1e-3


@needs_ref
@pytest.mark.parametrize("ngauss,seed", [(1, 3), (2, 5)])
def test_rk2_composition_vs_reference(ngauss, seed):
    """The RK2 reaction-Burgers step of the oracle (tt_oracle.rxn_burgers_rk2_step)
    against the same composition run on the reference's own C routines
    (ref_lib.ref_rxn_burgers_rk2_step: paratt_truncate, pattacHadamard,
    attac_tt_axpby); the midpoint step follows paratt_ode.h:77-112.  This pins
    the composition that the GPU step, the oracle and the reference arm share."""
    d, n, maxr, dt = 4, 16, 12, 1e-3
    u = O.config_ic(d, n, ngauss, seed)
    tol = 1e-8 * O.norm(u)
    uo, ur = u, u
    for _ in range(3):
        uo = O.rxn_burgers_rk2_step(uo, dt, tol, maxr)
        ur = R.ref_rxn_burgers_rk2_step(ur, dt, tol, maxr)
        assert O.ranks_of(uo) == O.ranks_of(ur)
        assert O.rel_diff_exact(uo, ur) <= 1e-12
