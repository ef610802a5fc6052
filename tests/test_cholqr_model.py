"""CPU model of the Cholesky-QR stage sequence that the cluster kernel
(paratt_b200/csrc/ptt_cholqr.cuh) runs for unfoldings with <= 32 columns:
plain Cholesky QR, shifted Cholesky QR (shift 11 (m c + c (c+1)) u ||Q||_F^2)
when the pivots span more than 12 decades, the first-order factor
I + striu(E) + diag(E)/2 once max|Q^T Q - I| <= 1e-7 (final without another
Gram stage when <= 1e-8), done at max|Q^T Q - I| <= 1e-13, at most 7 Gram
stages.  The model checks the numerical claims the kernel relies on: the
sequence converges within the stage limit for condition numbers up to 1e20
and for exactly repeated columns, Q is orthonormal and A = Q R to working
precision, and R carries A's singular values to working precision.  The
16384 x 64 case is the rank-64 rounding's unfolding, which the kernel does
not take yet (more than 32 columns): the sequence itself holds there too."""
import numpy as np
import pytest
from scipy.linalg import solve_triangular

U = 1.1102230246251565e-16


def _chol(G, shift):
    c = G.shape[0]
    g = G + shift * np.eye(c)
    R = np.zeros_like(G)
    piv = []
    ok = True
    for j in range(c):
        d = g[j, j]
        piv.append(d)
        if not d > 0:
            ok = False
            d = 1.0
        r = np.sqrt(d)
        R[j, j] = r
        R[j, j + 1:] = g[j, j + 1:] / r
        g[j + 1:, j + 1:] -= np.outer(R[j, j + 1:], R[j, j + 1:])
    piv = np.array(piv)
    return ok, R, (piv.min() / piv.max() if piv.max() > 0 else 0.0)


def cholqr_sequence(A, maxst=7, tau=1e-13, first=1e-7, first_done=1e-8):
    m, c = A.shape
    Q = A.copy()
    Rtot = np.eye(c)
    for st in range(maxst):
        G = Q.T @ Q
        tr = np.trace(G)
        E = G - np.eye(c)
        e = np.abs(E).max()
        if not np.isfinite(tr) or tr <= 0:
            return None
        if st >= 1 and e <= tau:
            return Q, Rtot, st + 1
        if st >= 1 and e <= first:
            R = np.eye(c) + np.triu(E, 1) + np.diag(np.diag(E)) / 2
        elif st == maxst - 1:
            return None
        else:
            ok, R, ratio = _chol(G, 0.0)
            if not ok or ratio < 1e-12:
                ok, R, _ = _chol(G, 11 * (m * c + c * (c + 1)) * U * tr)
            if not ok:
                return None
        Q = solve_triangular(R, Q.T, trans="T", lower=False).T
        Rtot = R @ Rtot
        if st >= 1 and e <= first_done:
            return Q, Rtot, st + 1
    return None


def _matrix(rng, m, c, kappa):
    X, _ = np.linalg.qr(rng.standard_normal((m, c)))
    Y, _ = np.linalg.qr(rng.standard_normal((c, c)))
    return (X * np.logspace(0, -np.log10(kappa), c)) @ Y.T


@pytest.mark.parametrize("m,c", [(7000, 28), (3072, 16), (640, 24), (16384, 64)])
@pytest.mark.parametrize("kappa", [1e1, 1e6, 1e8, 1e12, 1e20])
def test_sequence_converges_and_is_accurate(m, c, kappa):
    rng = np.random.default_rng(int(np.log10(kappa)) * 100 + c)
    A = _matrix(rng, m, c, kappa)
    out = cholqr_sequence(A)
    assert out is not None
    Q, R, stages = out
    assert stages <= 7
    assert np.abs(Q.T @ Q - np.eye(c)).max() <= 1e-13
    assert np.linalg.norm(A - Q @ R) <= 1e-15 * np.linalg.norm(A) * 8
    sa = np.linalg.svd(A, compute_uv=False)
    sr = np.linalg.svd(R, compute_uv=False)
    assert np.abs(sa - sr).max() <= 1e-14 * sa[0]


def test_repeated_columns():
    rng = np.random.default_rng(7)
    B = _matrix(rng, 2048, 10, 1e3)
    A = np.hstack([B, 0.5 * B])
    Q, R, stages = cholqr_sequence(A)
    assert stages <= 7
    assert np.abs(Q.T @ Q - np.eye(A.shape[1])).max() <= 1e-13
    assert np.linalg.norm(A - Q @ R) <= 1e-14 * np.linalg.norm(A)


def test_zero_columns_fall_back():
    """An exactly zero column stays zero under every stage, so the sequence
    cannot make Q orthonormal; the kernel then leaves the bond to the
    Householder TSQR."""
    rng = np.random.default_rng(8)
    A = np.hstack([_matrix(rng, 2048, 10, 1e3), np.zeros((2048, 4))])
    assert cholqr_sequence(A) is None
