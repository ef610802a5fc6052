"""CPU oracle for the paratt tensor-train hot path -- TEST INFRASTRUCTURE ONLY.

A numpy restatement of the reference algorithms, used by ``tests/`` and by
``bench.py``'s CPU-baseline leg as the checker.  The product (``paratt_b200``,
``libparatt_b200.so``) never imports this module.  It is pinned against the
reference itself: ``oracle/_ref/libparatt_ref.so`` is the reference's own C
compiled by ``oracle/Makefile``, and ``tests/test_oracle_vs_ref.py`` plus the
golden fixtures under ``tests/golden/`` check every function here against it.

Layout (source/paratt.h:36-42): core k is a numpy array of shape
(r_k, n_k, r_{k+1}); its Fortran-order ravel is the reference buffer, element
(i, j, l) at ``i + r_k*(j + n_k*l)``.
"""
from __future__ import annotations

import math

import numpy as np

EPS = np.finfo(np.float64).eps / 2  # LAPACK DLAMCH('E'): unit roundoff


# --------------------------------------------------------------------------
# helpers
# --------------------------------------------------------------------------
def ranks_of(cores):
    return [cores[0].shape[0]] + [c.shape[2] for c in cores]


def dims_of(cores):
    return [c.shape[1] for c in cores]


def left_unfold(c):
    r, n, r1 = c.shape
    return c.reshape(r * n, r1, order="F")


def right_unfold(c):
    r, n, r1 = c.shape
    return c.reshape(r, n * r1, order="F")


def full(cores):
    """Dense tensor (tiny cases only), index order (i_0, ..., i_{d-1})."""
    t = cores[0].reshape(cores[0].shape[1], cores[0].shape[2], order="F")
    for c in cores[1:]:
        r, n, r1 = c.shape
        t = np.tensordot(t, c, axes=([t.ndim - 1], [0]))
    return t.reshape(t.shape[:-1])


# --------------------------------------------------------------------------
# rank rule and numerical rank
# --------------------------------------------------------------------------
def svdq_numrank(L):
    """Numerical rank that LAPACK dgesvdq with JOBA='A' keeps (called from
    pattac.c:431-452): column-pivoted QR of L, then the leading diagonal run
    with |R_pp| >= sqrt(N)*eps*|R_11| (N = number of columns)."""
    import scipy.linalg as sl

    m, n = L.shape
    if n == 0:
        return 0
    R = sl.qr(L, mode="r", pivoting=True)[0]
    dg = np.abs(np.diag(R))
    thr = math.sqrt(n) * EPS * dg[0]
    nr = 1
    for p in range(1, min(m, n)):
        if dg[p] < thr:
            break
        nr += 1
    return nr


def rank_rule(sig, nsv, q, maxr, delta):
    """Tail-sum truncation rule, pattac.c:468-481: walk singular values from
    the smallest, drop while sqrt(tail sum of squares) < delta, then cap by q
    and maxr and floor at 1."""
    s = 0.0
    rank = nsv
    for j in range(nsv - 1, -1, -1):
        s += sig[j] * sig[j]
        if math.sqrt(s) < delta:
            rank = j
        else:
            break
    rank = min(rank, q)
    rank = min(rank, maxr)
    return max(rank, 1)


# --------------------------------------------------------------------------
# TT rounding (paratt_truncate -> pattacTruncate, ortho 'R', one rank)
# --------------------------------------------------------------------------
def left_orthogonalize(cores):
    """pattacLOrthogonalization (pattac.c:244-294) with one rank: QR of each
    left unfolding (tsqr_factorize, tsqr.c:541-714), R pushed into the next
    core (trapezoid_mult, utilities.c:233-308), Q kept (tsqr_make_q).
    Ranks become r_{i+1} <- min(r_i n_i, r_{i+1})."""
    x = [c.copy() for c in cores]
    d = len(x)
    for i in range(d - 1):
        r, n, r1 = x[i].shape
        Q, R = np.linalg.qr(left_unfold(x[i]), mode="reduced")
        q = Q.shape[1]
        x[i] = Q.reshape(r, n, q, order="F")
        nr1, n2, r2 = x[i + 1].shape
        x[i + 1] = (R @ right_unfold(x[i + 1])).reshape(q, n2, r2, order="F")
    return x


def truncate_sweep(x, delta, maxr, info=None):
    """pattacLTruncate (pattac.c:297-522) with one rank: for i = d-1..1, LQ of
    the right unfolding (wflq_factorize), SVD of L (dgesvdq), rank rule,
    x_i <- V_r^T Q, x_{i-1} <- x_{i-1} U_r S_r."""
    d = len(x)
    for i in range(d - 1, 0, -1):
        r, n, r1 = x[i].shape
        Cm = right_unfold(x[i])
        Qt, Rt = np.linalg.qr(Cm.T, mode="reduced")  # Cm = Rt^T Qt^T
        L = Rt.T  # r x q
        q = L.shape[1]
        U, s, Vt = np.linalg.svd(L, full_matrices=False)
        nsv = min(svdq_numrank(L), len(s))
        rank = rank_rule(s, nsv, q, maxr[i], delta)
        if info is not None:
            info.append({"bond": i, "sigma": s.copy(), "rank": rank, "nsv": nsv})
        x[i] = (Vt[:rank] @ Qt.T).reshape(rank, n, r1, order="F")
        rp, npv, _ = x[i - 1].shape
        x[i - 1] = (left_unfold(x[i - 1]) @ (U[:, :rank] * s[:rank])).reshape(
            rp, npv, rank, order="F")
    return x


def round_tt(cores, tol, maxrank, info=None):
    """paratt_truncate(x, tol, maxRank) (paratt.c:316-342 -> pattac.c:590-675).

    ``tol`` is ABSOLUTE on the grid-normalised (RMS) norm: every core is divided
    by sqrt(n_k) first (pattac.c:608-616) and the per-bond threshold is
    tol/sqrt(d-1) (pattac.c:315); cores are multiplied back afterwards
    (pattac.c:665-673).  ``maxrank`` is an int or a per-bond list of d+1."""
    d = len(cores)
    if not hasattr(maxrank, "__len__"):
        maxrank = [maxrank] * (d + 1)
    x = [c / math.sqrt(c.shape[1]) for c in cores]
    x = left_orthogonalize(x)
    delta = tol / math.sqrt(d - 1.0) if d > 1 else math.inf
    x = truncate_sweep(x, delta, maxrank, info)
    return [c * math.sqrt(c.shape[1]) for c in x]


# --------------------------------------------------------------------------
# formal arithmetic
# --------------------------------------------------------------------------
def axpby(a, x, b, y):
    """attac_tt_axpby (paratt.c:237-268) -> attacFormalAXPBY (attac.c:81-112):
    ranks add; a and b scale core 0 only; interior cores block-diagonal; the
    last core stacks x over y.  Requires d >= 2."""
    d = len(x)
    z = []
    for k in range(d):
        rx, n, rx1 = x[k].shape
        ry, _, ry1 = y[k].shape
        if k == 0:
            c = np.concatenate([a * x[0], b * y[0]], axis=2)
        elif k == d - 1:
            c = np.concatenate([x[k], y[k]], axis=0)
        else:
            c = np.zeros((rx + ry, n, rx1 + ry1))
            c[:rx, :, :rx1] = x[k]
            c[rx:, :, rx1:] = y[k]
        z.append(c)
    return z


def hadamard(x, y):
    """attacHadamard (attac.c:128-136) with attacKron (utilities.c:112-129):
    z_k[:, j, :] = kron(x_k[:, j, :], y_k[:, j, :]), row index k_y + r_y*i_x."""
    z = []
    for xc, yc in zip(x, y):
        rx, n, rx1 = xc.shape
        ry, _, ry1 = yc.shape
        c = np.einsum("ajb,cjd->acjbd", xc, yc).reshape(rx, ry, n, rx1, ry1)
        # row (a, c) -> c + ry*a ; col (b, d) -> d + ry1*b
        c = c.transpose(1, 0, 2, 4, 3).reshape(ry * rx, n, ry1 * rx1, order="F")
        z.append(c)
    return z


def scale(a, x):
    """attac_tt_scale (paratt.c:271-281): core 0 times a."""
    return [a * x[0]] + [c.copy() for c in x[1:]]


def mult_diag(x, mode, vec):
    """attac_mult_diag_mat (paratt.c:571-581): core[mode][:, j, :] *= vec[j]."""
    out = [c.copy() for c in x]
    out[mode] = out[mode] * np.asarray(vec)[None, :, None]
    return out


def periodic_stencil_core(core, sten):
    """Centred periodic stencil along the mode index of one core:
    out[i, a, l] = sum_t s_t f[i, (a + t - h) mod n, l], h = (s-1)/2, with an
    even length decremented first (paratt.c:586, 680).  This is what
    attac_apply_periodic_stencil (paratt.c:584-661) computes for every length
    and what pattac_apply_periodic_stencil (paratt.c:665-770) computes for
    3-point stencils; for h >= 2 the latter reads the wrong wrap-around ghost
    row at 0 < a < h (its ghost counter starts at the first negative index)."""
    s = len(sten)
    if s % 2 == 0:
        s -= 1
    h = (s - 1) // 2
    out = np.zeros_like(core)
    for t in range(s):
        out += sten[t] * np.roll(core, h - t, axis=1)
    return out


def periodic_stencil(x, mode, sten):
    out = [c.copy() for c in x]
    out[mode] = periodic_stencil_core(x[mode], sten)
    return out


# --------------------------------------------------------------------------
# contractions
# --------------------------------------------------------------------------
def inner_raw(x, y):
    """Unnormalised <X, Y> by transfer matrices (pattacInnerProduct logic,
    pattac.c:693-741)."""
    a = np.ones((1, 1))
    for xc, yc in zip(x, y):
        # a: rx x ry ; new a[b, d] = sum a[i, k] x[i, j, b] y[k, j, d]
        t = np.einsum("ik,kjd->ijd", a, yc)
        a = np.einsum("ijb,ijd->bd", xc, t)
    return float(a[0, 0])


def dot(x, y):
    """paratt_dotprod (paratt.c:412-469): <X, Y> / prod(n)."""
    p = 1.0
    for c in x:
        p *= c.shape[1]
    return inner_raw(x, y) / p


def norm(x):
    """paratt_norm (paratt.c:369-409): ||X||_F / sqrt(prod n)."""
    return math.sqrt(max(dot(x, x), 0.0))


def entry(x, idx):
    """paratt_entry (paratt.c:471-499 -> pattacValue, pattac.c:82-121)."""
    v = np.ones((1,))
    for c, j in zip(x, idx):
        v = v @ c[:, j, :]
    return float(v[0])


def rel_diff(x, y):
    """Gauge-free ||X - Y|| / ||Y|| through inner products."""
    xx = inner_raw(x, x)
    yy = inner_raw(y, y)
    xy = inner_raw(x, y)
    num = max(xx + yy - 2.0 * xy, 0.0)
    return math.sqrt(num) / math.sqrt(yy) if yy > 0 else math.sqrt(num)


def rel_diff_exact(x, y):
    """Same as rel_diff but with the difference formed as a TT (x - y) and
    left-orthogonalised, so it does not lose digits to cancellation."""
    dz = axpby(1.0, x, -1.0, y) if len(x) > 1 else [x[0] - y[0]]
    dz = left_orthogonalize(dz)
    yy = left_orthogonalize(y)
    return float(np.linalg.norm(dz[-1]) / max(np.linalg.norm(yy[-1]), 1e-300))


# --------------------------------------------------------------------------
# seeded synthetic inputs
# --------------------------------------------------------------------------
def random_tt(dims, ranks, seed, std=1.0):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((ranks[k], dims[k], ranks[k + 1])) * std
            for k in range(len(dims))]


# --------------------------------------------------------------------------
# reaction-Burgers step-truncation RK2 (composition of the primitives above)
# --------------------------------------------------------------------------
def op_sum_apply(x, stens, shift=0.0):
    """Y = sum_i S_i x + shift * x, S_i = periodic stencil stens[i] on mode i.

    Exact rank-2r TT of the sum of d mode-local operators (the formal sum of
    the d stencil applications of attac_apply_periodic_stencil, paratt.c:584,
    has rank d*r and represents the same tensor).  Core k has 2x2 blocks
    indexed by (applied-before-k, applied-up-to-k): [[x_k, S_k x_k], [0, x_k]];
    the first core keeps block row 0, the last keeps block column 1, and the
    shift is added to the block S_0 x_0.  For d == 1 it is (S_0 + shift) x_0."""
    d = len(x)
    if d == 1:
        return [periodic_stencil_core(x[0], stens[0]) + shift * x[0]]
    out = []
    for k in range(d):
        r, n, r1 = x[k].shape
        sx = periodic_stencil_core(x[k], stens[k])
        if k == 0:
            out.append(np.concatenate([x[0], sx + shift * x[0]], axis=2))
        elif k == d - 1:
            out.append(np.concatenate([sx, x[k]], axis=0))
        else:
            c = np.zeros((2 * r, n, 2 * r1))
            c[:r, :, :r1] = x[k]
            c[:r, :, r1:] = sx
            c[r:, :, r1:] = x[k]
            out.append(c)
    return out


def burgers_stencils(d, n, L=10.0, nu=0.05):
    """Second-order central differences on the periodic grid x_j = -L/2 + j h,
    h = L/n: nu*[1,-2,1]/h^2 (diffusion) and -(1/d)*[-1,0,1]/(2h) applied to
    u^2/2 (Burgers flux), i.e. -(1/(2d))*[-1,0,1]/(2h) applied to u*u."""
    h = L / n
    d2 = [nu / h**2, -2.0 * nu / h**2, nu / h**2]
    d1 = [1.0 / (4.0 * d * h), 0.0, -1.0 / (4.0 * d * h)]
    return d2, d1


def rxn_burgers_F(u, tol, maxr, L=10.0, nu=0.05):
    """F(u) = nu sum_i D2_i u - (1/d) sum_i D1_i (u^2/2) + u - u^2, every
    intermediate rounded with paratt_truncate semantics (absolute tol):
      w = T(u . u);  a = T(nu sum D2 u + u);  b = T(-(1/2d) sum D1 w - w)
      F = T(a + b)"""
    d = len(u)
    n = u[0].shape[1]
    d2, d1 = burgers_stencils(d, n, L, nu)
    w = round_tt(hadamard(u, u), tol, maxr)
    a = round_tt(op_sum_apply(u, [d2] * d, 1.0), tol, maxr)
    b = round_tt(op_sum_apply(w, [d1] * d, -1.0), tol, maxr)
    return round_tt(axpby(1.0, a, 1.0, b), tol, maxr)


def rxn_burgers_rk2_step(u, dt, tol, maxr, L=10.0, nu=0.05):
    """Step-truncation explicit midpoint (paratt_ode.h:77-112) with the stage
    rounded too: f_s = T(u + dt/2 F(u)); u+ = T(u + dt F(f_s))."""
    k1 = rxn_burgers_F(u, tol, maxr, L, nu)
    us = round_tt(axpby(1.0, u, 0.5 * dt, k1), tol, maxr)
    k2 = rxn_burgers_F(us, tol, maxr, L, nu)
    return round_tt(axpby(1.0, u, dt, k2), tol, maxr)


def grid(n, L=10.0):
    return -L / 2 + np.arange(n) * (L / n)


def gaussian_sum_ic(d, n, centres, widths, L=10.0):
    """sum_g prod_i exp(-(x_i - c_gi)^2 / (2 w_g^2)) as a rank-G TT
    (attac_sum_of_product layout: core 0 = [v_0 | v_1 | ...], diagonal
    interior cores, stacked last core; paratt.c:517-568)."""
    x = grid(n, L)
    G = len(widths)
    cores = []
    for k in range(d):
        vecs = [np.exp(-(x - centres[g][k]) ** 2 / (2 * widths[g] ** 2)) for g in range(G)]
        if G == 1:
            cores.append(vecs[0].reshape(1, n, 1))
        elif k == 0:
            cores.append(np.stack(vecs, axis=1).reshape(1, n, G))
        elif k == d - 1:
            cores.append(np.stack(vecs, axis=0).reshape(G, n, 1))
        else:
            c = np.zeros((G, n, G))
            for g in range(G):
                c[g, :, g] = vecs[g]
            cores.append(c)
    return cores


def config_ic(d, n, ngauss, seed, L=10.0):
    """Seeded sum of Gaussians: centres U[-2,2]^d, widths U[0.3,0.8]."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-2.0, 2.0, size=(ngauss, d))
    widths = rng.uniform(0.3, 0.8, size=ngauss)
    return gaussian_sum_ic(d, n, centres, widths, L)


# --------------------------------------------------------------------------
# CDF-problem stencils and marginals (one process: the reference's ghost
# cells are rows of the same core).  Each works on the fibers core[i, :, k]
# of one mode.
# --------------------------------------------------------------------------
def _fibers(core):
    """(r, n, r1) -> (r * r1 fibers, n) view order and back."""
    r, n, r1 = core.shape
    return core.transpose(0, 2, 1).reshape(r * r1, n)


def _unfibers(f, shape):
    r, n, r1 = shape
    return f.reshape(r, r1, n).transpose(0, 2, 1).copy()


def cdf_stencil(x, mode, sten):
    """pattac_apply_cdf_stencil (paratt.c:772-923) with one process.  An even
    length drops its last tap; h = (s - 1) / 2.  Outside the grid the
    reference reads ghost rows: for j < 0 the value it uses at output a is
    f[a - j - 1] (its above-ghost counter restarts at every a, paratt.c:
    896-903, with the ghost rows f[h - 1 - g] set at 836-842), for j >= n it
    is f[2n - 1 - j] (the mirrored last rows, 866-872)."""
    s = len(sten)
    if s % 2 == 0:
        s -= 1
    h = (s - 1) // 2
    out = [c.copy() for c in x]
    f = _fibers(x[mode])
    n = f.shape[1]
    g = np.zeros_like(f)
    for a in range(n):
        acc = np.zeros(f.shape[0])
        for t in range(s):
            j = a - h + t
            if j < 0:
                v = f[:, a - j - 1]
            elif j >= n:
                v = f[:, 2 * n - 1 - j]
            else:
                v = f[:, j]
            acc = acc + sten[t] * v
        g[:, a] = acc
    out[mode] = _unfibers(g, x[mode].shape)
    return out


def cdf_lf_flux(x, mode, wave_speed, gc_wave_speed, source_coef, dt, dx):
    """pattac_apply_cdf_lf_flux (paratt.c:926-1093) with one process: the
    centred difference [-1/(2dx), 0, 1/(2dx)] of -w f, with the ghost
    neighbours -gc_w[0] f[0] below the grid and -gc_w[1] f[n-1] above it
    (1043-1082), plus source_coef * f (1083-1090).  dt is not used by the
    reference."""
    out = [c.copy() for c in x]
    f = _fibers(x[mode])
    n = f.shape[1]
    w = np.asarray(wave_speed, dtype=float)
    s0, s2 = -0.5 / dx, 0.5 / dx
    g = np.zeros_like(f)
    for a in range(n):
        left = -gc_wave_speed[0] * f[:, 0] if a - 1 < 0 else -w[a - 1] * f[:, a - 1]
        right = -gc_wave_speed[1] * f[:, n - 1] if a + 1 >= n else -w[a + 1] * f[:, a + 1]
        acc = np.zeros(f.shape[0])
        acc = acc + s0 * left
        acc = acc + s2 * right
        g[:, a] = acc + source_coef[a] * f[:, a]
    out[mode] = _unfibers(g, x[mode].shape)
    return out


def cdf_lw_rhs(x, mode, wave_speed, gc_wave_speed, bdry_wave_speed, source_coef, dt, dx):
    """pattac_apply_cdf_lw_rhs (paratt.c:1096-1250) with one process:
    Lax-Wendroff half-step values u_{a+1/2} (ghosts f[0] below, f[n-1]
    above, 1207-1230), then -(b_{a+1} u_{a+1/2} - b_a u_{a-1/2}) / dx +
    source_coef_a f_a (1231-1235)."""
    out = [c.copy() for c in x]
    f = _fibers(x[mode])
    n = f.shape[1]
    w = np.asarray(wave_speed, dtype=float)
    b = np.asarray(bdry_wave_speed, dtype=float)
    k = dt / (2.0 * dx)
    g = np.zeros_like(f)
    gca, gcb = f[:, 0], f[:, n - 1]
    uh0 = 0.5 * (gca + f[:, 0]) - (w[0] * f[:, 0] - gca * gc_wave_speed[0]) * k
    for a in range(n):
        if a + 1 < n:
            uh1 = 0.5 * (f[:, a + 1] + f[:, a]) - (w[a + 1] * f[:, a + 1] - w[a] * f[:, a]) * k
        else:
            uh1 = 0.5 * (gcb + f[:, a]) - (gcb * gc_wave_speed[1] - w[a] * f[:, a]) * k
        g[:, a] = -(b[a + 1] * uh1 - b[a] * uh0) / dx + source_coef[a] * f[:, a]
        uh0 = uh1
    out[mode] = _unfibers(g, x[mode].shape)
    return out


def marginal_cusum(x, mode, w):
    """pattac_marginal_cusum (paratt.c:1393-1445) with one process:
    f[j] <- sum_{m <= j} w[m] f[m] along the mode."""
    out = [c.copy() for c in x]
    f = _fibers(x[mode]) * np.asarray(w, dtype=float)[None, :]
    out[mode] = _unfibers(np.cumsum(f, axis=1), x[mode].shape)
    return out


def marginal_trap(x, mode, w):
    """pattac_marginal_trap (paratt.c:1448-1524) with one process: the
    trapezoid cumulative integral f[j] <- sum_{m=1..j} w[m] (f[m-1] + f[m]) / 2
    (f[0] <- 0)."""
    out = [c.copy() for c in x]
    f = _fibers(x[mode])
    n = f.shape[1]
    g = np.zeros_like(f)
    cum = np.zeros(f.shape[0])
    for j in range(1, n):
        delta = 0.5 * w[j] * (f[:, j - 1] + f[:, j])
        g[:, j - 1] = cum
        cum = cum + delta
    g[:, n - 1] = cum
    out[mode] = _unfibers(g, x[mode].shape)
    return out


def scale_weight_sum(x, mode, scale, sum_w):
    """pattac_scale_weight_sum (paratt.c:1527-1618) with one process: the
    trapezoid cumulative integral with weights sum_w plus scale[j] f[j]."""
    f = _fibers(x[mode])
    t = _fibers(marginal_trap(x, mode, sum_w)[mode])
    out = [c.copy() for c in x]
    out[mode] = _unfibers(t + f * np.asarray(scale, dtype=float)[None, :], x[mode].shape)
    return out


def apply_marginal(x, mode, w):
    """pattac_apply_marginal (paratt.c:1252-1390) with one process: contract
    mode `mode` with the row vector w; the d-1 mode train folds W = sum_j
    w[j] x_mode[:, j, :] into the next core (mode < d-1, 1342-1350) or the
    previous one (mode = d-1, 1366-1373)."""
    d = len(x)
    W = np.einsum("j,ajb->ab", np.asarray(w, dtype=float), x[mode])
    if mode < d - 1:
        nxt = x[mode + 1]
        folded = np.einsum("ab,bjc->ajc", W, nxt)
        return [c.copy() for c in x[:mode]] + [folded] + [c.copy() for c in x[mode + 2:]]
    prev = x[mode - 1]
    folded = np.einsum("ajb,b->aj", prev, W[:, 0]).reshape(prev.shape[0], prev.shape[1], 1)
    return [c.copy() for c in x[:mode - 1]] + [folded]
