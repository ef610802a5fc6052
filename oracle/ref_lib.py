"""ctypes binding to the reference paratt library built by ``oracle/Makefile``.

TEST INFRASTRUCTURE ONLY.  ``oracle/_ref/libparatt_ref.so`` is the reference's
own C (source/paratt.c, source/paratt_ode.c, mpi_attac/pattac.c,
mpi_attac/tsqr.c, serial_attac/attac.c, serial_attac/utilities.c) compiled
unmodified against a single-process ``mpi.h`` and an LP64 OpenBLAS.  It is used
to pin the numpy restatement in ``tt_oracle.py`` and as the timed CPU baseline;
no product code path imports this module.

Struct layouts mirror source/paratt.h:25-63 (``attac_tt`` and ``paratt``).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(_HERE, "_ref", "libparatt_ref.so")


class AttacTT(C.Structure):
    # source/paratt.h:25-54
    _fields_ = [
        ("numDim", C.c_int),
        ("dim", C.POINTER(C.c_int)),
        ("ttRank", C.POINTER(C.c_int)),
        ("coreList", C.POINTER(C.POINTER(C.c_double))),
        ("coreMem", C.POINTER(C.c_int)),
        ("wk", C.POINTER(C.c_double)),
        ("wksz", C.c_int),
    ]


class Paratt(C.Structure):
    # source/paratt.h:56-65
    _fields_ = [
        ("x", C.POINTER(AttacTT)),
        ("mpi_rk", C.c_int),
        ("mpi_sz", C.c_int),
        ("distrib_dim_mat", C.POINTER(C.c_int)),
        ("dim", C.POINTER(C.c_int)),
        ("numDim", C.c_int),
        ("iwk", C.POINTER(C.c_int)),
        ("iwksz", C.c_int),
        ("orthog_wk", C.c_void_p),
    ]


_lib = None


def available() -> bool:
    return os.path.exists(REF_SO)


def lib():
    """Load the reference library (RTLD_LOCAL so its symbols never shadow the
    product library's identically named exports)."""
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(
                f"{REF_SO} missing: run `make -C oracle` (needs the reference sources)")
        L = C.CDLL(REF_SO, mode=os.RTLD_LOCAL)
        P = C.POINTER(Paratt)
        T = C.POINTER(AttacTT)
        ip = C.POINTER(C.c_int)
        dp = C.POINTER(C.c_double)
        L.alloc_ptt.restype = P
        L.alloc_ptt.argtypes = [C.c_int, ip, ip]
        L.free_ptt.argtypes = [P]
        L.paratt_truncate.argtypes = [P, C.c_double, ip]
        L.attac_tt_axpby.argtypes = [C.c_double, T, C.c_double, T, T]
        L.attac_tt_scale.argtypes = [C.c_double, T]
        L.paratt_norm.restype = C.c_double
        L.paratt_norm.argtypes = [P]
        L.paratt_dotprod.restype = C.c_double
        L.paratt_dotprod.argtypes = [P, P]
        L.paratt_entry.restype = C.c_double
        L.paratt_entry.argtypes = [P, ip]
        L.pattac_apply_periodic_stencil.argtypes = [P, C.c_int, dp, C.c_int]
        L.attac_apply_periodic_stencil.argtypes = [T, C.c_int, dp, C.c_int]
        L.attac_mult_diag_mat.argtypes = [T, C.c_int, dp]
        L.pattacHadamard.argtypes = [C.c_int, ip, ip, C.POINTER(dp), ip,
                                     C.POINTER(dp), ip, C.POINTER(dp)]
        L.rank_change_tt.restype = T
        L.rank_change_tt.argtypes = [T, ip]
        L.pattac_write_tt_folder.argtypes = [C.c_char_p, P]
        L.pattac_load_tt_folder.restype = P
        L.pattac_load_tt_folder.argtypes = [C.c_char_p, C.c_int]
        _lib = L
    return _lib


def _iarr(v):
    return (C.c_int * len(v))(*[int(t) for t in v])


class RefTT:
    """A ``paratt`` owned by the reference library, filled from numpy cores.

    Cores are numpy arrays of shape (r_k, n_k, r_{k+1}); the flat buffer is
    their Fortran-order ravel, which is the reference layout
    ``i + r_k*(j + n_k*l)`` (source/paratt.h:36-42)."""

    def __init__(self, cores=None, dims=None, ranks=None, ptr=None):
        L = lib()
        if ptr is not None:
            self.p = ptr
            return
        if cores is not None:
            dims = [c.shape[1] for c in cores]
            ranks = [cores[0].shape[0]] + [c.shape[2] for c in cores]
        d = len(dims)
        self.p = L.alloc_ptt(d, _iarr(dims), _iarr(ranks))
        if cores is not None:
            self.set_cores(cores)

    @property
    def d(self):
        return self.p.contents.numDim

    def ranks(self):
        x = self.p.contents.x.contents
        return [x.ttRank[k] for k in range(self.d + 1)]

    def dims(self):
        x = self.p.contents.x.contents
        return [x.dim[k] for k in range(self.d)]

    def set_cores(self, cores):
        L = lib()
        x = self.p.contents.x
        rk = [cores[0].shape[0]] + [c.shape[2] for c in cores]
        L.rank_change_tt(x, _iarr(rk))
        xc = x.contents
        for k, c in enumerate(cores):
            flat = np.ascontiguousarray(c.ravel(order="F"), dtype=np.float64)
            C.memmove(xc.coreList[k], flat.ctypes.data, flat.nbytes)

    def cores(self):
        xc = self.p.contents.x.contents
        r = self.ranks()
        n = self.dims()
        out = []
        for k in range(self.d):
            cnt = r[k] * n[k] * r[k + 1]
            buf = np.ctypeslib.as_array(xc.coreList[k], shape=(cnt,)).copy()
            out.append(buf.reshape((r[k], n[k], r[k + 1]), order="F"))
        return out

    def free(self):
        if self.p:
            lib().free_ptt(self.p)
            self.p = None


def ref_truncate(cores, tol, maxrank):
    """Round with the reference's ``paratt_truncate`` (paratt.c:316-342)."""
    t = RefTT(cores)
    try:
        mr = maxrank if hasattr(maxrank, "__len__") else [maxrank] * (len(cores) + 1)
        mr = _iarr(mr)
        lib().paratt_truncate(t.p, C.c_double(tol), mr)
        return t.cores()
    finally:
        t.free()


def ref_axpby(a, xc, b, yc):
    """``attac_tt_axpby`` (paratt.c:237-268)."""
    x, y = RefTT(xc), RefTT(yc)
    z = RefTT(dims=x.dims(), ranks=[1] * (x.d + 1))
    try:
        lib().attac_tt_axpby(a, x.p.contents.x, b, y.p.contents.x, z.p.contents.x)
        return z.cores()
    finally:
        x.free(); y.free(); z.free()


def ref_hadamard(xc, yc):
    """``pattacHadamard`` (pattac.c:175-177 -> attac.c:128-136) into a target
    allocated at ranks r_x*r_y (the caller's job in the reference)."""
    x, y = RefTT(xc), RefTT(yc)
    rx, ry = x.ranks(), y.ranks()
    rz = [a * b for a, b in zip(rx, ry)]
    z = RefTT(dims=x.dims(), ranks=rz)
    try:
        d = x.d
        xs, ys, zs = x.p.contents.x.contents, y.p.contents.x.contents, z.p.contents.x.contents
        lib().pattacHadamard(d, xs.dim, xs.ttRank, xs.coreList, ys.ttRank,
                             ys.coreList, zs.ttRank, zs.coreList)
        return z.cores()
    finally:
        x.free(); y.free(); z.free()


def ref_stencil(cores, mode, sten):
    """``pattac_apply_periodic_stencil`` (paratt.c:665-770)."""
    t = RefTT(cores)
    try:
        s = np.ascontiguousarray(sten, dtype=np.float64)
        lib().pattac_apply_periodic_stencil(
            t.p, mode, s.ctypes.data_as(C.POINTER(C.c_double)), len(s))
        return t.cores()
    finally:
        t.free()


def ref_norm(cores):
    """``paratt_norm`` (paratt.c:369-409): RMS norm ||X||_F / sqrt(prod n)."""
    t = RefTT(cores)
    try:
        return lib().paratt_norm(t.p)
    finally:
        t.free()


def ref_dot(xc, yc):
    """``paratt_dotprod`` (paratt.c:412-469): <X, Y> / prod n."""
    x, y = RefTT(xc), RefTT(yc)
    try:
        return lib().paratt_dotprod(x.p, y.p)
    finally:
        x.free(); y.free()


def ref_entry(cores, idx):
    t = RefTT(cores)
    try:
        return lib().paratt_entry(t.p, _iarr(idx))
    finally:
        t.free()


def ref_rxn_burgers_F(u, tol, maxr, L=10.0, nu=0.05):
    """F(u) of the reaction-Burgers step composed from the reference's own C
    routines in the order of ``tt_oracle.rxn_burgers_F``: paratt_truncate
    after every intermediate, the product u.u by pattacHadamard (rank r^2),
    the sum by attac_tt_axpby.  The operator sums sum_i S_i x + shift x are
    the rank-2r trains of ``tt_oracle.op_sum_apply`` (the reference has no
    such operator)."""
    from oracle import tt_oracle as O

    d, n = len(u), u[0].shape[1]
    d2, d1 = O.burgers_stencils(d, n, L, nu)
    w = ref_truncate(ref_hadamard(u, u), tol, maxr)
    a = ref_truncate(O.op_sum_apply(u, [d2] * d, 1.0), tol, maxr)
    b = ref_truncate(O.op_sum_apply(w, [d1] * d, -1.0), tol, maxr)
    return ref_truncate(ref_axpby(1.0, a, 1.0, b), tol, maxr)


def ref_rxn_burgers_rk2_step(u, dt, tol, maxr, L=10.0, nu=0.05):
    """Step-truncation midpoint step (paratt_ode.h:77-112, stage rounded) on
    the reference routines, as ``tt_oracle.rxn_burgers_rk2_step``."""
    k1 = ref_rxn_burgers_F(u, tol, maxr, L, nu)
    us = ref_truncate(ref_axpby(1.0, u, 0.5 * dt, k1), tol, maxr)
    k2 = ref_rxn_burgers_F(us, tol, maxr, L, nu)
    return ref_truncate(ref_axpby(1.0, u, dt, k2), tol, maxr)


# CDF-problem stencils and marginals (paratt.c:772-1618), one process
def _dp(v):
    a = np.ascontiguousarray(v, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


def _bind_cdf():
    L = lib()
    P = C.POINTER(Paratt)
    dp = C.POINTER(C.c_double)
    L.pattac_apply_cdf_stencil.argtypes = [P, C.c_int, dp, C.c_int]
    L.pattac_apply_cdf_lf_flux.argtypes = [P, C.c_int, dp, dp, dp, C.c_double, C.c_double]
    L.pattac_apply_cdf_lw_rhs.argtypes = [P, C.c_int, dp, dp, dp, dp, C.c_double, C.c_double]
    L.pattac_apply_marginal.argtypes = [P, C.POINTER(P), C.c_int, dp]
    L.pattac_marginal_cusum.argtypes = [P, C.c_int, dp]
    L.pattac_marginal_trap.argtypes = [P, C.c_int, dp]
    L.pattac_scale_weight_sum.argtypes = [P, C.c_int, dp, dp]
    return L


def ref_cdf_op(name, cores, mode, *vecs, scalars=()):
    """Run one of the in-place CDF/marginal routines on a copy of `cores`:
    name in cdf_stencil, cdf_lf_flux, cdf_lw_rhs, marginal_cusum,
    marginal_trap, scale_weight_sum; vecs are the double arrays in the
    reference's argument order, scalars the trailing doubles (dt, dx)."""
    L = _bind_cdf()
    t = RefTT(cores)
    keep = [_dp(v) for v in vecs]
    args = [k[1] for k in keep]
    try:
        if name == "cdf_stencil":
            L.pattac_apply_cdf_stencil(t.p, mode, args[0], len(keep[0][0]))
        elif name == "cdf_lf_flux":
            L.pattac_apply_cdf_lf_flux(t.p, mode, *args, *scalars)
        elif name == "cdf_lw_rhs":
            L.pattac_apply_cdf_lw_rhs(t.p, mode, *args, *scalars)
        elif name == "marginal_cusum":
            L.pattac_marginal_cusum(t.p, mode, args[0])
        elif name == "marginal_trap":
            L.pattac_marginal_trap(t.p, mode, args[0])
        elif name == "scale_weight_sum":
            L.pattac_scale_weight_sum(t.p, mode, args[0], args[1])
        else:
            raise ValueError(name)
        return t.cores()
    finally:
        t.free()


def ref_apply_marginal(cores, mode, w):
    """pattac_apply_marginal (paratt.c:1252-1390): the d-1 mode train."""
    L = _bind_cdf()
    t = RefTT(cores)
    a, p = _dp(w)
    out = C.POINTER(Paratt)()
    try:
        L.pattac_apply_marginal(t.p, C.byref(out), mode, p)
        m = RefTT(ptr=out)
        res = m.cores()
        m.free()
        return res
    finally:
        t.free()
