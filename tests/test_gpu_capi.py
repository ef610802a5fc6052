"""The reference-signature C API of libparatt_b200.so (include/paratt.h,
include/paratt_ode.h) on the GPU, called the way a driver written against the
reference calls it: host cores in library-owned `paratt` structs, every call
uploading to the HBM mirror of its arguments and downloading what it wrote.
Each call is compared with the same call into the reference's own compiled C
(oracle/_ref/libparatt_ref.so) on identical inputs:

  paratt_truncate (paratt.c:316-342), attac_tt_axpby (paratt.c:237-268),
  pattac_apply_periodic_stencil (paratt.c:665-770), paratt_norm /
  paratt_dotprod / paratt_entry (paratt.c:369-499), pattac_exp_euler_st
  (paratt_ode.c:25-36) with a vector field passed as a C function pointer,
  and pattac_exp_midpoint_st (declared at paratt_ode.h:113-120, never defined
  by the reference) against its documented composition of reference calls.

rank_change_tt between calls grows the host cores (realloc moves them), so
the mirror registry meets reallocated core pointers."""
import ctypes as C

import numpy as np
import pytest

from oracle import tt_oracle as O

pytestmark = pytest.mark.gpu

try:
    from oracle import ref_lib as R

    HAVE_REF = R.available()
except Exception:  # pragma: no cover
    HAVE_REF = False

if not HAVE_REF:
    pytest.skip("oracle/_ref not built (make -C oracle)", allow_module_level=True)

from paratt_b200 import capi as A  # noqa: E402

DP = C.POINTER(C.c_double)
STEN = np.array([0.7, -1.4, 0.7])


def ours(cores):
    return A.HostTT(cores)


def gapped(dims, ranks, keep, seed):
    rng = np.random.default_rng(seed)
    out = []
    for k, n in enumerate(dims):
        q, _ = np.linalg.qr(rng.standard_normal((ranks[k] * n, ranks[k + 1])))
        s = np.ones(ranks[k + 1])
        if k < len(dims) - 1:
            s[keep[k + 1]:] = 1e-9
        out.append((q * s).reshape(ranks[k], n, ranks[k + 1], order="F"))
    return out


def test_truncate_axpby_stencil_vs_reference():
    dims, ranks = [9, 7, 11, 8, 6], [1, 5, 9, 8, 4, 1]
    x = gapped(dims, ranks, [1, 3, 5, 4, 2, 1], 1)
    y = O.random_tt(dims, [1, 2, 3, 3, 2, 1], 2)
    L = A.capi()
    # axpby: z = 0.5 x - 2 y
    tx, ty = ours(x), ours(y)
    tz = A.HostTT(dims=dims, ranks=[1] * 6)
    L.attac_tt_axpby(0.5, tx.p.contents.x, -2.0, ty.p.contents.x, tz.p.contents.x)
    ref = R.ref_axpby(0.5, x, -2.0, y)
    for a, b in zip(tz.cores(), ref):
        np.testing.assert_array_equal(a, b)
    # stencil along every mode, in place on the host cores
    for m in range(len(dims)):
        t = ours(x)
        L.pattac_apply_periodic_stencil(t.p, m, STEN.ctypes.data_as(DP), 3)
        for a, b in zip(t.cores(), R.ref_stencil(x, m, STEN)):
            assert np.abs(a - b).max() <= 1e-14 * np.abs(b).max()
        t.free()
    # truncate with a per-bond cap
    tol = 1e-6 * O.norm(x)
    mr = [1, 64, 64, 3, 64, 1]
    tx2 = ours(x)
    L.paratt_truncate(tx2.p, tol, A._iarr(mr))
    ref = R.ref_truncate(x, tol, mr)
    got = tx2.cores()
    assert O.ranks_of(got) == O.ranks_of(ref)
    assert O.rel_diff_exact(got, ref) <= 1e-12
    for t in (tx, ty, tz, tx2):
        t.free()


def test_norm_dot_entry_and_reallocated_cores():
    dims = [10, 12, 9, 11]
    x = O.random_tt(dims, [1, 3, 4, 3, 1], 5)
    y = O.random_tt(dims, [1, 2, 5, 2, 1], 6)
    L = A.capi()
    tx, ty = ours(x), ours(y)
    assert abs(L.paratt_norm(tx.p) - R.ref_norm(x)) <= 1e-13 * R.ref_norm(x)
    assert abs(L.paratt_dotprod(tx.p, ty.p) - R.ref_dot(x, y)) <= 1e-13 * O.norm(x) * O.norm(y)
    idx = [3, 7, 1, 10]
    assert abs(L.paratt_entry(tx.p, A._iarr(idx)) - R.ref_entry(x, idx)) <= 1e-13 * np.abs(O.full(x)).max()
    # grow the ranks: the host cores are reallocated (new addresses) and refilled
    x2 = O.random_tt(dims, [1, 8, 14, 9, 1], 7)
    before = [C.cast(tx.p.contents.x.contents.coreList[k], C.c_void_p).value for k in range(4)]
    L.rank_change_tt(tx.p.contents.x, A._iarr(O.ranks_of(x2)))
    tx.set_cores(x2)
    after = [C.cast(tx.p.contents.x.contents.coreList[k], C.c_void_p).value for k in range(4)]
    assert before != after  # at least one core moved
    assert abs(L.paratt_norm(tx.p) - R.ref_norm(x2)) <= 1e-13 * R.ref_norm(x2)
    assert abs(L.paratt_dotprod(tx.p, ty.p) - R.ref_dot(x2, y)) <= 1e-13 * O.norm(x2) * O.norm(y)
    tol = 1e-3 * O.norm(x2)
    L.paratt_truncate(tx.p, tol, A._iarr([1, 64, 64, 64, 1]))
    ref = R.ref_truncate(x2, tol, 64)
    got = tx.cores()
    assert O.ranks_of(got) == O.ranks_of(ref)
    assert O.rel_diff_exact(got, ref) <= 1e-12
    tx.free()
    ty.free()


# vector field F(u) = S_0 u (periodic stencil along mode 0), written against
# each library's own API as a reference-style driver would write it
VF = C.CFUNCTYPE(None, C.POINTER(A.Paratt), C.POINTER(A.Paratt), C.c_int)


def _field(lib):
    def f(u, out, _n):
        lib.copy_rank_change_tt(out.contents.x, u.contents.x)
        lib.pattac_apply_periodic_stencil(out, 0, STEN.ctypes.data_as(DP), 3)
    return VF(f)


def _bind_ode(lib, T, Pp):
    lib.copy_rank_change_tt.argtypes = [T, T]
    lib.pattac_apply_periodic_stencil.argtypes = [Pp, C.c_int, DP, C.c_int]
    lib.pattac_exp_euler_st.argtypes = [Pp, Pp, Pp, VF, C.c_double, C.c_double, C.c_double]


def test_euler_and_midpoint_steps_vs_reference():
    dims, dt = [16, 12, 10], 0.05
    u = gapped(dims, [1, 4, 6, 1], [1, 4, 6, 1], 9)
    ours_lib, ref_lib = A.capi(), R.lib()
    _bind_ode(ours_lib, C.POINTER(A.AttacTT), C.POINTER(A.Paratt))
    ours_lib.pattac_exp_midpoint_st.argtypes = [C.POINTER(A.Paratt)] * 3 + [VF] + [C.c_double] * 4
    # the reference library's own struct types (same layout)
    ref_lib.copy_rank_change_tt.argtypes = [C.POINTER(R.AttacTT)] * 2
    ref_lib.pattac_apply_periodic_stencil.argtypes = [C.POINTER(R.Paratt), C.c_int, DP, C.c_int]
    RVF = C.CFUNCTYPE(None, C.POINTER(R.Paratt), C.POINTER(R.Paratt), C.c_int)
    ref_lib.pattac_exp_euler_st.argtypes = [C.POINTER(R.Paratt)] * 3 + [RVF] + [C.c_double] * 3

    def rfield(uu, out, _n):
        ref_lib.copy_rank_change_tt(out.contents.x, uu.contents.x)
        ref_lib.pattac_apply_periodic_stencil(out, 0, STEN.ctypes.data_as(DP), 3)

    rf, of = RVF(rfield), _field(ours_lib)
    tol = 1e-9 * O.norm(u)
    # Euler: the reference defines it (paratt_ode.c:25-36)
    ro, rn, rw = R.RefTT(u), R.RefTT(u), R.RefTT(u)
    ref_lib.pattac_exp_euler_st(ro.p, rn.p, rw.p, rf, dt, tol, tol)
    oo, on, ow = ours(u), ours(u), ours(u)
    ours_lib.pattac_exp_euler_st(oo.p, on.p, ow.p, of, dt, tol, tol)
    ref, got = rn.cores(), on.cores()
    assert O.ranks_of(got) == O.ranks_of(ref)
    assert O.rel_diff_exact(got, ref) <= 1e-12
    # midpoint: the documented composition (paratt_ode.h:77-112) of reference
    # calls, the stage rounded with eps_1 as in this library
    k1 = R.ref_truncate(R.ref_stencil(u, 0, STEN), tol, O.ranks_of(u))
    us = R.ref_axpby(1.0, u, 0.5 * dt, k1)
    us = R.ref_truncate(us, tol, O.ranks_of(us))
    k2 = R.ref_truncate(R.ref_stencil(us, 0, STEN), tol, O.ranks_of(us))
    un = R.ref_axpby(1.0, u, dt, k2)
    un = R.ref_truncate(un, tol, O.ranks_of(un))
    mo, mn, mw = ours(u), ours(u), ours(u)
    ours_lib.pattac_exp_midpoint_st(mo.p, mn.p, mw.p, of, dt, tol, tol, tol)
    got = mn.cores()
    assert O.ranks_of(got) == O.ranks_of(un)
    assert O.rel_diff_exact(got, un) <= 1e-12
    for t in (ro, rn, rw):
        t.free()
    for t in (oo, on, ow, mo, mn, mw):
        t.free()
