"""Host-side parts of the reference-compatible API that need no GPU:
allocation with reference ownership and the .cr core files
(paratt.c:1621-1892), checked against files written by the reference."""
import ctypes as C
import os

import numpy as np

from oracle import tt_oracle as O
from paratt_b200.capi import HostTT, capi

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def unpack(z, prefix):
    r, n = z[f"{prefix}_ranks"], z[f"{prefix}_dims"]
    return [z[f"{prefix}_{k}"].reshape((r[k], n[k], r[k + 1]), order="F") for k in range(len(n))]


def test_load_reference_written_folder():
    folder = os.path.join(GOLD, "cr_written_by_reference").encode()
    p = capi().pattac_load_tt_folder(folder, 3)
    t = HostTT(ptr=p)
    ref = unpack(np.load(os.path.join(GOLD, "cr_values.npz")), "x")
    got = t.cores()
    for a, b in zip(got, ref):
        assert a.shape == b.shape
        np.testing.assert_array_equal(a, b)
    t.free()


def test_write_matches_reference_bytes(tmp_path):
    ref_dir = os.path.join(GOLD, "cr_written_by_reference")
    cores = unpack(np.load(os.path.join(GOLD, "cr_values.npz")), "x")
    t = HostTT(cores)
    out = str(tmp_path / "tt")
    capi().pattac_write_tt_folder(out.encode(), t.p)
    for k in range(1, 4):
        a = open(os.path.join(out, f"core_{k}.cr")).read()
        b = open(os.path.join(ref_dir, f"core_{k}.cr")).read()
        assert a == b
    t.free()


def test_read_core_size_and_slice(tmp_path):
    x = O.random_tt([5, 6, 3], [1, 2, 4, 1], 3)
    t = HostTT(x)
    out = str(tmp_path / "s")
    capi().pattac_write_tt_folder(out.encode(), t.p)
    rl, n, rr = C.c_int(), C.c_int(), C.c_int()
    capi().read_core_size(os.path.join(out, "core_2.cr").encode(), C.byref(rl), C.byref(n), C.byref(rr))
    assert (rl.value, n.value, rr.value) == (2, 6, 4)
    L = capi()
    L.load_core_slice.argtypes = [C.c_char_p, C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.c_int),
                                  C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.c_int]
    buf = C.POINTER(C.c_double)()
    sz = C.c_int(0)
    L.load_core_slice(os.path.join(out, "core_2.cr").encode(), C.byref(buf), C.byref(sz), C.byref(rl),
                      C.byref(n), C.byref(rr), 2, 5)
    got = np.ctypeslib.as_array(buf, shape=(2 * 3 * 4,)).reshape((2, 3, 4), order="F")
    np.testing.assert_array_equal(got, x[1][:, 2:5, :])
    t.free()


def test_sum_of_product_layout():
    """attac_sum_of_product (paratt.c:517-568): rank-R sum of rank-1 terms."""
    L = capi()
    L.attac_sum_of_product.restype = C.c_void_p
    d, n, R = 3, [4, 5, 3], 2
    rng = np.random.default_rng(0)
    vecs = [[rng.standard_normal(n[k]) for k in range(d)] for _ in range(R)]
    keep = [[np.ascontiguousarray(v) for v in term] for term in vecs]
    arr = (C.POINTER(C.POINTER(C.c_double)) * R)()
    for t in range(R):
        inner = (C.POINTER(C.c_double) * d)(*[keep[t][k].ctypes.data_as(C.POINTER(C.c_double)) for k in range(d)])
        arr[t] = C.cast(inner, C.POINTER(C.POINTER(C.c_double)))
        keep[t].append(inner)
    from paratt_b200.capi import AttacTT
    L.attac_sum_of_product.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_int]
    ptr = L.attac_sum_of_product(C.cast(arr, C.c_void_p), d, (C.c_int * d)(*n), R)
    tt = C.cast(ptr, C.POINTER(AttacTT)).contents
    r = [tt.ttRank[k] for k in range(d + 1)]
    cores = []
    for k in range(d):
        cnt = r[k] * n[k] * r[k + 1]
        cores.append(np.ctypeslib.as_array(tt.coreList[k], shape=(cnt,)).reshape((r[k], n[k], r[k + 1]), order="F").copy())
    full = O.full(cores)
    ref = sum(np.einsum("i,j,k->ijk", *term[:3]) for term in vecs)
    np.testing.assert_allclose(full, ref, rtol=1e-14, atol=1e-14)
    L.free_tt.argtypes = [C.c_void_p]
    L.free_tt(ptr)
