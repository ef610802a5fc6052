"""ctypes binding of the reference-compatible C API (include/paratt.h,
include/paratt_ode.h) exported by libparatt_b200.so -- the calls a driver
written against the reference makes, with host-resident cores."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import LIB_PATH


class AttacTT(C.Structure):
    # include/paratt.h (same layout as the reference, source/paratt.h:25-54)
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


_capi = None


def capi():
    global _capi
    if _capi is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not built: run `make -C paratt_b200`")
        L = C.CDLL(LIB_PATH, mode=os.RTLD_LOCAL)
        P, T = C.POINTER(Paratt), C.POINTER(AttacTT)
        ip, dp = C.POINTER(C.c_int), C.POINTER(C.c_double)
        L.alloc_ptt.restype = P
        L.alloc_ptt.argtypes = [C.c_int, ip, ip]
        L.free_ptt.argtypes = [P]
        L.alloc_tt.restype = T
        L.alloc_tt.argtypes = [C.c_int, ip, ip]
        L.free_tt.argtypes = [T]
        L.rank_change_tt.restype = T
        L.rank_change_tt.argtypes = [T, ip]
        L.paratt_truncate.argtypes = [P, C.c_double, ip]
        L.attac_tt_truncate.argtypes = [T, C.c_double, ip]
        L.attac_tt_axpby.argtypes = [C.c_double, T, C.c_double, T, T]
        L.attac_tt_hadamard.argtypes = [T, T, T]
        L.attac_tt_scale.argtypes = [C.c_double, T]
        L.paratt_norm.restype = C.c_double
        L.paratt_norm.argtypes = [P]
        L.attac_tt_norm.restype = C.c_double
        L.attac_tt_norm.argtypes = [T]
        L.paratt_dotprod.restype = C.c_double
        L.paratt_dotprod.argtypes = [P, P]
        L.paratt_entry.restype = C.c_double
        L.paratt_entry.argtypes = [P, ip]
        L.pattac_apply_periodic_stencil.argtypes = [P, C.c_int, dp, C.c_int]
        L.attac_apply_periodic_stencil.argtypes = [T, C.c_int, dp, C.c_int]
        L.attac_mult_diag_mat.argtypes = [T, C.c_int, dp]
        L.pattac_write_tt_folder.argtypes = [C.c_char_p, P]
        L.pattac_load_tt_folder.restype = P
        L.pattac_load_tt_folder.argtypes = [C.c_char_p, C.c_int]
        L.read_core_size.argtypes = [C.c_char_p, ip, ip, ip]
        L.pattac_rxn_burgers_midpoint_st.argtypes = [P, C.c_double, C.c_double, C.c_int]
        L.paratt_last_error.restype = C.c_int
        L.ptt_host_pin.argtypes = [C.c_void_p, C.c_ulonglong]
        L.ptt_host_pin.restype = C.c_int
        L.ptt_host_unpin.argtypes = [C.c_void_p]
        L.ptt_host_unpin.restype = C.c_int
        _capi = L
    return _capi


def _iarr(v):
    return (C.c_int * len(v))(*[int(t) for t in v])


class HostTT:
    """A `paratt` allocated by the library (host cores, reference semantics).

    ``capacity`` (rank list) preallocates the cores large enough that no call
    has to realloc them, so they can stay page-locked with ``pin()``."""

    def __init__(self, cores=None, dims=None, ranks=None, capacity=None, ptr=None):
        L = capi()
        self.pinned = []
        if ptr is not None:
            self.p = ptr
            return
        if cores is not None:
            dims = [c.shape[1] for c in cores]
            ranks = [cores[0].shape[0]] + [c.shape[2] for c in cores]
        self.p = L.alloc_ptt(len(dims), _iarr(dims), _iarr(capacity or ranks))
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
        x = self.p.contents.x
        rk = [cores[0].shape[0]] + [c.shape[2] for c in cores]
        capi().rank_change_tt(x, _iarr(rk))
        xc = x.contents
        for k, c in enumerate(cores):
            flat = np.ascontiguousarray(c.ravel(order="F"), dtype=np.float64)
            C.memmove(xc.coreList[k], flat.ctypes.data, flat.nbytes)

    def cores(self):
        xc = self.p.contents.x.contents
        r, n = self.ranks(), self.dims()
        out = []
        for k in range(self.d):
            cnt = r[k] * n[k] * r[k + 1]
            buf = np.ctypeslib.as_array(xc.coreList[k], shape=(cnt,)).copy()
            out.append(buf.reshape((r[k], n[k], r[k + 1]), order="F"))
        return out

    def core_bytes(self):
        r, n = self.ranks(), self.dims()
        return sum(8 * r[k] * n[k] * r[k + 1] for k in range(self.d))

    def pin(self):
        """Page-lock the current core buffers (they must not be reallocated)."""
        xc = self.p.contents.x.contents
        for k in range(self.d):
            ptr = C.cast(xc.coreList[k], C.c_void_p).value
            if capi().ptt_host_pin(ptr, 8 * xc.coreMem[k]) == 0:
                self.pinned.append(ptr)

    def unpin(self):
        for ptr in self.pinned:
            capi().ptt_host_unpin(ptr)
        self.pinned = []

    def free(self):
        if self.p:
            self.unpin()
            capi().free_ptt(self.p)
            self.p = None
