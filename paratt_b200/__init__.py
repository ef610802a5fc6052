"""paratt_b200 -- B200 tensor-train hot path (rounding, axpby, Hadamard,
stencils, step-truncation RK2) behind the reference paratt C API.

The product is the C ABI library ``libparatt_b200.so`` built in this folder
(``make -C paratt_b200``); this module is a thin ctypes binding used by the
tests and the benchmark.  There is no CPU implementation: importing works
without a GPU, but every operation raises ``PttError`` (PTT_ERR_NOGPU) when no
CUDA device is present, and ``lib()`` raises if the library was not built.

Cores are numpy arrays of shape (r_k, n_k, r_{k+1}); their Fortran-order
ravel is the reference layout ``i + r_k*(j + n_k*l)`` (source/paratt.h:36-42).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libparatt_b200.so")

TIME_TSQR, TIME_SVD, TIME_GEMM = 1, 2, 3
STAT_NSIG = 16
STAT_LEN = 8 + STAT_NSIG
# rounding kinds of the reaction-Burgers step (PTT_RXN_KIND_*)
KIND_PRODUCT, KIND_FIELD, KIND_STAGE = 0, 1, 2
KINDS = 3

PTT_OK, PTT_ERR_ARG, PTT_ERR_CUDA, PTT_ERR_CAPACITY, PTT_ERR_NUMERIC, PTT_ERR_NOGPU, PTT_ERR_TIMEOUT = range(7)


class PttError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"paratt_b200 error {code}: {msg}")
        self.code = code


_lib = None

_i = C.c_int
_d = C.c_double
_p = C.c_void_p
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)
_dpp = C.POINTER(_dp)

# name -> (restype, argtypes) for the device ABI (include/paratt_b200.h)
_SIGS = {
    "ptt_last_error": (_i, []),
    "ptt_last_error_message": (C.c_char_p, []),
    "ptt_ctx_create": (_p, [_i]),
    "ptt_ctx_destroy": (None, [_p]),
    "ptt_ctx_synchronize": (_i, [_p]),
    "ptt_ctx_stream": (_p, [_p]),
    "ptt_ctx_launch_count": (C.c_longlong, [_p]),
    "ptt_tt_create": (_p, [_p, _i, _ip, _ip]),
    "ptt_tt_destroy": (None, [_p]),
    "ptt_tt_shape": (_i, [_p, _ip, _ip, _ip]),
    "ptt_tt_reserve": (_i, [_p, _ip]),
    "ptt_tt_set": (_i, [_p, _ip, _dpp]),
    "ptt_tt_get": (_i, [_p, _ip, _dpp]),
    "ptt_tt_get_ranks": (_i, [_p, _ip]),
    "ptt_tt_copy": (_i, [_p, _p]),
    "ptt_tt_device_cores": (_i, [_p, _dpp, C.POINTER(_ip)]),
    "ptt_round": (_i, [_p, _d, _ip]),
    "ptt_round_stats": (_i, [_p, _i, _dp]),
    "ptt_axpby": (_i, [_d, _p, _d, _p, _p]),
    "ptt_hadamard": (_i, [_p, _p, _p]),
    "ptt_square_sym": (_i, [_p, _p]),
    "ptt_round_batch": (_i, [C.POINTER(_p), _i, _dp, C.POINTER(_ip), _i]),
    "ptt_scale": (_i, [_d, _p]),
    "ptt_mult_diag": (_i, [_p, _i, _dp]),
    "ptt_stencil": (_i, [_p, _i, _dp, _i]),
    "ptt_dot": (_i, [_p, _p, _dp]),
    "ptt_dot_noalloc": (_i, [_p, _p, _dp]),
    "ptt_norm": (_i, [_p, _dp]),
    "ptt_entry": (_i, [_p, _ip, _dp]),
    "ptt_op_sum": (_i, [_p, _dp, _i, _d, _p]),
    "ptt_ctx_mark": (_i, [_p, _i]),
    "ptt_ctx_fixed_plans": (_i, [_p, _i]),
    "ptt_ctx_graphs": (_i, [_p, _i]),
    "ptt_ctx_cholqr": (_i, [_p, _i]),
    "ptt_ctx_ozaki": (_i, [_p, _i]),
    "ptt_gram": (_i, [_p, _p, C.c_longlong, _i, C.c_longlong, _p, _i]),
    "ptt_ctx_pdl": (_i, [_p, _i]),
    "ptt_ctx_autotune": (_i, [_p]),
    "ptt_checkpoint_begin": (_p, [_p, C.c_char_p]),
    "ptt_checkpoint_wait": (_i, [_p]),
    "ptt_tt_load_folder": (_i, [_p, C.c_char_p]),
    "ptt_ctx_autotune_table": (_i, [_p, C.POINTER(C.c_int)]),
    "ptt_ctx_autotune_gemm": (_i, [_p, C.POINTER(C.c_int)]),
    "ptt_ctx_qr_counts": (_i, [_p, C.POINTER(C.c_longlong)]),
    "ptt_ctx_workspace_bytes": (_i, [_p, C.POINTER(C.c_ulonglong)]),
    "ptt_cdf_stencil": (_i, [_p, _i, _dp, _i]),
    "ptt_cdf_lf_flux": (_i, [_p, _i, _dp, _dp, _dp, _d, _d]),
    "ptt_cdf_lw_rhs": (_i, [_p, _i, _dp, _dp, _dp, _dp, _d, _d]),
    "ptt_marginal_cusum": (_i, [_p, _i, _dp]),
    "ptt_marginal_trap": (_i, [_p, _i, _dp]),
    "ptt_scale_weight_sum": (_i, [_p, _i, _dp, _dp]),
    "ptt_apply_marginal": (_i, [_p, _i, _dp, _p]),
    "ptt_ctx_mem_info": (_i, [_p, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]),
    "ptt_ctx_elapsed": (_i, [_p, _i, _i, _dp]),
    "ptt_ctx_time_kernels": (_i, [_p, _i]),
    "ptt_ctx_kernel_time": (_i, [_p, _dp, C.POINTER(C.c_longlong)]),
    "ptt_ctx_kernel_work": (_i, [_p, _dp]),
    "ptt_ctx_flush_l2": (_i, [_p]),
    "ptt_host_pin": (_i, [_p, C.c_ulonglong]),
    "ptt_host_unpin": (_i, [_p]),
    "ptt_round_hadamard": (_i, [_p, _p, _p, _ip, C.c_ulonglong, _d, _ip]),
    "ptt_rxn_ws_create": (_p, [_p, _i, _ip, _i]),
    "ptt_rxn_ws_destroy": (None, [_p]),
    "ptt_rxn_ws_counts": (_i, [_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "ptt_rxn_burgers_F": (_i, [_p, _p, _p, _p]),
    "ptt_rxn_burgers_rk2_step": (_i, [_p, _p, _p]),
    "ptt_round_sketch": (_i, [_p, _p, _p, _ip, C.c_ulonglong, _d, _ip, _i, _ip]),
    "ptt_rxn_burgers_rk2_step_sketch": (_i, [_p, _p, _p, _ip, _i]),
    "ptt_rxn_ws_sketch_counts": (_i, [_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "ptt_rxn_ws_log": (_i, [_p, _i]),
    "ptt_rxn_ws_last_step": (_i, [_p, _ip, _dp, _dp]),
    "ptt_rxn_ws_last_step_kind": (_i, [_p, _i, _ip, _dp, _dp]),
    "ptt_rxn_burgers_rk2_step_sketch_kinds": (_i, [_p, _p, _p, _ip, _i]),
    "ptt_mlp_create": (_p, [_p, _i, _i, C.c_ulonglong]),
    "ptt_mlp_destroy": (None, [_p]),
    "ptt_mlp_num_params": (C.c_longlong, [_p]),
    "ptt_mlp_get_params": (_i, [_p, C.POINTER(C.c_float)]),
    "ptt_mlp_set_params": (_i, [_p, C.POINTER(C.c_float)]),
    "ptt_mlp_forward": (_i, [_p, C.POINTER(C.c_float), _i, C.POINTER(C.c_float)]),
    "ptt_mlp_grads": (_i, [_p, C.POINTER(C.c_float), C.POINTER(C.c_float), _i, C.POINTER(C.c_float),
                           C.POINTER(C.c_float)]),
    "ptt_mlp_train_step": (_i, [_p, C.POINTER(C.c_float), C.POINTER(C.c_float), _i, C.c_float,
                                C.POINTER(C.c_float)]),
    "ptt_mlp_set_under_weight": (_i, [_p, C.c_float]),
}


class RxnParams(C.Structure):
    """ptt_rxn_params (include/paratt_b200.h)."""
    _fields_ = [("dt", C.c_double), ("tol", C.c_double), ("nu", C.c_double), ("L", C.c_double),
                ("maxrank", C.c_int), ("sketch_pad", C.c_int), ("seed", C.c_ulonglong)]


def lib():
    """Load libparatt_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not built: run `make -C paratt_b200`")
        L = C.CDLL(LIB_PATH, mode=os.RTLD_LOCAL)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc != PTT_OK:
        msg = lib().ptt_last_error_message()
        raise PttError(rc, msg.decode() if msg else "")


def _iarr(v):
    return (C.c_int * len(v))(*[int(t) for t in v])


def _vec(v):
    return np.ascontiguousarray(v, dtype=np.float64)


class Context:
    """One device + stream + workspace (ptt_ctx)."""

    def __init__(self, device: int = 0):
        self.device = int(device)
        self.h = lib().ptt_ctx_create(device)
        if not self.h:
            _check(lib().ptt_last_error() or PTT_ERR_CUDA)

    def sync(self):
        _check(lib().ptt_ctx_synchronize(self.h))

    def round_stats(self, d):
        """Per-bond records of the last rounding on this context: array of
        shape (d, PTT_STAT_LEN) (row i = bond i; row 0 unused)."""
        out = np.zeros((d, STAT_LEN))
        _check(lib().ptt_round_stats(self.h, d, out.ctypes.data_as(_dp)))
        return out

    def fixed_plans(self, on=True):
        """Size rounding plans by capacity (no rank read-back) when on."""
        _check(lib().ptt_ctx_fixed_plans(self.h, 1 if on else 0))

    def cholqr(self, on=True):
        """Cholesky-QR factorisation of unfoldings with <= 32 columns (default
        on; off = Householder TSQR only)."""
        _check(lib().ptt_ctx_cholqr(self.h, 1 if on else 0))

    def ozaki(self, on=True):
        """Gram matrices of the 33-64-column Cholesky QR by the Ozaki split on
        the fifth-generation tensor cores (default off = FP64 mma)."""
        _check(lib().ptt_ctx_ozaki(self.h, 1 if on else 0))

    def gram(self, a_ptr, m, c, lda, g_ptr, method=0):
        """G = A^T A of device arrays (column-major m x c at a_ptr, c x c at
        g_ptr); method 0 FP64 mma, 1 Ozaki split; synchronises the context."""
        _check(lib().ptt_gram(self.h, C.c_void_p(a_ptr), m, c, lda, C.c_void_p(g_ptr), method))
        _check(lib().ptt_ctx_synchronize(self.h))

    def autotune(self):
        """Pick the Cholesky-QR cluster size per (columns, rows) bucket by
        timing; returns the 3 x 6 table (columns 16/24/32 x rows 512..16384)."""
        _check(lib().ptt_ctx_autotune(self.h))
        return self.autotune_table()

    def autotune_table(self):
        v = (C.c_int * 18)()
        _check(lib().ptt_ctx_autotune_table(self.h, v))
        return np.array(list(v)).reshape(3, 6)

    def autotune_gemm(self):
        """(smallest M, N of 64-wide contraction tiles, split-K tile target)."""
        out = (C.c_int * 2)()
        _check(lib().ptt_ctx_autotune_gemm(self.h, out))
        return int(out[0]), int(out[1])

    def pdl(self, on=True):
        """Programmatic dependent launch of the rounding chain (default on)."""
        _check(lib().ptt_ctx_pdl(self.h, 1 if on else 0))

    def qr_counts(self):
        """(finished by Cholesky QR, fell back to Householder, Gram stages)."""
        v = (C.c_longlong * 3)()
        _check(lib().ptt_ctx_qr_counts(self.h, v))
        return tuple(int(a) for a in v)

    def workspace_bytes(self) -> int:
        """Device bytes held by the context's grow-on-demand workspaces."""
        v = C.c_ulonglong(0)
        _check(lib().ptt_ctx_workspace_bytes(self.h, C.byref(v)))
        return int(v.value)

    def mem_info(self):
        """(free, total) device bytes of the context's device (cudaMemGetInfo)."""
        f, t = C.c_ulonglong(0), C.c_ulonglong(0)
        _check(lib().ptt_ctx_mem_info(self.h, C.byref(f), C.byref(t)))
        return int(f.value), int(t.value)

    def graphs(self, on=True):
        """Replay roundings from cached CUDA graphs when on (same results)."""
        _check(lib().ptt_ctx_graphs(self.h, 1 if on else 0))

    def mark(self, slot):
        _check(lib().ptt_ctx_mark(self.h, slot))

    def elapsed_ms(self, a, b):
        v = C.c_double()
        _check(lib().ptt_ctx_elapsed(self.h, a, b, C.byref(v)))
        return v.value

    def time_kernels(self, kind):
        """Event-time every launch of one kernel class (TIME_TSQR/SVD/GEMM)."""
        _check(lib().ptt_ctx_time_kernels(self.h, kind))

    def kernel_time(self):
        ms, n = C.c_double(), C.c_longlong()
        _check(lib().ptt_ctx_kernel_time(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def kernel_work(self):
        w = C.c_double()
        _check(lib().ptt_ctx_kernel_work(self.h, C.byref(w)))
        return w.value

    def flush_l2(self):
        _check(lib().ptt_ctx_flush_l2(self.h))

    @property
    def stream(self):
        return lib().ptt_ctx_stream(self.h)

    @property
    def launches(self) -> int:
        return int(lib().ptt_ctx_launch_count(self.h))

    def close(self):
        if self.h:
            lib().ptt_ctx_destroy(self.h)
            self.h = None


class TT:
    """A device-resident tensor train (ptt_tt)."""

    def __init__(self, ctx: Context, dims, rank_cap, cores=None):
        self.ctx = ctx
        self.dims = [int(n) for n in dims]
        self.d = len(self.dims)
        rc = list(rank_cap)
        self.h = lib().ptt_tt_create(ctx.h, self.d, _iarr(self.dims), _iarr(rc))
        if not self.h:
            _check(lib().ptt_last_error() or PTT_ERR_ARG)
        if cores is not None:
            self.set(cores)

    @classmethod
    def from_cores(cls, ctx, cores, rank_cap=None):
        dims = [c.shape[1] for c in cores]
        ranks = [cores[0].shape[0]] + [c.shape[2] for c in cores]
        return cls(ctx, dims, rank_cap or ranks, cores)

    def set(self, cores):
        ranks = [cores[0].shape[0]] + [c.shape[2] for c in cores]
        bufs = [np.ascontiguousarray(c.ravel(order="F"), dtype=np.float64) for c in cores]
        ptrs = (_dp * self.d)(*[b.ctypes.data_as(_dp) for b in bufs])
        _check(lib().ptt_tt_set(self.h, _iarr(ranks), ptrs))

    def set_device(self, ranks, ptrs):
        """Set the cores from device (or any CUDA-addressable) memory: ptrs[k]
        is the address of core k, ranks[k] x n_k x ranks[k+1] column-major."""
        arr = (_dp * self.d)(*[C.cast(C.c_void_p(int(p)), _dp) for p in ptrs])
        _check(lib().ptt_tt_set(self.h, _iarr(ranks), arr))

    def ranks(self):
        r = (C.c_int * (self.d + 1))()
        _check(lib().ptt_tt_get_ranks(self.h, r))
        return list(r)

    def get(self):
        r = self.ranks()
        bufs = [np.empty(r[k] * self.dims[k] * r[k + 1]) for k in range(self.d)]
        ptrs = (_dp * self.d)(*[b.ctypes.data_as(_dp) for b in bufs])
        _check(lib().ptt_tt_get(self.h, _iarr(r), ptrs))
        return [b.reshape((r[k], self.dims[k], r[k + 1]), order="F") for k, b in enumerate(bufs)]

    def reserve(self, rank_cap):
        _check(lib().ptt_tt_reserve(self.h, _iarr(rank_cap)))

    def round(self, tol, maxrank=None):
        mr = None
        if maxrank is not None:
            mr = _iarr(maxrank if hasattr(maxrank, "__len__") else [maxrank] * (self.d + 1))
        _check(lib().ptt_round(self.h, float(tol), mr))
        return self

    def scale(self, a):
        _check(lib().ptt_scale(float(a), self.h))
        return self

    def mult_diag(self, mode, vec):
        v = np.ascontiguousarray(vec, dtype=np.float64)
        _check(lib().ptt_mult_diag(self.h, int(mode), v.ctypes.data_as(_dp)))
        return self

    def stencil(self, mode, sten):
        s = np.ascontiguousarray(sten, dtype=np.float64)
        _check(lib().ptt_stencil(self.h, int(mode), s.ctypes.data_as(_dp), len(s)))
        return self

    # CDF-problem stencils and marginals of the reference (paratt.c:772-1618)
    def cdf_stencil(self, mode, sten):
        s = _vec(sten)
        _check(lib().ptt_cdf_stencil(self.h, int(mode), s.ctypes.data_as(_dp), len(s)))

    def cdf_lf_flux(self, mode, wave_speed, gc_wave_speed, source_coef, dt, dx):
        v = [_vec(t) for t in (wave_speed, gc_wave_speed, source_coef)]
        _check(lib().ptt_cdf_lf_flux(self.h, int(mode), *[t.ctypes.data_as(_dp) for t in v], float(dt), float(dx)))

    def cdf_lw_rhs(self, mode, wave_speed, gc_wave_speed, bdry_wave_speed, source_coef, dt, dx):
        v = [_vec(t) for t in (wave_speed, gc_wave_speed, bdry_wave_speed, source_coef)]
        _check(lib().ptt_cdf_lw_rhs(self.h, int(mode), *[t.ctypes.data_as(_dp) for t in v], float(dt), float(dx)))

    def marginal_cusum(self, mode, w):
        v = _vec(w)
        _check(lib().ptt_marginal_cusum(self.h, int(mode), v.ctypes.data_as(_dp)))

    def marginal_trap(self, mode, w):
        v = _vec(w)
        _check(lib().ptt_marginal_trap(self.h, int(mode), v.ctypes.data_as(_dp)))

    def scale_weight_sum(self, mode, scale, sum_w):
        a, b = _vec(scale), _vec(sum_w)
        _check(lib().ptt_scale_weight_sum(self.h, int(mode), a.ctypes.data_as(_dp), b.ctypes.data_as(_dp)))

    def apply_marginal(self, mode, w, out):
        """out (d - 1 modes) <- this train contracted along `mode` with w."""
        v = _vec(w)
        _check(lib().ptt_apply_marginal(self.h, int(mode), v.ctypes.data_as(_dp), out.h))

    def dot(self, other):
        v = C.c_double()
        _check(lib().ptt_dot(self.h, other.h, C.byref(v)))
        return v.value

    def dot_noalloc(self, other):
        """ptt_dot using the fixed device scratch array (no allocation)."""
        v = C.c_double()
        _check(lib().ptt_dot_noalloc(self.h, other.h, C.byref(v)))
        return v.value

    def norm(self):
        v = C.c_double()
        _check(lib().ptt_norm(self.h, C.byref(v)))
        return v.value

    def entry(self, idx):
        v = C.c_double()
        _check(lib().ptt_entry(self.h, _iarr(idx), C.byref(v)))
        return v.value

    def copy_from(self, other):
        _check(lib().ptt_tt_copy(self.h, other.h))
        return self

    def checkpoint(self, folder):
        """Start writing this train to `folder` as reference .cr core files
        (write-behind); returns a Checkpoint whose wait() finishes it."""
        h = lib().ptt_checkpoint_begin(self.h, os.fsencode(folder))
        if not h:
            raise RuntimeError(f"checkpoint of the train to {folder} could not start")
        return Checkpoint(h)

    def load_folder(self, folder):
        """Resume: read reference .cr core files from `folder` into this train."""
        _check(lib().ptt_tt_load_folder(self.h, os.fsencode(folder)))
        return self

    def close(self):
        if self.h:
            lib().ptt_tt_destroy(self.h)
            self.h = None


class Checkpoint:
    """A checkpoint being written in the background (TT.checkpoint)."""

    def __init__(self, h):
        self.h = h

    def wait(self):
        if self.h:
            h, self.h = self.h, None
            _check(lib().ptt_checkpoint_wait(h))


class HostTrain:
    """Page-locked host copy of a tensor train: one flat buffer per core,
    sized for the rank capacity, column-major cores as in the reference.
    upload() / download() move the whole train with one copy per core."""

    def __init__(self, dims, rank_cap, cores=None):
        self.dims = [int(n) for n in dims]
        self.d = len(self.dims)
        self.cap = list(rank_cap)
        self.bufs = [np.zeros(self.cap[k] * self.dims[k] * self.cap[k + 1]) for k in range(self.d)]
        for b in self.bufs:
            _check(lib().ptt_host_pin(C.c_void_p(b.ctypes.data), C.c_ulonglong(b.nbytes)))
        self._ptrs = (_dp * self.d)(*[b.ctypes.data_as(_dp) for b in self.bufs])
        self.r = [1] * (self.d + 1)
        if cores is not None:
            self.r = [cores[0].shape[0]] + [c.shape[2] for c in cores]
            for k, c in enumerate(cores):
                self.bufs[k][: c.size] = c.ravel(order="F")

    def nbytes(self):
        """Bytes of the train at its current ranks."""
        return 8 * sum(self.r[k] * self.dims[k] * self.r[k + 1] for k in range(self.d))

    def upload(self, tt: TT):
        _check(lib().ptt_tt_set(tt.h, _iarr(self.r), self._ptrs))

    def download(self, tt: TT):
        r = (C.c_int * (self.d + 1))()
        _check(lib().ptt_tt_get(tt.h, r, self._ptrs))
        self.r = list(r)

    def cores(self):
        return [self.bufs[k][: self.r[k] * self.dims[k] * self.r[k + 1]].reshape(
            (self.r[k], self.dims[k], self.r[k + 1]), order="F").copy() for k in range(self.d)]

    def close(self):
        for b in self.bufs:
            lib().ptt_host_unpin(C.c_void_p(b.ctypes.data))
        self.bufs = []


def axpby(a, x: TT, b, y: TT, z: TT):
    _check(lib().ptt_axpby(float(a), x.h, float(b), y.h, z.h))
    return z


def hadamard(x: TT, y: TT, z: TT):
    _check(lib().ptt_hadamard(x.h, y.h, z.h))
    return z


def round_batch(tts, tols, maxranks=None, lanes=8):
    """Round independent trains concurrently (ptt_round_batch); maxranks is
    None or one entry per train (None, an int or d+1 ints)."""
    n = len(tts)
    hs = (_p * n)(*[t.h for t in tts])
    tv = np.ascontiguousarray(tols, dtype=np.float64)
    mr = None
    keep = []
    if maxranks is not None:
        mr = (_ip * n)()
        for i, (t, m) in enumerate(zip(tts, maxranks)):
            if m is None:
                mr[i] = _ip()
                continue
            a = _iarr(m if hasattr(m, "__len__") else [m] * (t.d + 1))
            keep.append(a)
            mr[i] = C.cast(a, _ip)
    _check(lib().ptt_round_batch(hs, n, tv.ctypes.data_as(_dp), mr, int(lanes)))
    return tts


def square_sym(x: TT, z: TT):
    """z = x (.) x at ranks r (r + 1) / 2 (same tensor as hadamard(x, x))."""
    _check(lib().ptt_square_sym(x.h, z.h))
    return z


def op_sum(x: TT, sten, shift, y: TT):
    s = np.ascontiguousarray(sten, dtype=np.float64)
    _check(lib().ptt_op_sum(x.h, s.ctypes.data_as(_dp), len(s), float(shift), y.h))
    return y


def round_hadamard(x: TT, y: TT, z: TT, ell, seed, tol, maxrank=None):
    e = _iarr(ell if hasattr(ell, "__len__") else [ell] * (x.d + 1))
    mr = None if maxrank is None else _iarr(maxrank if hasattr(maxrank, "__len__") else [maxrank] * (x.d + 1))
    _check(lib().ptt_round_hadamard(x.h, y.h, z.h, e, C.c_ulonglong(seed), float(tol), mr))
    return z


class RxnBurgers:
    """Device workspace + parameters of the reaction-Burgers RK2 step."""

    def __init__(self, ctx: Context, d, n, maxrank, dt, tol, nu=0.05, L=10.0, sketch_pad=8, seed=1):
        self.ctx = ctx
        self.p = RxnParams(dt, tol, nu, L, maxrank, sketch_pad, seed)
        self.h = lib().ptt_rxn_ws_create(ctx.h, d, _iarr([n] * d), maxrank)
        if not self.h:
            _check(lib().ptt_last_error() or PTT_ERR_ARG)

    def F(self, u: TT, out: TT):
        _check(lib().ptt_rxn_burgers_F(u.h, out.h, self.h, C.byref(self.p)))
        return out

    def step(self, u: TT):
        _check(lib().ptt_rxn_burgers_rk2_step(u.h, self.h, C.byref(self.p)))
        return u

    def step_sketch(self, u: TT, ell, pad=4):
        e = _iarr(ell)
        _check(lib().ptt_rxn_burgers_rk2_step_sketch(u.h, self.h, C.byref(self.p), e, int(pad)))
        return u

    def step_sketch_kinds(self, u: TT, ell, pad=4):
        """ell: KINDS x (d+1) sketch ranks, row t for the roundings of kind t."""
        e = _iarr(np.asarray(ell, dtype=np.int64).ravel())
        _check(lib().ptt_rxn_burgers_rk2_step_sketch_kinds(u.h, self.h, C.byref(self.p), e, int(pad)))
        return u

    def sketch_counts(self):
        c, f = C.c_longlong(), C.c_longlong()
        _check(lib().ptt_rxn_ws_sketch_counts(self.h, C.byref(c), C.byref(f)))
        return c.value, f.value

    def log(self, on=True):
        _check(lib().ptt_rxn_ws_log(self.h, 1 if on else 0))

    def last_step(self, d):
        """(max kept rank per bond over the last step's roundings [d+1],
        top-16 singular values per bond of the last rounding [d+1, 16], threshold)"""
        r = (C.c_int * (d + 1))()
        sig = np.zeros((d + 1, STAT_NSIG))
        dl = C.c_double()
        _check(lib().ptt_rxn_ws_last_step(self.h, r, sig.ctypes.data_as(_dp), C.byref(dl)))
        return list(r), sig, dl.value

    def last_step_kind(self, kind, d):
        """last_step restricted to the roundings of one kind (KIND_*)."""
        r = (C.c_int * (d + 1))()
        sig = np.zeros((d + 1, STAT_NSIG))
        dl = C.c_double()
        _check(lib().ptt_rxn_ws_last_step_kind(self.h, int(kind), r, sig.ctypes.data_as(_dp), C.byref(dl)))
        return list(r), sig, dl.value

    def counts(self):
        f, s = C.c_longlong(), C.c_longlong()
        _check(lib().ptt_rxn_ws_counts(self.h, C.byref(f), C.byref(s)))
        return f.value, s.value

    def close(self):
        if self.h:
            lib().ptt_rxn_ws_destroy(self.h)
            self.h = None


def round_sketch(x: TT, y, z: TT, ell, seed, tol, maxrank=None, pad=4):
    """Sketch rounding of x (y None) or x (.) y; returns whether accepted."""
    e = _iarr(ell if hasattr(ell, "__len__") else [ell] * (x.d + 1))
    mr = None if maxrank is None else _iarr(maxrank if hasattr(maxrank, "__len__") else [maxrank] * (x.d + 1))
    ok = C.c_int()
    _check(lib().ptt_round_sketch(x.h, y.h if y is not None else None, z.h, e, C.c_ulonglong(seed), float(tol), mr,
                                  int(pad), C.byref(ok)))
    return bool(ok.value)


_fp = C.POINTER(C.c_float)


class MLP:
    """Sketch-rank proposer (ptt_mlp): nin -> width -> width -> 1."""

    def __init__(self, ctx: Context, nin, width=64, seed=1):
        self.ctx, self.nin, self.width = ctx, nin, width
        self.h = lib().ptt_mlp_create(ctx.h, nin, width, C.c_ulonglong(seed))
        if not self.h:
            _check(lib().ptt_last_error() or PTT_ERR_ARG)
        self.np = int(lib().ptt_mlp_num_params(self.h))

    def params(self):
        out = np.zeros(self.np, dtype=np.float32)
        _check(lib().ptt_mlp_get_params(self.h, out.ctypes.data_as(_fp)))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(lib().ptt_mlp_set_params(self.h, p.ctypes.data_as(_fp)))

    def forward(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros(x.shape[0], dtype=np.float32)
        _check(lib().ptt_mlp_forward(self.h, x.ctypes.data_as(_fp), x.shape[0], y.ctypes.data_as(_fp)))
        return y

    def grads(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(self.np, dtype=np.float32)
        loss = C.c_float()
        _check(lib().ptt_mlp_grads(self.h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp), x.shape[0],
                                   g.ctypes.data_as(_fp), C.byref(loss)))
        return g, loss.value

    def train_step(self, x, t, lr):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = C.c_float()
        _check(lib().ptt_mlp_train_step(self.h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp), x.shape[0],
                                        C.c_float(lr), C.byref(loss)))
        return loss.value

    def set_under_weight(self, w):
        _check(lib().ptt_mlp_set_under_weight(self.h, C.c_float(w)))

    def close(self):
        if self.h:
            lib().ptt_mlp_destroy(self.h)
            self.h = None
