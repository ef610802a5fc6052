// Internal definitions shared by the paratt_b200 CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include <math.h>

#include "../../include/paratt_b200.h"

// ---------------------------------------------------------------------------
// Device-side descriptor of one tensor train.  It lives in device memory so
// kernels read the current ranks and buffer pointers at run time: a sequence
// of launches is independent of the data and can be captured in a graph.
// ---------------------------------------------------------------------------
struct DevDesc {
    int d;
    int n[PTT_MAX_DIM];
    int r[PTT_MAX_DIM + 1];        // actual ranks
    int rcap[PTT_MAX_DIM + 1];     // rank capacity (for on-device checks)
    long long cap[PTT_MAX_DIM];    // doubles allocated per core buffer
    double* core[PTT_MAX_DIM];     // current cores
    double* alt[PTT_MAX_DIM];      // second buffer per core (out-of-place ops)
};

// Device status word codes (mirrors PTT_ERR_*).
#define PTT_STATUS_SET(st, code) atomicCAS((st), 0, (code))

struct ptt_ctx {
    int device;
    cudaStream_t stream;
    cudaStream_t side;            // second stream for overlapped work
    cudaEvent_t ev_fork, ev_join;
    int* d_status;                // device status word (first error wins)
    long long launches;
    // generic device workspace (grown on demand, never shrunk)
    void* ws;
    size_t ws_bytes;
    int* d_counters;              // zeroed, self-resetting tree counters
    size_t counters_n;
    double* d_scalars;            // small scratch for reductions
    double* h_scalars;            // pinned mirror
};

struct ptt_tt {
    ptt_ctx* ctx;
    int d;
    int n[PTT_MAX_DIM];
    int rcap[PTT_MAX_DIM + 1];
    long long cap[PTT_MAX_DIM];
    DevDesc* dd;                  // device descriptor
    DevDesc hd;                   // host shadow: pointers, n, caps (ranks stale)
};

// ---------------------------------------------------------------------------
// Error handling (host)
// ---------------------------------------------------------------------------
int ptt_set_error(int code, const char* fmt, ...);
int ptt_cuda_check(cudaError_t e, const char* what);

#define PTT_CUDA(call)                                                   \
    do {                                                                 \
        cudaError_t e_ = (call);                                         \
        if (e_ != cudaSuccess) return ptt_cuda_check(e_, #call);         \
    } while (0)

#define PTT_LAUNCHED(ctx)                                                \
    do {                                                                 \
        (ctx)->launches++;                                               \
        cudaError_t e_ = cudaGetLastError();                             \
        if (e_ != cudaSuccess) return ptt_cuda_check(e_, "kernel launch"); \
    } while (0)

// Workspace: returns a device pointer with at least `bytes`, 256-aligned.
int ptt_ws_reserve(ptt_ctx* ctx, size_t bytes);
int ptt_counters_reserve(ptt_ctx* ctx, size_t n);

// Swap core[k] <-> alt[k] for k in [k0, k1).
int ptt_swap(ptt_tt* t, int k0, int k1);

// Round a size up to a multiple of 256 bytes.
static inline size_t ptt_align(size_t b) { return (b + 255) & ~(size_t)255; }

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over groups of G consecutive lanes (G a power of two <= 32).
template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ int ldcg(const int* p) { return __ldcg(p); }
