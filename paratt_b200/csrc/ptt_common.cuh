// Internal definitions shared by the paratt_b200 CUDA sources.
#pragma once
#include <atomic>
#include <functional>

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

#define PTT_MAX_LANES 16

struct ptt_ctx {
    int device;
    int nsm;                      // streaming multiprocessors of the device
    cudaStream_t stream;
    cudaStream_t side;            // second stream for overlapped work
    cudaEvent_t ev_fork, ev_join;
    cudaEvent_t ev_svd[2], ev_tail[2];  // truncation sweep: a bond's SVD done / its tail done, per slot
    int* d_status;                // device status word (first error wins)
    int fixed_plans;              // 1: size rounding plans by capacity (no rank read-back)
    long long launches;
    // generic device workspace (grown on demand, never shrunk)
    void* ws;
    size_t ws_bytes;
    void* ws2;                    // second workspace (sketch contractions)
    size_t ws2_bytes;
    void* ws3;                    // split-K partial products of the batched GEMMs
    size_t ws3_bytes;
    int* d_counters;              // zeroed, self-resetting tree counters
    size_t counters_n;
    double* d_scalars;            // small scratch for reductions
    double* h_scalars;            // pinned mirror
    double* d_stats;              // per-bond record of the last rounding (PTT_STAT_LEN doubles each)
    // measurement: user marks and per-launch timing of one kernel class
    cudaEvent_t marks[64];
    int tkind;                    // PTT_TIME_* class being timed (0 = none)
    cudaEvent_t* tev;             // 2 events per timed launch
    int tcount, tcap;
    double tms;                   // accumulated milliseconds of resolved launches
    long long tlaunches;
    double* d_work;               // device accumulators of algorithmic work per class [4]
    double hwork[4];              // host-known algorithmic work per class
    double* d_ones;               // vector of ones (the all-ones rank-1 train)
    int ones_n;
    void* flush;                  // L2 flush buffer
    size_t flush_bytes;
    // whole-train transfers of pageable host cores (ptt_tt_set / ptt_tt_get):
    // page-locked and device staging buffers, grown on demand
    double* h_stage;
    size_t h_stage_n;
    double* d_stage;
    size_t d_stage_n;
    // worker contexts of batched calls (own stream and workspaces, the
    // parent's status word)
    struct ptt_ctx* lanes[PTT_MAX_LANES];
    int nlanes;
    int shared_status;            // d_status belongs to the parent context
    // captured launch sequences (ptt_graph_run): on/off and the cache
    int graphs;
    void* graph_cache;
    // Cholesky-QR factorisation of unfoldings with <= 32 columns: 0 = used
    // (default), 1 = Householder TSQR only; device counters [finished,
    // fell back, Gram stages of the finished ones]
    int no_cholqr;
    long long* d_qrstat;
    // Gram matrices of the grid Cholesky QR (33-64 columns) by the Ozaki
    // split on the fifth-generation tensor cores: 0 = FP64 mma (default)
    int ozaki;
    // a worker context of ptt_round_batch: the batch already overlaps whole
    // roundings, so a lane runs each rounding's chain on its one stream
    int lane;
    // programmatic dependent launch of the rounding chain: 0 = used (default)
    int no_pdl;
    int capturing;                // inside ptt_graph_run's own capture
    // Cholesky-QR cluster sizes chosen by ptt_ctx_autotune: [column bound
    // 16/24/32][rows bucket 512 .. 16384]; 0 = not tuned (size heuristic)
    unsigned char cq_cs[3][6];
    int cq_tuned;                 // generation of the table (0 = none)
    int cq_cs_force;              // cluster size while tuning (0 = table/heuristic)
    // sketch contractions (ptt_sketch.cu): smallest M and N of a 64 x 64
    // output tile, and the tile count split-K aims at when the tiles alone
    // cannot fill the device (0 = built-in 48 / 2 x SMs; set by the autotuner)
    int gemm_tm64;
    int gemm_fill;
};

// Per-device one-time set-up (kernel attributes are per device): returns the
// current device's bit of `mask` and whether it was already set.
static inline bool ptt_device_done(std::atomic<unsigned long long>& mask, unsigned long long* bit) {
    int dev = 0;
    cudaGetDevice(&dev);
    *bit = 1ull << (dev & 63);
    return (mask.load() & *bit) != 0;
}

// Programmatic dependent launch.  A kernel launched through ptt_launch may be
// scheduled while the previous kernel on the stream is still running; it must
// start with PTT_PDL_ENTRY(), which waits (griddepcontrol.wait) until the
// previous grid has completed and its writes are visible -- before any memory
// access -- and then lets the next kernel be scheduled in turn.  Launched
// without the attribute, the two instructions have no effect.
#define PTT_PDL_ENTRY()                                          \
    do {                                                         \
        asm volatile("griddepcontrol.wait;" ::: "memory");       \
        asm volatile("griddepcontrol.launch_dependents;" ::: ); \
    } while (0)

template <typename... KArgs, typename... Args>
static inline cudaError_t ptt_launch(const ptt_ctx* c, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                     Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = (c->no_pdl || c->capturing) ? 0 : 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Event pair around a launch of kind `kind` when that class is being timed.
void ptt_time_begin(ptt_ctx* c, int kind);
void ptt_time_end(ptt_ctx* c, int kind);

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
int ptt_ws2_reserve(ptt_ctx* ctx, size_t bytes);
int ptt_pull_desc(ptt_tt* t);
int ptt_ws3_reserve(ptt_ctx* c, size_t bytes);
int ptt_push_desc(ptt_tt* t);
int ptt_set_ranks_async(ptt_tt* t, int k0, const int* vals, int cnt);
int ptt_ones(ptt_ctx* c, int n);  // make c->d_ones hold at least n ones
// Device address of ptt_dot_noalloc's fixed scratch array on `device`
// (looked up once per device; the caller's current device is kept).
int ptt_dot_scratch_init(int device, double** out);
// Autotuner of the sketch contractions' tile and split-K choices (sets
// ctx->gemm_tm64 / gemm_fill; synchronises).
int ptt_gemm_autotune(ptt_ctx* c);

// Swap core[k] <-> alt[k] for k in [k0, k1).
int ptt_swap(ptt_tt* t, int k0, int k1);

// Rounding stages (ptt_round.cu): phases 1 = orthogonalise, 2 = truncate
// (input left-orthogonal), 4 = QR of core `only` alone.
int ptt_round_phases(ptt_tt* x, double tol, const int* maxrank, int phases, int only);
// Run issue() (kernel launches on c->stream only: no allocation, no
// synchronisation) directly, or -- with graphs on and no kernel timing --
// through a CUDA graph cached under `key`, which must hold every value the
// launches bake in (pointers, sizes, scalars): captured on the first call,
// replayed afterwards.
int ptt_graph_run(ptt_ctx* c, const void* key, size_t keylen, const std::function<int()>& issue);
void ptt_graph_clear(ptt_ctx* c);
int ptt_round_phases_rk(ptt_tt* x, const int* rk, double tol, const int* maxrank, int phases, int only);
double ptt_round_threshold(const ptt_tt* x, double tol);

// Blocks per core of a grid-stride launch over d cores (grid y = core): a
// few waves over the device (32 blocks of 256 threads per SM in total).
static inline int ptt_core_grid_cap(const ptt_ctx* c, int d) {
    const int cap = 32 * c->nsm / (d > 0 ? d : 1);
    return cap < 1 ? 1 : cap;
}

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
