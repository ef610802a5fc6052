// Context, device-resident tensor-train container, host<->device transfer.
//
// The reference allocates every core with malloc and grows it with realloc
// (paratt.c:73-162); here the cores of a tensor train live in one HBM
// allocation sized for a rank capacity, with a second buffer per core for
// out-of-place kernels.  Actual ranks are kept on the device (DevDesc).
#include "ptt_common.cuh"

#include <string>
#include <unordered_map>

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static __thread int g_last_error = 0;
static __thread char g_last_msg[512];

int ptt_set_error(int code, const char* fmt, ...) {
    g_last_error = code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_msg, sizeof(g_last_msg), fmt, ap);
    va_end(ap);
    if (code != PTT_OK && getenv("PTT_VERBOSE")) fprintf(stderr, "paratt_b200: %s\n", g_last_msg);
    return code;
}

int ptt_cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return PTT_OK;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return ptt_set_error(PTT_ERR_NOGPU, "%s: %s (this library has no CPU path)", what,
                             cudaGetErrorString(e));
    return ptt_set_error(PTT_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

extern "C" int ptt_last_error(void) { return g_last_error; }
extern "C" const char* ptt_last_error_message(void) { return g_last_msg; }

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
extern "C" ptt_ctx* ptt_ctx_create(int device) {
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        ptt_set_error(PTT_ERR_NOGPU, "no CUDA device (%s): paratt_b200 has no CPU fallback",
                      e == cudaSuccess ? "count 0" : cudaGetErrorString(e));
        return NULL;
    }
    if (device < 0 || device >= ndev) {
        ptt_set_error(PTT_ERR_ARG, "device %d out of range (%d devices)", device, ndev);
        return NULL;
    }
    if (ptt_cuda_check(cudaSetDevice(device), "cudaSetDevice")) return NULL;
    ptt_ctx* c = (ptt_ctx*)calloc(1, sizeof(ptt_ctx));
    c->device = device;
    if (cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || c->nsm < 1) {
        cudaGetLastError();
        c->nsm = 148;
    }
    if (ptt_cuda_check(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream") ||
        ptt_cuda_check(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking), "stream") ||
        ptt_cuda_check(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming), "event") ||
        ptt_cuda_check(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming), "event") ||
        ptt_cuda_check(cudaEventCreateWithFlags(&c->ev_svd[0], cudaEventDisableTiming), "event") ||
        ptt_cuda_check(cudaEventCreateWithFlags(&c->ev_svd[1], cudaEventDisableTiming), "event") ||
        ptt_cuda_check(cudaEventCreateWithFlags(&c->ev_tail[0], cudaEventDisableTiming), "event") ||
        ptt_cuda_check(cudaEventCreateWithFlags(&c->ev_tail[1], cudaEventDisableTiming), "event") ||
        ptt_cuda_check(cudaMalloc(&c->d_status, sizeof(int)), "cudaMalloc status") ||
        ptt_cuda_check(cudaMemset(c->d_status, 0, sizeof(int)), "memset") ||
        ptt_cuda_check(cudaMalloc(&c->d_scalars, 512 * sizeof(double)), "cudaMalloc scalars") ||
        ptt_cuda_check(cudaMallocHost(&c->h_scalars, 512 * sizeof(double)), "cudaMallocHost") ||
        ptt_cuda_check(cudaMalloc(&c->d_stats, sizeof(double) * PTT_STAT_LEN * (PTT_MAX_DIM + 1)), "cudaMalloc stats") ||
        ptt_cuda_check(cudaMalloc(&c->d_work, sizeof(double) * 4), "cudaMalloc work") ||
        ptt_cuda_check(cudaMemset(c->d_work, 0, sizeof(double) * 4), "memset") ||
        ptt_cuda_check(cudaMalloc(&c->d_qrstat, sizeof(long long) * 4), "cudaMalloc qr counters") ||
        ptt_cuda_check(cudaMemset(c->d_qrstat, 0, sizeof(long long) * 4), "memset") ||
        ptt_cuda_check(cudaMemset(c->d_stats, 0, sizeof(double) * PTT_STAT_LEN * (PTT_MAX_DIM + 1)), "memset") ||
        // ptt_dot_noalloc's fixed array: loaded and located now, so its calls
        // never load a module or allocate later
        ptt_dot_scratch_init(device, NULL)) {
        free(c);
        return NULL;
    }
    return c;
}

// ---------------------------------------------------------------------------
// graph cache
// ---------------------------------------------------------------------------
namespace {
struct GraphEntry {
    cudaGraphExec_t exec;
    long long kernels;  // kernel launches the graph holds
};
struct GraphCache {
    std::unordered_map<std::string, GraphEntry> map;
};
constexpr size_t GRAPH_CACHE_MAX = 512;
}  // namespace

void ptt_graph_clear(ptt_ctx* c) {
    GraphCache* g = (GraphCache*)c->graph_cache;
    if (!g) return;
    for (auto& e : g->map) cudaGraphExecDestroy(e.second.exec);
    g->map.clear();
}

int ptt_graph_run(ptt_ctx* c, const void* key, size_t keylen, const std::function<int()>& issue) {
    if (!c->graphs || c->tkind) return issue();
    // inside a capture the caller makes, the launches join the caller's graph
    cudaStreamCaptureStatus cs;
    PTT_CUDA(cudaStreamIsCapturing(c->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return issue();
    GraphCache* g = (GraphCache*)c->graph_cache;
    if (!g) c->graph_cache = g = new GraphCache();
    std::string k((const char*)key, keylen);
    auto it = g->map.find(k);
    if (it != g->map.end()) {
        PTT_CUDA(cudaGraphLaunch(it->second.exec, c->stream));
        c->launches += it->second.kernels;
        return PTT_OK;
    }
    if (g->map.size() >= GRAPH_CACHE_MAX) ptt_graph_clear(c);
    PTT_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const long long l0 = c->launches;
    c->capturing = 1;  // plain launches inside the graph
    int rc = issue();
    c->capturing = 0;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (rc || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return rc ? rc : ptt_cuda_check(e, "graph capture");
    }
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return ptt_cuda_check(e, "graph instantiate");
    g->map.emplace(std::move(k), GraphEntry{exec, c->launches - l0});
    PTT_CUDA(cudaGraphLaunch(exec, c->stream));
    return PTT_OK;
}

extern "C" int ptt_ctx_pdl(ptt_ctx* c, int on) {
    if (!c) return ptt_set_error(PTT_ERR_ARG, "null context");
    c->no_pdl = on ? 0 : 1;
    return PTT_OK;
}

extern "C" int ptt_ctx_cholqr(ptt_ctx* c, int on) {
    if (!c) return ptt_set_error(PTT_ERR_ARG, "null context");
    c->no_cholqr = on ? 0 : 1;
    return PTT_OK;
}

extern "C" int ptt_ctx_qr_counts(ptt_ctx* c, long long* out) {
    if (!c || !out) return ptt_set_error(PTT_ERR_ARG, "ptt_ctx_qr_counts: bad arguments");
    long long v[4] = {0, 0, 0, 0};
    for (int i = -1; i < c->nlanes; i++) {
        ptt_ctx* l = i < 0 ? c : c->lanes[i];
        long long w[4];
        PTT_CUDA(cudaStreamSynchronize(l->stream));
        PTT_CUDA(cudaMemcpy(w, l->d_qrstat, sizeof(w), cudaMemcpyDeviceToHost));
        for (int j = 0; j < 3; j++) v[j] += w[j];
    }
    for (int j = 0; j < 3; j++) out[j] = v[j];
    return PTT_OK;
}

extern "C" int ptt_ctx_graphs(ptt_ctx* c, int on) {
    if (!c) return ptt_set_error(PTT_ERR_ARG, "null context");
    c->graphs = on ? 1 : 0;
    return PTT_OK;
}

extern "C" void ptt_ctx_destroy(ptt_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    cudaStreamSynchronize(c->side);
    ptt_graph_clear(c);
    delete (GraphCache*)c->graph_cache;
    cudaFree(c->ws);
    cudaFree(c->ws2);
    cudaFree(c->ws3);
    cudaFree(c->d_ones);
    cudaFree(c->d_counters);
    for (int i = 0; i < c->nlanes; i++) ptt_ctx_destroy(c->lanes[i]);
    if (!c->shared_status) cudaFree(c->d_status);
    cudaFree(c->d_scalars);
    cudaFree(c->d_stats);
    cudaFree(c->d_work);
    cudaFree(c->d_qrstat);
    cudaFreeHost(c->h_scalars);
    cudaFreeHost(c->h_stage);
    cudaFree(c->d_stage);
    for (int i = 0; i < 64; i++)
        if (c->marks[i]) cudaEventDestroy(c->marks[i]);
    for (int i = 0; i < 2 * c->tcap; i++) cudaEventDestroy(c->tev[i]);
    free(c->tev);
    cudaFree(c->flush);
    cudaEventDestroy(c->ev_fork);
    cudaEventDestroy(c->ev_join);
    for (int i = 0; i < 2; i++) {
        cudaEventDestroy(c->ev_svd[i]);
        cudaEventDestroy(c->ev_tail[i]);
    }
    cudaStreamDestroy(c->stream);
    cudaStreamDestroy(c->side);
    free(c);
}

extern "C" void* ptt_ctx_stream(ptt_ctx* c) { return c ? (void*)c->stream : NULL; }

// ---------------------------------------------------------------------------
// measurement helpers
// ---------------------------------------------------------------------------
extern "C" int ptt_ctx_mark(ptt_ctx* c, int slot) {
    if (!c || slot < 0 || slot >= 64) return ptt_set_error(PTT_ERR_ARG, "ptt_ctx_mark: bad slot");
    if (!c->marks[slot]) PTT_CUDA(cudaEventCreate(&c->marks[slot]));
    PTT_CUDA(cudaEventRecord(c->marks[slot], c->stream));
    return PTT_OK;
}

extern "C" int ptt_ctx_elapsed(ptt_ctx* c, int a, int b, double* ms) {
    if (!c || a < 0 || a >= 64 || b < 0 || b >= 64 || !c->marks[a] || !c->marks[b] || !ms)
        return ptt_set_error(PTT_ERR_ARG, "ptt_ctx_elapsed: bad slots");
    PTT_CUDA(cudaEventSynchronize(c->marks[b]));
    float f = 0.f;
    PTT_CUDA(cudaEventElapsedTime(&f, c->marks[a], c->marks[b]));
    *ms = f;
    return PTT_OK;
}

void ptt_time_begin(ptt_ctx* c, int kind) {
    if (c->tkind != kind || kind == 0) return;
    if (c->tcount >= c->tcap) {
        int ncap = c->tcap ? 2 * c->tcap : 1024;
        cudaEvent_t* ev = (cudaEvent_t*)realloc(c->tev, sizeof(cudaEvent_t) * 2 * ncap);
        for (int i = 2 * c->tcap; i < 2 * ncap; i++) cudaEventCreate(&ev[i]);
        c->tev = ev;
        c->tcap = ncap;
    }
    cudaEventRecord(c->tev[2 * c->tcount], c->stream);
}

void ptt_time_end(ptt_ctx* c, int kind) {
    if (c->tkind != kind || kind == 0) return;
    cudaEventRecord(c->tev[2 * c->tcount + 1], c->stream);
    c->tcount++;
}

extern "C" int ptt_ctx_time_kernels(ptt_ctx* c, int kind) {
    if (!c) return ptt_set_error(PTT_ERR_ARG, "null context");
    c->tkind = kind;
    c->tcount = 0;
    c->tms = 0.0;
    c->tlaunches = 0;
    for (int i = 0; i < 4; i++) c->hwork[i] = 0.0;
    PTT_CUDA(cudaMemsetAsync(c->d_work, 0, sizeof(double) * 4, c->stream));
    return PTT_OK;
}

// Resolve the recorded launches: total milliseconds and launch count since
// ptt_ctx_time_kernels (synchronises).
extern "C" int ptt_ctx_kernel_work(ptt_ctx* c, double* work) {
    if (!c || !work) return ptt_set_error(PTT_ERR_ARG, "bad arguments");
    double w[4];
    PTT_CUDA(cudaStreamSynchronize(c->stream));
    PTT_CUDA(cudaMemcpy(w, c->d_work, sizeof(w), cudaMemcpyDeviceToHost));
    const int k = c->tkind;
    *work = (k >= 0 && k < 4) ? w[k] + c->hwork[k] : 0.0;
    return PTT_OK;
}

extern "C" int ptt_ctx_kernel_time(ptt_ctx* c, double* ms, long long* count) {
    if (!c) return ptt_set_error(PTT_ERR_ARG, "null context");
    PTT_CUDA(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < c->tcount; i++) {
        float f = 0.f;
        PTT_CUDA(cudaEventElapsedTime(&f, c->tev[2 * i], c->tev[2 * i + 1]));
        c->tms += f;
    }
    c->tlaunches += c->tcount;
    c->tcount = 0;
    if (ms) *ms = c->tms;
    if (count) *count = c->tlaunches;
    return PTT_OK;
}

__global__ void k_flush(double* p, long long n, double v) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = v;
}

// Overwrite a buffer twice the size of L2 so the next kernel starts cold.
extern "C" int ptt_ctx_flush_l2(ptt_ctx* c) {
    if (!c) return ptt_set_error(PTT_ERR_ARG, "null context");
    if (!c->flush) {
        int l2 = 0;
        PTT_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, c->device));
        c->flush_bytes = (size_t)(l2 > 0 ? l2 : (128 << 20)) * 2;
        PTT_CUDA(cudaMalloc(&c->flush, c->flush_bytes));
    }
    k_flush<<<1184, 256, 0, c->stream>>>((double*)c->flush, (long long)(c->flush_bytes / 8), 0.0);
    PTT_LAUNCHED(c);
    return PTT_OK;
}

extern "C" int ptt_host_pin(void* p, unsigned long long bytes) {
    PTT_CUDA(cudaHostRegister(p, bytes, cudaHostRegisterDefault));
    return PTT_OK;
}

extern "C" int ptt_host_unpin(void* p) {
    PTT_CUDA(cudaHostUnregister(p));
    return PTT_OK;
}
extern "C" long long ptt_ctx_launch_count(const ptt_ctx* c) { return c ? c->launches : 0; }

extern "C" int ptt_ctx_synchronize(ptt_ctx* c) {
    if (!c) return ptt_set_error(PTT_ERR_ARG, "null context");
    PTT_CUDA(cudaStreamSynchronize(c->side));
    PTT_CUDA(cudaStreamSynchronize(c->stream));
    int st = 0;
    PTT_CUDA(cudaMemcpy(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st) {
        PTT_CUDA(cudaMemset(c->d_status, 0, sizeof(int)));
        const char* what = st == PTT_ERR_CAPACITY ? "rank exceeds capacity"
                         : st == PTT_ERR_TIMEOUT  ? "device wait timed out"
                         : st == PTT_ERR_NUMERIC  ? "non-finite value or solver did not converge"
                                                  : "device error";
        return ptt_set_error(st, "device status %d: %s", st, what);
    }
    return PTT_OK;
}

int ptt_ws_reserve(ptt_ctx* c, size_t bytes) {
    if (bytes <= c->ws_bytes) return PTT_OK;
    PTT_CUDA(cudaStreamSynchronize(c->stream));
    PTT_CUDA(cudaStreamSynchronize(c->side));
    if (c->ws) PTT_CUDA(cudaFree(c->ws));
    c->ws = NULL;
    c->ws_bytes = 0;
    size_t b = ptt_align(bytes + bytes / 4);
    PTT_CUDA(cudaMalloc(&c->ws, b));
    c->ws_bytes = b;
    return PTT_OK;
}

int ptt_ws3_reserve(ptt_ctx* c, size_t bytes) {
    if (bytes <= c->ws3_bytes) return PTT_OK;
    PTT_CUDA(cudaStreamSynchronize(c->stream));
    PTT_CUDA(cudaStreamSynchronize(c->side));
    if (c->ws3) PTT_CUDA(cudaFree(c->ws3));
    c->ws3 = NULL;
    c->ws3_bytes = 0;
    size_t b = ptt_align(bytes + bytes / 4);
    PTT_CUDA(cudaMalloc(&c->ws3, b));
    c->ws3_bytes = b;
    return PTT_OK;
}

int ptt_ws2_reserve(ptt_ctx* c, size_t bytes) {
    if (bytes <= c->ws2_bytes) return PTT_OK;
    PTT_CUDA(cudaStreamSynchronize(c->stream));
    PTT_CUDA(cudaStreamSynchronize(c->side));
    if (c->ws2) PTT_CUDA(cudaFree(c->ws2));
    c->ws2 = NULL;
    c->ws2_bytes = 0;
    size_t b = ptt_align(bytes + bytes / 4);
    PTT_CUDA(cudaMalloc(&c->ws2, b));
    c->ws2_bytes = b;
    return PTT_OK;
}

// Write ranks r[k0 .. k0+cnt) of the device descriptor (stream-ordered).
// The values travel as a kernel argument, so the call neither stages through
// host memory nor waits for the stream.
struct RankVals {
    int v[PTT_MAX_DIM + 1];
};

__global__ void k_set_ranks(DevDesc* D, int k0, int cnt, RankVals rv) {
    PTT_PDL_ENTRY();
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) D->r[k0 + i] = rv.v[i];
}

int ptt_set_ranks_async(ptt_tt* t, int k0, const int* vals, int cnt) {
    if (k0 < 0 || cnt < 0 || k0 + cnt > t->d + 1) return ptt_set_error(PTT_ERR_ARG, "rank range");
    RankVals rv;
    memcpy(rv.v, vals, sizeof(int) * cnt);
    PTT_CUDA(ptt_launch(t->ctx, k_set_ranks, dim3(1), dim3(128), 0, t->dd, k0, cnt, rv));
    PTT_LAUNCHED(t->ctx);
    return PTT_OK;
}

__global__ void k_ones(double* p, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = 1.0;
}

int ptt_ones(ptt_ctx* c, int n) {
    if (n <= c->ones_n) return PTT_OK;
    PTT_CUDA(cudaStreamSynchronize(c->stream));
    if (c->d_ones) PTT_CUDA(cudaFree(c->d_ones));
    PTT_CUDA(cudaMalloc(&c->d_ones, sizeof(double) * (size_t)n));
    k_ones<<<(n + 255) / 256, 256, 0, c->stream>>>(c->d_ones, n);
    PTT_LAUNCHED(c);
    c->ones_n = n;
    return PTT_OK;
}

int ptt_counters_reserve(ptt_ctx* c, size_t n) {
    if (n <= c->counters_n) return PTT_OK;
    PTT_CUDA(cudaStreamSynchronize(c->stream));
    PTT_CUDA(cudaStreamSynchronize(c->side));
    if (c->d_counters) PTT_CUDA(cudaFree(c->d_counters));
    size_t m = n < 4096 ? 4096 : 2 * n;
    PTT_CUDA(cudaMalloc(&c->d_counters, m * sizeof(int)));
    PTT_CUDA(cudaMemset(c->d_counters, 0, m * sizeof(int)));
    c->counters_n = m;
    return PTT_OK;
}

// ---------------------------------------------------------------------------
// tensor trains
// ---------------------------------------------------------------------------
static int alloc_cores(ptt_tt* t) {
    for (int k = 0; k < t->d; k++) {
        long long cap = (long long)t->rcap[k] * t->n[k] * t->rcap[k + 1];
        t->cap[k] = cap;
        t->hd.cap[k] = cap;
        PTT_CUDA(cudaMalloc(&t->hd.core[k], ptt_align(cap * sizeof(double))));
        PTT_CUDA(cudaMalloc(&t->hd.alt[k], ptt_align(cap * sizeof(double))));
    }
    return PTT_OK;
}

extern "C" ptt_tt* ptt_tt_create(ptt_ctx* ctx, int d, const int* n, const int* rank_cap) {
    if (!ctx || d < 1 || d > PTT_MAX_DIM || !n || !rank_cap) {
        ptt_set_error(PTT_ERR_ARG, "ptt_tt_create: bad arguments (d=%d)", d);
        return NULL;
    }
    if (rank_cap[0] != 1 || rank_cap[d] != 1) {
        ptt_set_error(PTT_ERR_ARG, "ptt_tt_create: boundary ranks must be 1");
        return NULL;
    }
    for (int k = 0; k < d; k++)
        if (n[k] < 1 || rank_cap[k] < 1 || rank_cap[k + 1] < 1) {
            ptt_set_error(PTT_ERR_ARG, "ptt_tt_create: bad size at mode %d", k);
            return NULL;
        }
    if (ptt_cuda_check(cudaSetDevice(ctx->device), "cudaSetDevice")) return NULL;
    ptt_tt* t = (ptt_tt*)calloc(1, sizeof(ptt_tt));
    t->ctx = ctx;
    t->d = d;
    t->hd.d = d;
    for (int k = 0; k < d; k++) t->n[k] = t->hd.n[k] = n[k];
    for (int k = 0; k <= d; k++) {
        t->rcap[k] = t->hd.rcap[k] = rank_cap[k];
        t->hd.r[k] = 1;
    }
    if (alloc_cores(t) || ptt_cuda_check(cudaMalloc(&t->dd, sizeof(DevDesc)), "cudaMalloc desc") ||
        ptt_cuda_check(cudaMemcpyAsync(t->dd, &t->hd, sizeof(DevDesc), cudaMemcpyHostToDevice, ctx->stream),
                       "desc upload") ||
        ptt_cuda_check(cudaStreamSynchronize(ctx->stream), "sync")) {
        ptt_tt_destroy(t);
        return NULL;
    }
    return t;
}

extern "C" void ptt_tt_destroy(ptt_tt* t) {
    if (!t) return;
    cudaStreamSynchronize(t->ctx->stream);
    cudaStreamSynchronize(t->ctx->side);
    for (int k = 0; k < t->d; k++) {
        cudaFree(t->hd.core[k]);
        cudaFree(t->hd.alt[k]);
    }
    cudaFree(t->dd);
    free(t);
}

extern "C" int ptt_tt_shape(const ptt_tt* t, int* d, int* n, int* rank_cap) {
    if (!t) return ptt_set_error(PTT_ERR_ARG, "null tt");
    if (d) *d = t->d;
    if (n) memcpy(n, t->n, sizeof(int) * t->d);
    if (rank_cap) memcpy(rank_cap, t->rcap, sizeof(int) * (t->d + 1));
    return PTT_OK;
}

// Pull the device descriptor (current buffer order and ranks) to the host.
int ptt_pull_desc(ptt_tt* t) {
    PTT_CUDA(cudaStreamSynchronize(t->ctx->side));
    PTT_CUDA(cudaMemcpyAsync(&t->hd, t->dd, sizeof(DevDesc), cudaMemcpyDeviceToHost, t->ctx->stream));
    PTT_CUDA(cudaStreamSynchronize(t->ctx->stream));
    return PTT_OK;
}

int ptt_push_desc(ptt_tt* t) {
    PTT_CUDA(cudaMemcpyAsync(t->dd, &t->hd, sizeof(DevDesc), cudaMemcpyHostToDevice, t->ctx->stream));
    return PTT_OK;
}

extern "C" int ptt_tt_reserve(ptt_tt* t, const int* rank_cap) {
    if (!t || !rank_cap) return ptt_set_error(PTT_ERR_ARG, "ptt_tt_reserve: bad arguments");
    int grow = 0;
    for (int k = 0; k <= t->d; k++) grow |= rank_cap[k] > t->rcap[k];
    if (!grow) return PTT_OK;
    if (rank_cap[0] != 1 || rank_cap[t->d] != 1)
        return ptt_set_error(PTT_ERR_ARG, "ptt_tt_reserve: boundary ranks must be 1");
    int rc = ptt_pull_desc(t);
    if (rc) return rc;
    for (int k = 0; k <= t->d; k++)
        if (rank_cap[k] > t->rcap[k]) t->rcap[k] = t->hd.rcap[k] = rank_cap[k];
    for (int k = 0; k < t->d; k++) {
        long long cap = (long long)t->rcap[k] * t->n[k] * t->rcap[k + 1];
        if (cap <= t->cap[k]) continue;
        double *nc = NULL, *na = NULL;
        PTT_CUDA(cudaMalloc(&nc, ptt_align(cap * sizeof(double))));
        PTT_CUDA(cudaMalloc(&na, ptt_align(cap * sizeof(double))));
        PTT_CUDA(cudaMemcpyAsync(nc, t->hd.core[k], t->cap[k] * sizeof(double), cudaMemcpyDeviceToDevice,
                                 t->ctx->stream));
        PTT_CUDA(cudaStreamSynchronize(t->ctx->stream));
        cudaFree(t->hd.core[k]);
        cudaFree(t->hd.alt[k]);
        t->hd.core[k] = nc;
        t->hd.alt[k] = na;
        t->cap[k] = t->hd.cap[k] = cap;
    }
    rc = ptt_push_desc(t);
    if (rc) return rc;
    PTT_CUDA(cudaStreamSynchronize(t->ctx->stream));
    return PTT_OK;
}

// Whole-train host transfers.  Cores in pageable host memory (the reference
// API's malloc'd cores) go through one page-locked staging buffer: the host
// packs them contiguously, one bulk copy crosses PCIe, and one kernel
// scatters them to (or gathers them from) the device cores -- instead of a
// pageable copy per core, each with its own staging and, device to host, its
// own synchronisation.  Other memory (device, managed, page-locked) is copied
// core by core.
struct StageMap {
    double* core[PTT_MAX_DIM];
    long long off[PTT_MAX_DIM + 1];
};
__global__ void k_stage_scatter(const double* src, StageMap m) {
    const int k = blockIdx.y;
    const long long a = m.off[k], n = m.off[k + 1] - a;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        m.core[k][e] = src[a + e];
}
__global__ void k_stage_gather(double* dst, StageMap m) {
    const int k = blockIdx.y;
    const long long a = m.off[k], n = m.off[k + 1] - a;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        dst[a + e] = m.core[k][e];
}

static bool all_pageable(const void* const* p, int d) {
    for (int k = 0; k < d; k++) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, p[k]) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        if (a.type != cudaMemoryTypeUnregistered) return false;
    }
    return true;
}

// staging for n doubles; callers leave no transfer in flight on the buffers
// (ptt_tt_set and ptt_tt_get end with a stream synchronisation)
static int stage_reserve(ptt_ctx* c, size_t n) {
    if (n > c->h_stage_n) {
        cudaFreeHost(c->h_stage);
        c->h_stage = nullptr;
        c->h_stage_n = 0;
        const size_t m = n < (1u << 16) ? (1u << 16) : n + n / 2;
        PTT_CUDA(cudaMallocHost(&c->h_stage, m * sizeof(double)));
        c->h_stage_n = m;
    }
    if (n > c->d_stage_n) {
        PTT_CUDA(cudaStreamSynchronize(c->stream));
        cudaFree(c->d_stage);
        c->d_stage = nullptr;
        c->d_stage_n = 0;
        const size_t m = n < (1u << 16) ? (1u << 16) : n + n / 2;
        PTT_CUDA(cudaMalloc(&c->d_stage, m * sizeof(double)));
        c->d_stage_n = m;
    }
    return PTT_OK;
}

static int stage_grid(const StageMap& m, int d) {
    long long mx = 0;
    for (int k = 0; k < d; k++) mx = (m.off[k + 1] - m.off[k]) > mx ? (m.off[k + 1] - m.off[k]) : mx;
    long long g = (mx + 255) / 256;
    return (int)(g < 1 ? 1 : (g > 64 ? 64 : g));
}

extern "C" int ptt_tt_set(ptt_tt* t, const int* ranks, const double* const* cores) {
    if (!t || !ranks || !cores) return ptt_set_error(PTT_ERR_ARG, "ptt_tt_set: bad arguments");
    if (ranks[0] != 1 || ranks[t->d] != 1) return ptt_set_error(PTT_ERR_ARG, "ptt_tt_set: boundary ranks must be 1");
    int need = 0;
    for (int k = 0; k <= t->d; k++) {
        if (ranks[k] < 1) return ptt_set_error(PTT_ERR_ARG, "ptt_tt_set: rank %d < 1", k);
        need |= ranks[k] > t->rcap[k];
    }
    if (need) {
        int rc[PTT_MAX_DIM + 1];
        for (int k = 0; k <= t->d; k++) rc[k] = ranks[k] > t->rcap[k] ? ranks[k] : t->rcap[k];
        int e = ptt_tt_reserve(t, rc);
        if (e) return e;
    }
    int rc = ptt_pull_desc(t);
    if (rc) return rc;
    StageMap m;
    m.off[0] = 0;
    for (int k = 0; k < t->d; k++) {
        m.core[k] = t->hd.core[k];
        m.off[k + 1] = m.off[k] + (long long)ranks[k] * t->n[k] * ranks[k + 1];
    }
    ptt_ctx* c = t->ctx;
    if (m.off[t->d] > 0 && all_pageable((const void* const*)cores, t->d)) {
        if ((rc = stage_reserve(c, (size_t)m.off[t->d]))) return rc;
        for (int k = 0; k < t->d; k++)
            memcpy(c->h_stage + m.off[k], cores[k], sizeof(double) * (size_t)(m.off[k + 1] - m.off[k]));
        PTT_CUDA(cudaMemcpyAsync(c->d_stage, c->h_stage, sizeof(double) * (size_t)m.off[t->d],
                                 cudaMemcpyHostToDevice, c->stream));
        k_stage_scatter<<<dim3(stage_grid(m, t->d), t->d), 256, 0, c->stream>>>(c->d_stage, m);
        PTT_LAUNCHED(c);
    } else {
        for (int k = 0; k < t->d; k++) {
            size_t cnt = (size_t)ranks[k] * t->n[k] * ranks[k + 1];
            PTT_CUDA(cudaMemcpyAsync(t->hd.core[k], cores[k], cnt * sizeof(double), cudaMemcpyDefault,
                                     t->ctx->stream));
        }
    }
    for (int k = 0; k <= t->d; k++) t->hd.r[k] = ranks[k];
    rc = ptt_push_desc(t);
    if (rc) return rc;
    PTT_CUDA(cudaStreamSynchronize(t->ctx->stream));
    return PTT_OK;
}

extern "C" int ptt_tt_get_ranks(ptt_tt* t, int* ranks) {
    if (!t || !ranks) return ptt_set_error(PTT_ERR_ARG, "ptt_tt_get_ranks: bad arguments");
    PTT_CUDA(cudaStreamSynchronize(t->ctx->side));
    PTT_CUDA(cudaMemcpyAsync(t->ctx->h_scalars, t->dd->r, sizeof(int) * (t->d + 1), cudaMemcpyDeviceToHost,
                             t->ctx->stream));
    PTT_CUDA(cudaStreamSynchronize(t->ctx->stream));
    memcpy(ranks, t->ctx->h_scalars, sizeof(int) * (t->d + 1));
    return PTT_OK;
}

extern "C" int ptt_tt_get(ptt_tt* t, int* ranks, double* const* cores) {
    if (!t) return ptt_set_error(PTT_ERR_ARG, "ptt_tt_get: null tt");
    int rc = ptt_pull_desc(t);
    if (rc) return rc;
    if (ranks) memcpy(ranks, t->hd.r, sizeof(int) * (t->d + 1));
    if (cores) {
        StageMap m;
        m.off[0] = 0;
        for (int k = 0; k < t->d; k++) {
            m.core[k] = t->hd.core[k];
            m.off[k + 1] = m.off[k] + (long long)t->hd.r[k] * t->n[k] * t->hd.r[k + 1];
        }
        ptt_ctx* c = t->ctx;
        if (m.off[t->d] > 0 && all_pageable((const void* const*)cores, t->d)) {
            if ((rc = stage_reserve(c, (size_t)m.off[t->d]))) return rc;
            k_stage_gather<<<dim3(stage_grid(m, t->d), t->d), 256, 0, c->stream>>>(c->d_stage, m);
            PTT_LAUNCHED(c);
            PTT_CUDA(cudaMemcpyAsync(c->h_stage, c->d_stage, sizeof(double) * (size_t)m.off[t->d],
                                     cudaMemcpyDeviceToHost, c->stream));
            rc = ptt_ctx_synchronize(c);
            for (int k = 0; k < t->d; k++)
                memcpy(cores[k], c->h_stage + m.off[k], sizeof(double) * (size_t)(m.off[k + 1] - m.off[k]));
            return rc;
        }
        for (int k = 0; k < t->d; k++) {
            size_t cnt = (size_t)t->hd.r[k] * t->n[k] * t->hd.r[k + 1];
            PTT_CUDA(cudaMemcpyAsync(cores[k], t->hd.core[k], cnt * sizeof(double), cudaMemcpyDefault,
                                     t->ctx->stream));
        }
        // the data is on the host: report (and clear) a device-side error of
        // the work that produced it, as ptt_ctx_synchronize does
        return ptt_ctx_synchronize(t->ctx);
    }
    return PTT_OK;
}

extern "C" ptt_ctx* ptt_tt_context(const ptt_tt* t) { return t ? t->ctx : NULL; }

extern "C" int ptt_tt_device_cores(const ptt_tt* t, double** cores, int** ranks) {
    if (!t) return ptt_set_error(PTT_ERR_ARG, "null tt");
    int rc = ptt_pull_desc((ptt_tt*)t);
    if (rc) return rc;
    if (cores)
        for (int k = 0; k < t->d; k++) cores[k] = t->hd.core[k];
    if (ranks) *ranks = t->dd->r;
    return PTT_OK;
}

// ---------------------------------------------------------------------------
// copy and swap kernels
// ---------------------------------------------------------------------------
__global__ void k_swap(DevDesc* D, int k0, int k1) {
    int k = k0 + threadIdx.x;
    if (k < k1) {
        double* a = D->core[k];
        D->core[k] = D->alt[k];
        D->alt[k] = a;
    }
}

int ptt_swap(ptt_tt* t, int k0, int k1) {
    if (k1 <= k0) return PTT_OK;
    k_swap<<<1, 128, 0, t->ctx->stream>>>(t->dd, k0, k1);
    PTT_LAUNCHED(t->ctx);
    return PTT_OK;
}

__global__ void k_copy_tt(DevDesc* S, DevDesc* Dst, int* status) {
    int k = blockIdx.y;
    int d = S->d;
    if (k >= d) return;
    long long cnt = (long long)S->r[k] * S->n[k] * S->r[k + 1];
    if (S->r[k] > Dst->rcap[k] || S->r[k + 1] > Dst->rcap[k + 1] || cnt > Dst->cap[k]) {
        if (threadIdx.x == 0 && blockIdx.x == 0) PTT_STATUS_SET(status, PTT_ERR_CAPACITY);
        return;
    }
    const double* s = S->core[k];
    double* o = Dst->core[k];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
         i += (long long)gridDim.x * blockDim.x)
        o[i] = s[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        Dst->r[k] = S->r[k];
        if (k == d - 1) Dst->r[d] = S->r[d];
    }
}

extern "C" int ptt_tt_copy(ptt_tt* dst, const ptt_tt* src) {
    if (!dst || !src || dst->d != src->d) return ptt_set_error(PTT_ERR_ARG, "ptt_tt_copy: shape mismatch");
    for (int k = 0; k < src->d; k++)
        if (dst->n[k] != src->n[k]) return ptt_set_error(PTT_ERR_ARG, "ptt_tt_copy: mode %d differs", k);
    if (dst == src) return PTT_OK;
    int rc = ptt_tt_reserve(dst, src->rcap);
    if (rc) return rc;
    ptt_ctx* c = dst->ctx;
    long long mx = 0;
    for (int k = 0; k < src->d; k++) mx = src->cap[k] > mx ? src->cap[k] : mx;
    int bx = (int)((mx + 255) / 256);
    // a few waves over the GPU in total; the loop strides over any core size
    const int bcap = ptt_core_grid_cap(c, src->d);
    if (bx > bcap) bx = bcap;
    if (src->ctx != c) {
        PTT_CUDA(cudaEventRecord(src->ctx->ev_fork, src->ctx->stream));
        PTT_CUDA(cudaStreamWaitEvent(c->stream, src->ctx->ev_fork, 0));
    }
    k_copy_tt<<<dim3(bx, src->d), 256, 0, c->stream>>>(src->dd, dst->dd, c->d_status);
    PTT_LAUNCHED(c);
    return PTT_OK;
}

extern "C" int ptt_ctx_workspace_bytes(const ptt_ctx* c, unsigned long long* bytes) {
    if (!c || !bytes) return ptt_set_error(PTT_ERR_ARG, "ptt_ctx_workspace_bytes: bad arguments");
    unsigned long long b = (unsigned long long)(c->ws_bytes + c->ws2_bytes + c->ws3_bytes + c->flush_bytes) +
                           (unsigned long long)c->counters_n * sizeof(int) + (unsigned long long)c->ones_n * sizeof(double);
    for (int i = 0; i < c->nlanes; i++) {
        unsigned long long lb = 0;
        if (c->lanes[i] && ptt_ctx_workspace_bytes(c->lanes[i], &lb) == PTT_OK) b += lb;
    }
    *bytes = b;
    return PTT_OK;
}

extern "C" int ptt_ctx_mem_info(const ptt_ctx* c, unsigned long long* free_bytes, unsigned long long* total_bytes) {
    if (!c) return ptt_set_error(PTT_ERR_ARG, "ptt_ctx_mem_info: null context");
    int prev = 0;
    PTT_CUDA(cudaGetDevice(&prev));
    size_t f = 0, t = 0;
    cudaError_t e = cudaSetDevice(c->device);
    if (e == cudaSuccess) e = cudaMemGetInfo(&f, &t);
    const cudaError_t e2 = cudaSetDevice(prev);
    if (e != cudaSuccess) return ptt_cuda_check(e, "cudaMemGetInfo");
    if (e2 != cudaSuccess) return ptt_cuda_check(e2, "cudaSetDevice (restore)");
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
    return PTT_OK;
}
