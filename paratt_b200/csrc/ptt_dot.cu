// Contractions: inner product, norm, single entry.
//
//  ptt_dot    paratt_dotprod (paratt.c:412-469) via transfer matrices as in
//             pattacInnerProduct (pattac.c:693-741); each step is divided by
//             n_k, which is the reference's 1/sqrt(n_k) scaling of both
//             arguments, so the result is <X, Y> / prod(n).
//  ptt_norm   paratt_norm (paratt.c:369-409) returns ||X||_F / sqrt(prod n);
//             computed here as sqrt(<X,X>/prod n) without touching the gauge
//             (the reference left-orthogonalises its argument in place).
//  ptt_entry  paratt_entry (paratt.c:471-499) -> pattacValue (pattac.c:82-121).
#include "ptt_common.cuh"

#include <mutex>

// T[i, j, e] = sum_k a[i, k] * y[k, j, e]      (a: rx x ry, column-major ld rx)
__global__ void k_dot_t(const DevDesc* X, const DevDesc* Y, int k, const double* a, double* T) {
    const int rx = X->r[k], ry = Y->r[k], n = X->n[k], ry1 = Y->r[k + 1];
    const long long cnt = (long long)rx * n * ry1;
    const double* y = Y->core[k];
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cnt;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % rx);
        const long long je = e / rx;  // j + n*e'
        double acc = 0.0;
        for (int kk = 0; kk < ry; kk++) acc += a[i + (long long)rx * kk] * y[kk + (long long)ry * je];
        T[e] = acc;
    }
}

// a'[b, e] = (1/n) sum_{i,j} x[i, j, b] * T[i, j, e]; one block per (b, e).
__global__ void k_dot_a(const DevDesc* X, const DevDesc* Y, int k, const double* T, double* anew) {
    const int rx = X->r[k], n = X->n[k], rx1 = X->r[k + 1], ry1 = Y->r[k + 1];
    const int b = blockIdx.y, e = blockIdx.x;
    if (b >= rx1 || e >= ry1) return;
    const long long len = (long long)rx * n;
    const double* xb = X->core[k] + len * b;
    const double* te = T + len * e;
    double acc = 0.0;
    for (long long t = threadIdx.x; t < len; t += blockDim.x) acc += xb[t] * te[t];
    __shared__ double red[32];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) anew[b + (long long)rx1 * e] = v / (double)n;
    }
}

__global__ void k_set_one(double* a) { a[0] = 1.0; }

extern "C" int ptt_dot(const ptt_tt* x, const ptt_tt* y, double* out) {
    if (!x || !y || !out || x->d != y->d) return ptt_set_error(PTT_ERR_ARG, "ptt_dot: bad arguments");
    for (int k = 0; k < x->d; k++)
        if (x->n[k] != y->n[k]) return ptt_set_error(PTT_ERR_ARG, "ptt_dot: mode %d differs", k);
    ptt_ctx* c = x->ctx;
    if (y->ctx != c) {
        PTT_CUDA(cudaEventRecord(y->ctx->ev_fork, y->ctx->stream));
        PTT_CUDA(cudaStreamWaitEvent(c->stream, y->ctx->ev_fork, 0));
    }
    long long amax = 1, tmax = 1;
    for (int k = 0; k <= x->d; k++) amax = (long long)x->rcap[k] * y->rcap[k] > amax ? (long long)x->rcap[k] * y->rcap[k] : amax;
    for (int k = 0; k < x->d; k++) {
        long long t = (long long)x->rcap[k] * x->n[k] * y->rcap[k + 1];
        tmax = t > tmax ? t : tmax;
    }
    size_t bytes = sizeof(double) * (size_t)(2 * amax + tmax) + 1024;
    int rc = ptt_ws_reserve(c, bytes);
    if (rc) return rc;
    double* A0 = (double*)c->ws;
    double* A1 = A0 + amax;
    double* T = A1 + amax;
    k_set_one<<<1, 1, 0, c->stream>>>(A0);
    PTT_LAUNCHED(c);
    for (int k = 0; k < x->d; k++) {
        long long tc = (long long)x->rcap[k] * x->n[k] * y->rcap[k + 1];
        int bx = (int)((tc + 255) / 256);
        if (bx > 4096) bx = 4096;
        k_dot_t<<<bx, 256, 0, c->stream>>>(x->dd, y->dd, k, A0, T);
        PTT_LAUNCHED(c);
        k_dot_a<<<dim3(y->rcap[k + 1], x->rcap[k + 1]), 256, 0, c->stream>>>(x->dd, y->dd, k, T, A1);
        PTT_LAUNCHED(c);
        double* s = A0;
        A0 = A1;
        A1 = s;
    }
    PTT_CUDA(cudaMemcpyAsync(c->h_scalars, A0, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    rc = ptt_ctx_synchronize(c);
    if (rc) return rc;
    *out = c->h_scalars[0];
    return PTT_OK;
}

extern "C" int ptt_norm(const ptt_tt* x, double* out) {
    double v = 0.0;
    int rc = ptt_dot(x, x, &v);
    if (rc) return rc;
    *out = sqrt(v > 0.0 ? v : 0.0);
    return PTT_OK;
}

// v <- v * core[k][:, idx, :]  (one block; v has r_k entries)
__global__ void k_entry_step(const DevDesc* X, int k, int idx, const double* vin, double* vout) {
    const int r = X->r[k], n = X->n[k], r1 = X->r[k + 1];
    const double* ck = X->core[k];
    for (int l = threadIdx.x; l < r1; l += blockDim.x) {
        double acc = 0.0;
        for (int i = 0; i < r; i++) acc += vin[i] * ck[i + (long long)r * (idx + (long long)n * l)];
        vout[l] = acc;
    }
}

extern "C" int ptt_entry(const ptt_tt* x, const int* idx, double* out) {
    if (!x || !idx || !out) return ptt_set_error(PTT_ERR_ARG, "ptt_entry: bad arguments");
    for (int k = 0; k < x->d; k++)
        if (idx[k] < 0 || idx[k] >= x->n[k]) return ptt_set_error(PTT_ERR_ARG, "ptt_entry: index %d out of range", k);
    ptt_ctx* c = x->ctx;
    int rmax = 1;
    for (int k = 0; k <= x->d; k++) rmax = x->rcap[k] > rmax ? x->rcap[k] : rmax;
    int rc = ptt_ws_reserve(c, sizeof(double) * 2 * (size_t)rmax + 256);
    if (rc) return rc;
    double* v0 = (double*)c->ws;
    double* v1 = v0 + rmax;
    k_set_one<<<1, 1, 0, c->stream>>>(v0);
    PTT_LAUNCHED(c);
    for (int k = 0; k < x->d; k++) {
        k_entry_step<<<1, 128, 0, c->stream>>>(x->dd, k, idx[k], v0, v1);
        PTT_LAUNCHED(c);
        double* s = v0;
        v0 = v1;
        v1 = s;
    }
    PTT_CUDA(cudaMemcpyAsync(c->h_scalars, v0, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    rc = ptt_ctx_synchronize(c);
    if (rc) return rc;
    *out = c->h_scalars[0];
    return PTT_OK;
}

// ---------------------------------------------------------------------------
// ptt_dot_noalloc: the same inner product with no device allocation.
//
// Some callers cannot let a library call cudaMalloc: a host framework that
// has already reserved the GPU's memory for its own pool, a latency-bound
// loop where cudaMalloc's implicit device-wide synchronisation would stall
// work on other streams, or an embedding that forbids allocation after
// start-up.  This variant keeps its scratch (two transfer matrices and the
// partial contraction T) in a fixed file-scope device array instead of the
// context workspace.  The array is PTT_DOT_NOALLOC_MAX_DOUBLES doubles
// (4 MiB) and exists on every GPU that loads the library until the process
// exits.  Requests that do not fit are rejected with PTT_ERR_CAPACITY.
//
// The array is shared by every call: it keeps the last call's contents, and
// nothing in it has to start at zero (the start value of the transfer matrix
// is written by a kernel of each call).  Two calls whose kernels overlap on
// the GPU (different streams or contexts on one device) race on it.
//
// Host code cannot use the array's name as a device address, so its address
// is looked up once per device (cudaGetSymbolAddress, with that device
// current).  ptt_ctx_create does that lookup for its device, which also loads
// this module (and so reserves the array) while the context is created:
// create the context before handing the GPU's memory to another allocator.
// A call on a device whose address is not known yet (not possible through
// ptt_ctx_create) looks it up itself, so make the first call before any
// stream capture.  The lookup restores the caller's current device and is
// serialised by a mutex, so threads making their first calls at once agree.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double g_dot_scratch[PTT_DOT_NOALLOC_MAX_DOUBLES];

#define PTT_NOALLOC_MAX_DEVICES 64
static std::atomic<double*> g_dot_scratch_addr[PTT_NOALLOC_MAX_DEVICES];
static std::mutex g_dot_scratch_mu;

int ptt_dot_scratch_init(int device, double** out) {
    if (device < 0 || device >= PTT_NOALLOC_MAX_DEVICES)
        return ptt_set_error(PTT_ERR_ARG, "ptt_dot_noalloc: device %d out of range", device);
    double* a = g_dot_scratch_addr[device].load(std::memory_order_acquire);
    if (!a) {
        std::lock_guard<std::mutex> lock(g_dot_scratch_mu);
        a = g_dot_scratch_addr[device].load(std::memory_order_acquire);
        if (!a) {
            int prev = 0;
            PTT_CUDA(cudaGetDevice(&prev));
            void* p = NULL;
            cudaError_t e = cudaSetDevice(device);
            if (e == cudaSuccess) e = cudaGetSymbolAddress(&p, g_dot_scratch);
            const cudaError_t e2 = cudaSetDevice(prev);  // the caller's device, whatever happened
            if (e != cudaSuccess) return ptt_cuda_check(e, "cudaGetSymbolAddress(g_dot_scratch)");
            if (e2 != cudaSuccess) return ptt_cuda_check(e2, "cudaSetDevice (restore)");
            a = (double*)p;
            g_dot_scratch_addr[device].store(a, std::memory_order_release);
        }
    }
    if (out) *out = a;
    return PTT_OK;
}

extern "C" int ptt_dot_noalloc(const ptt_tt* x, const ptt_tt* y, double* out) {
    if (!x || !y || !out || x->d != y->d) return ptt_set_error(PTT_ERR_ARG, "ptt_dot_noalloc: bad arguments");
    for (int k = 0; k < x->d; k++)
        if (x->n[k] != y->n[k]) return ptt_set_error(PTT_ERR_ARG, "ptt_dot_noalloc: mode %d differs", k);
    ptt_ctx* c = x->ctx;
    if (y->ctx != c) {
        PTT_CUDA(cudaEventRecord(y->ctx->ev_fork, y->ctx->stream));
        PTT_CUDA(cudaStreamWaitEvent(c->stream, y->ctx->ev_fork, 0));
    }
    double* scratch = NULL;
    int rc = ptt_dot_scratch_init(c->device, &scratch);
    if (rc) return rc;
    // size the scratch from the actual ranks (reading them synchronises)
    int rx[PTT_MAX_DIM + 1], ry[PTT_MAX_DIM + 1];
    if ((rc = ptt_tt_get_ranks((ptt_tt*)x, rx)) || (rc = ptt_tt_get_ranks((ptt_tt*)y, ry))) return rc;
    long long amax = 1, tmax = 1;
    for (int k = 0; k <= x->d; k++) amax = (long long)rx[k] * ry[k] > amax ? (long long)rx[k] * ry[k] : amax;
    for (int k = 0; k < x->d; k++) {
        const long long t = (long long)rx[k] * x->n[k] * ry[k + 1];
        tmax = t > tmax ? t : tmax;
    }
    if (2 * amax + tmax > PTT_DOT_NOALLOC_MAX_DOUBLES)
        return ptt_set_error(PTT_ERR_CAPACITY,
                             "ptt_dot_noalloc: needs %lld doubles of scratch, the fixed array holds %d "
                             "(use ptt_dot, which allocates)",
                             2 * amax + tmax, (int)PTT_DOT_NOALLOC_MAX_DOUBLES);
    double* A0 = scratch;
    double* A1 = A0 + amax;
    double* T = A1 + amax;
    k_set_one<<<1, 1, 0, c->stream>>>(A0);
    PTT_LAUNCHED(c);
    for (int k = 0; k < x->d; k++) {
        const long long tc = (long long)rx[k] * x->n[k] * ry[k + 1];
        int bx = (int)((tc + 255) / 256);
        if (bx > 4096) bx = 4096;
        k_dot_t<<<bx, 256, 0, c->stream>>>(x->dd, y->dd, k, A0, T);
        PTT_LAUNCHED(c);
        k_dot_a<<<dim3(ry[k + 1], rx[k + 1]), 256, 0, c->stream>>>(x->dd, y->dd, k, T, A1);
        PTT_LAUNCHED(c);
        double* s = A0;
        A0 = A1;
        A1 = s;
    }
    PTT_CUDA(cudaMemcpyAsync(c->h_scalars, A0, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    rc = ptt_ctx_synchronize(c);
    if (rc) return rc;
    *out = c->h_scalars[0];
    return PTT_OK;
}
