// Formal TT arithmetic and mode-local operators (HBM-bound kernels).
//
//  axpby     attacFormalAXPBY   attac.c:81-112, wrapper paratt.c:237-268
//  hadamard  attacHadamard      attac.c:128-136 with attacKron utilities.c:112-129
//  square_sym  x (.) x at rank r(r+1)/2 (no reference counterpart; same tensor)
//  scale     attac_tt_scale     paratt.c:271-281
//  diag      attac_mult_diag_mat paratt.c:571-581
//  stencil   attac_apply_periodic_stencil paratt.c:584-661
//
// Every kernel reads ranks from the device descriptors, writes its result to
// the output's second buffer and the new ranks to a scratch array; a one-block
// finalize kernel then swaps the buffers and publishes the ranks.  This keeps
// the ops safe when the output aliases an input and free of host syncs.
#include "ptt_common.cuh"

#include <string.h>

#define PTT_MAX_STENCIL 15

struct Stencil {
    double s[PTT_MAX_STENCIL];
    int len;
};

// grid: (blocks, cores). One block per (slab chunk, core).
static inline int elem_blocks(long long maxcnt) {
    long long b = (maxcnt + 255) / 256;
    if (b > 2048) b = 2048;
    if (b < 1) b = 1;
    return (int)b;
}

// Blocks per core of an element-wise launch over all d cores (grid y =
// core): sized by the largest capacity, capped at a few waves over the
// device; the grid-stride loops cover any core with any grid.
static inline int core_blocks(const ptt_ctx* c, long long maxcnt, int d) {
    const int b = elem_blocks(maxcnt);
    const int cap = ptt_core_grid_cap(c, d);
    return b < cap ? b : cap;
}

// Fibers of a core: element (i, f) at i + R f, f = j + n l (the column-major
// core seen as R x (n R1)).  A group of G lanes (a power of two; 32 once
// R >= 32) takes one fiber at a time, so a fiber's rows are contiguous
// accesses of consecutive lanes and (j, l) cost one 32-bit division per
// fiber instead of 64-bit divisions per element.
struct FiberIter {
    int G, li;
    long long f0, fstep;
};
__device__ __forceinline__ FiberIter fiber_iter(int R) {
    FiberIter it;
    int G = 32;
    if (R < 32) {
        G = 1;
        while (G < R) G <<= 1;
    }
    const int lane = threadIdx.x & 31;
    const int per = 32 / G;
    it.G = G;
    it.li = lane & (G - 1);
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    it.f0 = warp * per + lane / G;
    it.fstep = nw * per;
    return it;
}

// Blocks per core of a fiber launch over d cores (grid y = core): enough for
// the largest core's fibers at 8 per block (one per warp of 256 threads),
// capped at 32 blocks per SM over the whole grid.
static inline int fiber_blocks(const ptt_ctx* c, const ptt_tt* z, int d) {
    long long nf = 1;
    for (int k = 0; k < d; k++) {
        const long long f = (long long)z->n[k] * z->rcap[k + 1];
        nf = f > nf ? f : nf;
    }
    long long b = (nf + 7) / 8;
    const long long cap = ptt_core_grid_cap(c, d);
    if (b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

// ---------------------------------------------------------------------------
// finalize: publish ranks computed by a kernel and swap the written cores
// ---------------------------------------------------------------------------
__global__ void k_finalize(DevDesc* Z, const int* newr, int k0, int k1, int set_ranks) {
    int d = Z->d;
    for (int k = threadIdx.x; k <= d; k += blockDim.x)
        if (set_ranks) Z->r[k] = newr[k];
    for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        double* a = Z->core[k];
        Z->core[k] = Z->alt[k];
        Z->alt[k] = a;
    }
}

static int finalize(ptt_tt* z, int* newr, int k0, int k1, int set_ranks) {
    k_finalize<<<1, 128, 0, z->ctx->stream>>>(z->dd, newr, k0, k1, set_ranks);
    PTT_LAUNCHED(z->ctx);
    return PTT_OK;
}

// new ranks of an op, published by the finalize kernel (512 doubles = 1024 ints)
static int* ranks_scratch(ptt_ctx* c, int d) {
    if (d + 1 <= 1024) return (int*)c->d_scalars;
    return NULL;
}

// ---------------------------------------------------------------------------
// axpby
// ---------------------------------------------------------------------------
__global__ void k_axpby(const DevDesc* X, const DevDesc* Y, DevDesc* Z, double a, double b, int* newr,
                        int* status) {
    const int k = blockIdx.y;
    const int d = X->d;
    const int rx = X->r[k], rx1 = X->r[k + 1], ry = Y->r[k], ry1 = Y->r[k + 1];
    const int n = X->n[k];
    int rz, rz1;
    if (d == 1) {
        rz = 1;
        rz1 = 1;
    } else {
        rz = (k == 0) ? 1 : rx + ry;
        rz1 = (k == d - 1) ? 1 : rx1 + ry1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        newr[k] = rz;
        if (k == d - 1) newr[d] = 1;
    }
    const long long cnt = (long long)rz * n * rz1;
    if (rz > Z->rcap[k] || rz1 > Z->rcap[k + 1] || cnt > Z->cap[k]) {
        if (blockIdx.x == 0 && threadIdx.x == 0) PTT_STATUS_SET(status, PTT_ERR_CAPACITY);
        return;
    }
    const double* xc = X->core[k];
    const double* yc = Y->core[k];
    double* zc = Z->alt[k];
    if (d == 1) {
        const long long stride = (long long)gridDim.x * blockDim.x;
        for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += stride)
            zc[e] = a * xc[e] + b * yc[e];
        return;
    }
    // fiber (j, l) of z: x's fiber over zeros (l < rx1), zeros over y's fiber
    // (l >= rx1); core 0 is [a x_0 | b y_0], the last core stacks x over y
    const int NF = n * rz1;
    const FiberIter it = fiber_iter(rz);
    for (long long f = it.f0; f < NF; f += it.fstep) {
        const int fi = (int)f, l = fi / n, j = fi - l * n;
        double* zf = zc + (long long)rz * fi;
        if (k == 0) {
            if (it.li == 0) zf[0] = (l < rx1) ? a * xc[j + (long long)n * l] : b * yc[j + (long long)n * (l - rx1)];
        } else if (k == d - 1) {
#pragma unroll 4
            for (int i = it.li; i < rz; i += it.G)
                zf[i] = (i < rx) ? xc[i + (long long)rx * j] : yc[(i - rx) + (long long)ry * j];
        } else if (l < rx1) {
            const double* src = xc + (long long)rx * (j + (long long)n * l);
#pragma unroll 4
            for (int i = it.li; i < rz; i += it.G) zf[i] = (i < rx) ? src[i] : 0.0;
        } else {
            const double* src = yc + (long long)ry * (j + (long long)n * (l - rx1));
#pragma unroll 4
            for (int i = it.li; i < rz; i += it.G) zf[i] = (i >= rx) ? src[i - rx] : 0.0;
        }
    }
}

// Make z's rank capacity cover an op's output.  need[] is the bound from the
// inputs' capacities; when z already covers it nothing happens (no sync).
// Otherwise the inputs' actual ranks are read back (synchronises) and z is
// grown only to the exact output ranks: op 0 = sum (r_x + r_y), 1 = product,
// 2 = operator sum (2 r_x; y unused), 3 = symmetric square (r_x (r_x + 1) / 2).
static int fit_output(ptt_tt* z, const int* need, const ptt_tt* x, const ptt_tt* y, int op) {
    const int d = z->d;
    int ok = 1;
    for (int k = 0; k <= d; k++) ok &= need[k] <= z->rcap[k];
    if (ok) return PTT_OK;
    int rx[PTT_MAX_DIM + 1], ry[PTT_MAX_DIM + 1], ex[PTT_MAX_DIM + 1];
    int rc;
    if ((rc = ptt_tt_get_ranks((ptt_tt*)x, rx))) return rc;
    if (op < 2 && (rc = ptt_tt_get_ranks((ptt_tt*)y, ry))) return rc;
    for (int k = 0; k <= d; k++) {
        if (op == 0)
            ex[k] = (k == 0 || k == d) ? 1 : rx[k] + ry[k];
        else if (op == 1)
            ex[k] = rx[k] * ry[k];
        else if (op == 3)
            ex[k] = rx[k] * (rx[k] + 1) / 2;
        else
            ex[k] = (k == 0 || k == d) ? 1 : 2 * rx[k];
        if (ex[k] < z->rcap[k]) ex[k] = z->rcap[k];
    }
    return ptt_tt_reserve(z, ex);
}

static int check_same_modes(const ptt_tt* x, const ptt_tt* y) {
    if (!x || !y || x->d != y->d) return ptt_set_error(PTT_ERR_ARG, "mode count mismatch");
    for (int k = 0; k < x->d; k++)
        if (x->n[k] != y->n[k]) return ptt_set_error(PTT_ERR_ARG, "mode %d size mismatch", k);
    return PTT_OK;
}

extern "C" int ptt_axpby(double a, const ptt_tt* x, double b, const ptt_tt* y, ptt_tt* z) {
    int rc = check_same_modes(x, y);
    if (rc || (rc = check_same_modes(x, z))) return rc;
    const int d = x->d;
    int need[PTT_MAX_DIM + 1];
    need[0] = need[d] = 1;
    for (int k = 1; k < d; k++) need[k] = x->rcap[k] + y->rcap[k];
    if ((rc = fit_output(z, need, x, y, 0))) return rc;
    ptt_ctx* c = z->ctx;
    int* newr = ranks_scratch(c, d);
    if (!newr) return ptt_set_error(PTT_ERR_ARG, "d too large");
    long long mx = 0;
    for (int k = 0; k < d; k++) mx = z->cap[k] > mx ? z->cap[k] : mx;
    (void)mx;
    k_axpby<<<dim3(fiber_blocks(c, z, d), d), 256, 0, c->stream>>>(x->dd, y->dd, z->dd, a, b, newr, c->d_status);
    PTT_LAUNCHED(c);
    return finalize(z, newr, 0, d, 1);
}

// ---------------------------------------------------------------------------
// hadamard: z_k[(ky + ry*ix), j, (ly + ry1*jx)] = x_k[ix, j, jx] * y_k[ky, j, ly]
// ---------------------------------------------------------------------------
__global__ void k_hadamard(const DevDesc* X, const DevDesc* Y, DevDesc* Z, int* newr, int* status) {
    const int k = blockIdx.y;
    const int d = X->d;
    const int rx = X->r[k], rx1 = X->r[k + 1], ry = Y->r[k], ry1 = Y->r[k + 1];
    const int n = X->n[k];
    const int rz = rx * ry, rz1 = rx1 * ry1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        newr[k] = rz;
        if (k == d - 1) newr[d] = rz1;
    }
    const long long cnt = (long long)rz * n * rz1;
    if (rz > Z->rcap[k] || rz1 > Z->rcap[k + 1] || cnt > Z->cap[k]) {
        if (blockIdx.x == 0 && threadIdx.x == 0) PTT_STATUS_SET(status, PTT_ERR_CAPACITY);
        return;
    }
    const double* xc = X->core[k];
    const double* yc = Y->core[k];
    double* zc = Z->alt[k];
    // fiber (j, lz), lz = ly + ry1 jx: rows iz = ky + ry ix
    const int NF = n * rz1;
    const FiberIter it = fiber_iter(rz);
    for (long long f = it.f0; f < NF; f += it.fstep) {
        const int fi = (int)f, lz = fi / n, j = fi - lz * n;
        const int jx = lz / ry1, ly = lz - jx * ry1;
        const double* xf = xc + (long long)rx * (j + (long long)n * jx);
        const double* yf = yc + (long long)ry * (j + (long long)n * ly);
        double* zf = zc + (long long)rz * fi;
        for (int iz = it.li; iz < rz; iz += it.G) {
            const int ix = iz / ry, ky = iz - ix * ry;
            zf[iz] = xf[ix] * yf[ky];
        }
    }
}

extern "C" int ptt_hadamard(const ptt_tt* x, const ptt_tt* y, ptt_tt* z) {
    int rc = check_same_modes(x, y);
    if (rc || (rc = check_same_modes(x, z))) return rc;
    const int d = x->d;
    int need[PTT_MAX_DIM + 1];
    for (int k = 0; k <= d; k++) need[k] = x->rcap[k] * y->rcap[k];
    if ((rc = fit_output(z, need, x, y, 1))) return rc;
    ptt_ctx* c = z->ctx;
    int* newr = ranks_scratch(c, d);
    if (!newr) return ptt_set_error(PTT_ERR_ARG, "d too large");
    long long mx = 0;
    for (int k = 0; k < d; k++) mx = z->cap[k] > mx ? z->cap[k] : mx;
    (void)mx;
    k_hadamard<<<dim3(fiber_blocks(c, z, d), d), 256, 0, c->stream>>>(x->dd, y->dd, z->dd, newr, c->d_status);
    PTT_LAUNCHED(c);
    return finalize(z, newr, 0, d, 1);
}

// ---------------------------------------------------------------------------
// symmetric square: x (.) x restricted to the symmetric subspace.
// The formal core x_k (x) x_k (per mode index j) maps Sym^2(R^r) into
// Sym^2(R^r') and both interface vectors of x (.) x are symmetric, so with
// the orthonormal basis e_(a,a) and (e_(a,b) + e_(b,a))/sqrt2 (a < b) of
// Sym^2 the compressed core
//   z[s, j, s'] = (x[a,j,a'] x[b,j,b'] + x[a,j,b'] x[b,j,a']) f(s) f(s'),
//   f(s) = 1/sqrt2 if a == b else 1,
// gives exactly the same tensor at rank r (r + 1) / 2 instead of r^2.
// Pairs are packed s = b (b + 1) / 2 + a, a <= b.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void sym_pair(int s, int* a, int* b) {
    int bb = (int)((sqrt(8.0 * s + 1.0) - 1.0) * 0.5);
    while ((bb + 1) * (bb + 2) / 2 <= s) bb++;
    while (bb * (bb + 1) / 2 > s) bb--;
    *b = bb;
    *a = s - bb * (bb + 1) / 2;
}

__global__ void k_square_sym(const DevDesc* X, DevDesc* Z, int* newr, int* status) {
    const int k = blockIdx.y;
    const int d = X->d;
    const int rx = X->r[k], rx1 = X->r[k + 1];
    const int n = X->n[k];
    const int rz = rx * (rx + 1) / 2, rz1 = rx1 * (rx1 + 1) / 2;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        newr[k] = rz;
        if (k == d - 1) newr[d] = rz1;
    }
    const long long cnt = (long long)rz * n * rz1;
    if (rz > Z->rcap[k] || rz1 > Z->rcap[k + 1] || cnt > Z->cap[k]) {
        if (blockIdx.x == 0 && threadIdx.x == 0) PTT_STATUS_SET(status, PTT_ERR_CAPACITY);
        return;
    }
    const double* xc = X->core[k];
    double* zc = Z->alt[k];
    const long long rzn = (long long)rz * n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const double h = 0.70710678118654752440;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += stride) {
        const int sz1 = (int)(e / rzn);
        const long long rem = e - sz1 * rzn;
        const int j = (int)(rem / rz);
        const int sz = (int)(rem - (long long)j * rz);
        int a, b, a1, b1;
        sym_pair(sz, &a, &b);
        sym_pair(sz1, &a1, &b1);
        const double* xj = xc + (long long)rx * j;
        const long long ls = (long long)rx * n;
        const double v = xj[a + ls * a1] * xj[b + ls * b1] + xj[a + ls * b1] * xj[b + ls * a1];
        zc[e] = v * (a == b ? h : 1.0) * (a1 == b1 ? h : 1.0);
    }
}

extern "C" int ptt_square_sym(const ptt_tt* x, ptt_tt* z) {
    int rc = check_same_modes(x, z);
    if (rc) return rc;
    const int d = x->d;
    int need[PTT_MAX_DIM + 1];
    for (int k = 0; k <= d; k++) need[k] = x->rcap[k] * (x->rcap[k] + 1) / 2;
    if ((rc = fit_output(z, need, x, x, 3))) return rc;
    ptt_ctx* c = z->ctx;
    int* newr = ranks_scratch(c, d);
    if (!newr) return ptt_set_error(PTT_ERR_ARG, "d too large");
    long long mx = 0;
    for (int k = 0; k < d; k++) mx = z->cap[k] > mx ? z->cap[k] : mx;
    k_square_sym<<<dim3(core_blocks(c, mx, d), d), 256, 0, c->stream>>>(x->dd, z->dd, newr, c->d_status);
    PTT_LAUNCHED(c);
    return finalize(z, newr, 0, d, 1);
}

// ---------------------------------------------------------------------------
// scale core 0, diagonal multiply along one mode (in place)
// ---------------------------------------------------------------------------
__global__ void k_scale_core(DevDesc* X, int k, double a) {
    const long long cnt = (long long)X->r[k] * X->n[k] * X->r[k + 1];
    double* xc = X->core[k];
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cnt;
         e += (long long)gridDim.x * blockDim.x)
        xc[e] *= a;
}

extern "C" int ptt_scale(double a, ptt_tt* x) {
    if (!x) return ptt_set_error(PTT_ERR_ARG, "null tt");
    k_scale_core<<<elem_blocks(x->cap[0]), 256, 0, x->ctx->stream>>>(x->dd, 0, a);
    PTT_LAUNCHED(x->ctx);
    return PTT_OK;
}

__global__ void k_diag(DevDesc* X, int k, const double* vec) {
    const int r = X->r[k], n = X->n[k];
    const long long cnt = (long long)r * n * X->r[k + 1];
    double* xc = X->core[k];
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cnt;
         e += (long long)gridDim.x * blockDim.x) {
        const int j = (int)((e / r) % n);
        xc[e] *= vec[j];
    }
}

extern "C" int ptt_mult_diag(ptt_tt* x, int mode, const double* vec) {
    if (!x || !vec || mode < 0 || mode >= x->d) return ptt_set_error(PTT_ERR_ARG, "ptt_mult_diag: bad arguments");
    ptt_ctx* c = x->ctx;
    size_t bytes = sizeof(double) * x->n[mode];
    int rc = ptt_ws_reserve(c, bytes);
    if (rc) return rc;
    PTT_CUDA(cudaMemcpyAsync(c->ws, vec, bytes, cudaMemcpyHostToDevice, c->stream));
    k_diag<<<elem_blocks(x->cap[mode]), 256, 0, c->stream>>>(x->dd, mode, (const double*)c->ws);
    PTT_LAUNCHED(c);
    return PTT_OK;
}

// ---------------------------------------------------------------------------
// periodic centred stencil along one mode:
//   out[i, a, l] = sum_t s_t f[i, (a + t - h) mod n, l],  h = (len-1)/2
// Block = one (l) slab of r*n contiguous doubles; i fastest -> coalesced.
// ---------------------------------------------------------------------------
__global__ void k_stencil(DevDesc* X, int k, Stencil st) {
    const int r = X->r[k], n = X->n[k], r1 = X->r[k + 1];
    const int h = (st.len - 1) / 2;
    const double* in = X->core[k];
    double* out = X->alt[k];
    // fiber (a, l): out[:, a, l] = sum_t s_t in[:, (a + t - h) mod n, l]
    const int NF = n * r1;
    const FiberIter it = fiber_iter(r);
    for (long long f = it.f0; f < NF; f += it.fstep) {
        const int fi = (int)f, l = fi / n, a = fi - l * n;
        const double* fl = in + (long long)r * n * l;
        double* fo = out + (long long)r * fi;
        for (int i = it.li; i < r; i += it.G) {
            double acc = 0.0;
            for (int t = 0; t < st.len; t++) {
                int src = a + t - h;
                src = src < 0 ? src + n : (src >= n ? src - n : src);
                acc += st.s[t] * fl[i + (long long)r * src];
            }
            fo[i] = acc;
        }
    }
}

int ptt_make_stencil(const double* sten, int slen, Stencil* st) {
    if (slen % 2 == 0) slen -= 1;  // paratt.c:586: even lengths drop the last tap
    if (slen < 1 || slen > PTT_MAX_STENCIL) return ptt_set_error(PTT_ERR_ARG, "stencil length %d", slen);
    memset(st, 0, sizeof(*st));
    st->len = slen;
    for (int t = 0; t < slen; t++) st->s[t] = sten[t];
    return PTT_OK;
}

extern "C" int ptt_stencil(ptt_tt* x, int mode, const double* sten, int slen) {
    if (!x || !sten || mode < 0 || mode >= x->d) return ptt_set_error(PTT_ERR_ARG, "ptt_stencil: bad arguments");
    Stencil st;
    int rc = ptt_make_stencil(sten, slen, &st);
    if (rc) return rc;
    if ((st.len - 1) / 2 >= x->n[mode] && st.len > 1)
        return ptt_set_error(PTT_ERR_ARG, "stencil half-width exceeds mode size");
    ptt_ctx* c = x->ctx;
    long long bx = ((long long)x->n[mode] * x->rcap[mode + 1] + 7) / 8;  // 8 fibers per block
    if (bx > 8LL * c->nsm) bx = 8LL * c->nsm;
    if (bx < 1) bx = 1;
    k_stencil<<<dim3((unsigned)bx), 256, 0, c->stream>>>(x->dd, mode, st);
    PTT_LAUNCHED(c);
    k_finalize<<<1, 32, 0, c->stream>>>(x->dd, NULL, mode, mode + 1, 0);
    PTT_LAUNCHED(c);
    return PTT_OK;
}

// ---------------------------------------------------------------------------
// Y = sum_i S_i X + shift * X, S_i = the periodic stencil on mode i.
// Exact rank-2r TT (the formal sum of the d single-mode stencil applications,
// attac_apply_periodic_stencil paratt.c:584-661 summed with attacFormalSum,
// represents the same tensor at rank d*r).  Core k in 2x2 blocks indexed by
// (applied-before-k, applied-up-to-k): [[x_k, S x_k], [0, x_k]]; the first
// core keeps block row 0 with the shift added to S x_0, the last core keeps
// block column 1.  For d == 1: (S + shift) x_0.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double sten_at(const double* xc, int r, int n, int i, int j, int l, const Stencil& st) {
    const int h = (st.len - 1) / 2;
    double acc = 0.0;
    for (int t = 0; t < st.len; t++) {
        int s = j + t - h;
        s = s < 0 ? s + n : (s >= n ? s - n : s);
        acc += st.s[t] * xc[i + (long long)r * (s + (long long)n * l)];
    }
    return acc;
}

__global__ void k_opsum(const DevDesc* X, DevDesc* Y, Stencil st, double shift, int* newr, int* status) {
    const int k = blockIdx.y;
    const int d = X->d;
    const int r = X->r[k], r1 = X->r[k + 1], n = X->n[k];
    const int ry = (d == 1 || k == 0) ? 1 : 2 * r;
    const int ry1 = (d == 1 || k == d - 1) ? 1 : 2 * r1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        newr[k] = ry;
        if (k == d - 1) newr[d] = 1;
    }
    const long long cnt = (long long)ry * n * ry1;
    if (ry > Y->rcap[k] || ry1 > Y->rcap[k + 1] || cnt > Y->cap[k]) {
        if (blockIdx.x == 0 && threadIdx.x == 0) PTT_STATUS_SET(status, PTT_ERR_CAPACITY);
        return;
    }
    const double* xc = X->core[k];
    double* yc = Y->alt[k];
    // fiber (j, l) of y; l' = l - r1 for the second block column
    const int NF = n * ry1;
    const FiberIter it = fiber_iter(ry);
    for (long long f = it.f0; f < NF; f += it.fstep) {
        const int fi = (int)f, l = fi / n, j = fi - l * n;
        double* yf = yc + (long long)ry * fi;
        if (d == 1) {
            if (it.li == 0) yf[0] = sten_at(xc, 1, n, 0, j, 0, st) + shift * xc[j];
        } else if (k == 0) {
            if (it.li == 0)
                yf[0] = (l < r1) ? xc[j + (long long)n * l]
                                 : sten_at(xc, 1, n, 0, j, l - r1, st) + shift * xc[j + (long long)n * (l - r1)];
        } else if (k == d - 1) {
            for (int i = it.li; i < ry; i += it.G)
                yf[i] = (i < r) ? sten_at(xc, r, n, i, j, 0, st) : xc[(i - r) + (long long)r * j];
        } else if (l < r1) {
            const double* src = xc + (long long)r * (j + (long long)n * l);
#pragma unroll 4
            for (int i = it.li; i < ry; i += it.G) yf[i] = (i < r) ? src[i] : 0.0;
        } else {
            const int lp = l - r1;
            const double* src = xc + (long long)r * (j + (long long)n * lp);
            for (int i = it.li; i < ry; i += it.G) yf[i] = (i < r) ? sten_at(xc, r, n, i, j, lp, st) : src[i - r];
        }
    }
}

extern "C" int ptt_op_sum(const ptt_tt* x, const double* sten, int slen, double shift, ptt_tt* y) {
    int rc = check_same_modes(x, y);
    if (rc) return rc;
    Stencil st;
    if ((rc = ptt_make_stencil(sten, slen, &st))) return rc;
    const int d = x->d;
    for (int k = 0; k < d; k++)
        if ((st.len - 1) / 2 >= x->n[k] && st.len > 1)
            return ptt_set_error(PTT_ERR_ARG, "stencil half-width exceeds mode %d size", k);
    int need[PTT_MAX_DIM + 1];
    for (int k = 0; k <= d; k++) need[k] = (k == 0 || k == d) ? 1 : 2 * x->rcap[k];
    if ((rc = fit_output(y, need, x, x, 2))) return rc;
    ptt_ctx* c = y->ctx;
    int* newr = ranks_scratch(c, d);
    long long mx = 0;
    for (int k = 0; k < d; k++) mx = y->cap[k] > mx ? y->cap[k] : mx;
    (void)mx;
    k_opsum<<<dim3(fiber_blocks(c, y, d), d), 256, 0, c->stream>>>(x->dd, y->dd, st, shift, newr, c->d_status);
    PTT_LAUNCHED(c);
    return finalize(y, newr, 0, d, 1);
}
