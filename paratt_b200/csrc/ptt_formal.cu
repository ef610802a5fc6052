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

// Blocks per core of a launch over all d cores (grid y = core).  The count is
// sized by the capacity, which can be far above the actual ranks: a few
// waves over the GPU (148 SMs x 32 blocks) are enough at full size, and the
// grid-stride loops cover any core with any grid.
static inline int core_blocks(long long maxcnt, int d) {
    const int b = elem_blocks(maxcnt);
    int cap = 4736 / (d > 0 ? d : 1);
    if (cap < 1) cap = 1;
    return b < cap ? b : cap;
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
    const long long stride = (long long)gridDim.x * blockDim.x;
    if (d == 1) {
        for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += stride)
            zc[e] = a * xc[e] + b * yc[e];
        return;
    }
    const long long rzn = (long long)rz * n;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += stride) {
        const int l = (int)(e / rzn);
        const long long rem = e - l * rzn;
        const int j = (int)(rem / rz);
        const int i = (int)(rem - (long long)j * rz);
        double v;
        if (k == 0) {
            v = (l < rx1) ? a * xc[j + (long long)n * l] : b * yc[j + (long long)n * (l - rx1)];
        } else if (k == d - 1) {
            v = (i < rx) ? xc[i + (long long)rx * j] : yc[(i - rx) + (long long)ry * j];
        } else if (i < rx && l < rx1) {
            v = xc[i + (long long)rx * (j + (long long)n * l)];
        } else if (i >= rx && l >= rx1) {
            v = yc[(i - rx) + (long long)ry * (j + (long long)n * (l - rx1))];
        } else {
            v = 0.0;
        }
        zc[e] = v;
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
    k_axpby<<<dim3(core_blocks(mx, d), d), 256, 0, c->stream>>>(x->dd, y->dd, z->dd, a, b, newr, c->d_status);
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
    const long long rzn = (long long)rz * n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += stride) {
        const int lz = (int)(e / rzn);
        const long long rem = e - lz * rzn;
        const int j = (int)(rem / rz);
        const int iz = (int)(rem - (long long)j * rz);
        const int ix = iz / ry, ky = iz - ix * ry;
        const int jx = lz / ry1, ly = lz - jx * ry1;
        zc[e] = xc[ix + (long long)rx * (j + (long long)n * jx)] * yc[ky + (long long)ry * (j + (long long)n * ly)];
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
    k_hadamard<<<dim3(core_blocks(mx, d), d), 256, 0, c->stream>>>(x->dd, y->dd, z->dd, newr, c->d_status);
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
    k_square_sym<<<dim3(core_blocks(mx, d), d), 256, 0, c->stream>>>(x->dd, z->dd, newr, c->d_status);
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
    const long long slab = (long long)r * n;
    const double* in = X->core[k];
    double* out = X->alt[k];
    for (int l = blockIdx.y; l < r1; l += gridDim.y) {
        const double* fi = in + slab * l;
        double* fo = out + slab * l;
        for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < slab;
             e += (long long)gridDim.x * blockDim.x) {
            const int a = (int)(e / r);
            const int i = (int)(e - (long long)a * r);
            double acc = 0.0;
            for (int t = 0; t < st.len; t++) {
                int src = a + t - h;
                src = src < 0 ? src + n : (src >= n ? src - n : src);
                acc += st.s[t] * fi[i + (long long)r * src];
            }
            fo[e] = acc;
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
    long long slab = (long long)x->rcap[mode] * x->n[mode];
    int bx = (int)((slab + 255) / 256);
    int by = x->rcap[mode + 1];
    if (bx > 64) bx = 64;
    if (by > 1024) by = 1024;
    k_stencil<<<dim3(bx, by), 256, 0, c->stream>>>(x->dd, mode, st);
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
    const long long ryn = (long long)ry * n;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cnt;
         e += (long long)gridDim.x * blockDim.x) {
        const int l = (int)(e / ryn);
        const long long rem = e - l * ryn;
        const int j = (int)(rem / ry);
        const int i = (int)(rem - (long long)j * ry);
        double v;
        if (d == 1) {
            v = sten_at(xc, 1, n, 0, j, 0, st) + shift * xc[j];
        } else if (k == 0) {
            v = (l < r1) ? xc[j + (long long)n * l]
                         : sten_at(xc, 1, n, 0, j, l - r1, st) + shift * xc[j + (long long)n * (l - r1)];
        } else if (k == d - 1) {
            v = (i < r) ? sten_at(xc, r, n, i, j, 0, st) : xc[(i - r) + (long long)r * j];
        } else {
            const bool a = i >= r, b = l >= r1;
            if (!a && !b)
                v = xc[i + (long long)r * (j + (long long)n * l)];
            else if (!a && b)
                v = sten_at(xc, r, n, i, j, l - r1, st);
            else if (a && b)
                v = xc[(i - r) + (long long)r * (j + (long long)n * (l - r1))];
            else
                v = 0.0;
        }
        yc[e] = v;
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
    k_opsum<<<dim3(core_blocks(mx, d), d), 256, 0, c->stream>>>(x->dd, y->dd, st, shift, newr, c->d_status);
    PTT_LAUNCHED(c);
    return finalize(y, newr, 0, d, 1);
}
