// Randomised TT rounding of a Hadamard product without forming it.
//
// z ~= round(x (.) y), where the formal product (attacHadamard, attac.c:
// 128-136) would have ranks r_x r_y: a Gaussian TT sketch G with ranks l_k
// is contracted with the product right-to-left, W_k = sum_j (x_k[:,j,:] (x)
// y_k[:,j,:]) W_{k+1} G_k[:,j,:]^T  (r_x r_y x l_k), then the product is
// orthogonalised left-to-right against the sketch (Y = Z_k W_{k+1}, QR,
// carry Q^T Z_k), which is the "randomize-then-orthogonalize" rounding of
// Al Daas, Ballard, Cazeaux, Hallman, Miedlar, Pasha, Reid and Saibaba,
// "Randomized algorithms for rounding in the tensor-train format", SISC 2023.
// The result is left-orthogonal with ranks <= l_k and is finished by the
// deterministic right-to-left SVD truncation of ptt_round (tol, maxrank).
//
// Every contraction is a batched strided FP64 GEMM over the Kronecker
// structure, so no r_x r_y x n x r_x r_y core is ever stored.
#include "ptt_common.cuh"

#include <stddef.h>
#include <stdio.h>
#include <string.h>

namespace {

struct GemmB {
    const double* A;
    long long ars, acs, ab1, ab2;
    const double* B;
    long long brs, bcs, bb1, bb2;
    double* C;
    long long crs, ccs, cb1, cb2;
    int M, N, K, nb1, nb2;
    double alpha, beta;
    // optional: the first kernel of the product also writes the ranks
    // rset[rk0] = rv0, rset[rk0 + 1] = rv1 (a train's device descriptor), so
    // that bookkeeping needs no launch of its own
    int* rset;
    int rk0, rv0, rv1;
};

__device__ __forceinline__ void gemm_set_ranks(const GemmB& g, bool first) {
    if (g.rset && first && threadIdx.x == 0) {
        g.rset[g.rk0] = g.rv0;
        g.rset[g.rk0 + 1] = g.rv1;
    }
}

// C[b] = alpha * A[b] B[b] + beta * C[b]; batch b = b1 + nb1 * b2.
// With split-K (part != NULL) grid z runs over (batch, slice): slice s sums
// k in [s kper, (s+1) kper) and writes its tile to part[s][b][M][N]; a
// second kernel adds the slices in order (deterministic).
template <int TM>
__global__ void __launch_bounds__(256) k_gemm_b(GemmB g, long long zoff, int kper, double* part) {
    PTT_PDL_ENTRY();
    gemm_set_ranks(g, blockIdx.x == 0 && blockIdx.y == 0 && zoff + blockIdx.z == 0);
    constexpr int BK = 32;
    constexpr int NL = TM * BK / 256;  // elements of each operand tile per thread
    __shared__ double sA[BK][TM + 1];
    __shared__ double sB[BK][TM + 1];
    const long long nb = (long long)g.nb1 * g.nb2;
    const long long zz = blockIdx.z + zoff;
    const int sl = (int)(zz / nb);
    const int bz = (int)(zz - (long long)sl * nb);
    const int b1 = bz % g.nb1, b2 = bz / g.nb1;
    const int kbeg = sl * kper;
    const int kend = (kbeg + kper) < g.K ? (kbeg + kper) : g.K;
    const double* A = g.A + b1 * g.ab1 + b2 * g.ab2;
    const double* B = g.B + b1 * g.bb1 + b2 * g.bb2;
    double* C = g.C + b1 * g.cb1 + b2 * g.cb2;
    const int tid = threadIdx.x;
    const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TM;
    const bool a_colmajor = (g.ars == 1);
    const bool b_rowfast = (g.bcs == 1);
    // the product on the FP64 tensor cores: warp w owns TPW of the
    // (TM / 8)^2 8 x 8 output tiles, all in one tile row (shared A fragment)
    constexpr int TD = TM / 8, TPW = TD * TD / 8;
    const int warp = tid >> 5, lane = tid & 31, li = lane >> 2, lk = lane & 3;
    const int t0 = warp * TPW, tr = t0 / TD, tc0 = t0 - tr * TD;
    double d0[TPW], d1[TPW];
#pragma unroll
    for (int t = 0; t < TPW; t++) {
        d0[t] = 0.0;
        d1[t] = 0.0;
    }
    for (int k0 = kbeg; k0 < kend; k0 += BK) {
        // every element of both tiles is requested before the first store
        double va[NL], vb[NL];
#pragma unroll
        for (int u = 0; u < NL; u++) {
            const int e = tid + u * 256;
            int r, kk;
            if (a_colmajor) {
                r = e % TM;
                kk = e / TM;
            } else {
                kk = e % BK;
                r = e / BK;
            }
            const int gr = m0 + r, gk = k0 + kk;
            va[u] = (gr < g.M && gk < kend) ? A[(long long)gr * g.ars + (long long)gk * g.acs] : 0.0;
            int cn, kb;
            if (b_rowfast) {
                cn = e % TM;
                kb = e / TM;
            } else {
                kb = e % BK;
                cn = e / BK;
            }
            const int gkb = k0 + kb, gc = n0 + cn;
            vb[u] = (gkb < kend && gc < g.N) ? B[(long long)gkb * g.brs + (long long)gc * g.bcs] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < NL; u++) {
            const int e = tid + u * 256;
            if (a_colmajor)
                sA[e / TM][e % TM] = va[u];
            else
                sA[e % BK][e / BK] = va[u];
            if (b_rowfast)
                sB[e / TM][e % TM] = vb[u];
            else
                sB[e % BK][e / BK] = vb[u];
        }
        __syncthreads();
#pragma unroll
        for (int k4 = 0; k4 < BK; k4 += 4) {
            const double av = sA[k4 + lk][8 * tr + li];
#pragma unroll
            for (int t = 0; t < TPW; t++) {
                const double bv = sB[k4 + lk][8 * (tc0 + t) + li];
                asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                             : "+d"(d0[t]), "+d"(d1[t])
                             : "d"(av), "d"(bv));
            }
        }
        __syncthreads();
    }
    const int gr = m0 + 8 * tr + li;
    if (gr < g.M) {
#pragma unroll
        for (int t = 0; t < TPW; t++) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int gc = n0 + 8 * (tc0 + t) + 2 * lk + h;
                if (gc >= g.N) continue;
                const double v = h ? d1[t] : d0[t];
                if (part) {
                    part[(((long long)sl * nb + bz) * g.M + gr) * g.N + gc] = v;
                    continue;
                }
                double* cp = C + (long long)gr * g.crs + (long long)gc * g.ccs;
                *cp = (g.beta != 0.0) ? fma(g.alpha, v, g.beta * *cp) : g.alpha * v;
            }
        }
    }
}

// Split-K for C small (M, N <= 32) and K long: slice blockIdx.x of batch
// blockIdx.y multiplies the KS-long chunk of K; every element of the chunk is
// requested before the first product (the loads of one slice are in flight
// together), and the slice's partial C goes to part[slice][b][M][N].
constexpr int KS = 128;
constexpr size_t SKINNY_SMEM = sizeof(double) * 2 * KS * 33;

__global__ void __launch_bounds__(256) k_gemm_skinny(GemmB g, int ns, double* part) {
    PTT_PDL_ENTRY();
    gemm_set_ranks(g, blockIdx.x == 0 && blockIdx.y == 0);
    extern __shared__ double ssm[];
    double* sA = ssm;            // [KS][33]: sA[k][i] = A(i, k0 + k)
    double* sB = ssm + KS * 33;  // [KS][33]: sB[k][j] = B(k0 + k, j)
    const int sl = blockIdx.x, bz = blockIdx.y;
    const int b1 = bz % g.nb1, b2 = bz / g.nb1;
    const double* A = g.A + b1 * g.ab1 + b2 * g.ab2;
    const double* B = g.B + b1 * g.bb1 + b2 * g.bb2;
    const int k0 = sl * KS;
    const int kn = (g.K - k0) < KS ? (g.K - k0) : KS;
    const int tid = threadIdx.x;
    // A chunk: M x kn, walked along whichever index is contiguous
    {
        const int tot = g.M * KS;
        for (int base = tid; base < tot; base += 256 * 8) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int e = base + u * 256;
                int i, k;
                if (g.acs == 1) {
                    k = e % KS;
                    i = e / KS;
                } else {
                    i = e % g.M;
                    k = e / g.M;
                }
                v[u] = (e < tot && k < kn) ? A[(long long)i * g.ars + (long long)(k0 + k) * g.acs] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int e = base + u * 256;
                if (e < tot) {
                    int i, k;
                    if (g.acs == 1) {
                        k = e % KS;
                        i = e / KS;
                    } else {
                        i = e % g.M;
                        k = e / g.M;
                    }
                    sA[k * 33 + i] = v[u];
                }
            }
        }
    }
    {
        const int tot = g.N * KS;
        for (int base = tid; base < tot; base += 256 * 8) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int e = base + u * 256;
                int j, k;
                if (g.brs == 1) {
                    k = e % KS;
                    j = e / KS;
                } else {
                    j = e % g.N;
                    k = e / g.N;
                }
                v[u] = (e < tot && k < kn) ? B[(long long)(k0 + k) * g.brs + (long long)j * g.bcs] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int e = base + u * 256;
                if (e < tot) {
                    int j, k;
                    if (g.brs == 1) {
                        k = e % KS;
                        j = e / KS;
                    } else {
                        j = e % g.N;
                        k = e / g.N;
                    }
                    sB[k * 33 + j] = v[u];
                }
            }
        }
    }
    __syncthreads();
    const int tx = tid & 15, ty = tid >> 4;
    double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll 8
    for (int k = 0; k < KS; k++) {
        const double a0 = sA[k * 33 + ty], a1 = sA[k * 33 + ty + 16];
        const double c0 = sB[k * 33 + tx], c1 = sB[k * 33 + tx + 16];
        acc[0][0] = fma(a0, c0, acc[0][0]);
        acc[0][1] = fma(a0, c1, acc[0][1]);
        acc[1][0] = fma(a1, c0, acc[1][0]);
        acc[1][1] = fma(a1, c1, acc[1][1]);
    }
    const long long nb = (long long)g.nb1 * g.nb2;
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 2; b++) {
            const int i = ty + 16 * a, j = tx + 16 * b;
            if (i < g.M && j < g.N) part[(((long long)sl * nb + bz) * g.M + i) * g.N + j] = acc[a][b];
        }
}

// C[b][r][c] = alpha * sum_s part[s][b][r][c] + beta * C.  Eight lanes per
// output: lane l sums the slices l, l + 8, ... in order (eight loads in
// flight), then the eight sums are added by a fixed butterfly -- the same
// bits in every lane and on every run.
__global__ void k_gemm_red(GemmB g, int ns, const double* part) {
    PTT_PDL_ENTRY();
    const long long nb = (long long)g.nb1 * g.nb2;
    const long long per = (long long)g.M * g.N, tot = per * nb;
    const int lane = threadIdx.x & 31, sub = lane & 7;
    const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = wid * 4; base < tot; base += nw * 4) {  // uniform over the warp
        const long long e = base + (lane >> 3);
        const bool ok = e < tot;
        double acc = 0.0;
        if (ok) {
            for (int s = sub; s < ns; s += 64) {
                double v[8];
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const int ss = s + 8 * u;
                    v[u] = ss < ns ? part[(long long)ss * tot + e] : 0.0;
                }
#pragma unroll
                for (int u = 0; u < 8; u++) acc += v[u];
            }
        }
        acc += __shfl_xor_sync(0xffffffffu, acc, 1);
        acc += __shfl_xor_sync(0xffffffffu, acc, 2);
        acc += __shfl_xor_sync(0xffffffffu, acc, 4);
        if (ok && sub == 0) {
            const int bz = (int)(e / per);
            const long long rc = e - (long long)bz * per;
            const int gr = (int)(rc / g.N), gc = (int)(rc - (long long)gr * g.N);
            const int b1 = bz % g.nb1, b2 = bz / g.nb1;
            double* cp = g.C + b1 * g.cb1 + b2 * g.cb2 + (long long)gr * g.crs + (long long)gc * g.ccs;
            *cp = (g.beta != 0.0) ? fma(g.alpha, acc, g.beta * *cp) : g.alpha * acc;
        }
    }
}

int gemm(ptt_ctx* c, const GemmB& g) {
    if (g.M <= 0 || g.N <= 0 || g.nb1 <= 0 || g.nb2 <= 0) {  // nothing to multiply; the ranks still go out
        if (!g.rset) return PTT_OK;
        GemmB h = g;
        h.M = h.N = h.K = 0;
        h.nb1 = h.nb2 = 1;
        PTT_CUDA(ptt_launch(c, k_gemm_b<32>, dim3(1, 1, 1), dim3(256), 0, h, 0LL, 0, (double*)nullptr));
        PTT_LAUNCHED(c);
        return PTT_OK;
    }
    const long long nb = (long long)g.nb1 * g.nb2;
    if (c->tkind == PTT_TIME_GEMM) c->hwork[PTT_TIME_GEMM] += 2.0 * g.M * (double)g.N * g.K * (double)nb;
    if (g.M <= 32 && g.N <= 32 && g.K >= 2 * KS) {
        // small C, long K: one block per KS-long slice of K, then the ordered sum
        const int ns = (g.K + KS - 1) / KS;
        if (nb > 65535) return ptt_set_error(PTT_ERR_CAPACITY, "sketch contraction: %lld batches", nb);
        const size_t need = sizeof(double) * (size_t)ns * (size_t)nb * (size_t)g.M * (size_t)g.N;
        int rc = ptt_ws3_reserve(c, need);
        if (rc) return rc;
        double* part = (double*)c->ws3;
        static std::atomic<unsigned long long> attr{0};
        unsigned long long bit;
        if (!ptt_device_done(attr, &bit)) {
            PTT_CUDA(cudaFuncSetAttribute(k_gemm_skinny, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SKINNY_SMEM));
            attr.fetch_or(bit);
        }
        ptt_time_begin(c, PTT_TIME_GEMM);
        PTT_CUDA(ptt_launch(c, k_gemm_skinny, dim3(dim3(ns, (unsigned)nb)), dim3(256), SKINNY_SMEM, g, ns, part));
        PTT_LAUNCHED(c);
        const long long tot = (long long)g.M * g.N * nb;
        long long nbk = (8 * tot + 255) / 256;  // eight lanes per output
        if (nbk > 1184) nbk = 1184;
        PTT_CUDA(ptt_launch(c, k_gemm_red, dim3((int)nbk), dim3(256), 0, g, ns, part));
        PTT_LAUNCHED(c);
        ptt_time_end(c, PTT_TIME_GEMM);
        return PTT_OK;
    }
    const int tm64 = c->gemm_tm64 > 0 ? c->gemm_tm64 : 48;
    const long long fill = c->gemm_fill > 0 ? c->gemm_fill : 2LL * c->nsm;
    const bool big = g.M >= tm64 && g.N >= tm64;
    const int TM = big ? 64 : 32;
    dim3 grid((g.M + TM - 1) / TM, (g.N + TM - 1) / TM, 1);
    // split K when the tiles alone cannot fill the GPU and K is long
    const long long tiles = (long long)grid.x * grid.y * nb;
    int ns = 1, kper = g.K;
    if (tiles < fill && g.K >= 512) {
        long long want = (fill + tiles - 1) / tiles;
        const long long kmax = (g.K + 255) / 256;
        ns = (int)(want < kmax ? want : kmax);
        if (ns > 64) ns = 64;
        kper = (g.K + ns - 1) / ns;
        kper = (kper + 31) / 32 * 32;
        ns = (g.K + kper - 1) / kper;
    }
    double* part = nullptr;
    if (ns > 1) {
        const size_t need = sizeof(double) * (size_t)ns * (size_t)nb * (size_t)g.M * (size_t)g.N;
        int rc = ptt_ws3_reserve(c, need);
        if (rc) return rc;
        part = (double*)c->ws3;
    }
    const long long nz = nb * ns;
    ptt_time_begin(c, PTT_TIME_GEMM);
    for (long long z0 = 0; z0 < nz; z0 += 65535) {
        grid.z = (unsigned)((nz - z0) < 65535 ? (nz - z0) : 65535);
        if (big)
            PTT_CUDA(ptt_launch(c, k_gemm_b<64>, dim3(grid), dim3(256), 0, g, z0, kper, part));
        else
            PTT_CUDA(ptt_launch(c, k_gemm_b<32>, dim3(grid), dim3(256), 0, g, z0, kper, part));
        PTT_LAUNCHED(c);
    }
    if (part) {
        const long long tot = (long long)g.M * g.N * nb;
        long long nbk = (8 * tot + 255) / 256;  // eight lanes per output
        if (nbk > 1184) nbk = 1184;
        PTT_CUDA(ptt_launch(c, k_gemm_red, dim3((int)nbk), dim3(256), 0, g, ns, part));
        PTT_LAUNCHED(c);
    }
    ptt_time_end(c, PTT_TIME_GEMM);
    return PTT_OK;
}

// ---------------------------------------------------------------------------
// Gaussian sketch cores from a counter-based generator: splitmix64 (Vigna)
// hashes (seed, core, index); Box-Muller turns two uniforms into a normal.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// The Gaussian sketch cores G_1 .. G_{d-1} in one launch: core k fills
// [off[k], off[k+1]) of G from its own counter-based stream (splitmix64 of
// the seed and the core index, Box-Muller), so a core's values do not
// depend on the other cores or on the launch shape.
struct GaussOff {
    long long off[PTT_MAX_DIM + 1];
};
__global__ void k_gauss_all(double* G, GaussOff o, int k0, int k1, unsigned long long seed) {
    PTT_PDL_ENTRY();
    const long long tot = o.off[k1] - o.off[k0];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < tot;
         i += (long long)gridDim.x * blockDim.x) {
        const long long e = o.off[k0] + i;
        int lo = k0, hi = k1;  // the core: largest k with off[k] <= e
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (o.off[mid] <= e)
                lo = mid;
            else
                hi = mid;
        }
        const int k = lo;
        const unsigned long long base = splitmix64(seed ^ (0xD1B54A32D192ED03ull * (unsigned long long)(k + 1)));
        const long long el = e - o.off[k];
        const unsigned long long h1 = splitmix64(base + 2ull * (unsigned long long)el);
        const unsigned long long h2 = splitmix64(base + 2ull * (unsigned long long)el + 1ull);
        const double u1 = ((double)(h1 >> 11) + 0.5) * 1.1102230246251565e-16;  // (0,1)
        const double u2 = (double)(h2 >> 11) * 1.1102230246251565e-16;          // [0,1)
        G[e] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    }
}

__global__ void k_fill(double* p, long long cnt, double v) {
    PTT_PDL_ENTRY();
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cnt;
         e += (long long)gridDim.x * blockDim.x)
        p[e] = v;
}

static int blocks_for(long long cnt) {
    long long b = (cnt + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 2048 ? 2048 : b));
}

}  // namespace

// Sketch-round x (.) y (y == NULL: the all-ones rank-1 train, i.e. x
// itself).  On return used[k] holds the sketch rank of bond k.
static int sketch_round(const ptt_tt* x, const ptt_tt* y, ptt_tt* z, const int* ell, unsigned long long seed,
                        double tol, const int* maxrank, int* used) {
    if (!x || !z || x->d != z->d || (y && y->d != x->d))
        return ptt_set_error(PTT_ERR_ARG, "sketch rounding: shape mismatch");
    if (z == x || z == y) return ptt_set_error(PTT_ERR_ARG, "sketch rounding: output aliases an input");
    const int d = x->d;
    for (int k = 0; k < d; k++)
        if ((y && x->n[k] != y->n[k]) || x->n[k] != z->n[k])
            return ptt_set_error(PTT_ERR_ARG, "sketch rounding: mode %d differs", k);
    ptt_ctx* c = z->ctx;
    int rc;
    int rx[PTT_MAX_DIM + 1], ry[PTT_MAX_DIM + 1], L[PTT_MAX_DIM + 1];
    long long R[PTT_MAX_DIM + 1];
    if ((rc = ptt_tt_get_ranks((ptt_tt*)x, rx))) return rc;
    if (y) {
        if ((rc = ptt_tt_get_ranks((ptt_tt*)y, ry))) return rc;
    } else {
        for (int k = 0; k <= d; k++) ry[k] = 1;
    }
    const int* n = x->n;
    for (int k = 0; k <= d; k++) R[k] = (long long)rx[k] * ry[k];
    L[0] = L[d] = 1;
    for (int k = 1; k < d; k++) {
        long long l = ell ? ell[k] : 72;
        if (l > R[k]) l = R[k];
        if (l > 128) l = 128;
        if (l < 1) l = 1;
        L[k] = (int)l;
    }
    // z capacity: ranks <= L
    {
        int cap[PTT_MAX_DIM + 1];
        for (int k = 0; k <= d; k++) cap[k] = L[k] > z->rcap[k] ? L[k] : z->rcap[k];
        if ((rc = ptt_tt_reserve(z, cap))) return rc;
    }
    // workspace: G_1..G_{d-1}, W_1..W_d, then temporaries
    long long oG[PTT_MAX_DIM + 1], oW[PTT_MAX_DIM + 1], off = 0;
    for (int k = 1; k < d; k++) {
        oG[k] = off;
        off += (long long)L[k] * n[k] * L[k + 1];
    }
    for (int k = 1; k <= d; k++) {
        oW[k] = off;
        off += R[k] * L[k];
    }
    long long szA = 1, szB = 1, szP = 1, szZ = 1, szM = 1;
    for (int k = 0; k < d; k++) {
        const long long Rp = R[k + 1];
        szA = (long long)n[k] * Rp * L[k] > szA ? (long long)n[k] * Rp * L[k] : szA;
        szB = (long long)rx[k] * L[k] * n[k] * ry[k + 1] > szB ? (long long)rx[k] * L[k] * n[k] * ry[k + 1] : szB;
        szP = (long long)rx[k] * n[k] * ry[k + 1] * L[k] > szP ? (long long)rx[k] * n[k] * ry[k + 1] * L[k] : szP;
        szZ = (long long)L[k] * n[k] * Rp > szZ ? (long long)L[k] * n[k] * Rp : szZ;
        szM = (long long)L[k] * R[k] > szM ? (long long)L[k] * R[k] : szM;
    }
    const long long oA = off, oB = oA + szA, oP = oB + szB, oZ = oP + szP, oM0 = oZ + szZ, oM1 = oM0 + szM;
    const long long total = oM1 + szM + 64;
    if ((rc = ptt_ws2_reserve(c, (size_t)total * sizeof(double)))) return rc;
    double* ws = (double*)c->ws2;
    // input core pointers (the ones train points every core at one ones vector)
    if ((rc = ptt_pull_desc((ptt_tt*)x))) return rc;
    const double* const* xc = x->hd.core;
    const double* yones[PTT_MAX_DIM];
    const double* const* yc;
    if (y) {
        if ((rc = ptt_pull_desc((ptt_tt*)y))) return rc;
        yc = y->hd.core;
    } else {
        int nmax = 1;
        for (int k = 0; k < d; k++) nmax = n[k] > nmax ? n[k] : nmax;
        if ((rc = ptt_ones(c, nmax))) return rc;
        for (int k = 0; k < d; k++) yones[k] = c->d_ones;
        yc = yones;
    }

    if (d > 1) {  // G_k at ws + oG[k], contiguous from oG[1] = 0
        GaussOff go;
        for (int k = 1; k < d; k++) go.off[k] = oG[k];
        go.off[d] = oG[d - 1] + (long long)L[d - 1] * n[d - 1] * L[d];
        PTT_CUDA(ptt_launch(c, k_gauss_all, dim3(blocks_for(go.off[d] - go.off[1])), dim3(256), 0, ws, go, 1, d,
                            seed));
        PTT_LAUNCHED(c);
    }
    PTT_CUDA(ptt_launch(c, k_fill, dim3(1), dim3(32), 0, ws + oW[d], 1, 1.0));
    PTT_LAUNCHED(c);

    // ---- right-to-left sketch contractions -------------------------------
    for (int k = d - 1; k >= 1; k--) {
        const long long Rp = R[k + 1];
        const int Lk = L[k], Lp = L[k + 1], nk = n[k];
        const int rxk = rx[k], ryk = ry[k], rxp = rx[k + 1], ryp = ry[k + 1];
        GemmB g;
        if (!y) {
            // x alone (the partner is the ones train): A_j = W_{k+1} G_j^T
            // stored with row index j + n jx, so that
            // W_k[ix, c] = sum_{j, jx} x[ix, j, jx] A_j[jx, c] is one GEMM
            // with K = n r_{k+1} over the core's right unfolding
            g = GemmB{ws + oW[k + 1], 1, Rp, 0, 0,
                      ws + oG[k], (long long)Lk * nk, 1, Lk, 0,
                      ws + oA, nk, (long long)nk * Rp, 1, 0,
                      (int)Rp, Lk, Lp, nk, 1, 1.0, 0.0};
            if ((rc = gemm(c, g))) return rc;
            g = GemmB{xc[k], 1, rxk, 0, 0,
                      ws + oA, 1, (long long)nk * Rp, 0, 0,
                      ws + oW[k], 1, R[k], 0, 0,
                      rxk, Lk, (int)(nk * Rp), 1, 1, 1.0, 0.0};
            if ((rc = gemm(c, g))) return rc;
            continue;
        }
        // A_j = W_{k+1} G_j^T   (Rp x Lk), j < n
        g = GemmB{ws + oW[k + 1], 1, Rp, 0, 0,
                  ws + oG[k], (long long)Lk * nk, 1, Lk, 0,
                  ws + oA, 1, Rp, Rp * Lk, 0,
                  (int)Rp, Lk, Lp, nk, 1, 1.0, 0.0};
        if ((rc = gemm(c, g))) return rc;
        // Bt[ix][c][j + n ly] = sum_jx x[ix, j, jx] A_j[ly + ryp jx, c]
        g = GemmB{xc[k], 1, (long long)rxk * nk, rxk, 0,
                  ws + oA, ryp, Rp, Rp * Lk, 1,
                  ws + oB, (long long)Lk * nk * ryp, (long long)nk * ryp, 1, nk,
                  rxk, Lk, rxp, nk, ryp, 1.0, 0.0};
        if ((rc = gemm(c, g))) return rc;
        // W_k[ky + ryk ix, c] = sum_q y_right[ky, q] Bt[ix][c][q]
        g = GemmB{yc[k], 1, ryk, 0, 0,
                  ws + oB, 1, (long long)nk * ryp, (long long)Lk * nk * ryp, 0,
                  ws + oW[k], 1, R[k], ryk, 0,
                  ryk, Lk, nk * ryp, rxk, 1, 1.0, 0.0};
        if ((rc = gemm(c, g))) return rc;
    }

    // ---- left-to-right orthogonalisation against the sketch ----------------
    double* M = ws + oM0;
    double* Mn = ws + oM1;
    PTT_CUDA(ptt_launch(c, k_fill, dim3(1), dim3(32), 0, M, 1, 1.0));
    PTT_LAUNCHED(c);
    int r = 1;
    int zr[PTT_MAX_DIM + 1];
    zr[0] = 1;
    if ((rc = ptt_pull_desc(z))) return rc;
    for (int k = 0; k < d; k++) {
        const long long Rp = R[k + 1];
        const int nk = n[k], rxk = rx[k], ryk = ry[k], rxp = rx[k + 1], ryp = ry[k + 1];
        GemmB g;
        double* Zp = (k == d - 1) ? z->hd.core[k] : ws + oZ;
        if (!y) {
            // x alone: Z = M x_k, (r x r_k) times the core's right unfolding
            g = GemmB{M, 1, r, 0, 0,
                      xc[k], 1, rxk, 0, 0,
                      Zp, 1, r, 0, 0,
                      r, nk * rxp, rxk, 1, 1, 1.0, 0.0};
            if ((rc = gemm(c, g))) return rc;
        } else {
            // P[ix][q][c] = sum_ky M[c, ky + ryk ix] y_right[ky, q]
            g = GemmB{M, 1, r, (long long)r * ryk, 0,
                      yc[k], 1, ryk, 0, 0,
                      ws + oP, 1, r, (long long)r * nk * ryp, 0,
                      r, nk * ryp, ryk, rxk, 1, 1.0, 0.0};
            if ((rc = gemm(c, g))) return rc;
            // Z[c + r j, ly + ryp jx] = sum_ix P[ix][j + n ly][c] x[ix, j, jx]
            g = GemmB{ws + oP, 1, (long long)r * nk * ryp, r, (long long)r * nk,
                      xc[k], 1, (long long)rxk * nk, rxk, 0,
                      Zp, 1, (long long)r * nk * ryp, r, (long long)r * nk,
                      r, rxp, rxk, nk, ryp, 1.0, 0.0};
            if ((rc = gemm(c, g))) return rc;
        }
        if (k == d - 1) {
            zr[k] = r;
            zr[d] = 1;
            break;
        }
        const int Lp = L[k + 1];
        // Y = Z W_{k+1} into z core k, then QR in place (core k <- Q)
        // its first kernel also sets z's ranks r_k = r, r_{k+1} = Lp for the QR
        g = GemmB{ws + oZ, 1, (long long)r * nk, 0, 0,
                  ws + oW[k + 1], 1, Rp, 0, 0,
                  z->hd.core[k], 1, (long long)r * nk, 0, 0,
                  r * nk, Lp, (int)Rp, 1, 1, 1.0, 0.0,
                  (int*)((char*)z->dd + offsetof(DevDesc, r)), k, r, Lp};
        if ((rc = gemm(c, g))) return rc;
        {
            // QR of core k: ranks known here (no read-back); the QR swaps
            // core k with its second buffer, mirrored in the host shadow
            int rk[PTT_MAX_DIM + 1];
            for (int i = 0; i <= d; i++) rk[i] = 1;  // only core k is factored
            rk[k] = r;
            rk[k + 1] = Lp;
            if ((rc = ptt_round_phases_rk(z, rk, 0.0, NULL, 4, k))) return rc;
            double* t = z->hd.core[k];
            z->hd.core[k] = z->hd.alt[k];
            z->hd.alt[k] = t;
        }
        const int q = r * nk < Lp ? r * nk : Lp;
        // M' = Q^T Z   (q x Rp)
        g = GemmB{z->hd.core[k], (long long)r * nk, 1, 0, 0,
                  ws + oZ, 1, (long long)r * nk, 0, 0,
                  Mn, 1, q, 0, 0,
                  q, (int)Rp, r * nk, 1, 1, 1.0, 0.0};
        if ((rc = gemm(c, g))) return rc;
        double* t = M;
        M = Mn;
        Mn = t;
        zr[k] = r;
        r = q;
    }
    if ((rc = ptt_set_ranks_async(z, 0, zr, d + 1))) return rc;
    if (used)
        for (int k = 0; k <= d; k++) used[k] = L[k];
    return ptt_round_phases_rk(z, zr, tol, maxrank, 2, 0);
}

extern "C" int ptt_round_hadamard(const ptt_tt* x, const ptt_tt* y, ptt_tt* z, const int* ell, unsigned long long seed,
                                  double tol, const int* maxrank) {
    if (!y) return ptt_set_error(PTT_ERR_ARG, "ptt_round_hadamard: null factor");
    return sketch_round(x, y, z, ell, seed, tol, maxrank, NULL);
}

// Accept the sketch when every bond kept at most used[k] - pad ranks after
// the deterministic truncation, or when the sketch spanned the full bond
// rank (then nothing was lost).  Randomized range finding with oversampling
// p loses ~sigma_{l-p+1}; a truncation that stops p below l shows that
// sigma_{l-p+1} already lies in the dropped tail, below the threshold.
static int check_sketch(ptt_tt* z, const int* used, const int* full, int pad, int* accepted) {
    int r[PTT_MAX_DIM + 1];
    int rc = ptt_tt_get_ranks(z, r);
    if (rc) return rc;
    int ok = 1;
    for (int k = 1; k < z->d; k++)
        if (used[k] < full[k] && r[k] > used[k] - pad) ok = 0;
    *accepted = ok;
    return PTT_OK;
}

extern "C" int ptt_round_sketch(const ptt_tt* x, const ptt_tt* y, ptt_tt* z, const int* ell, unsigned long long seed,
                                double tol, const int* maxrank, int pad, int* accepted) {
    int used[PTT_MAX_DIM + 1], rx[PTT_MAX_DIM + 1], ry[PTT_MAX_DIM + 1], full[PTT_MAX_DIM + 1];
    if (!x || !z) return ptt_set_error(PTT_ERR_ARG, "ptt_round_sketch: null tensor");
    int rc = ptt_tt_get_ranks((ptt_tt*)x, rx);
    if (rc) return rc;
    if (y) {
        if ((rc = ptt_tt_get_ranks((ptt_tt*)y, ry))) return rc;
    } else {
        for (int k = 0; k <= x->d; k++) ry[k] = 1;
    }
    for (int k = 0; k <= x->d; k++) full[k] = rx[k] * ry[k];
    if ((rc = sketch_round(x, y, z, ell, seed, tol, maxrank, used))) return rc;
    if (accepted) return check_sketch(z, used, full, pad, accepted);
    return PTT_OK;
}

// ---------------------------------------------------------------------------
// autotuner of the contractions' tile width and split-K target: times the
// shapes the sketch rounding meets (a batch of 48 x 48 x 48 products, tiles
// of 32 or 64; one 40 x 40 product over K = 8192, split to fill 1, 2 or 4
// times the SM count) and keeps a setting only when it is >= 10 % faster
// than the built-in one.  Allocates its own operands; synchronises.
// ---------------------------------------------------------------------------
namespace {
__global__ void k_tune_val(double* p, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        p[e] = 1.0 / (double)(1 + (e * 7919) % 1021) - 0.0005;
}
}  // namespace

int ptt_gemm_autotune(ptt_ctx* c) {
    const int tm0 = c->gemm_tm64, fill0 = c->gemm_fill, tk = c->tkind;
    c->tkind = 0;
    double* buf = nullptr;
    const long long nA = 48LL * 48 * 256 * 3, nB = 40LL * 8192 * 2 + 40 * 40;
    const long long tot = nA > nB ? nA : nB;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = PTT_OK;
    PTT_CUDA(cudaMalloc(&buf, sizeof(double) * (size_t)tot));
    if ((rc = ptt_cuda_check(cudaEventCreate(&e0), "event")) || (rc = ptt_cuda_check(cudaEventCreate(&e1), "event"))) {
        cudaFree(buf);
        return rc;
    }
    k_tune_val<<<296, 256, 0, c->stream>>>(buf, tot);
    auto time_it = [&](const GemmB& g, float* best) -> int {
        float tmin = 1e30f;
        for (int rep = 0; rep < 6; rep++) {
            PTT_CUDA(cudaEventRecord(e0, c->stream));
            int r2 = gemm(c, g);
            if (r2) return r2;
            PTT_CUDA(cudaEventRecord(e1, c->stream));
            PTT_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            PTT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (rep > 0 && ms < tmin) tmin = ms;
        }
        *best = tmin;
        return PTT_OK;
    };
    // (1) a batch of 256 products of 48 x 48 x 48: 64-wide tiles from 48 on, or 32-wide
    GemmB ga = {};
    ga.A = buf; ga.ars = 1; ga.acs = 48; ga.ab1 = 48 * 48; ga.ab2 = 0;
    ga.B = buf + 48LL * 48 * 256; ga.brs = 1; ga.bcs = 48; ga.bb1 = 48 * 48; ga.bb2 = 0;
    ga.C = buf + 2LL * 48 * 48 * 256; ga.crs = 1; ga.ccs = 48; ga.cb1 = 48 * 48; ga.cb2 = 0;
    ga.M = ga.N = ga.K = 48; ga.nb1 = 256; ga.nb2 = 1; ga.alpha = 1.0; ga.beta = 0.0;
    float t64 = 0.f, t32 = 0.f;
    c->gemm_tm64 = 48;
    if (!rc) rc = time_it(ga, &t64);
    c->gemm_tm64 = 65;  // 48-wide products take 32-wide tiles
    if (!rc) rc = time_it(ga, &t32);
    const int tm_best = (t32 < 0.9f * t64) ? 65 : 48;
    // (2) one 40 x 40 product over K = 8192: split-K fill targets
    GemmB gb = {};
    gb.A = buf; gb.ars = 8192; gb.acs = 1;  // A row-major 40 x 8192
    gb.B = buf + 40LL * 8192; gb.brs = 1; gb.bcs = 8192;  // B column-major 8192 x 40
    gb.C = buf + 80LL * 8192; gb.crs = 40; gb.ccs = 1;
    gb.M = gb.N = 40; gb.K = 8192; gb.nb1 = gb.nb2 = 1; gb.alpha = 1.0; gb.beta = 0.0;
    const int fills[3] = {2 * c->nsm, c->nsm, 4 * c->nsm};
    float tf[3] = {1e30f, 1e30f, 1e30f};
    c->gemm_tm64 = tm_best;
    for (int i = 0; i < 3 && !rc; i++) {
        c->gemm_fill = fills[i];
        rc = time_it(gb, &tf[i]);
    }
    int fbest = 0;
    for (int i = 1; i < 3; i++)
        if (tf[i] < 0.9f * tf[0] && tf[i] < tf[fbest]) fbest = i;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamSynchronize(c->stream);
    cudaFree(buf);
    c->tkind = tk;
    if (rc) {
        c->gemm_tm64 = tm0;
        c->gemm_fill = fill0;
        return rc;
    }
    c->gemm_tm64 = tm_best;
    c->gemm_fill = fills[fbest];
    return PTT_OK;
}

extern "C" int ptt_ctx_autotune_gemm(const ptt_ctx* c, int* out2) {
    if (!c || !out2) return ptt_set_error(PTT_ERR_ARG, "ptt_ctx_autotune_gemm: bad arguments");
    out2[0] = c->gemm_tm64 > 0 ? c->gemm_tm64 : 48;
    out2[1] = c->gemm_fill > 0 ? c->gemm_fill : 2 * c->nsm;
    return PTT_OK;
}
