// Householder factorisation kernels of the TSQR tree (included by
// ptt_round.cu inside its anonymous namespace).
//
// Thread layout (256 threads): column slot cs = tid/8 owns columns
// l = cs + 32u, row part p = tid%8 owns rows t = p + 8v.  The tile being
// factored lives in registers a[u][v]; the current reflector's vector is
// published to a double-buffered shared vector, so each reflector costs one
// block barrier and no shared-memory traffic for the tile itself.  The
// triangle R of a TSQRT lives in shared memory (row-major, CT x CT).
#pragma once

template <int CT>
struct FCfg {
    static constexpr int NU = CT / 32;        // columns per thread
    static constexpr int NV = H / 8;          // chunk rows per thread
    static constexpr int NG = CT / 8;         // GEQRT block rows per thread
    static constexpr int NR = NG > NV ? NG : NV;
    static constexpr int VB = CT > H ? CT : H;  // reflector buffer length
};

// Householder vector of (alpha; x) with ||x||^2 = s2 (LAPACK dlarfg convention:
// no reflection when x == 0).
// With nrm = sqrt(alpha^2 + s2) and beta = -sign(alpha) nrm:
//   tau = (beta - alpha)/beta = 1 + |alpha|/nrm,  1/(alpha - beta) = sign(alpha)/(|alpha| + nrm)
// so one reciprocal square root and one reciprocal replace a square root and
// two divisions on the critical path of every reflector.
__device__ __forceinline__ void hh_params(double alpha, double s2, double* beta, double* tau, double* sc) {
    if (s2 > 0.0) {
        const double n2 = fma(alpha, alpha, s2);
        const double rs = rsqrt(n2);
        const double nrm = n2 * rs;
        const double aa = fabs(alpha);
        *beta = -copysign(nrm, alpha);
        *tau = fma(aa, rs, 1.0);
        *sc = copysign(__drcp_rn(aa + nrm), alpha);
    } else {
        *beta = alpha;
        *tau = 0.0;
        *sc = 0.0;
    }
}

// QR of the CT x CT tile in registers (rows >= valid rows are zero).
// On exit rows t <= l hold R, rows t > l hold the vectors (unit diagonal).
template <int CT>
__device__ void geqrt_reg(double (&a)[FCfg<CT>::NU][FCfg<CT>::NR], double* vbuf, double* tau_s, int c, int tid) {
    constexpr int NU = FCfg<CT>::NU, NG = FCfg<CT>::NG, VB = FCfg<CT>::VB;
    const int cs = tid >> 3, p = tid & 7;
    const unsigned gm = group_mask8(tid);
    for (int j = 0; j < c; j++) {
        double* vb = vbuf + (j & 1) * VB;
        if ((j & 31) == cs) {
            const int uo = j >> 5;
            double s2 = 0.0, cand = 0.0;
#pragma unroll
            for (int u = 0; u < NU; u++)
                if (u == uo) {
#pragma unroll
                    for (int v = 0; v < NG; v++) {
                        const int t = p + 8 * v;
                        const double x = a[u][v];
                        if (t > j) s2 += x * x;
                        if (t == j) cand = x;
                    }
                }
            s2 = gsum8(s2, gm);
            const double alpha = __shfl_sync(gm, cand, ((tid & 31) & ~7) | (j & 7));
            double beta, tau, sc;
            hh_params(alpha, s2, &beta, &tau, &sc);
#pragma unroll
            for (int u = 0; u < NU; u++)
                if (u == uo) {
#pragma unroll
                    for (int v = 0; v < NG; v++) {
                        const int t = p + 8 * v;
                        double x = a[u][v];
                        if (t > j) {
                            x *= sc;
                            a[u][v] = x;
                            vb[t] = x;
                        } else if (t == j) {
                            a[u][v] = beta;
                            vb[t] = 1.0;
                        } else {
                            vb[t] = 0.0;
                        }
                    }
                }
            if (p == 0) tau_s[j] = tau;
        }
        __syncthreads();
        const double tau = tau_s[j];
        if (tau != 0.0) {
#pragma unroll
            for (int u = 0; u < NU; u++) {
                const int l = cs + 32 * u;
                const bool act = (l > j) && (l < c);
                double da = 0.0, db = 0.0;
                if (act) {
#pragma unroll
                    for (int v = 0; v < NG; v += 2) {
                        da = fma(vb[p + 8 * v], a[u][v], da);
                        db = fma(vb[p + 8 * v + 8], a[u][v + 1], db);
                    }
                }
                const double dot = gsum8(da + db, 0xffffffffu);
                if (act) {
                    const double tw = tau * dot;
#pragma unroll
                    for (int v = 0; v < NG; v++) a[u][v] -= tw * vb[p + 8 * v];
                }
            }
        }
    }
}

// Eliminate an H-row chunk (registers) into the triangle Rb (TSQRT).
// Reflector j: pivot Rb[j][j], vector = chunk column j; on exit the chunk
// holds the vectors.
template <int CT>
__device__ void tsqrt_reg(double (&a)[FCfg<CT>::NU][FCfg<CT>::NR], double* Rb, double* vbuf, double* tau_s, int c,
                          int tid) {
    constexpr int NU = FCfg<CT>::NU, NV = FCfg<CT>::NV, VB = FCfg<CT>::VB;
    const int cs = tid >> 3, p = tid & 7;
    const unsigned gm = group_mask8(tid);
    for (int j = 0; j < c; j++) {
        double* vb = vbuf + (j & 1) * VB;
        if ((j & 31) == cs) {
            const int uo = j >> 5;
            double s2a = 0.0, s2b = 0.0;
#pragma unroll
            for (int u = 0; u < NU; u++)
                if (u == uo) {
#pragma unroll
                    for (int v = 0; v < NV; v += 2) {
                        s2a = fma(a[u][v], a[u][v], s2a);
                        s2b = fma(a[u][v + 1], a[u][v + 1], s2b);
                    }
                }
            const double s2 = gsum8(s2a + s2b, gm);
            const double alpha = Rb[j * CT + j];
            double beta, tau, sc;
            hh_params(alpha, s2, &beta, &tau, &sc);
#pragma unroll
            for (int u = 0; u < NU; u++)
                if (u == uo) {
#pragma unroll
                    for (int v = 0; v < NV; v++) {
                        const double x = a[u][v] * sc;
                        a[u][v] = x;
                        vb[p + 8 * v] = x;
                    }
                }
            __syncwarp(gm);
            if (p == 0) {
                Rb[j * CT + j] = beta;
                tau_s[j] = tau;
            }
        }
        __syncthreads();
        const double tau = tau_s[j];
        if (tau != 0.0) {
#pragma unroll
            for (int u = 0; u < NU; u++) {
                const int l = cs + 32 * u;
                const bool act = (l > j) && (l < c);
                double da = 0.0, db = 0.0, rjl = 0.0;
                if (act) {
                    rjl = Rb[j * CT + l];
#pragma unroll
                    for (int v = 0; v < NV; v += 2) {
                        da = fma(vb[p + 8 * v], a[u][v], da);
                        db = fma(vb[p + 8 * v + 8], a[u][v + 1], db);
                    }
                }
                const double dot = gsum8(da + db, 0xffffffffu);
                if (act) {
                    const double tw = tau * (rjl + dot);
#pragma unroll
                    for (int v = 0; v < NV; v++) a[u][v] -= tw * vb[p + 8 * v];
                    if (p == 0) Rb[j * CT + l] = rjl - tw;
                }
            }
        }
    }
}

// Load rows [r0, r0+h) x columns [0, c) of the view into registers (zero pad).
template <int CT, int NROW>
__device__ __forceinline__ void load_tile(double (&a)[FCfg<CT>::NU][FCfg<CT>::NR], const View& A, int r0, int h, int c,
                                          int tid) {
    constexpr int NU = FCfg<CT>::NU;
    const int cs = tid >> 3, p = tid & 7;
#pragma unroll
    for (int u = 0; u < NU; u++) {
        const int l = cs + 32 * u;
#pragma unroll
        for (int v = 0; v < NROW; v++) {
            const int t = p + 8 * v;
            a[u][v] = (t < h && l < c) ? A.p[(long long)(r0 + t) * A.rs + (long long)l * A.cs] : 0.0;
        }
    }
}

template <int CT, int NROW>
__device__ __forceinline__ void store_tile(const double (&a)[FCfg<CT>::NU][FCfg<CT>::NR], const View& A, int r0, int h,
                                           int c, int tid, bool strict_lower) {
    constexpr int NU = FCfg<CT>::NU;
    const int cs = tid >> 3, p = tid & 7;
#pragma unroll
    for (int u = 0; u < NU; u++) {
        const int l = cs + 32 * u;
#pragma unroll
        for (int v = 0; v < NROW; v++) {
            const int t = p + 8 * v;
            if (t < h && l < c && (!strict_lower || t > l)) A.p[(long long)(r0 + t) * A.rs + (long long)l * A.cs] = a[u][v];
        }
    }
}

// ---------------------------------------------------------------------------
// factor kernel: one block per leaf, then the last-arriving block of every
// node eliminates its sibling's triangle (no waiting on other blocks).
// ---------------------------------------------------------------------------
template <int CT>
__global__ void __launch_bounds__(NT, 1) k_tsqr_factor(const DevDesc* D, int kcore, int mode, Plan pl, double* ws,
                                                       int* status) {
    constexpr int NU = FCfg<CT>::NU, NV = FCfg<CT>::NV, NG = FCfg<CT>::NG, NR = FCfg<CT>::NR, VB = FCfg<CT>::VB;
    PTT_PDL_ENTRY();
    if (gq_finished(pl)) return;  // factored by the grid Cholesky QR
    extern __shared__ double sm[];
    double* Rb = sm;                 // CT x CT, row-major
    double* vbuf = Rb + CT * CT;     // 2 x VB
    double* tau_s = vbuf + 2 * VB;   // CT
    __shared__ int s_flag;
    const int tid = threadIdx.x;
    const int cs = tid >> 3, p = tid & 7;
    const View A = make_view(D, kcore, mode, false);
    const int m = A.m, c = A.c;
    const int P = pl.P, leaf = blockIdx.x;
    double* Rn = ws + pl.o_Rn;
    const bool bad = (c > CT || c < 1 || m < 1);
    // algorithmic bytes of this factorisation: read the m x c unfolding and
    // write the Householder vectors back in place (16 m c bytes)
    if (leaf == 0 && tid == 0 && !bad && pl.work) atomicAdd(pl.work, 16.0 * (double)m * (double)c);
    if (leaf == 0 && tid == 0) {
        pl.info->m = m;
        pl.info->c = c;
        pl.info->q = m < c ? m : c;
        pl.info->rank = 0;
        pl.info->status = bad ? 1 : 0;
        if (bad) PTT_STATUS_SET(status, PTT_ERR_CAPACITY);
    }
    if (bad) return;
    int r0, r1;
    leaf_range(m, pl.L, P, leaf, &r0, &r1);
    const int rows = r1 - r0;
    const int slot = P - 1 + leaf;
    double* tau_leaf = ws + pl.o_tau_leaf + (long long)leaf * pl.KL * CT;
    double a[NU][NR];
    if (rows > 0) {
        const int rb = rows < c ? rows : c;
        load_tile<CT, NG>(a, A, r0, rb, c, tid);
        geqrt_reg<CT>(a, vbuf, tau_s, c, tid);
        store_tile<CT, NG>(a, A, r0, rb, c, tid, true);
        // R to shared memory (zero below the diagonal and outside c)
#pragma unroll
        for (int u = 0; u < NU; u++) {
            const int l = cs + 32 * u;
#pragma unroll
            for (int v = 0; v < NG; v++) {
                const int t = p + 8 * v;
                Rb[t * CT + l] = (t <= l && l < c) ? a[u][v] : 0.0;
            }
        }
        for (int j = tid; j < CT; j += NT) tau_leaf[j] = j < c ? tau_s[j] : 0.0;
        __syncthreads();
        int s = 0;
        for (int t0 = r0 + rb; t0 < r1; t0 += H, s++) {
            const int h = (r1 - t0) < H ? (r1 - t0) : H;
            load_tile<CT, NV>(a, A, t0, h, c, tid);
            tsqrt_reg<CT>(a, Rb, vbuf, tau_s, c, tid);
            store_tile<CT, NV>(a, A, t0, h, c, tid, false);
            __syncthreads();
            for (int j = tid; j < CT; j += NT) tau_leaf[(long long)(1 + s) * CT + j] = j < c ? tau_s[j] : 0.0;
        }
        __syncthreads();
        double* Ro = Rn + (long long)slot * CT * CT;
        for (int e = tid; e < CT * CT; e += NT) Ro[e] = Rb[e];
    }
    if (tid == 0) pl.qn[slot] = rows > 0 ? (rows < c ? rows : c) : 0;

    int node = slot;
    while (node > 0) {
        const int par = (node - 1) >> 1;
        __threadfence();
        __syncthreads();
        if (tid == 0) s_flag = atomicAdd(&pl.cnt[par], 1);
        __syncthreads();
        if (s_flag == 0) return;
        __threadfence();
        if (tid == 0) pl.cnt[par] = 0;
        const int cl = 2 * par + 1, cr = 2 * par + 2;
        const int qL = ldcg(&pl.qn[cl]), qR = ldcg(&pl.qn[cr]);
        double* Rp = Rn + (long long)par * CT * CT;
        if (qL > 0 && qR > 0) {
            if ((qL != c || qR != c) && tid == 0) PTT_STATUS_SET(status, PTT_ERR_NUMERIC);
            const double* RL = Rn + (long long)cl * CT * CT;
            double* RR = Rn + (long long)cr * CT * CT;
            for (int e = tid; e < CT * CT; e += NT) Rb[e] = ldcg(RL + e);
            View RV;
            RV.p = RR;
            RV.rs = CT;
            RV.cs = 1;
            RV.m = CT;
            RV.c = CT;
            for (int half = 0; half < pl.NH; half++) {
                const int h0 = half * H;
                if (h0 >= c) break;
                const int h = (c - h0) < H ? (c - h0) : H;
                __syncthreads();
#pragma unroll
                for (int u = 0; u < NU; u++) {
                    const int l = cs + 32 * u;
#pragma unroll
                    for (int v = 0; v < NV; v++) {
                        const int t = p + 8 * v;
                        a[u][v] = (t < h && l < c) ? ldcg(RR + (long long)(h0 + t) * CT + l) : 0.0;
                    }
                }
                tsqrt_reg<CT>(a, Rb, vbuf, tau_s, c, tid);
                store_tile<CT, NV>(a, RV, h0, h, CT, tid, false);
                __syncthreads();
                double* tn = ws + pl.o_tau_node + ((long long)par * pl.NH + half) * CT;
                for (int j = tid; j < CT; j += NT) tn[j] = j < c ? tau_s[j] : 0.0;
            }
            __syncthreads();
            for (int e = tid; e < CT * CT; e += NT) Rp[e] = Rb[e];
            if (tid == 0) {
                pl.qn[par] = c;
                pl.pass[par] = 0;
            }
        } else {
            const int which = qL > 0 ? 1 : (qR > 0 ? 2 : 3);
            if (which != 3) {
                const double* src = Rn + (long long)(which == 1 ? cl : cr) * CT * CT;
                for (int e = tid; e < CT * CT; e += NT) Rp[e] = ldcg(src + e);
            }
            if (tid == 0) {
                pl.qn[par] = which == 1 ? qL : (which == 2 ? qR : 0);
                pl.pass[par] = which;
            }
        }
        node = par;
    }
}
