// Cholesky QR of unfoldings with up to 64 columns by the whole GPU (included
// by ptt_round.cu inside its anonymous namespace, after ptt_cholqr.cuh).
//
// At 64 columns a bond's unfolding (16384 x 64 doubles at d = 40, n = 256,
// rank 64: 8.4 MB) no longer fits in one cluster's shared memory, and the
// Householder TSQR costs one block barrier per reflector and tree level.
// Here the rows are spread over all SMs and the same Gram-stage sequence as
// the cluster kernel (ptt_cholqr.cuh) runs as one launch per stage:
//
//   stage 0        CTA b loads rows [b rpb, (b+1) rpb) of A, forms the
//                  partial Gram matrix of its rows;
//   stage s >= 1   CTA b loads its rows of Q_{s-1} (A for s = 1), applies the
//                  factor of the previous stage by a row-wise triangular solve
//                  (Q_s = Q_{s-1} R_s^{-1}), writes Q_s and forms the partial
//                  Gram matrix of Q_s;
//
// and the partials are summed in a fixed order by the last-arriving CTA of
// each group of GROUP CTAs (atomic ticket, no waiting), then by the
// last-arriving group, which takes the decision of the stage exactly as the
// cluster kernel does: done (max|Q^T Q - I| <= 1e-13), a first-order factor
// I + striu(E) + diag(E)/2 (finishing without another Gram stage when
// max|E| <= 1e-8), a Cholesky factor of G, or of G + sigma I when a pivot is
// not positive or the pivots span more than 12 decades (shifted Cholesky QR,
// Fukaya, Kannan, Nakatsukasa, Yamamoto, Yanagisawa, SIAM J. Sci. Comput. 42
// (2020), sigma = 11 (m c + c (c + 1)) u ||Q||_F^2).  The host launches MAXST
// stages; a stage finds the state left by the previous one and returns at
// once when the factorisation is finished or has fallen back.  The row-wise
// triangular solve changes A = Q R by O(u ||A||) per stage, so R carries the
// singular values to the accuracy of a Householder R.
//
// Q is written to Qbuf: LEFT -> alt[k] (m x c, column-major, its final place);
// RIGHT_T -> a scratch region (row-major rows of c), from which k_gq_write
// forms Q V_r after the bond's SVD.  A never changes, so a bond that falls
// back (NaN, zero matrix or column, no convergence in MAXST stages) is
// factored by the Householder TSQR from the same input; those kernels skip
// the bonds finished here (Plan::gqstate).
#pragma once

namespace gq {

constexpr int NT = 256;
constexpr int CB = 64;                 // column bound
constexpr int XP = CB + 8;             // pitch of the rows in shared memory: 8 mod 16 doubles, so the
                                       // four rows of an mma fragment load fall in the two halves of the banks
constexpr int RP = CB + 2;             // pitch of a factor R (row-major, upper triangular)
constexpr int GP = CB + 1;             // pitch of the Gram matrix of the deciding CTA
constexpr int TS = CB / 8;             // Gram tiles are TS x TS, 8 x 8 of them
constexpr int UP = 36 * TS * TS;       // entries of the 36 upper tiles
constexpr int GROUP = 8;               // CTAs summed by the first level
constexpr int RPB_MAX = 112;           // rows per CTA
constexpr int RPB_MIN = 16;
constexpr int MAXST = 8;               // stage launches per factorisation: an unfolding of condition ~1e16
                                       // (numerically rank-deficient) takes three shifted stages, a plain
                                       // one and a first-order finish -- seven launches
constexpr double TAU = 1e-13;
constexpr double FIRST = 1e-7;
constexpr double FIRST_DONE = 1e-8;
constexpr double U = 1.1102230246251565e-16;
constexpr int FSZ = CB * RP + CB;      // a factor and its inverse pivots
constexpr int SCR = CB * GP + 2 * FSZ + 64;  // Gram, two candidate factors, row broadcasts of the deciding CTA
constexpr size_t SMEM = sizeof(double) * ((size_t)RPB_MAX * XP + (size_t)SCR);
// the Ozaki Gram (ptt_ozaki.cuh): the digit slices take the scratch region
// and beyond once the rows are solved; its 64 x 65 sum buffer the rows' region
constexpr size_t SMEM_OZ = sizeof(double) * (size_t)RPB_MAX * XP + oz::SMEM;
static_assert(RPB_MAX == oz::KMAX, "one CTA's rows are one exact FP32 accumulation");
static_assert(SMEM_OZ >= SMEM && RPB_MAX * XP >= 64 * 65, "Ozaki buffers");
static_assert(CB * GP <= FSZ, "the accumulated R fits a factor buffer");
static_assert(CB * RP + CB <= SCR, "factor fits the scratch");

enum { RUN = 0, DONE = 1, FALLBACK = 2, FINISH = 4, CHOL = 8 };

__host__ __device__ __forceinline__ bool finished(int s) { return s == DONE || s == FINISH; }

// Record of the factorisation in flight (rec[0..)):
struct State {
    int state;   // RUN, DONE, FALLBACK, FINISH
    int fin;     // FINISH: the stage launch that applies the last factor
    int nst;     // factors applied
    int nshift;  // shifted stages (diagnostic)
    int m, c;
    int pad[2];
};

struct GQ {
    double* rec;         // State, then the factor and the accumulated R
    double* part;        // per-CTA partial Gram matrices (UP each)
    double* gpart;       // per-group sums
    double* qscr;        // Q rows of a RIGHT_T factorisation (row-major, pitch c)
    int* cnt;            // tickets: [group] ... [ngroups] = top; zero between launches
    int rpb;             // rows per CTA
};
constexpr long long O_FAC = 8;                   // CB x RP factor, then CB inverse pivots
constexpr long long O_T = O_FAC + CB * RP + CB;  // CB x CB accumulated R (row-major)
constexpr long long REC = O_T + CB * CB;

// rows per CTA and CTAs for an unfolding of at most mcap rows
__host__ __forceinline__ int rows_per_cta(long long mcap, int nsm) {
    long long r = (mcap + nsm - 1) / nsm;
    if (r < RPB_MIN) r = RPB_MIN;
    if (r > RPB_MAX) r = RPB_MAX;
    return (int)r;
}
__host__ __forceinline__ int ctas(long long mcap, int rpb) {
    long long b = (mcap + rpb - 1) / rpb;
    return (int)(b < 1 ? 1 : b);
}

// x <- x R^{-1} for the CTA's rows (h of them, zero rows up to a multiple of
// 8), one warp per 8-row tile, by 8-column blocks in order: the update of
// block J by the solved blocks, X_J - Y_{<J} R_{<J,J}, on the FP64 tensor
// cores (mma.m8n8k4, four columns of Y a step), then forward substitution in
// the 8 x 8 diagonal block, the row's four lanes passing each solved entry by
// a shuffle.  Rows are independent, so a warp needs no barrier.  R upper
// triangular (pitch RP), zero outside the c x c triangle; iv = inverse
// pivots, zero beyond c.
__device__ __forceinline__ void tile_solve(double* Xs, int h, const double* R, const double* iv, int c) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int li = lane >> 2, lk = lane & 3;
    const int ntile = (h + 7) >> 3, nb = (c + 7) >> 3;
    constexpr int NW = NT / 32;
    // two tiles at a time (t and t + NW), their dependent chains interleaved;
    // a warp with one tile left solves it twice and stores it once
    for (int t = warp; t < ntile; t += 2 * NW) {
        const bool two = t + NW < ntile;
        double* xa = Xs + (t * 8 + li) * XP;  // this lane's rows
        double* xb = two ? Xs + ((t + NW) * 8 + li) * XP : xa;
        for (int J = 0; J < nb; J++) {
            const double2 ca = *(const double2*)(xa + 8 * J + 2 * lk);
            const double2 cb = *(const double2*)(xb + 8 * J + 2 * lk);
            double a0 = ca.x, a1 = ca.y, b0 = cb.x, b1 = cb.y;  // columns 8J + 2lk, 8J + 2lk + 1
            for (int kk = 0; kk < 2 * J; kk++) {
                const double bv = R[(4 * kk + lk) * RP + 8 * J + li];
                const double ava = -xa[4 * kk + lk], avb = -xb[4 * kk + lk];
                asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                             : "+d"(a0), "+d"(a1)
                             : "d"(ava), "d"(bv));
                asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                             : "+d"(b0), "+d"(b1)
                             : "d"(avb), "d"(bv));
            }
            const double* Rb = R + 8 * J * RP + 8 * J;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int own = j >> 1;
                const double ivj = iv[8 * J + j];
                if (lk == own) {
                    if (j & 1) {
                        a1 *= ivj;
                        b1 *= ivj;
                    } else {
                        a0 *= ivj;
                        b0 *= ivj;
                    }
                }
                const double ya = __shfl_sync(0xffffffffu, (j & 1) ? a1 : a0, (lane & ~3) | own);
                const double yb = __shfl_sync(0xffffffffu, (j & 1) ? b1 : b0, (lane & ~3) | own);
                if (2 * lk > j) {
                    const double r = Rb[j * RP + 2 * lk];
                    a0 = fma(-ya, r, a0);
                    b0 = fma(-yb, r, b0);
                }
                if (2 * lk + 1 > j) {
                    const double r = Rb[j * RP + 2 * lk + 1];
                    a1 = fma(-ya, r, a1);
                    b1 = fma(-yb, r, b1);
                }
            }
            *(double2*)(xa + 8 * J + 2 * lk) = make_double2(a0, a1);
            if (two) *(double2*)(xb + 8 * J + 2 * lk) = make_double2(b0, b1);
            __syncwarp();
        }
    }
}

// Cholesky of one 32-column panel by one warp, lane = column: g[t] holds
// entry (t, lane) of the panel's symmetric block (rows t < 32); row j of the
// factor is broadcast through sRow.  Writes R[off + j][off + lane] (pitch RP)
// and iv[off + j] = 1 / R[off + j][off + j] for j < cc; tracks the pivots.
__device__ __forceinline__ void chol_panel(double (&g)[32], int cc, int off, double* R, double* iv, double* sRow,
                                           bool& ok, double& dmin, double& dmax) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < 32; j++) {
        if (j >= cc) continue;
        const double d = __shfl_sync(0xffffffffu, g[j], j);
        ok = ok && (d > 0.0);  // false for NaN
        dmin = fmin(dmin, d);
        dmax = fmax(dmax, d);
        const double dd = d > 0.0 ? d : 1.0;
        const double inv = rsqrt(dd);
        const double rj = (lane == j) ? dd * inv : ((lane > j && lane < cc) ? g[j] * inv : 0.0);
        sRow[lane] = rj;
        __syncwarp();
        if (lane > j && lane < cc) {
#pragma unroll
            for (int t = j + 1; t < 32; t++) g[t] = fma(-sRow[t], rj, g[t]);
        }
        if (lane >= j && lane < cc) R[(off + j) * RP + off + lane] = rj;
        if (lane == j) iv[off + j] = inv;
        __syncwarp();
    }
}

// Cholesky factor of G + shift I (c x c, pitch GP) by ONE warp in two
// 32-column panels: R11 = chol(G11); R12 = R11^{-T} G12 (forward
// substitution, lane = column); S = G22 - R12^T R12 (lane = column, in
// registers); R22 = chol(S).  Result R (row-major, pitch RP, zero outside the
// upper c x c triangle), iv[j] = 1 / R[j][j].  Returns false when a pivot is
// not positive (NaN included); *ratio = min/max pivot.  Two warps can form
// the plain and the shifted factor at once into different R buffers.
__device__ bool warp_chol64(const double* G, int c, double shift, double* R, double* iv, double* sRow, double* ratio) {
    const int lane = threadIdx.x & 31;
    for (int e = lane; e < CB * RP; e += 32) R[e] = 0.0;
    for (int e = lane; e < CB; e += 32) iv[e] = 0.0;
    __syncwarp();
    bool ok = true;
    double dmin = 1.0 / 0.0, dmax = 0.0;
    const int c1 = c < 32 ? c : 32;
    double g[32];
#pragma unroll
    for (int t = 0; t < 32; t++) g[t] = (t < c1 && lane < c1) ? G[t * GP + lane] + (t == lane ? shift : 0.0) : 0.0;
    chol_panel(g, c1, 0, R, iv, sRow, ok, dmin, dmax);
    if (c > 32) {
        const int c2 = c - 32, k = 32 + lane;
        const bool mine = lane < c2;
        // R12[:, k]: R11^T y = G[0:32, k]
        double y[32];
#pragma unroll
        for (int i = 0; i < 32; i++) y[i] = mine ? G[i * GP + k] : 0.0;
#pragma unroll
        for (int i = 0; i < 32; i++) {
            const double yi = y[i] * iv[i];
            y[i] = yi;
#pragma unroll
            for (int t = i + 1; t < 32; t++) y[t] = fma(-R[i * RP + t], yi, y[t]);
        }
        if (mine) {
#pragma unroll
            for (int i = 0; i < 32; i++) R[i * RP + k] = y[i];
        }
        __syncwarp();
        // P = R12^T R12 on the FP64 tensor cores (the 10 upper 8 x 8 tiles, k
        // over the 32 rows of R12), parked in the lower-left quarter of R,
        // which is zero in the result; S[32 + t][k] = G[32 + t][k] + shift
        // [t == lane] - P[t][lane] (only the upper entries t <= lane are used)
        {
            const int li = lane >> 2, lk = lane & 3;
            double p0[10], p1[10];
#pragma unroll
            for (int q = 0; q < 10; q++) {
                p0[q] = 0.0;
                p1[q] = 0.0;
            }
#pragma unroll
            for (int k0 = 0; k0 < 32; k0 += 4) {
                double f[4];
#pragma unroll
                for (int bb = 0; bb < 4; bb++) f[bb] = R[(k0 + lk) * RP + 32 + 8 * bb + li];
                int q = 0;
#pragma unroll
                for (int I = 0; I < 4; I++)
#pragma unroll
                    for (int J = I; J < 4; J++, q++)
                        asm volatile(
                            "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                            : "+d"(p0[q]), "+d"(p1[q])
                            : "d"(f[I]), "d"(f[J]));
            }
            int q = 0;
#pragma unroll
            for (int I = 0; I < 4; I++)
#pragma unroll
                for (int J = I; J < 4; J++, q++) {
                    R[(32 + 8 * I + li) * RP + 8 * J + 2 * lk] = p0[q];
                    R[(32 + 8 * I + li) * RP + 8 * J + 2 * lk + 1] = p1[q];
                }
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < 32; t++) {
            const double pt = R[(32 + t) * RP + lane];
            g[t] = (mine && t < c2) ? G[(32 + t) * GP + k] + (t == lane ? shift : 0.0) - pt : 0.0;
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < 32; t++) R[(32 + t) * RP + lane] = 0.0;
        __syncwarp();
        chol_panel(g, c2, 32, R, iv, sRow, ok, dmin, dmax);
    }
    __syncwarp();
    *ratio = dmax > 0.0 ? dmin / dmax : 0.0;
    return ok;
}

// Partial Gram matrix (upper 8 x 8 tiles) of the CTA's rows on the FP64
// tensor cores: warp w accumulates tiles w, w + 8, ... over all rows, four
// rows per mma.m8n8k4 (A = the tile's row-block columns transposed, B = its
// column-block columns), and writes them straight to P (tile q at P + 64 q).
__device__ __forceinline__ void gram_fp64(const double* Xs, int h, double* P) {
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int li = lane >> 2, lk = lane & 3;
    constexpr int NWP = NT / 32, TPW = (36 + NWP - 1) / NWP;
    double c0[TPW], c1[TPW];
    int oa[TPW], ob[TPW];
#pragma unroll
    for (int t = 0; t < TPW; t++) {
        int ti = 0, tj = 0;
        if (warp + NWP * t < 36) cq::upper_tile(warp + NWP * t, &ti, &tj);
        oa[t] = ti * TS + li;
        ob[t] = tj * TS + li;
        c0[t] = 0.0;
        c1[t] = 0.0;
    }
    for (int r = 0; r < h; r += 4) {
        const int row = r + lk;
        const double* xr = Xs + row * XP;
        const bool ok = row < h;
#pragma unroll
        for (int t = 0; t < TPW; t++) {
            if (warp + NWP * t < 36) {
                const double av = ok ? xr[oa[t]] : 0.0;
                const double bv = ok ? xr[ob[t]] : 0.0;
                asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                             : "+d"(c0[t]), "+d"(c1[t])
                             : "d"(av), "d"(bv));
            }
        }
    }
#pragma unroll
    for (int t = 0; t < TPW; t++)
        if (warp + NWP * t < 36)
            *(double2*)(P + (warp + NWP * t) * TS * TS + li * TS + 2 * lk) = make_double2(c0[t], c1[t]);
}

// One stage of the factorisation of core k's unfolding (mode); gridDim.x CTAs
// of g.rpb rows each.  OZ: the Gram partials by the Ozaki split on the
// fifth-generation tensor cores (ptt_ozaki.cuh) instead of FP64 mma.
template <bool OZ>
__global__ void __launch_bounds__(NT, 1) k_gq_stage(const DevDesc* D, int k, int mode, Plan pl, GQ g, double* ws,
                                                    int stage, long long* qstat) {
    PTT_PDL_ENTRY();
    extern __shared__ __align__(128) double gsm[];
    double* Xs = gsm;                     // rpb x XP rows
    double* sScr = Xs + RPB_MAX * XP;     // factor; Gram partials; decision arrays
    __shared__ int s_state, s_fin, s_ticket, s_flags, s_cok[2];
    __shared__ double s_cratio[2];
    __shared__ double s_red[NT / 32][2];
    State* st = (State*)g.rec;
    const View A = make_view(D, k, mode, false);
    const int m = A.m, c = A.c;
    const int tid = threadIdx.x;
    const int rpb = g.rpb, nb = (int)gridDim.x, b = (int)blockIdx.x;
    if (stage == 0) {
        if (c > CB || c < 1 || m < c || (long long)m > (long long)rpb * nb) {  // uniform
            if (b == 0 && tid == 0) {
                st->state = FALLBACK;
                st->nst = 0;
                st->m = m;
                st->c = c;
                if (qstat) atomicAdd((unsigned long long*)(qstat + 1), 1ull);
            }
            return;
        }
        if (pl.work && b == 0 && tid == 0) atomicAdd(pl.work, 16.0 * (double)m * (double)c);
    } else {
        if (tid == 0) {
            s_state = ldcg(&st->state);
            s_fin = ldcg(&st->fin);
        }
        __syncthreads();
        if (!(s_state == RUN || (s_state == FINISH && s_fin == stage))) return;
    }
    const int r0 = b * rpb;
    const int h = (m - r0) < rpb ? ((m - r0) > 0 ? (m - r0) : 0) : rpb;
    // Qbuf: where the Q_s rows live
    View Qv;
    if (mode == LEFT) {
        Qv.p = D->alt[k];
        Qv.rs = 1;
        Qv.cs = m;
    } else {
        Qv.p = g.qscr;
        Qv.rs = c;
        Qv.cs = 1;
    }
    const View& src = (stage <= 1) ? A : Qv;
    // this CTA's rows (zero beyond c), every element in flight by cp.async
    for (int e = tid; e < ((h + 7) & ~7) * XP; e += NT) Xs[e] = 0.0;  // whole 8-row tiles
    if (stage >= 1) {  // the factor of the previous stage (all loads in flight first)
        const double* F = g.rec + O_FAC;
        constexpr int FL = CB * RP + CB, FPT = (FL + NT - 1) / NT;
        double f[FPT];
#pragma unroll
        for (int k = 0; k < FPT; k++) f[k] = (tid + k * NT < FL) ? ldcg(F + tid + k * NT) : 0.0;
#pragma unroll
        for (int k = 0; k < FPT; k++)
            if (tid + k * NT < FL) sScr[tid + k * NT] = f[k];
    }
    __syncthreads();
    {
        const unsigned xs0 = (unsigned)__cvta_generic_to_shared(Xs);
        if (src.rs == 1) {
            // column-major: a warp copies 4 rows x 8 columns at a time (32
            // contiguous bytes of each column; the 4 rows fall in different
            // bank halves)
            const int nrb = (h + 3) / 4, ncb = (c + 7) / 8;
            const int lr = (tid & 31) & 3, lc = (tid & 31) >> 2;
            for (int t = tid >> 5; t < nrb * ncb; t += NT / 32) {
                const int cb = t / nrb, rb = t - cb * nrb;
                const int row = rb * 4 + lr, col = cb * 8 + lc;
                if (row < h && col < c) {
                    const double* gp = src.p + (long long)(r0 + row) + (long long)col * src.cs;
                    const unsigned sa = xs0 + 8u * (unsigned)(row * XP + col);
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gp) : "memory");
                }
            }
        } else {  // row-major rows of c: element f = row c + col, stepped without divisions
            const int dq = NT / c, dr = NT - dq * c;
            int row = tid / c, col = tid - row * c;
            for (; row < h;) {
                const double* gp = src.p + (long long)(r0 + row) * src.rs + (long long)col * src.cs;
                const unsigned sa = xs0 + 8u * (unsigned)(row * XP + col);
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gp) : "memory");
                row += dq;
                col += dr;
                if (col >= c) {
                    col -= c;
                    row++;
                }
            }
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
    }
    __syncthreads();
    if (stage >= 1) {
        tile_solve(Xs, h, sScr, sScr + CB * RP, c);
        __syncthreads();
        if (Qv.rs == 1) {  // column-major, in the load's 4 x 8 warp tiles
            const int nrb = (h + 3) / 4, ncb = (c + 7) / 8;
            const int lr = (tid & 31) & 3, lc = (tid & 31) >> 2;
            for (int t = tid >> 5; t < nrb * ncb; t += NT / 32) {
                const int cb = t / nrb, rb = t - cb * nrb;
                const int row = rb * 4 + lr, col = cb * 8 + lc;
                if (row < h && col < c) Qv.p[(long long)(r0 + row) + (long long)col * Qv.cs] = Xs[row * XP + col];
            }
        } else {
            const int dq = NT / c, dr = NT - dq * c;
            int row = tid / c, col = tid - row * c;
            for (; row < h;) {
                Qv.p[(long long)(r0 + row) * Qv.rs + (long long)col * Qv.cs] = Xs[row * XP + col];
                row += dq;
                col += dr;
                if (col >= c) {
                    col -= c;
                    row++;
                }
            }
        }
        if (s_state == FINISH) return;  // the last factor is applied: Q is final
    }
    // partial Gram matrix (upper 8 x 8 tiles) of this CTA's rows
    if constexpr (OZ)
        oz::gram_partial<NT>(Xs, XP, h, c, (unsigned char*)sScr, Xs, g.part + (long long)b * UP);
    else
        gram_fp64(Xs, h, g.part + (long long)b * UP);
    // first level: the last CTA of each group sums the group's partials
    const int ngroups = (nb + GROUP - 1) / GROUP;
    const int grp = b / GROUP;
    const int gsize = (nb - grp * GROUP) < GROUP ? (nb - grp * GROUP) : GROUP;
    __threadfence();
    __syncthreads();
    if (tid == 0) s_ticket = atomicAdd(&g.cnt[grp], 1);
    __syncthreads();
    if (s_ticket != gsize - 1) return;
    if (tid == 0) g.cnt[grp] = 0;
    __threadfence();
    {
        // every load of the thread's entries in flight before the sums (in
        // CTA order; absent CTAs add exact zeros)
        const double* P = g.part + (long long)grp * GROUP * UP;
        double* Gp = g.gpart + (long long)grp * UP;
        constexpr int UPT = (UP + NT - 1) / NT;
        double v[UPT][GROUP];
#pragma unroll
        for (int k = 0; k < UPT; k++) {
            const int u = tid + k * NT;
#pragma unroll
            for (int t = 0; t < GROUP; t++) v[k][t] = (u < UP && t < gsize) ? ldcg(P + (long long)t * UP + u) : 0.0;
        }
#pragma unroll
        for (int k = 0; k < UPT; k++) {
            const int u = tid + k * NT;
            double a = 0.0;
#pragma unroll
            for (int t = 0; t < GROUP; t++) a += v[k][t];
            if (u < UP) Gp[u] = a;
        }
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) s_ticket = atomicAdd(&g.cnt[ngroups], 1);
    __syncthreads();
    if (s_ticket != ngroups - 1) return;
    if (tid == 0) g.cnt[ngroups] = 0;
    __threadfence();
    // ---- the deciding CTA: G = sum of the groups in order --------------------
    double* sG = sScr;              // CB x GP
    double* sFa = sG + CB * GP;     // CB x RP factor + CB inverse pivots: plain Cholesky (or first order)
    double* sFb = sFa + FSZ;        // the same for the shifted Cholesky
    double* sRow = sFb + FSZ;       // 2 x 32 row broadcasts of the two Cholesky warps
    for (int e = tid; e < CB * GP; e += NT) sG[e] = 0.0;
    if (tid == 0) s_flags = 0;
    __syncthreads();
    {
        // the groups' sums in order, all of a thread's entries of eight groups
        // in flight at a time
        constexpr int UPT = (UP + NT - 1) / NT;
        double vs[UPT];
#pragma unroll
        for (int k = 0; k < UPT; k++) vs[k] = 0.0;
        for (int t0 = 0; t0 < ngroups; t0 += 8) {
            double w8[UPT][8];
#pragma unroll
            for (int k = 0; k < UPT; k++) {
                const int u = tid + k * NT;
#pragma unroll
                for (int t = 0; t < 8; t++)
                    w8[k][t] = (u < UP && t0 + t < ngroups) ? ldcg(g.gpart + (long long)(t0 + t) * UP + u) : 0.0;
            }
#pragma unroll
            for (int k = 0; k < UPT; k++)
#pragma unroll
                for (int t = 0; t < 8; t++) vs[k] += w8[k][t];
        }
#pragma unroll
        for (int k = 0; k < UPT; k++) {
            const int u = tid + k * NT;
            if (u >= UP) continue;
            const int qq = u / (TS * TS), w = u - qq * (TS * TS);
            int a0, b0;
            cq::upper_tile(qq, &a0, &b0);
            const int gi = a0 * TS + w / TS, gj = b0 * TS + w % TS;
            if (gi < c && gj < c) {
                sG[gi * GP + gj] = vs[k];
                sG[gj * GP + gi] = vs[k];
            }
        }
    }
    __syncthreads();
    // trace, max |G - I|, NaN, zero column
    double tr = 0.0, emax = 0.0;
    int fl = 0;  // bit 0: NaN, bit 1: a zero diagonal entry (an exactly zero column)
    for (int u = tid; u < c * c; u += NT) {
        const int i = u / c, j = u - (u / c) * c;
        const double v = sG[i * GP + j] - (i == j ? 1.0 : 0.0);
        if (!(v == v)) fl |= 1;
        emax = fmax(emax, fabs(v));
        if (i == j) {
            tr += sG[i * GP + j];
            if (sG[i * GP + j] == 0.0) fl |= 2;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        tr += __shfl_xor_sync(0xffffffffu, tr, o);
        emax = fmax(emax, __shfl_xor_sync(0xffffffffu, emax, o));
        fl |= __shfl_xor_sync(0xffffffffu, fl, o);
    }
    if ((tid & 31) == 0) {
        s_red[tid >> 5][0] = tr;
        s_red[tid >> 5][1] = emax;
        if (fl) atomicOr(&s_flags, fl);
    }
    __syncthreads();
    tr = 0.0;
    emax = 0.0;
    for (int w = 0; w < NT / 32; w++) {  // every thread, same order: same values
        tr += s_red[w][0];
        emax = fmax(emax, s_red[w][1]);
    }
    const bool nan = (s_flags & 1) || !(emax == emax);
    const bool zcol = (s_flags & 2) != 0;
    int nst = (stage == 0) ? 0 : ldcg(&st->nst);
    int nshift = (stage == 0) ? 0 : ldcg(&st->nshift);
    int dec;
    if (nan || !(tr > 0.0) || !(tr < 1.0 / 0.0) || (stage == 0 && zcol)) {
        dec = FALLBACK;
    } else if (stage >= 1 && emax <= TAU) {
        dec = DONE;
    } else if (stage >= 1 && emax <= FIRST) {
        for (int e = tid; e < CB * RP; e += NT) {
            const int j = e / RP, l = e - (e / RP) * RP;
            double v = 0.0;
            if (j < c && l < c) {
                if (l > j)
                    v = sG[j * GP + l];
                else if (l == j)
                    v = 1.0 + 0.5 * (sG[j * GP + j] - 1.0);
            }
            sFa[e] = v;
        }
        for (int j = tid; j < CB; j += NT) sFa[CB * RP + j] = j < c ? 1.0 / (1.0 + 0.5 * (sG[j * GP + j] - 1.0)) : 0.0;
        dec = emax <= FIRST_DONE ? FINISH : RUN;
    } else if (stage == MAXST - 1) {
        dec = FALLBACK;
    } else {
        // plain (warp 0) and shifted (warp 1) Cholesky at once; the plain one
        // is kept when its pivots span less than 12 decades
        if (tid < 64) {
            const int w = tid >> 5;
            const double sigma = w ? 11.0 * ((double)m * c + (double)c * (c + 1)) * U * tr : 0.0;
            double ratio;
            double* F = w ? sFb : sFa;
            const bool ok = warp_chol64(sG, c, sigma, F, F + CB * RP, sRow + 32 * w, &ratio);
            if ((tid & 31) == 0) {
                s_cok[w] = ok;
                s_cratio[w] = ratio;
            }
        }
        dec = CHOL;
    }
    __syncthreads();
    bool use_b = false;
    if (dec == CHOL) {
        if (s_cok[0] && s_cratio[0] >= 1e-12) {
            dec = RUN;
        } else if (s_cok[1]) {
            dec = RUN;
            use_b = true;
            nshift++;
        } else {
            dec = FALLBACK;
        }
    }
    if (stage == MAXST - 1 && (dec == RUN || dec == FINISH)) dec = FALLBACK;  // no launch left to apply it
    double* sF = use_b ? sFb : sFa;  // the factor applied next
    double* sT = use_b ? sFa : sFb;  // the accumulated R of the factors applied so far
    {
        constexpr int TPT = (CB * GP + NT - 1) / NT;
        double tv[TPT];
#pragma unroll
        for (int k = 0; k < TPT; k++) {
            const int e = tid + k * NT;
            const int i = e / GP, j = e - (e / GP) * GP;
            tv[k] = (e >= CB * GP) ? 0.0
                    : (stage == 0) ? ((i == j && i < c) ? 1.0 : 0.0)
                    : ((j < CB) ? ldcg(g.rec + O_T + i * CB + j) : 0.0);
        }
#pragma unroll
        for (int k = 0; k < TPT; k++)
            if (tid + k * NT < CB * GP) sT[tid + k * NT] = tv[k];
    }
    __syncthreads();
    if (dec == RUN || dec == FINISH) {
        // new accumulated R = F T (both upper triangular) into sG: each thread
        // a 4 x 4 block; at stage 0 T = I and it is F itself
        {
            const int bi = (tid >> 4) * 4, bj = (tid & 15) * 4;
            double acc[4][4];
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
            if (stage == 0) {
#pragma unroll
                for (int a = 0; a < 4; a++)
#pragma unroll
                    for (int b = 0; b < 4; b++) acc[a][b] = sF[(bi + a) * RP + bj + b];
            } else if (bj + 3 >= bi) {
                for (int t = bi; t <= bj + 3 && t < CB; t++) {
                    double fa[4], tb[4];
#pragma unroll
                    for (int a = 0; a < 4; a++) fa[a] = sF[(bi + a) * RP + t];
#pragma unroll
                    for (int b = 0; b < 4; b++) tb[b] = sT[t * GP + bj + b];
#pragma unroll
                    for (int a = 0; a < 4; a++)
#pragma unroll
                        for (int b = 0; b < 4; b++) acc[a][b] = fma(fa[a], tb[b], acc[a][b]);
                }
            }
            // F and T are upper triangular and zero beyond c: the products
            // outside the upper c x c triangle are exact zeros
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int b = 0; b < 4; b++) sG[(bi + a) * GP + bj + b] = (bj + b >= bi + a) ? acc[a][b] : 0.0;
        }
        __syncthreads();
        double* F = g.rec + O_FAC;
        for (int e = tid; e < CB * RP + CB; e += NT) F[e] = sF[e];
        double* T = g.rec + O_T;
        for (int e = tid; e < CB * CB; e += NT) T[e] = sG[(e / CB) * GP + (e % CB)];
        nst++;
    }
    const double* Rfin = (dec == DONE) ? sT : sG;  // FINISH: the new accumulated R
    if (dec == DONE || dec == FINISH) {
        double* Rs = ws + pl.o_Rn;  // root slot (row-major CT x CT)
        for (int e = tid; e < pl.CT * pl.CT; e += NT) {
            const int i = e / pl.CT, j = e - (e / pl.CT) * pl.CT;
            Rs[e] = (i < c && j < c && j >= i) ? Rfin[i * GP + j] : 0.0;
        }
        if (tid == 0) {
            Info* info = pl.info;
            info->m = m;
            info->c = c;
            info->q = c;
            info->rank = 0;
            info->status = 0;
            if (qstat) {
                atomicAdd((unsigned long long*)qstat, 1ull);
                atomicAdd((unsigned long long*)(qstat + 2), (unsigned long long)(stage + 1));
            }
        }
    }
    if (tid == 0) {
        if (dec == FALLBACK && qstat) atomicAdd((unsigned long long*)(qstat + 1), 1ull);
        st->fin = stage + 1;
        st->nst = nst;
        st->nshift = nshift;
        st->m = m;
        st->c = c;
        __threadfence();
        st->state = dec;
    }
}

// alt[k][row * rank + col] = (Q V_r)(row, col) for a RIGHT_T bond this path
// finished: Q rows in g.qscr (row-major, pitch c), V_r at the root B slot
// (row-major CT x KC).  One block per WROWS rows; the writes of a block are
// one contiguous range.
constexpr int WROWS = 16;
__global__ void __launch_bounds__(NT) k_gq_write(const DevDesc* D, int k, Plan pl, GQ g, double* ws) {
    PTT_PDL_ENTRY();
    __shared__ double sB[CB * (CB + 1)];
    __shared__ double sQ[WROWS * (CB + 1)];
    if (!finished(ldcg((const int*)g.rec))) return;
    const Info* info = pl.info;
    if (info->status) return;
    const int m = info->m, c = info->c, rank = info->rank;
    const int tid = threadIdx.x;
    const double* Bn = ws + pl.o_Bn;
    for (int e = tid; e < CB * CB; e += NT) {
        const int t = e / CB, l = e - (e / CB) * CB;
        sB[t * (CB + 1) + l] = (t < c && l < rank) ? Bn[(long long)t * pl.KC + l] : 0.0;
    }
    double* out = D->alt[k];
    for (int r0 = blockIdx.x * WROWS; r0 < m; r0 += gridDim.x * WROWS) {
        const int h = (m - r0) < WROWS ? (m - r0) : WROWS;
        __syncthreads();
        for (int e = tid; e < WROWS * CB; e += NT) {
            const int row = e / CB, t = e - (e / CB) * CB;
            sQ[row * (CB + 1) + t] = (row < h && t < c) ? g.qscr[(long long)(r0 + row) * c + t] : 0.0;
        }
        __syncthreads();
        for (int e = tid; e < h * rank; e += NT) {
            const int row = e / rank, col = e - (e / rank) * rank;
            double y0 = 0.0, y1 = 0.0;
#pragma unroll 8
            for (int t = 0; t < CB; t += 2) {
                y0 = fma(sQ[row * (CB + 1) + t], sB[t * (CB + 1) + col], y0);
                y1 = fma(sQ[row * (CB + 1) + t + 1], sB[(t + 1) * (CB + 1) + col], y1);
            }
            out[(long long)r0 * rank + e] = y0 + y1;
        }
    }
}

// G = A^T A of a column-major m x c matrix (c <= CB, leading dimension lda),
// the Gram matrix of an unfolding on its own (ptt_gram): CTA b forms the
// partial of rows [b RPB_MAX, (b + 1) RPB_MAX) -- on the FP64 tensor cores,
// or by the Ozaki split on tcgen05 when OZ -- the last-arriving CTA of each
// group of GROUP sums the group's partials in CTA order, the last-arriving
// group sums the groups in order and writes G (c x c, column-major, both
// triangles).  Deterministic; no CTA waits for another.
template <bool OZ>
__global__ void __launch_bounds__(NT, 1) k_gram(const double* A, long long m, int c, long long lda, double* part,
                                                double* gpart, int* cnt, double* G) {
    extern __shared__ __align__(128) double gsm[];
    double* Xs = gsm;
    __shared__ int s_ticket;
    const int tid = threadIdx.x, b = (int)blockIdx.x, nb = (int)gridDim.x;
    const long long r0 = (long long)b * RPB_MAX;
    const int h = (m - r0) < RPB_MAX ? (int)(m - r0) : RPB_MAX;
    for (int e = tid; e < RPB_MAX * XP; e += NT) Xs[e] = 0.0;
    __syncthreads();
    for (int e = tid; e < h * c; e += NT) {
        const int col = e / h, row = e - col * h;
        Xs[row * XP + col] = A[r0 + row + (long long)col * lda];
    }
    __syncthreads();
    if constexpr (OZ)
        oz::gram_partial<NT>(Xs, XP, h, c, (unsigned char*)(Xs + RPB_MAX * XP), Xs, part + (long long)b * UP);
    else
        gram_fp64(Xs, h, part + (long long)b * UP);
    const int ngroups = (nb + GROUP - 1) / GROUP, grp = b / GROUP;
    const int gsize = (nb - grp * GROUP) < GROUP ? (nb - grp * GROUP) : GROUP;
    __threadfence();
    __syncthreads();
    if (tid == 0) s_ticket = atomicAdd(&cnt[grp], 1);
    __syncthreads();
    if (s_ticket != gsize - 1) return;
    if (tid == 0) cnt[grp] = 0;
    __threadfence();
    for (int u = tid; u < UP; u += NT) {
        double a = 0.0;
        for (int t = 0; t < gsize; t++) a += ldcg(part + (long long)(grp * GROUP + t) * UP + u);
        gpart[(long long)grp * UP + u] = a;
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) s_ticket = atomicAdd(&cnt[ngroups], 1);
    __syncthreads();
    if (s_ticket != ngroups - 1) return;
    if (tid == 0) cnt[ngroups] = 0;
    __threadfence();
    for (int u = tid; u < UP; u += NT) {
        double a = 0.0;
        for (int t = 0; t < ngroups; t++) a += ldcg(gpart + (long long)t * UP + u);
        int ti = 0, tj = 0;
        cq::upper_tile(u >> 6, &ti, &tj);
        const int i = ti * TS + ((u >> 3) & 7), j = tj * TS + (u & 7);
        if (i < c && j < c && (ti < tj || i <= j)) {  // a diagonal tile's upper half
            G[i + (long long)j * c] = a;
            G[j + (long long)i * c] = a;
        }
    }
}

}  // namespace gq
