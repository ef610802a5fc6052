// Cholesky QR of unfoldings with at most 32 columns (included by ptt_round.cu
// inside its anonymous namespace, after the warp-level TSQR).
//
// The Householder TSQR is a chain of c x (tree depth + 1) dependent reflector
// steps; here the only sequential work is a c-step Cholesky of a c x c Gram
// matrix per stage.  A = Q R is computed as a sequence of Gram stages: stage
// s holds the rows of Q_s = A R_1^{-1} ... R_s^{-1} (Q_0 = A; each stage
// applies its new factor to the rows by a triangular solve), forms their Gram
// matrix G_s = Q_s^T Q_s, and from it
//   * s >= 1 and max|G_s - I| <= TAU: Q_s is orthonormal -- done, R = R_s ... R_1;
//   * s >= 1 and max|G_s - I| <= FIRST: R_{s+1} = I + striu(E) + diag(E)/2 with
//     E = G_s - I, the Cholesky factor of I + E to first order (Q_s R_{s+1}^{-1}
//     is then orthonormal to O(c^2 max|E|^2)); when max|E| <= FIRST_DONE that
//     is below TAU and Q_s R_{s+1}^{-1} is final without another Gram stage;
//   * otherwise R_{s+1} = chol(G_s), or chol(G_s + sigma I) when a pivot is not
//     positive or the pivots span more than 12 decades (condition > 1e6) --
//     two warps form both factors at once and the plain one is kept if valid:
//     shifted Cholesky QR (Fukaya, Kannan, Nakatsukasa, Yamamoto, Yanagisawa,
//     SIAM J. Sci. Comput. 42 (2020)) with their shift
//     sigma = 11 (m c + c (c + 1)) u ||Q_s||_F^2, which cannot break down and
//     shrinks the condition number by ~sqrt(sigma) / ||Q_s||.
// An unshifted stage on a matrix of condition kappa < 1e6 leaves an error
// O(u kappa^2) that the next stages remove (repeated Cholesky QR, Yamamoto,
// Nakatsukasa, Yanagisawa, Fukaya, ETNA 44 (2015)).  Each stage changes A = Q R
// by O(u ||A||), so the R handed to the SVD carries the singular values of A to
// the same absolute accuracy as a Householder R.  Condition numbers up to
// 1e20 and exactly repeated columns converge within six stages.
//
// One thread-block cluster factors one unfolding: CTA b of the cluster keeps
// rows [b h, (b+1) h) (h = ceil(m / CS)) in shared memory for all stages, every CTA writes
// the partial Gram matrix of its rows into its shared memory, and after a
// cluster barrier every CTA sums all partials (distributed shared memory, CTA
// order 0..CS-1) and runs the same Cholesky -- identical data and arithmetic,
// so all CTAs take the same decisions and nothing is broadcast.  The partials
// alternate between two buffers, so one barrier per stage suffices.  Only the
// upper TS x TS tiles of the symmetric Gram matrix are formed (36 tiles x 7
// row groups of threads), and the rows arrive by cp.async.
//
// On success Q is written once: LEFT -> alt[k] (m x c, column-major), RIGHT_T
// -> core[k] in place (row-major rows of c; k_cq_write forms Q V_r from it
// after the bond's SVD).  A bond that does not converge within MAXST stages or
// meets a NaN, a zero matrix or an exactly zero column is left untouched and
// falls back to the Householder TSQR: k_wfactor / k_wapply skip the bonds
// finished here and k_cq_write skips the others.
#pragma once

namespace cq {

namespace cg = cooperative_groups;

constexpr int NT = 256;       // threads per CTA
constexpr int MAXST = 7;      // Gram stages per factorisation
constexpr int CSMAX = 16;     // CTAs per cluster (non-portable size)
constexpr int RTARGET = 384;  // rows per CTA the cluster size aims at
constexpr int NG = 7;         // row groups of the Gram threads (36 tiles x 7 = 252)
constexpr double TAU = 1e-13;
constexpr double FIRST = 1e-7;
constexpr double FIRST_DONE = 1e-8;
constexpr double U = 1.1102230246251565e-16;  // unit roundoff of double

enum { RUN = 0, DONE = 1, FALLBACK = 2, CHOL = 3, FINISH = 4 };
static_assert(DONE == wt::CQ_DONE, "state code shared with the TSQR kernels");

// Per-bond record at wsb + o_cq (REGION doubles).
struct State {
    int state;   // RUN, DONE or FALLBACK
    int nst;     // factors applied to Q
    int m, c;    // size of the factored unfolding
    int nshift;  // shifted stages (diagnostic)
    int pad[3];
};
constexpr long long REGION = 32;

template <int CB>
struct Cfg {
    static constexpr int XP = CB + 2;        // shared row pitch (even)
    static constexpr int TS = CB / 8;        // Gram tiles are TS x TS, 8 x 8 of them
    static constexpr int UP = 36 * TS * TS;  // entries of the 36 upper tiles
    static constexpr int EPT = (UP + NT - 1) / NT;
};

// shared memory (doubles): row-group partials, 2 folded partials, Gram, two
// factors, two accumulated R, scalars, then the CTA's rows
template <int CB>
__host__ __device__ constexpr long long fixed_smem() {
    return (long long)(NG + 2) * Cfg<CB>::UP + 33 * 32 + 2 * (33 * 32 + 32) + 2 * 33 * 32 + 64;
}
template <int CB>
__host__ __device__ constexpr size_t smem(int rpb) {
    return sizeof(double) * (size_t)(fixed_smem<CB>() + (long long)rpb * Cfg<CB>::XP);
}
constexpr size_t SMEM_MAX = 226 * 1024;  // dynamic; leaves room for the static variables
template <int CB>
__host__ __device__ constexpr int rpb_max() {
    return (int)(((long long)(SMEM_MAX / sizeof(double)) - fixed_smem<CB>()) / Cfg<CB>::XP);
}

// upper tile q (0..35) of the 8 x 8 tile grid -> tile row and column
__device__ __forceinline__ void upper_tile(int q, int* ti, int* tj) {
    int r = 0;
    while (q >= 8 - r) {
        q -= 8 - r;
        r++;
    }
    *ti = r;
    *tj = r + q;
}

// x <- x R^{-1} for the rows at x0 and (if two) x1 (R upper triangular c x c
// in sR, pitch 33, inverse pivots at sR[33 * 32 + j]); each R entry read
// serves both rows.
template <int CB>
__device__ __forceinline__ void row_solve2(double* x0s, double* x1s, bool two, const double* sR, int c) {
    double x0[CB], x1[CB];
    const double* s1 = two ? x1s : x0s;  // a single row is solved twice, stored once
#pragma unroll
    for (int j = 0; j < CB; j++) {
        x0[j] = x0s[j];
        x1[j] = s1[j];
    }
#pragma unroll
    for (int j = 0; j < CB; j++) {
        if (j >= c) continue;
        const double iv = sR[33 * 32 + j];
        const double y0 = x0[j] * iv, y1 = x1[j] * iv;
        x0[j] = y0;
        x1[j] = y1;
#pragma unroll
        for (int l = j + 1; l < CB; l++) {
            const double r = sR[j * 33 + l];
            x0[l] = fma(-y0, r, x0[l]);
            x1[l] = fma(-y1, r, x1[l]);
        }
    }
#pragma unroll
    for (int j = 0; j < CB; j++) x0s[j] = x0[j];
    if (two) {
#pragma unroll
        for (int j = 0; j < CB; j++) x1s[j] = x1[j];
    }
}

// Cholesky factor of G + shift I (c x c in sG, pitch 33) by one warp, lane =
// column, into sR (row-major, pitch 33, zero outside c x c; inverse pivots at
// sR[33 * 32 + j]).  Row j of R is broadcast through sRow.  Returns false
// when a pivot is not positive; *ratio = min / max pivot.
template <int CB>
__device__ bool warp_chol(const double* sG, int c, double shift, double* sR, double* sRow, double* ratio) {
    const int lane = threadIdx.x & 31;
    double g[CB];
#pragma unroll
    for (int t = 0; t < CB; t++) g[t] = (t < c && lane < c) ? sG[t * 33 + lane] + (t == lane ? shift : 0.0) : 0.0;
    bool ok = true;
    double dmin = 1.0 / 0.0, dmax = 0.0;
#pragma unroll
    for (int j = 0; j < CB; j++) {
        if (j >= c) continue;
        const double d = __shfl_sync(0xffffffffu, g[j], j);
        ok = ok && (d > 0.0);  // false for NaN
        dmin = fmin(dmin, d);
        dmax = fmax(dmax, d);
        const double dd = d > 0.0 ? d : 1.0;
        const double inv = rsqrt(dd);
        const double rj = (lane == j) ? dd * inv : ((lane > j && lane < c) ? g[j] * inv : 0.0);
        sRow[lane] = rj;
        __syncwarp();
        if (lane > j && lane < c) {
#pragma unroll
            for (int t = j + 1; t < CB; t++) g[t] = fma(-sRow[t], rj, g[t]);
        }
        sR[j * 33 + lane] = rj;
        if (lane == j) sR[33 * 32 + j] = inv;
        __syncwarp();
    }
    for (int j = c; j < 32; j++) {
        sR[j * 33 + lane] = 0.0;
        if (lane == j) sR[33 * 32 + j] = 0.0;
    }
    __syncwarp();
    *ratio = dmax > 0.0 ? dmin / dmax : 0.0;
    return ok;
}

// First-order Cholesky factor of G = I + E by one warp (lane = column).
__device__ __forceinline__ void warp_first_order(const double* sG, int c, double* sR) {
    const int lane = threadIdx.x & 31;
    for (int j = 0; j < 32; j++) {
        double v = 0.0;
        if (j < c && lane < c) {
            if (lane > j)
                v = sG[j * 33 + lane];
            else if (lane == j)
                v = 1.0 + 0.5 * (sG[j * 33 + j] - 1.0);
        }
        sR[j * 33 + lane] = v;
    }
    sR[33 * 32 + lane] = lane < c ? 1.0 / (1.0 + 0.5 * (sG[lane * 33 + lane] - 1.0)) : 0.0;
    __syncwarp();
}

// Factor core k's unfolding (mode) by the Cholesky sequence above.  Launched
// as one cluster of CS CTAs with room for rpb rows each (m <= CS rpb, else
// fallback); CTA b takes rows [b ceil(m / CS), ...).
template <int CB>
__global__ void __launch_bounds__(NT, 1) k_cq_factor(const DevDesc* D, int k, int mode, Plan pl, wt::WP wp,
                                                  double* wsb, int rpb, long long* qstat) {
    PTT_PDL_ENTRY();
    constexpr int XP = Cfg<CB>::XP, TS = Cfg<CB>::TS, UP = Cfg<CB>::UP, EPT = Cfg<CB>::EPT;
    cg::cluster_group cl = cg::this_cluster();
    const int CS = (int)cl.num_blocks();
    const int crank = (int)cl.block_rank();
    extern __shared__ double csm[];
    double* sScr = csm;                // NG row-group partials (UP each)
    double* sP = sScr + NG * UP;       // 2 folded partials, read by the other CTAs
    double* sG = sP + 2 * UP;          // 32 x 33 Gram of the whole unfolding
    double* sRa = sG + 33 * 32;        // factor (32 x 33) + 32 inverse pivots: plain Cholesky
    double* sRb = sRa + 33 * 32 + 32;  // the same for the shifted Cholesky
    double* sT = sRb + 33 * 32 + 32;   // 32 x 33 accumulated R = R_s ... R_1
    double* sTn = sT + 33 * 32;        // 32 x 33 the other buffer of it
    double* sRow = sTn + 33 * 32;      // 2 x 32 scalars
    double* Xs = sRow + 64;            // rpb x XP rows of this CTA
    double* sR = sRa;                  // factor of the current stage
    __shared__ int s_dec, s_ok[2];
    __shared__ double s_ratio[2];
    State* st = (State*)(wsb + wp.o_cq);
    const View A = make_view(D, k, mode, false);
    const int m = A.m, c = A.c;
    const int tid = threadIdx.x;
    if (c > CB || c < 1 || m < c || (long long)m > (long long)rpb * CS) {  // uniform: Householder TSQR
        if (crank == 0 && tid == 0) {
            st->state = FALLBACK;
            st->nst = 0;
            if (qstat) atomicAdd((unsigned long long*)(qstat + 1), 1ull);
        }
        return;
    }
    if (pl.work && crank == 0 && tid == 0) atomicAdd(pl.work, 16.0 * (double)m * (double)c);
    // the actual rows spread evenly: the host sized rpb (and the shared
    // memory) from a bound on m, which the truncation sweep's shrinking
    // ranks leave well above the rows a bond has
    const int rpbd = (m + CS - 1) / CS;  // <= rpb
    const int r0 = crank * rpbd;
    const int h = (m - r0) < rpbd ? ((m - r0) > 0 ? (m - r0) : 0) : rpbd;
    // this CTA's rows: zero, then every element by cp.async (all in flight)
    for (int e = tid; e < h * XP; e += NT) Xs[e] = 0.0;
    for (int e = tid; e < 32 * 33; e += NT) {
        sT[e] = ((e / 33) == (e % 33) && (e / 33) < c) ? 1.0 : 0.0;
        sTn[e] = 0.0;
    }
    __syncthreads();
    {
        const int tot = h * c;
        const unsigned xs0 = (unsigned)__cvta_generic_to_shared(Xs);
        for (int f = tid; f < tot; f += NT) {
            int row, col;
            const double* g;
            if (mode == LEFT) {  // column-major: a column's rows are contiguous
                col = f / h;
                row = f - col * h;
                g = A.p + (long long)(r0 + row) + (long long)col * m;
            } else {  // RIGHT_T: this CTA's rows are one contiguous range
                row = f / c;
                col = f - row * c;
                g = A.p + (long long)r0 * c + f;
            }
            const unsigned sa = xs0 + 8u * (unsigned)(row * XP + col);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(g) : "memory");
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
    }
    __syncthreads();
    // Gram warps: rows [4 ks0, 4 ks1) of this CTA, every 8 x 8 tile of the
    // NB column blocks (mma.m8n8k4: four rows a step, the block's fragment
    // serves as A and as B)
    constexpr int NB = CB / 8, NTL = NB * (NB + 1) / 2;
    static_assert(4 * NTL * 64 <= NG * UP, "the warp tiles fit the Gram scratch");
    const int warp = tid >> 5, lane = tid & 31, li = lane >> 2, lk = lane & 3;
    const int nks = (h + 3) / 4;
    const int ks0 = (nks * warp) / (NT / 32), ks1 = (nks * (warp + 1)) / (NT / 32);
    int dec = RUN, nst = 0, nshift = 0, stage = 0;
    for (stage = 0; stage < MAXST; stage++) {
        if (stage > 0) {  // Q_stage = Q_{stage-1} R_stage^{-1}
            for (int r = tid; r < h; r += 2 * NT) row_solve2<CB>(Xs + r * XP, Xs + (r + NT) * XP, r + NT < h, sR, c);
            __syncthreads();
        }
        // partial Gram of this CTA's rows on the FP64 tensor cores: each warp
        // its rows, all tiles; warps w and w + 4 are added in shared memory,
        // then the four sums in warp order into the grid layout of myP
        {
            double c0[NTL], c1[NTL];
#pragma unroll
            for (int t = 0; t < NTL; t++) {
                c0[t] = 0.0;
                c1[t] = 0.0;
            }
            for (int ks = ks0; ks < ks1; ks++) {
                const int row = 4 * ks + lk;
                double f[NB];
#pragma unroll
                for (int bb = 0; bb < NB; bb++) f[bb] = row < h ? Xs[row * XP + 8 * bb + li] : 0.0;
                int t = 0;
#pragma unroll
                for (int I = 0; I < NB; I++)
#pragma unroll
                    for (int J = I; J < NB; J++, t++)
                        asm volatile(
                            "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                            : "+d"(c0[t]), "+d"(c1[t])
                            : "d"(f[I]), "d"(f[J]));
            }
            double* slot = sScr + (warp & 3) * NTL * 64 + li * 8 + 2 * lk;
            if (warp < 4) {
#pragma unroll
                for (int t = 0; t < NTL; t++) {
                    slot[t * 64] = c0[t];
                    slot[t * 64 + 1] = c1[t];
                }
            }
            __syncthreads();
            if (warp >= 4) {
#pragma unroll
                for (int t = 0; t < NTL; t++) {
                    slot[t * 64] += c0[t];
                    slot[t * 64 + 1] += c1[t];
                }
            }
            __syncthreads();
        }
        double* myP = sP + (stage & 1) * UP;
        for (int u = tid; u < UP; u += NT) {
            // entry (gi, gj) of upper grid tile qq, from the 8 x 8 tile of its
            // column blocks (the symmetric entry when gi's block is the later)
            const int qq = u / (TS * TS), w = u - qq * (TS * TS);
            int a0, b0;
            upper_tile(qq, &a0, &b0);
            int gi = a0 * TS + w / TS, gj = b0 * TS + w % TS;
            if ((gi >> 3) > (gj >> 3)) {
                const int tmp = gi;
                gi = gj;
                gj = tmp;
            }
            const int I = gi >> 3, J = gj >> 3;
            const int e = (I * NB - (I * (I - 1)) / 2 + (J - I)) * 64 + (gi & 7) * 8 + (gj & 7);
            myP[u] = ((sScr[e] + sScr[NTL * 64 + e]) + sScr[2 * NTL * 64 + e]) + sScr[3 * NTL * 64 + e];
        }
        cl.sync();  // every CTA's partial is complete and visible
        // sum the CTAs' partials in CTA order (distributed shared memory),
        // every load issued before the sums
        {
            double v[EPT][CSMAX];
#pragma unroll
            for (int i = 0; i < EPT; i++) {
                const int u = tid + i * NT;
#pragma unroll
                for (int b = 0; b < CSMAX; b++) v[i][b] = (u < UP && b < CS) ? cl.map_shared_rank(myP, b)[u] : 0.0;
            }
#pragma unroll
            for (int i = 0; i < EPT; i++) {
                const int u = tid + i * NT;
                if (u < UP) {
                    double s2 = 0.0;
#pragma unroll
                    for (int b = 0; b < CSMAX; b++) s2 += v[i][b];  // zeros beyond CS leave the sum unchanged
                    const int qq = u / (TS * TS), w = u - qq * (TS * TS);
                    int a0, b0;
                    upper_tile(qq, &a0, &b0);
                    const int gi = a0 * TS + w / TS, gj = b0 * TS + w % TS;
                    sG[gi * 33 + gj] = s2;
                    sG[gj * 33 + gi] = s2;
                }
            }
        }
        __syncthreads();
        // decision; when a Cholesky factor is needed warp 0 forms the plain
        // and warp 1 the shifted one at the same time
        if (tid < 64) {
            const int lane = tid & 31, wq = tid >> 5;
            double tr = (lane < c) ? sG[lane * 33 + lane] : 0.0;
            double e = 0.0;
            bool nan = false;
            for (int t = 0; t < c; t++) {
                const double v2 = (lane < c) ? sG[t * 33 + lane] - (t == lane ? 1.0 : 0.0) : 0.0;
                nan = nan || !(v2 == v2);
                e = fmax(e, fabs(v2));
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                tr += __shfl_xor_sync(0xffffffffu, tr, o);
                e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
            }
            nan = __any_sync(0xffffffffu, nan);
            // an exactly zero column stays zero under every stage: leave the
            // bond to the Householder TSQR at once
            const bool zcol = __any_sync(0xffffffffu, lane < c && sG[lane * 33 + lane] == 0.0);
            int d;
            if (nan || !(tr > 0.0) || !(tr < 1.0 / 0.0) || (stage == 0 && zcol)) {
                d = FALLBACK;
            } else if (stage >= 1 && e <= TAU) {
                d = DONE;
            } else if (stage >= 1 && e <= FIRST) {
                if (wq == 0) warp_first_order(sG, c, sRa);
                d = e <= FIRST_DONE ? FINISH : RUN;
            } else if (stage == MAXST - 1) {
                d = FALLBACK;
            } else {
                const double sigma = wq ? 11.0 * ((double)m * c + (double)c * (c + 1)) * U * tr : 0.0;
                double ratio;
                const bool ok = warp_chol<CB>(sG, c, sigma, wq ? sRb : sRa, sRow + 32 * wq, &ratio);
                if (lane == 0) {
                    s_ok[wq] = ok;
                    s_ratio[wq] = ratio;
                }
                d = CHOL;
            }
            if (tid == 0) s_dec = d;
        }
        __syncthreads();
        dec = s_dec;
        sR = sRa;
        if (dec == CHOL) {
            if (s_ok[0] && s_ratio[0] >= 1e-12) {
                dec = RUN;
            } else if (s_ok[1]) {
                dec = RUN;
                sR = sRb;
                nshift++;
            } else {
                dec = FALLBACK;
            }
        }
        if (dec == DONE || dec == FALLBACK) break;
        nst = stage + 1;
        // R <- R_{stage+1} R (both upper triangular, zero beyond c) into the
        // other buffer on the FP64 tensor cores: warp w forms 8 x 8 tiles w and
        // w + 8 of the 10 upper tiles, k over the tile's triangle band; the
        // tiles below the diagonal of sTn stay zero from the start, the lower
        // halves of the diagonal tiles come out as exact zeros
        for (int t = warp; t < 10; t += NT / 32) {
            int I = 0, J = t;
            while (J >= 4 - I) {
                J -= 4 - I;
                I++;
            }
            J += I;
            double d0 = 0.0, d1 = 0.0;
            for (int k0 = 8 * I; k0 < 8 * J + 8; k0 += 4) {
                const double av = sR[(8 * I + li) * 33 + k0 + lk];
                const double bv = sT[(k0 + lk) * 33 + 8 * J + li];
                asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                             : "+d"(d0), "+d"(d1)
                             : "d"(av), "d"(bv));
            }
            sTn[(8 * I + li) * 33 + 8 * J + 2 * lk] = d0;
            sTn[(8 * I + li) * 33 + 8 * J + 2 * lk + 1] = d1;
        }
        {
            double* t2 = sT;
            sT = sTn;
            sTn = t2;
        }
        if (dec == FINISH) {  // apply the first-order factor; Q is final
            for (int r = tid; r < h; r += 2 * NT) row_solve2<CB>(Xs + r * XP, Xs + (r + NT) * XP, r + NT < h, sR, c);
            __syncthreads();
            dec = DONE;
            break;
        }
        __syncthreads();
    }
    cl.sync();  // no CTA leaves while another may still read its partials
    if (dec == DONE) {
        if (mode == LEFT) {
            double* out = D->alt[k];
            for (int e = tid; e < h * c; e += NT) {
                const int col = e / h, row = e - col * h;
                out[(long long)(r0 + row) + (long long)col * m] = Xs[row * XP + col];
            }
        } else {
            double* out = A.p + (long long)r0 * c;  // in place over A: this CTA's rows only
            for (int e = tid; e < h * c; e += NT) {
                const int row = e / c, col = e - row * c;
                out[e] = Xs[row * XP + col];
            }
        }
        if (crank == 0) {
            double* Rs = wsb + wp.o_R;  // root slot, row-major 32 x 32
            for (int e = tid; e < 1024; e += NT) {
                const int i = e >> 5, j = e & 31;
                Rs[e] = (i < c && j < c && j >= i) ? sT[i * 33 + j] : 0.0;
            }
            if (tid == 0) {
                Info* info = (Info*)(wsb + pl.o_info_d);
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
    }
    if (crank == 0 && tid == 0) {
        st->state = dec;
        st->nst = nst;
        st->m = m;
        st->c = c;
        st->nshift = nshift;
        if (dec == FALLBACK && qstat) atomicAdd((unsigned long long*)(qstat + 1), 1ull);
    }
}

// alt[k][row * rank + col] = (Q V_r)(row, col) for the RIGHT_T bonds k0 ..
// k0 + gridDim.y - 1 that the Cholesky sequence finished: Q is in core[k]
// (row-major rows of c), V_r in Bn (row-major 32 x KC).
template <int CB>
__global__ void __launch_bounds__(NT) k_cq_write(const DevDesc* D, int k0, Plan pl, wt::WP wp, double* ws) {
    PTT_PDL_ENTRY();
    __shared__ double sB[32 * 33];
    const int k = k0 + blockIdx.y;
    double* wsb = ws + (long long)k * wp.stride;
    const State* st = (const State*)(wsb + wp.o_cq);
    if (st->state != DONE) return;
    const Info* info = (const Info*)(wsb + pl.o_info_d);
    if (info->status) return;
    const int m = info->m, c = info->c, qB = info->rank;
    const int tid = threadIdx.x;
    const double* Bn = wsb + pl.o_Bn;
    for (int e = tid; e < 1024; e += NT) {
        const int t = e >> 5, l = e & 31;
        sB[t * 33 + l] = (t < c && l < qB) ? Bn[(long long)t * pl.KC + l] : 0.0;
    }
    __syncthreads();
    const double* Q = D->core[k];
    double* out = D->alt[k];
    for (int row = blockIdx.x * NT + tid; row < m; row += gridDim.x * NT) {
        double x[CB];
#pragma unroll
        for (int t = 0; t < CB; t++) x[t] = t < c ? Q[(long long)row * c + t] : 0.0;
        for (int l = 0; l < qB; l++) {
            double y = 0.0;
#pragma unroll
            for (int t = 0; t < CB; t++) y = fma(x[t], sB[t * 33 + l], y);
            out[(long long)row * qB + l] = y;
        }
    }
}

}  // namespace cq
