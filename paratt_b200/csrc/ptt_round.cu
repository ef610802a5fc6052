// TT rounding on the device, FP64: paratt_truncate (paratt.c:316-342) ->
// pattacTruncate (pattac.c:590-675) with ortho 'R':
//
//   left-to-right:  for i = 0..d-2   QR of the left unfolding of core i
//                   (pattacLOrthogonalization, pattac.c:244-294), R pushed into
//                   core i+1 (trapezoid_mult, utilities.c:233-308), Q kept.
//   right-to-left:  for i = d-1..1   LQ of the right unfolding (as QR of its
//                   transpose), SVD of L, tail-sum rank rule, core i <- V_r^T Q,
//                   core i-1 <- core i-1 * U_r S_r (pattacLTruncate,
//                   pattac.c:297-522).
//
// The grid normalisation of pattac.c:608-616/665-673 (divide every core by
// sqrt(n_k), multiply back afterwards) scales every bond's singular values by
// 1/sqrt(prod n_k); it is folded into the threshold instead of two passes
// over the cores: drop while sqrt(tail) < tol/sqrt(d-1) * sqrt(prod n_k).
//
// Every stage reads sizes from device memory (descriptor + Info record), so
// a rounding is a fixed launch sequence with no host synchronisation.
#include "ptt_tsqr.cuh"

#include <cooperative_groups.h>
#include <stdio.h>
#include <string.h>

using namespace tsqr;

namespace {

constexpr int MAXSW = 40;  // Jacobi sweep limit

__device__ __forceinline__ unsigned group_mask8(int tid) { return 0xFFu << ((tid & 31) & ~7); }

// the same for groups of LP lanes (LP = 2, 4, 8)
template <int LP>
__device__ __forceinline__ unsigned group_mask(int tid) {
    return ((1u << LP) - 1u) << ((tid & 31) & ~(LP - 1));
}
template <int LP>
__device__ __forceinline__ double gsum_g(double v, unsigned mask) {
#pragma unroll
    for (int o = LP / 2; o >= 1; o >>= 1) v += __shfl_xor_sync(mask, v, o);
    return v;
}

__device__ __forceinline__ double gsum8(double v, unsigned mask) {
    v += __shfl_xor_sync(mask, v, 4);
    v += __shfl_xor_sync(mask, v, 2);
    v += __shfl_xor_sync(mask, v, 1);
    return v;
}

#include "ptt_factor.cuh"

// ---------------------------------------------------------------------------
// Q application: out = Q * B, B = Bn[root] (q x k), k read from device.
// ---------------------------------------------------------------------------
template <int CT>
__device__ void replay_tsqrt(double* Rp, const double* Vs, const double* taus, int c, double* out, int col, int part) {
    constexpr int S = CT + 1;
    constexpr int NV = H / 8;
    const unsigned gm = 0xffffffffu;
    for (int j = c - 1; j >= 0; j--) {
        const double tau = taus[j];
        if (tau == 0.0) continue;
        double pr = 0.0;
#pragma unroll
        for (int v = 0; v < NV; v++) pr += Vs[(part + 8 * v) * S + j] * out[v];
        const double rj = Rp[j * KG + col];
        pr = gsum8(pr, gm);
        const double tw = tau * (rj + pr);
        if (part == 0) Rp[j * KG + col] = rj - tw;
#pragma unroll
        for (int v = 0; v < NV; v++) out[v] -= tw * Vs[(part + 8 * v) * S + j];
        __syncwarp();
    }
}

template <int CT>
__device__ void replay_geqrt(double* Rp, const double* Vb, const double* taus, int c, int col, int part) {
    constexpr int S = CT + 1;
    constexpr int NV = CT / 8;
    for (int j = c - 1; j >= 0; j--) {
        const double tau = taus[j];
        if (tau == 0.0) continue;
        double pr = 0.0;
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const int t = part + 8 * v;
            if (t >= j) pr += (t == j ? 1.0 : Vb[t * S + j]) * Rp[t * KG + col];
        }
        pr = gsum8(pr, 0xffffffffu);
        const double tw = tau * pr;
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const int t = part + 8 * v;
            if (t >= j) Rp[t * KG + col] -= tw * (t == j ? 1.0 : Vb[t * S + j]);
        }
        __syncwarp();
    }
}

template <int CT>
__global__ void __launch_bounds__(NT) k_apply_node(Plan pl, double* ws, int first, const int* kptr) {
    PTT_PDL_ENTRY();
    if (gq_finished(pl)) return;
    extern __shared__ double sm[];
    constexpr int S = CT + 1;
    double* Rp = sm;             // CT x KG
    double* Vs = Rp + CT * KG;   // H x S
    const int node = first + blockIdx.x;
    const int kg0 = blockIdx.y * KG;
    const int kk = *kptr;
    if (pl.info->status || kg0 >= kk) return;
    const int q = pl.qn[node];
    if (q == 0) return;
    const int tid = threadIdx.x, col = tid >> 3, part = tid & 7;
    const int c = pl.info->c;
    const int KC = pl.KC;
    double* Bn = ws + pl.o_Bn;
    const double* Bi = Bn + (long long)node * CT * KC;
    const int cl = 2 * node + 1, cr = 2 * node + 2;
    const int ps = pl.pass[node];
    if (ps == 1 || ps == 2) {
        double* Bo = Bn + (long long)(ps == 1 ? cl : cr) * CT * KC;
        for (int e = tid; e < CT * KG; e += NT) {
            const int a = e / KG, b = e - (e / KG) * KG;
            Bo[(long long)a * KC + kg0 + b] = Bi[(long long)a * KC + kg0 + b];
        }
        return;
    }
    if (ps != 0) return;
    for (int e = tid; e < CT * KG; e += NT) {
        const int a = e / KG, b = e - (e / KG) * KG;
        Rp[e] = Bi[(long long)a * KC + kg0 + b];
    }
    const double* RR = ws + pl.o_Rn + (long long)cr * CT * CT;
    double* Bcr = Bn + (long long)cr * CT * KC;
    for (int half = pl.NH - 1; half >= 0; half--) {
        const int h0 = half * H;
        if (h0 >= c) continue;
        __syncthreads();
        for (int e = tid; e < H * CT; e += NT) {
            const int t = e / CT, l = e - (e / CT) * CT;
            Vs[t * S + l] = (h0 + t < c) ? RR[(long long)(h0 + t) * CT + l] : 0.0;
        }
        __syncthreads();
        double out[H / 8];
#pragma unroll
        for (int v = 0; v < H / 8; v++) out[v] = 0.0;
        const double* taus = ws + pl.o_tau_node + ((long long)node * pl.NH + half) * CT;
        replay_tsqrt<CT>(Rp, Vs, taus, c, out, col, part);
#pragma unroll
        for (int v = 0; v < H / 8; v++) {
            const int t = h0 + part + 8 * v;
            if (t < CT) Bcr[(long long)t * KC + kg0 + col] = out[v];
        }
    }
    __syncthreads();
    double* Bcl = Bn + (long long)cl * CT * KC;
    for (int e = tid; e < CT * KG; e += NT) {
        const int a = e / KG, b = e - (e / KG) * KG;
        Bcl[(long long)a * KC + kg0 + b] = Rp[e];
    }
}

// out_mode LEFT: out(row, col) at alt[row + m*col];  RIGHT_T: alt[row*k + col]
template <int CT>
__global__ void __launch_bounds__(NT) k_apply_leaf(const DevDesc* D, int kcore, int mode, Plan pl, double* ws,
                                                   const int* kptr) {
    PTT_PDL_ENTRY();
    if (gq_finished(pl)) return;
    extern __shared__ double sm[];
    constexpr int S = CT + 1;
    constexpr int VR = CT > H ? CT : H;
    double* Rp = sm;             // CT x KG
    double* Vs = Rp + CT * KG;   // VR x S
    const int p = blockIdx.x;
    const int kg0 = blockIdx.y * KG;
    const int kk = *kptr;
    if (pl.info->status || kg0 >= kk) return;
    const int tid = threadIdx.x, col = tid >> 3, part = tid & 7;
    const int m = pl.info->m, c = pl.info->c;
    // the unfolding the factorisation recorded (m x c), not the descriptor's
    // ranks: in the truncation sweep this runs on the side stream while the
    // main stream has already published the bond's new rank
    View A;
    A.p = D->core[kcore];
    A.m = m;
    A.c = c;
    A.rs = (mode == LEFT) ? 1 : c;
    A.cs = (mode == LEFT) ? m : 1;
    double* outp = D->alt[kcore];
    const long long ors = (mode == LEFT) ? 1 : kk;
    const long long ocs = (mode == LEFT) ? m : 1;
    int r0, r1;
    leaf_range(m, pl.L, pl.P, p, &r0, &r1);
    const int rows = r1 - r0;
    if (rows <= 0) return;
    const int rb = rows < c ? rows : c;
    const int slot = pl.P - 1 + p;
    const int KC = pl.KC;
    const double* Bi = ws + pl.o_Bn + (long long)slot * CT * KC;
    const double* tau_leaf = ws + pl.o_tau_leaf + (long long)p * pl.KL * CT;
    for (int e = tid; e < CT * KG; e += NT) {
        const int a = e / KG, b = e - (e / KG) * KG;
        Rp[e] = Bi[(long long)a * KC + kg0 + b];
    }
    const int ocol = kg0 + col;
    const bool colok = ocol < kk;
    const int nch = (rows - rb + H - 1) / H;
    for (int s = nch - 1; s >= 0; s--) {
        const int t0 = r0 + rb + s * H;
        const int h = (r1 - t0) < H ? (r1 - t0) : H;
        __syncthreads();
        for (int e = tid; e < H * CT; e += NT) {
            const int t = e / CT, l = e - (e / CT) * CT;
            Vs[t * S + l] = (t < h && l < c) ? A.p[(long long)(t0 + t) * A.rs + (long long)l * A.cs] : 0.0;
        }
        __syncthreads();
        double out[H / 8];
#pragma unroll
        for (int v = 0; v < H / 8; v++) out[v] = 0.0;
        replay_tsqrt<CT>(Rp, Vs, tau_leaf + (long long)(1 + s) * CT, c, out, col, part);
#pragma unroll
        for (int v = 0; v < H / 8; v++) {
            const int t = part + 8 * v;
            if (t < h && colok) outp[(long long)(t0 + t) * ors + (long long)ocol * ocs] = out[v];
        }
    }
    __syncthreads();
    for (int e = tid; e < CT * CT; e += NT) {
        const int t = e / CT, l = e - (e / CT) * CT;
        Vs[t * S + l] = (t < rb && l < c && t > l) ? A.p[(long long)(r0 + t) * A.rs + (long long)l * A.cs] : 0.0;
    }
    __syncthreads();
    replay_geqrt<CT>(Rp, Vs, tau_leaf, c, col, part);
    __syncthreads();
    for (int e = tid; e < CT * KG; e += NT) {
        const int t = e / KG, b = e - (e / KG) * KG;
        if (t < rb && kg0 + b < kk) outp[(long long)(r0 + t) * ors + (long long)(kg0 + b) * ocs] = Rp[e];
    }
}

// B = I_q at the root, zero-padded to CT x KC.
__global__ void k_set_identity(Plan pl, double* ws) {
    PTT_PDL_ENTRY();
    if (pl.info->status || gq_finished(pl)) return;
    const int CT = pl.CT, KC = pl.KC;
    const int q = pl.info->q;
    double* B = ws + pl.o_Bn;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < CT * KC; e += gridDim.x * blockDim.x) {
        const int a = e / KC, b = e - (e / KC) * KC;
        B[e] = (a == b && a < q) ? 1.0 : 0.0;
    }
}

// ---------------------------------------------------------------------------
// one-sided Jacobi SVD of L = R^T (c x q), R = root factor of the LQ.
// Column pairs follow the circle (round-robin) order; rotations are recorded
// so V can be rebuilt row-parallel by k_svd_replay.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int circle_col(int pos, int round, int qq) {
    return pos == 0 ? 0 : 1 + (pos - 1 + round) % (qq - 1);
}

// Stationary-ring order, for G = qq / 2 a power of two.  Level l (block size
// hb = G >> l groups, rounds [2G - 2hb, 2G - hb)): block b of hb consecutive
// pairs owns columns [2 hb b, 2 hb (b + 1)); pair i of the block keeps column
// 2 hb b + i and meets 2 hb b + hb + (i + s) mod hb at shift s, so the second
// columns move one pair along a ring of hb pairs per round while the first
// ones stay.  Between levels each block splits in two: the first half pairs
// its first columns among themselves, the second half its second columns
// (a swap of one column between pairs i and i + hb / 2).  Every pair of
// columns meets once in 2G - 1 rounds.
__device__ __forceinline__ void stat_cols(int i, int rd, int G, int* pc, int* qc) {
    const int x = 2 * G - 1 - rd;  // in [hb, 2 hb - 1]
    const int hb = 1 << (31 - __clz(x));
    const int s = rd - (2 * G - 2 * hb);
    const int b = i / hb, ii = i - b * hb;
    *pc = 2 * hb * b + ii;
    *qc = 2 * hb * b + hb + (ii + s) % hb;
}

// threads of the SVD block: 8 lanes for each of the (CT+2)/2 column pairs
// of a round, rounded to a power of two (idle threads only slow the barriers)
template <int CT>
__host__ __device__ constexpr int svd_nt() {
    return CT <= 32 ? 128 : (CT <= 64 ? 256 : 512);
}

// One-sided Jacobi on the columns of L (c rows, q columns).  Each column pair
// is handled by LP lanes (rows p + LP v), NTH / LP pairs per pass: with the
// default 8 lanes and svd_nt threads one circle-order round is a single pass
// for q <= 128.  (A one-warp form, NTH = 32 and LP = 4, measured slower on
// the benchmark's bonds with q <= 16: 43.6 us against ~40 us, the
// rotation chain and not the block barrier being the cost.)  Column norms
// are tracked through the rotations (a_p' = a_p - t a_pq ...) and recomputed
// at the start of a sweep.
template <int CT, int NTH = svd_nt<CT>(), int LP = 8>
__global__ void __launch_bounds__(NTH) k_svd_jacobi(Plan pl, double* ws, double delta, int maxr, int bond,
                                                    int* status) {
    PTT_PDL_ENTRY();
    constexpr int SVD_NT = NTH;
    extern __shared__ double sm[];
    constexpr int S = CT + 1;
    constexpr int NG = CT / LP;
    double* Lc = sm;                   // (CT+1) columns x S
    __shared__ double s_nrm[CT + 2];
    __shared__ double s_sig[CT + 2];
    __shared__ int s_ord[CT + 2];
    __shared__ int s_rot;
    __shared__ double s_thr2;
    const int tid = threadIdx.x;
    const int grp = tid / LP, p = tid % LP;  // pair slots x LP lanes
    const unsigned gm = group_mask<LP>(tid);
    Info* info = pl.info;
    if (info->status) return;
    const int c = info->c, q = info->q;
    const int qq = q + (q & 1);
    const double* R = ws + pl.o_Rn;  // root factor, row-major CT x CT; L = R^T
    constexpr int LPT = (CT * S + SVD_NT - 1) / SVD_NT;  // qq <= CT
    if constexpr (LPT <= 16) {  // every element requested before the first is stored
        double v[LPT];
#pragma unroll
        for (int u = 0; u < LPT; u++) {
            const int e = tid + u * SVD_NT;
            const int j = e / S, t = e - (e / S) * S;
            v[u] = (e < qq * S && j < q && t < c) ? R[(long long)j * CT + t] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < LPT; u++) {
            const int e = tid + u * SVD_NT;
            if (e < qq * S) Lc[e] = v[u];
        }
    } else {
        for (int e = tid; e < qq * S; e += SVD_NT) {
            const int j = e / S, t = e - (e / S) * S;
            Lc[e] = (j < q && t < c) ? R[(long long)j * CT + t] : 0.0;
        }
    }
    __syncthreads();
    double2* rot = (double2*)(ws + pl.o_rot);
    const int npair = (CT + 2) / 2;
    const double tol = (double)(c < 16 ? 16 : c) * 2.220446049250313e-16;
    const double tol2 = tol * tol;  // |ga| > tol sqrt(al be), compared in squares
    int sweeps = 0;
    bool conv = (qq < 2);
    for (int sw = 0; sw < MAXSW && !conv; sw++) {
        // exact column norms at the start of every sweep
        for (int j = tid / LP; j < qq; j += SVD_NT / LP) {
            double s2 = 0.0;
#pragma unroll
            for (int v = 0; v < NG; v++) {
                const double x = Lc[j * S + p + LP * v];
                s2 += x * x;
            }
            s2 = gsum_g<LP>(s2, gm);
            if (p == 0) s_nrm[j] = s2;
        }
        if (tid == 0) s_rot = 0;
        __syncthreads();
        // Columns below the numerical-rank threshold (sqrt(q) eps_LAPACK times
        // the largest column norm) are rounding noise: rotating noise against
        // noise is a random walk that never meets the relative criterion, and
        // their values are discarded by the rank rule anyway, so pairs with
        // such a column are left alone.
        if (tid == 0) {
            double mx = 0.0;
            for (int j = 0; j < qq; j++) mx = fmax(mx, s_nrm[j]);
            s_thr2 = (double)q * 1.232595164407831e-32 * mx;  // (sqrt(q) * 2^-53)^2 * max |a_j|^2
        }
        __syncthreads();
        const double thr2 = s_thr2;
        int myrot = 0;
        for (int rd = 0; rd < qq - 1; rd++) {
            for (int i = grp; i < qq / 2; i += SVD_NT / LP) {
                const int pc = circle_col(i, rd, qq), qc = circle_col(qq - 1 - i, rd, qq);
                double* ap = Lc + pc * S;
                double* aq = Lc + qc * S;
                double xa[NG], xb[NG];
                double g0 = 0.0, g1 = 0.0;
#pragma unroll
                for (int v = 0; v < NG; v++) {
                    xa[v] = ap[p + LP * v];
                    xb[v] = aq[p + LP * v];
                }
#pragma unroll
                for (int v = 0; v < NG; v += 2) {
                    g0 = fma(xa[v], xb[v], g0);
                    g1 = fma(xa[v + 1], xb[v + 1], g1);
                }
                const double ga = gsum_g<LP>(g0 + g1, gm);
                const double al = s_nrm[pc], be = s_nrm[qc];
                double cs = 1.0, sn = 0.0;
                if (ga != 0.0 && al > thr2 && be > thr2 && ga * ga > tol2 * (al * be)) {
                    // the smaller rotation of the pair: with dd = be - al, g2 = 2 ga,
                    // cos 2theta = |dd| / r, sin 2theta = sign(dd) g2 / r,
                    // r = sqrt(dd^2 + g2^2); then cos theta = sqrt((1 + cos 2theta) / 2),
                    // sin theta = sin 2theta / (2 cos theta), t = tan theta -- two
                    // reciprocal square roots on the chain, no square root or division
                    const double dd = be - al, g2 = 2.0 * ga;
                    const double ri = rsqrt(fma(dd, dd, g2 * g2));
                    const double hc = fma(0.5 * fabs(dd), ri, 0.5);  // (1 + cos 2theta) / 2, in [1/2, 1]
                    const double ic = rsqrt(hc);                      // 1 / cos theta
                    cs = hc * ic;
                    sn = 0.5 * copysign(1.0, dd) * g2 * ri * ic;
                    const double t = sn * ic;
#pragma unroll
                    for (int v = 0; v < NG; v++) {
                        ap[p + LP * v] = cs * xa[v] - sn * xb[v];
                        aq[p + LP * v] = sn * xa[v] + cs * xb[v];
                    }
                    if (p == 0) {
                        s_nrm[pc] = al - t * ga;
                        s_nrm[qc] = be + t * ga;
                    }
                    // bit 1: a rotation of a pair whose cosine exceeded 1e-8
                    myrot |= (ga * ga > 1e-16 * (al * be)) ? 3 : 1;
                }
                if (p == 0) rot[((long long)sw * (CT + 1) + rd) * npair + i] = make_double2(cs, sn);
            }
            __syncthreads();
        }
        if (myrot) atomicOr(&s_rot, myrot);
        __syncthreads();
        if (s_rot == 0) {
            conv = true;
        } else {
            sweeps = sw + 1;
            // cyclic Jacobi converges quadratically at the end: after a sweep
            // whose cosines all stayed below 1e-8 the next one would only
            // meet cosines ~1e-16, so it is not run
            if (!(s_rot & 2)) conv = true;
        }
    }
    if (!conv && tid == 0) PTT_STATUS_SET(status, PTT_ERR_NUMERIC);
    // singular values (column norms) and descending order
    for (int j = tid / LP; j < qq; j += SVD_NT / LP) {
        double s2 = 0.0;
#pragma unroll
        for (int v = 0; v < NG; v++) {
            const double x = Lc[j * S + p + LP * v];
            s2 += x * x;
        }
        s2 = gsum_g<LP>(s2, gm);
        // a NaN (corrupt input) would break the strict order below and leave
        // order slots unset; it sorts last and is reported instead
        if (p == 0) {
            const bool nan = !(s2 == s2);
            if (nan && j < q) PTT_STATUS_SET(status, PTT_ERR_NUMERIC);
            s_sig[j] = (j < q && !nan) ? sqrt(s2) : -1.0;
        }
    }
    __syncthreads();
    for (int j = tid; j < qq; j += SVD_NT) {
        const double sj = s_sig[j];
        int pos = 0;
        for (int i = 0; i < qq; i++) {
            const double si = s_sig[i];
            pos += (si > sj) || (si == sj && i < j);
        }
        s_ord[pos] = j;
    }
    __syncthreads();
    double* sig_out = ws + pl.o_sig;
    if (tid == 0) {
        const double s0 = q > 0 ? s_sig[s_ord[0]] : 0.0;
        // numerical rank kept by LAPACK dgesvdq(JOBA='A'): sqrt(N)*eps*s0
        const double thr = sqrt((double)q) * 1.1102230246251565e-16 * s0;
        int nsv = q > 0 ? 1 : 0;
        while (nsv < q && s_sig[s_ord[nsv]] >= thr) nsv++;
        if (!(s0 == s0)) PTT_STATUS_SET(status, PTT_ERR_NUMERIC);
        // tail-sum rule, pattac.c:468-481
        double ssum = 0.0;
        int rank = nsv;
        for (int j = nsv - 1; j >= 0; j--) {
            const double sj = s_sig[s_ord[j]];
            ssum += sj * sj;
            if (sqrt(ssum) < delta)
                rank = j;
            else
                break;
        }
        if (rank > q) rank = q;
        if (rank > maxr) rank = maxr;
        if (rank < 1) rank = 1;
        info->rank = rank;
        info->nsv = nsv;
        info->sweeps = sweeps;
        info->order = 0;
        double tail = 0.0;
        for (int j = rank; j < q; j++) tail += s_sig[s_ord[j]] * s_sig[s_ord[j]];
        info->tail = tail;
        if (pl.stats) {
            double* st = pl.stats + (long long)bond * PTT_STAT_LEN;
            st[0] = rank;
            st[1] = nsv;
            st[2] = sweeps;
            st[3] = q;
            st[4] = c;
            st[5] = tail;
            st[6] = delta;
            st[7] = 0.0;
            for (int j = 0; j < PTT_STAT_NSIG; j++) st[8 + j] = j < q ? s_sig[s_ord[j]] : 0.0;
        }
    }
    for (int j = tid; j < CT; j += SVD_NT) {
        sig_out[j] = j < q ? s_sig[s_ord[j]] : 0.0;
        ((int*)(sig_out + CT))[j] = j < qq ? s_ord[j] : 0;
    }
    __syncthreads();
    const int rank = info->rank;
    double* US = ws + pl.o_US;  // c x rank, column-major ld CT
    for (int e = tid; e < CT * CT; e += SVD_NT) {
        const int b = e / CT, t = e - (e / CT) * CT;
        US[e] = (b < rank && t < c) ? Lc[s_ord[b] * S + t] : 0.0;
    }
}

// The same one-sided Jacobi with the columns kept in registers.  Group g of
// LP lanes holds the two columns of pair g (rows p + LP v), and after each
// round the columns move as the circle order moves them: pair g's top to
// pair g - 1 (pair 0's top, column 0, stays; pair 1's top goes to pair 0's
// bottom), pair g's bottom to pair g + 1 (the last pair's bottom becomes its
// own top) -- warp shuffles between neighbouring groups, shared memory only
// across warp boundaries (double-buffered, one block barrier per round).  The
// tracked column norms travel with the columns.  Rotations are logged for
// k_svd_replay(_b) exactly as by k_svd_jacobi, and after the last sweep the
// columns are written to shared memory for the same epilogue (order, rank
// rule, U S, statistics).
// LP lanes per column pair (4: a round's rotation math, the same instructions
// for every group of a warp, serves eight pairs per warp; the SVD is bound by
// the instructions it issues on its one SM).
template <int CT, int LP = 4>
__host__ __device__ constexpr int ring_nt() {
    return (CT / 2) * LP;
}
template <int CT, int LP = 4>
__global__ void __launch_bounds__(ring_nt<CT, LP>(), 1) k_svd_ring(Plan pl, double* ws, double delta, int maxr, int bond,
                                                               int* status) {
    PTT_PDL_ENTRY();
    constexpr int SVD_NT = ring_nt<CT, LP>();
    constexpr int GPW = 32 / LP;           // groups per warp
    constexpr int NG = CT / LP;            // rows per lane
    constexpr int NW = SVD_NT / 32;        // warps
    constexpr int S = CT + 1;
    extern __shared__ double sm[];
    double* Lc = sm;                                  // (CT + 2) columns x S, written after the sweeps
    double* xch = sm + (CT + 2) * S;                  // [2 buffers][NW][2 (top, bottom)][LP lanes][NG + 1]
    __shared__ double s_nrm[CT + 2];
    __shared__ double s_sig[CT + 2];
    __shared__ int s_ord[CT + 2];
    __shared__ int s_rot;
    __shared__ double s_wmax[NW];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int grp = tid / LP, p = tid % LP;
    const unsigned gm = group_mask<LP>(tid);
    Info* info = pl.info;
    if (info->status) return;
    const int c = info->c, q = info->q;
    const int qq = q + (q & 1);
    const int G = qq / 2;  // pairs of a round
    const double* R = ws + pl.o_Rn;  // root factor, row-major CT x CT; L = R^T: column j = row j of R
    // stationary-ring order (one column of each pair moves per round) over G2
    // pairs, G rounded up to a power of two (the extra columns are zero and
    // never rotated); circle order for a single pair
    const bool stat = G >= 2;
    const int G2 = stat ? 1 << (32 - __clz(G - 1)) : G;
    const bool act = grp < G2;
    // round 0: pair g holds columns g (top) and qq - 1 - g (circle) or G2 + g
    // (stationary ring) (bottom)
    double top[NG], bot[NG];
    {
        const int ct = grp, cb = stat ? G2 + grp : qq - 1 - grp;
#pragma unroll
        for (int v = 0; v < NG; v++) {
            const int t = p + LP * v;
            top[v] = (act && ct < q && t < c) ? R[(long long)ct * CT + t] : 0.0;
            bot[v] = (act && cb < q && cb >= 0 && t < c) ? R[(long long)cb * CT + t] : 0.0;
        }
    }
    double2* rot = (double2*)(ws + pl.o_rot);
    const int npair = (CT + 2) / 2;
    const double tol = (double)(c < 16 ? 16 : c) * 2.220446049250313e-16;
    const double tol2 = tol * tol;
    const int gw = lane / LP;  // group within the warp (0 .. GPW - 1)
    int sweeps = 0, buf = 0;
    bool conv = (qq < 2);
    for (int sw = 0; sw < MAXSW && !conv; sw++) {
        // exact column norms, and the noise threshold from the largest
        double al = 0.0, be = 0.0;
#pragma unroll
        for (int v = 0; v < NG; v++) {
            al = fma(top[v], top[v], al);
            be = fma(bot[v], bot[v], be);
        }
        al = gsum_g<LP>(al, gm);
        be = gsum_g<LP>(be, gm);
        double mx = act ? fmax(al, be) : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (lane == 0) s_wmax[warp] = mx;
        if (tid == 0) s_rot = 0;
        __syncthreads();
        mx = 0.0;
#pragma unroll
        for (int w = 0; w < NW; w++) mx = fmax(mx, s_wmax[w]);
        const double thr2 = (double)q * 1.232595164407831e-32 * mx;  // (sqrt(q) 2^-53)^2 max |a_j|^2
        int myrot = 0;
        // rotate the pair (top, bot) of this group; log it as pair grp of round rd
        auto rotate = [&](int rd) {
            double cs = 1.0, sn = 0.0;
            double g0 = 0.0, g1 = 0.0;
#pragma unroll
            for (int v = 0; v < NG; v += 2) {
                g0 = fma(top[v], bot[v], g0);
                g1 = fma(top[v + 1], bot[v + 1], g1);
            }
            const double ga = gsum_g<LP>(g0 + g1, gm);
            if (ga != 0.0 && al > thr2 && be > thr2 && ga * ga > tol2 * (al * be)) {
                const double dd = be - al, g2 = 2.0 * ga;
                const double ri = rsqrt(fma(dd, dd, g2 * g2));
                const double hc = fma(0.5 * fabs(dd), ri, 0.5);
                const double ic = rsqrt(hc);
                cs = hc * ic;
                sn = 0.5 * copysign(1.0, dd) * g2 * ri * ic;
                const double t = sn * ic;
#pragma unroll
                for (int v = 0; v < NG; v++) {
                    const double xa = top[v], xb = bot[v];
                    top[v] = cs * xa - sn * xb;
                    bot[v] = sn * xa + cs * xb;
                }
                al = al - t * ga;
                be = be + t * ga;
                myrot |= (ga * ga > 1e-16 * (al * be)) ? 3 : 1;
            }
            if (p == 0) rot[((long long)sw * (CT + 1) + rd) * npair + grp] = make_double2(cs, sn);
        };
        if (stat) {
            // levels of block size hb = G2, G2 / 2, ..., 1 (see stat_cols)
            int rd = 0;
            for (int hb = G2; hb >= 1; hb >>= 1) {
                const int i = grp & (hb - 1);
                const bool cross = hb > GPW;  // the ring of hb pairs spans warps
                const int wpb = cross ? hb / GPW : 1, wbase = warp - warp % wpb;
                const int src = cross ? ((lane + LP) & 31) : ((i + 1 == hb) ? lane - (hb - 1) * LP : lane + LP);
                for (int s = 0; s < hb; s++, rd++) {
                    if (act) rotate(rd);
                    if (hb == 1) continue;
                    // second columns one pair back along the ring: within the
                    // warp by shuffles, across warps through shared memory
                    double* xb0 = xch + (long long)buf * NW * 2 * LP * (NG + 1);
                    if (cross && gw == 0) {
                        double* d = xb0 + (warp * 2 * LP + p) * (NG + 1);
#pragma unroll
                        for (int v = 0; v < NG; v++) d[v] = bot[v];
                        d[NG] = be;
                    }
                    double nb[NG];
#pragma unroll
                    for (int v = 0; v < NG; v++) nb[v] = __shfl_sync(0xffffffffu, bot[v], src);
                    double nbe = __shfl_sync(0xffffffffu, be, src);
                    if (cross) {
                        __syncthreads();
                        if (gw == GPW - 1) {
                            const int wn = wbase + (warp - wbase + 1) % wpb;
                            const double* sx = xb0 + (wn * 2 * LP + p) * (NG + 1);
#pragma unroll
                            for (int v = 0; v < NG; v++) nb[v] = sx[v];
                            nbe = sx[NG];
                        }
                        buf ^= 1;
                    }
#pragma unroll
                    for (int v = 0; v < NG; v++) bot[v] = nb[v];
                    be = nbe;
                }
                if (hb >= 2) {
                    // split: pair i < h takes the first column of pair i + h
                    // as its second, pair i + h the second column of pair i
                    // as its first (h = hb / 2), through shared memory
                    const int h = hb >> 1;
                    const bool lo = i < h;
                    double* d = Lc + ((long long)grp * LP + p) * (NG + 1);
                    if (act) {
#pragma unroll
                        for (int v = 0; v < NG; v++) d[v] = lo ? bot[v] : top[v];
                        d[NG] = lo ? be : al;
                    }
                    __syncthreads();
                    if (act) {
                        const double* sx = Lc + ((long long)(grp ^ h) * LP + p) * (NG + 1);
                        if (lo) {
#pragma unroll
                            for (int v = 0; v < NG; v++) bot[v] = sx[v];
                            be = sx[NG];
                        } else {
#pragma unroll
                            for (int v = 0; v < NG; v++) top[v] = sx[v];
                            al = sx[NG];
                        }
                    }
                    __syncthreads();
                }
            }
            // back to the first arrangement: pair g holds columns 2g, 2g + 1
            // after the last level; it starts the next sweep with g, G2 + g
            if (act) {
#pragma unroll
                for (int v = 0; v < NG; v++) {
                    Lc[(2 * grp) * S + p + LP * v] = top[v];
                    Lc[(2 * grp + 1) * S + p + LP * v] = bot[v];
                }
            }
            __syncthreads();
            if (act) {
#pragma unroll
                for (int v = 0; v < NG; v++) {
                    top[v] = Lc[grp * S + p + LP * v];
                    bot[v] = Lc[(G2 + grp) * S + p + LP * v];
                }
            }
        } else {
            for (int rd = 0; rd < qq - 1; rd++) {
                if (act) rotate(rd);
                // move the columns to the next round's pairs
                double* xb0 = xch + (long long)buf * NW * 2 * LP * (NG + 1);
                if (gw == 0) {  // this warp's first top: to the previous warp's last group
                    double* d = xb0 + ((warp * 2 + 0) * LP + p) * (NG + 1);
#pragma unroll
                    for (int v = 0; v < NG; v++) d[v] = top[v];
                    d[NG] = al;
                }
                if (gw == GPW - 1) {  // this warp's last bottom: to the next warp's first group
                    double* d = xb0 + ((warp * 2 + 1) * LP + p) * (NG + 1);
#pragma unroll
                    for (int v = 0; v < NG; v++) d[v] = bot[v];
                    d[NG] = be;
                }
                double rt[NG], rb[NG];
#pragma unroll
                for (int v = 0; v < NG; v++) {
                    rt[v] = __shfl_down_sync(0xffffffffu, top[v], LP);  // top of group + 1
                    rb[v] = __shfl_up_sync(0xffffffffu, bot[v], LP);    // bottom of group - 1
                }
                double rta = __shfl_down_sync(0xffffffffu, al, LP);
                double rbb = __shfl_up_sync(0xffffffffu, be, LP);
                __syncthreads();
                if (gw == GPW - 1 && warp + 1 < NW) {
                    const double* sx = xb0 + (((warp + 1) * 2 + 0) * LP + p) * (NG + 1);
#pragma unroll
                    for (int v = 0; v < NG; v++) rt[v] = sx[v];
                    rta = sx[NG];
                }
                if (gw == 0 && warp > 0) {
                    const double* sx = xb0 + (((warp - 1) * 2 + 1) * LP + p) * (NG + 1);
#pragma unroll
                    for (int v = 0; v < NG; v++) rb[v] = sx[v];
                    rbb = sx[NG];
                }
                buf ^= 1;
                if (G == 1) {
                    // one pair: both positions are fixed points of the circle order
                } else if (grp == 0) {  // top fixed, bottom <- top of pair 1
#pragma unroll
                    for (int v = 0; v < NG; v++) bot[v] = rt[v];
                    be = rta;
                } else if (grp == G - 1) {  // top <- own bottom, bottom <- bottom of pair G - 2
#pragma unroll
                    for (int v = 0; v < NG; v++) {
                        top[v] = bot[v];
                        bot[v] = rb[v];
                    }
                    al = be;
                    be = rbb;
                } else if (act) {
#pragma unroll
                    for (int v = 0; v < NG; v++) {
                        top[v] = rt[v];
                        bot[v] = rb[v];
                    }
                    al = rta;
                    be = rbb;
                }
            }
        }
        if (myrot) atomicOr(&s_rot, myrot);
        __syncthreads();
        if (s_rot == 0) {
            conv = true;
        } else {
            sweeps = sw + 1;
            if (!(s_rot & 2)) conv = true;
        }
        __syncthreads();  // s_rot is reset at the next sweep's start
    }
    if (!conv && tid == 0) PTT_STATUS_SET(status, PTT_ERR_NUMERIC);
    // the columns back to shared memory: each sweep ends with pair g holding
    // columns g and qq - 1 - g (circle) or g and G2 + g (stationary ring)
    if (act) {
        const int cb = stat ? G2 + grp : qq - 1 - grp;
#pragma unroll
        for (int v = 0; v < NG; v++) {
            Lc[grp * S + p + LP * v] = top[v];
            Lc[cb * S + p + LP * v] = bot[v];
        }
    }
    __syncthreads();
    // singular values (column norms) and descending order
    for (int j = tid / LP; j < qq; j += SVD_NT / LP) {
        double s2 = 0.0;
#pragma unroll
        for (int v = 0; v < NG; v++) {
            const double x = Lc[j * S + p + LP * v];
            s2 += x * x;
        }
        s2 = gsum_g<LP>(s2, gm);
        if (p == 0) {
            const bool nan = !(s2 == s2);
            if (nan && j < q) PTT_STATUS_SET(status, PTT_ERR_NUMERIC);
            s_sig[j] = (j < q && !nan) ? sqrt(s2) : -1.0;
        }
    }
    __syncthreads();
    for (int j = tid; j < qq; j += SVD_NT) {
        const double sj = s_sig[j];
        int pos = 0;
        for (int i = 0; i < qq; i++) {
            const double si = s_sig[i];
            pos += (si > sj) || (si == sj && i < j);
        }
        s_ord[pos] = j;
    }
    __syncthreads();
    double* sig_out = ws + pl.o_sig;
    if (tid == 0) {
        const double s0 = q > 0 ? s_sig[s_ord[0]] : 0.0;
        const double thr = sqrt((double)q) * 1.1102230246251565e-16 * s0;
        int nsv = q > 0 ? 1 : 0;
        while (nsv < q && s_sig[s_ord[nsv]] >= thr) nsv++;
        if (!(s0 == s0)) PTT_STATUS_SET(status, PTT_ERR_NUMERIC);
        double ssum = 0.0;
        int rank = nsv;
        for (int j = nsv - 1; j >= 0; j--) {
            const double sj = s_sig[s_ord[j]];
            ssum += sj * sj;
            if (sqrt(ssum) < delta)
                rank = j;
            else
                break;
        }
        if (rank > q) rank = q;
        if (rank > maxr) rank = maxr;
        if (rank < 1) rank = 1;
        info->rank = rank;
        info->nsv = nsv;
        info->sweeps = sweeps;
        info->order = stat ? 1 : 0;
        double tail = 0.0;
        for (int j = rank; j < q; j++) tail += s_sig[s_ord[j]] * s_sig[s_ord[j]];
        info->tail = tail;
        if (pl.stats) {
            double* st = pl.stats + (long long)bond * PTT_STAT_LEN;
            st[0] = rank;
            st[1] = nsv;
            st[2] = sweeps;
            st[3] = q;
            st[4] = c;
            st[5] = tail;
            st[6] = delta;
            st[7] = 0.0;
            for (int j = 0; j < PTT_STAT_NSIG; j++) st[8 + j] = j < q ? s_sig[s_ord[j]] : 0.0;
        }
    }
    for (int j = tid; j < CT; j += SVD_NT) {
        sig_out[j] = j < q ? s_sig[s_ord[j]] : 0.0;
        ((int*)(sig_out + CT))[j] = j < qq ? s_ord[j] : 0;
    }
    __syncthreads();
    const int rank = info->rank;
    double* US = ws + pl.o_US;  // c x rank, column-major ld CT
    for (int e = tid; e < CT * CT; e += SVD_NT) {
        const int b = e / CT, t = e - (e / CT) * CT;
        US[e] = (b < rank && t < c) ? Lc[s_ord[b] * S + t] : 0.0;
    }
}

// The ring Jacobi is used for bonds of more than SVD_RING_MIN columns; below
// that the shared-memory Jacobi was faster on one B200 (the reaction-Burgers
// steps, whose bonds have <= ~40 columns: 105 vs 101 ms per plain step),
// above it the ring (64 columns: 13.2 vs 21.7 ms for 39 bonds).
constexpr int SVD_RING_MIN = 48;

template <int CT, int LP = 4>
static size_t ring_smem() {
    constexpr int NW = ring_nt<CT, LP>() / 32;
    return sizeof(double) * ((size_t)(CT + 2) * (CT + 1) + 2ull * NW * 2 * LP * (CT / LP + 1));
}

// Rebuild rows of V (q x q, V = product of the recorded rotations) and write
// V_r = V[:, order[0:rank]] into Bn[root].  One warp per row; each sweep's
// rotation table is staged in shared memory once per block, the column pair
// of each (round, pair) slot is tabulated once for all sweeps.
__device__ void svd_replay_body(const Plan& pl, double* ws, const Info* info, int bx) {
    extern __shared__ double sm[];
    const int CT = pl.CT, KC = pl.KC;
    const int SR = CT + 2;
    const int npair = (CT + 2) / 2;
    double* vrow = sm + (threadIdx.x >> 5) * SR;   // 8 rows
    double2* tab = (double2*)(sm + 8 * SR);         // (CT+1) rounds x npair
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int row = bx * 8 + warp;
    if (info->status) return;
    const int q = info->q, qq = q + (q & 1), sweeps = info->sweeps, rank = info->rank, order = info->order;
    // pairs and rounds of a sweep: the stationary ring runs over qq / 2
    // rounded up to a power of two
    const int npr = (order == 1 && qq >= 4) ? 1 << (32 - __clz(qq / 2 - 1)) : qq / 2;
    const int nrd = 2 * npr - 1;
    // the column pair of every (round, pair) slot, once for all sweeps
    unsigned char* pcol = (unsigned char*)(tab + (CT + 1) * npair);
    unsigned char* qcol = pcol + (CT + 1) * npair;
    for (int e = threadIdx.x; e < nrd * npr; e += blockDim.x) {
        const int rd = e / npr, i = e - (e / npr) * npr;
        int pc, qc;
        if (order == 1) {
            stat_cols(i, rd, npr, &pc, &qc);
        } else {
            pc = circle_col(i, rd, qq);
            qc = circle_col(qq - 1 - i, rd, qq);
        }
        pcol[rd * npair + i] = (unsigned char)pc;
        qcol[rd * npair + i] = (unsigned char)qc;
    }
    for (int j = lane; j < SR; j += 32) vrow[j] = (j == row) ? 1.0 : 0.0;
    const double2* rot = (const double2*)(ws + pl.o_rot);
    for (int sw = 0; sw < sweeps; sw++) {
        __syncthreads();
        const long long base = (long long)sw * (CT + 1) * npair;
        const int cnt = nrd * npair;
        for (int e = threadIdx.x; e < cnt; e += blockDim.x) tab[e] = rot[base + e];
        __syncthreads();
        if (row < q) {
            for (int rd = 0; rd < nrd; rd++) {
                for (int i = lane; i < npr; i += 32) {
                    const double2 r = tab[rd * npair + i];
                    if (r.y != 0.0) {
                        const int pc = pcol[rd * npair + i], qc = qcol[rd * npair + i];
                        const double x = vrow[pc], y = vrow[qc];
                        vrow[pc] = r.x * x - r.y * y;
                        vrow[qc] = r.y * x + r.x * y;
                    }
                }
                __syncwarp();
            }
        }
    }
    __syncthreads();
    if (row >= CT) return;
    const int* ord = (const int*)(ws + pl.o_sig + CT);
    double* B = ws + pl.o_Bn + (long long)row * KC;
    for (int b = lane; b < KC; b += 32) B[b] = (row < q && b < rank) ? vrow[ord[b]] : 0.0;
}

__global__ void __launch_bounds__(256) k_svd_replay(Plan pl, double* ws) {
    PTT_PDL_ENTRY();
    svd_replay_body(pl, ws, pl.info, blockIdx.x);
}

// the same for bonds k0 .. k0 + gridDim.y - 1, bond k's records at ws + k * stride
__global__ void __launch_bounds__(256) k_svd_replay_b(Plan pl, double* ws, long long stride, int k0) {
    PTT_PDL_ENTRY();
    double* wsb = ws + (long long)(k0 + blockIdx.y) * stride;
    svd_replay_body(pl, wsb, (const Info*)(wsb + pl.o_info_d), blockIdx.x);
}

// ---------------------------------------------------------------------------
// FP64 GEMM tiles: C[M x N] = A[M x K] * B[K x N], views with strides.
// ---------------------------------------------------------------------------
struct GV {
    const double* p;
    long long rs, cs;
};

constexpr int GT = 64, GK = 16;

__device__ void gemm_tile(GV A, GV B, double* C, long long crs, long long ccs, int M, int N, int K, int tm, int tn) {
    __shared__ double sA[GK][GT + 1];
    __shared__ double sB[GK][GT + 1];
    const int tid = threadIdx.x;
    const int m0 = tm * GT, n0 = tn * GT;
    // the tile product on the FP64 tensor cores: warp w owns the eight 8 x 8
    // output tiles of tile row w (mma.m8n8k4, four k a step)
    const int warp = tid >> 5, lane = tid & 31, li = lane >> 2, lk = lane & 3;
    double d0[8], d1[8];
#pragma unroll
    for (int t = 0; t < 8; t++) {
        d0[t] = 0.0;
        d1[t] = 0.0;
    }
    // every element of a K chunk requested before the first is stored, and the
    // next chunk's loads in flight during this chunk's products
    constexpr int PT = GT * GK / 256;
    double va[PT], vb[PT];
    auto load = [&](int k0) {
#pragma unroll
        for (int u = 0; u < PT; u++) {
            const int e = tid + 256 * u;
            {
                const int r = e % GT, kk = e / GT;
                const int gr = m0 + r, gk = k0 + kk;
                va[u] = (gr < M && gk < K) ? A.p[(long long)gr * A.rs + (long long)gk * A.cs] : 0.0;
            }
            {
                const int kk = e % GK, cn = e / GK;
                const int gk = k0 + kk, gc = n0 + cn;
                vb[u] = (gk < K && gc < N) ? B.p[(long long)gk * B.rs + (long long)gc * B.cs] : 0.0;
            }
        }
    };
    if (K > 0) load(0);
    for (int k0 = 0; k0 < K; k0 += GK) {
#pragma unroll
        for (int u = 0; u < PT; u++) {
            const int e = tid + 256 * u;
            sA[e / GT][e % GT] = va[u];
            sB[e % GK][e / GK] = vb[u];
        }
        __syncthreads();
        if (k0 + GK < K) load(k0 + GK);
#pragma unroll
        for (int k4 = 0; k4 < GK; k4 += 4) {
            const double av = sA[k4 + lk][8 * warp + li];
#pragma unroll
            for (int t = 0; t < 8; t++) {
                const double bv = sB[k4 + lk][8 * t + li];
                asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                             : "+d"(d0[t]), "+d"(d1[t])
                             : "d"(av), "d"(bv));
            }
        }
        __syncthreads();
    }
    const int gr = m0 + 8 * warp + li;
    if (gr < M) {
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const int gc = n0 + 8 * t + 2 * lk;
            if (gc < N) C[(long long)gr * crs + (long long)gc * ccs] = d0[t];
            if (gc + 1 < N) C[(long long)gr * crs + (long long)(gc + 1) * ccs] = d1[t];
        }
    }
}

// The bookkeeping that follows a bond's contraction: publish the bond's new
// rank (D->r[kq] = *val) and swap core[ka] with the buffer just written.
// With a ticket (a zero-initialised counter) the last block of the
// contraction does it, so it needs no launch of its own; without one the
// caller launches k_bond_finalize.
struct Fin {
    int* ticket;
    int kq, ka;
    const int* val;
};

__device__ __forceinline__ void fin_last_block(DevDesc* D, const Fin& f, const Info* info) {
    if (!f.ticket) return;
    __shared__ int s_last;
    __syncthreads();
    __threadfence();  // this block's output is visible before its ticket
    if (threadIdx.x == 0) s_last = atomicAdd(f.ticket, 1) == (int)(gridDim.x * gridDim.y) - 1;
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        *f.ticket = 0;
        __threadfence();
        if (info->status == 0) {
            D->r[f.kq] = *f.val;
            double* t = D->core[f.ka];
            D->core[f.ka] = D->alt[f.ka];
            D->alt[f.ka] = t;
        }
    }
}

// core[i+1] <- R * core[i+1]   (R = root factor, q x c, row-major CT)
__global__ void __launch_bounds__(256) k_gemm_rx(DevDesc* D, int i1, Plan pl, double* ws, Fin fin) {
    PTT_PDL_ENTRY();
    const int tm = blockIdx.x, tn = blockIdx.y;
    if (pl.info->status == 0) {
        const int q = pl.info->q, c = pl.info->c;
        const int N = D->n[i1] * D->r[i1 + 1];
        if (tm * GT < q) {
            for (int t = tn; t * GT < N; t += gridDim.y) {
                GV A{ws + pl.o_Rn, pl.CT, 1};
                GV B{D->core[i1], 1, c};
                gemm_tile(A, B, D->alt[i1], 1, q, q, N, c, tm, t);
            }
        }
    }
    fin_last_block(D, fin, pl.info);
}

// core[i-1] <- core[i-1] * US   (US = c x rank, column-major ld CT)
__global__ void __launch_bounds__(256) k_gemm_xm(DevDesc* D, int im1, Plan pl, double* ws, Fin fin) {
    PTT_PDL_ENTRY();
    const int tn = blockIdx.y;
    if (pl.info->status == 0) {
        const int c = pl.info->c, rank = pl.info->rank;
        const int M = D->r[im1] * D->n[im1];
        if (tn * GT < rank) {
            for (int t = blockIdx.x; t * GT < M; t += gridDim.x) {
                GV A{D->core[im1], 1, M};
                GV B{ws + pl.o_US, 1, pl.CT};
                gemm_tile(A, B, D->alt[im1], 1, M, M, rank, c, t, tn);
            }
        }
    }
    fin_last_block(D, fin, pl.info);
}

#include "ptt_ozaki.cuh"

// k_gemm_rx of the block-level path with the product as an Ozaki
// split-precision product on the fifth-generation tensor cores
// (oz::gemm_tiles): R (q x c, row-major, leading dimension CT) times core
// i1 (c x N, column-major) into alt[i1] (q x N); CTA y takes the 64-column
// tiles y, y + gridDim.y, ...
__global__ void __launch_bounds__(256, 1) k_gemm_rx_oz(DevDesc* D, int i1, Plan pl, double* ws) {
    PTT_PDL_ENTRY();
    extern __shared__ __align__(128) unsigned char osm[];
    if (pl.info->status != 0) return;
    const int q = pl.info->q, c = pl.info->c;
    const int N = D->n[i1] * D->r[i1 + 1];
    if (q > oz::KG || c > oz::KG || 64 * (int)blockIdx.y >= N) return;  // uniform
    oz::gemm_tiles<256>(ws + pl.o_Rn, pl.CT, 1, D->core[i1], 1, c, D->alt[i1], q, q, N, c, osm, false);
}

// k_gemm_xm of the block-level path as an Ozaki product: core[i-1] (M x c,
// column-major) times U_r S_r (c x rank, column-major, leading dimension CT)
// into alt[i-1], formed as its transpose (U_r S_r)^T core^T so that the
// 64-wide tiles run along the M rows
__global__ void __launch_bounds__(256, 1) k_gemm_xm_oz(DevDesc* D, int im1, Plan pl, double* ws) {
    PTT_PDL_ENTRY();
    extern __shared__ __align__(128) unsigned char osm[];
    if (pl.info->status != 0) return;
    const int c = pl.info->c, rank = pl.info->rank;
    const int M = D->r[im1] * D->n[im1];
    if (rank > oz::KG || c > oz::KG || 64 * (int)blockIdx.y >= M) return;  // uniform
    oz::gemm_tiles<256>(ws + pl.o_US, pl.CT, 1, D->core[im1], M, 1, D->alt[im1], M, rank, M, c, osm, true);
}

// publish a bond's new rank and swap the two rewritten cores
__global__ void k_bond_finalize(DevDesc* D, int kq, int ka, int kb, const int* val, const Info* info) {
    PTT_PDL_ENTRY();
    if (threadIdx.x == 0 && info->status == 0) {
        D->r[kq] = *val;
        double* t = D->core[ka];
        D->core[ka] = D->alt[ka];
        D->alt[ka] = t;
        if (kb >= 0) {
            t = D->core[kb];
            D->core[kb] = D->alt[kb];
            D->alt[kb] = t;
        }
    }
}

#include "ptt_wtsqr.cuh"
#include "ptt_cholqr.cuh"
#include "ptt_gridqr.cuh"

// ---------------------------------------------------------------------------
// host planning
// ---------------------------------------------------------------------------
static int next_pow2(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

struct Layout {
    Plan pl;
    long long bytes;
};

// pmax bounds the leaves (and so the tree levels, one apply launch each):
// the Householder TSQR behind the grid Cholesky QR only runs for a bond that
// falls back, so there it takes few, long leaves and its skipped launches
// stay few.
static void plan_bond(int CT, long long mcap, int KC, Plan* pl, int pmax = 512) {
    int L = 2 * CT;
    if (L < 128) L = 128;
    L = (L + H - 1) / H * H;
    long long P = (mcap + L - 1) / L;
    while (P > pmax) {
        L *= 2;
        P = (mcap + L - 1) / L;
    }
    pl->CT = CT;
    pl->L = L;
    pl->P = next_pow2((int)(P < 1 ? 1 : P));
    pl->KL = 1 + (2 * L - 1 + H - 1) / H;
    pl->NH = (CT + H - 1) / H;
    pl->KC = KC;
    pl->gqstate = nullptr;
}

static long long carve(Plan* pl, int PMAX, int LMAXKL) {
    const int CT = pl->CT, KC = pl->KC;
    long long o = 0;
    auto take = [&](long long n) {
        long long r = o;
        o += (n + 31) / 32 * 32;
        return r;
    };
    pl->o_tau_leaf = take((long long)PMAX * LMAXKL * CT);
    pl->o_Rn = take((long long)(2 * PMAX - 1) * CT * CT);
    pl->o_tau_node = take((long long)PMAX * pl->NH * CT);
    pl->o_Bn = take((long long)(2 * PMAX - 1) * CT * KC);
    pl->o_US = take((long long)CT * CT);
    pl->o_rot = take((long long)MAXSW * (CT + 1) * ((CT + 2) / 2) * 2);
    pl->o_sig = take(2LL * CT + 64);
    pl->o_info_d = take(64);
    pl->o_nodes = take((long long)(3 * PMAX + 64) / 2 + 1);  // qn [2P-1] and pass [P] as ints
    pl->total = o;
    return o;
}

template <int CT>
static size_t factor_smem() {
    return sizeof(double) * ((size_t)CT * CT + 2 * (size_t)FCfg<CT>::VB + CT);
}
template <int CT>
static size_t apply_smem() {
    const int VR = CT > H ? CT : H;
    return sizeof(double) * ((size_t)CT * KG + (size_t)VR * (CT + 1));
}
template <int CT>
static size_t svd_smem() {
    return sizeof(double) * (size_t)(CT + 2) * (CT + 1);
}

// 8 V rows + one sweep's rotation table ((CT+1) rounds x (CT+2)/2 pairs)
template <int CT>
static size_t replay_smem() {
    // 8 rows of V, one sweep's rotations, the two column tables (bytes)
    return sizeof(double) * (8 * (size_t)(CT + 2) + 2 * (size_t)(CT + 1) * ((CT + 2) / 2)) +
           2 * (size_t)(CT + 1) * ((CT + 2) / 2);
}

template <int CT>
static int set_attrs() {
    static std::atomic<unsigned long long> done{0};
    unsigned long long bit;
    if (ptt_device_done(done, &bit)) return PTT_OK;
    PTT_CUDA(cudaFuncSetAttribute(k_tsqr_factor<CT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)factor_smem<CT>()));
    PTT_CUDA(cudaFuncSetAttribute(k_apply_leaf<CT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)apply_smem<CT>()));
    PTT_CUDA(cudaFuncSetAttribute(k_apply_node<CT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)apply_smem<CT>()));
    PTT_CUDA(cudaFuncSetAttribute(k_svd_jacobi<CT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)svd_smem<CT>()));
    if (CT <= 64)
        PTT_CUDA(cudaFuncSetAttribute(k_svd_ring<CT <= 64 ? CT : 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)ring_smem<CT <= 64 ? CT : 64>()));
    PTT_CUDA(cudaFuncSetAttribute(k_svd_replay, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)replay_smem<128>()));
    PTT_CUDA(cudaFuncSetAttribute(gq::k_gq_stage<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gq::SMEM));
    PTT_CUDA(cudaFuncSetAttribute(gq::k_gq_stage<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)gq::SMEM_OZ));
    PTT_CUDA(cudaFuncSetAttribute(k_gemm_rx_oz, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)oz::SMEM_GEMM));
    PTT_CUDA(cudaFuncSetAttribute(k_gemm_xm_oz, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)oz::SMEM_GEMM));
    done.fetch_or(bit);
    return PTT_OK;
}

// Factor the unfolding (mode) of core k; R lands at the root slot.  With the
// grid Cholesky QR (g != null) its stage launches go first and the Householder
// TSQR only factors a bond they did not finish.
template <int CT>
static int launch_factor(ptt_ctx* c, ptt_tt* x, int k, int mode, Plan& pl, double* ws, gq::GQ* g, long long mcap) {
    ptt_time_begin(c, PTT_TIME_TSQR);
    if (g) {
        g->rpb = gq::rows_per_cta(mcap, c->nsm);
        const int nb = gq::ctas(mcap, g->rpb);
        pl.gqstate = (const int*)g->rec;
        for (int s = 0; s < gq::MAXST; s++) {
            if (c->ozaki)
                PTT_CUDA(ptt_launch(c, gq::k_gq_stage<true>, dim3(nb), dim3(gq::NT), gq::SMEM_OZ,
                                    (const DevDesc*)x->dd, k, mode, pl, *g, ws, s, c->d_qrstat));
            else
                PTT_CUDA(ptt_launch(c, gq::k_gq_stage<false>, dim3(nb), dim3(gq::NT), gq::SMEM,
                                    (const DevDesc*)x->dd, k, mode, pl, *g, ws, s, c->d_qrstat));
            PTT_LAUNCHED(c);
        }
    }
    PTT_CUDA(ptt_launch(c, k_tsqr_factor<CT>, dim3(pl.P), dim3(NT), factor_smem<CT>(), (const DevDesc*)x->dd, k, mode,
                        pl, ws, c->d_status));
    ptt_time_end(c, PTT_TIME_TSQR);
    PTT_LAUNCHED(c);
    return PTT_OK;
}

// out = Q * Bn[root]; k columns read from *kptr, at most kcap.
template <int CT>
static int launch_apply(ptt_ctx* c, ptt_tt* x, int k, int mode, Plan& pl, double* ws, const int* kptr, int kcap) {
    const int kgroups = (kcap + KG - 1) / KG;
    int first = 0, cnt = 1;
    while (first + cnt <= pl.P - 1) {  // internal levels: nodes [first, first+cnt)
        PTT_CUDA(ptt_launch(c, k_apply_node<CT>, dim3(cnt, kgroups), dim3(NT), apply_smem<CT>(), pl, ws, first, kptr));
        PTT_LAUNCHED(c);
        first += cnt;
        cnt *= 2;
    }
    PTT_CUDA(ptt_launch(c, k_apply_leaf<CT>, dim3(pl.P, kgroups), dim3(NT), apply_smem<CT>(), (const DevDesc*)x->dd, k,
                        mode, pl, ws, kptr));
    PTT_LAUNCHED(c);
    return PTT_OK;
}

// phases: 1 = left-to-right orthogonalisation, 2 = right-to-left truncation,
// 4 = QR of the single core `only` (left unfolding; core <- Q, r_{only+1} <- q).
// rk[k]: upper bound of rank k for the whole call (the capacity, or the
// actual ranks when they were read back; ranks only shrink while rounding).
// At CT = 64 every factorisation first runs the grid Cholesky QR
// (ptt_gridqr.cuh) unless the context is set to Householder only.
template <int CT>
static int round_impl(ptt_tt* x, const int* rk, double delta, const int* maxr, int phases, int only) {
    ptt_ctx* c = x->ctx;
    const int d = x->d;
    int rc = set_attrs<CT>();
    if (rc) return rc;
    const bool use_gq = (CT == gq::CB) && !c->no_cholqr;
    // plan: largest leaf count over all bonds decides the workspace
    const int KC = (CT + KG - 1) / KG * KG;
    int PMAX = 1, KLMAX = 1, NBMAX = 1;
    long long MQMAX = 1;
    const int pmax = use_gq ? 32 : 512;
    for (int i = 0; i < d; i++) {
        Plan t;
        long long ml = (long long)rk[i] * x->n[i], mr = (long long)x->n[i] * rk[i + 1];
        plan_bond(CT, ml > mr ? ml : mr, KC, &t, pmax);
        if (t.P > PMAX) PMAX = t.P;
        if (t.KL > KLMAX) KLMAX = t.KL;
        for (long long mm : {ml, mr}) {
            const int nb = gq::ctas(mm, gq::rows_per_cta(mm, c->nsm));
            NBMAX = nb > NBMAX ? nb : NBMAX;
        }
        MQMAX = mr > MQMAX ? mr : MQMAX;
    }
    Plan base;
    plan_bond(CT, 1, KC, &base);
    base.NH = (CT + H - 1) / H;
    long long total = carve(&base, PMAX, KLMAX);
    // grid Cholesky QR: record, partial Gram matrices, Q rows of RIGHT_T bonds
    const int NGMAX = (NBMAX + gq::GROUP - 1) / gq::GROUP;
    long long o_gq = (total + 31) / 32 * 32, gq_len = 0;
    if (use_gq) gq_len = gq::REC + (long long)(NBMAX + NGMAX) * gq::UP + MQMAX * gq::CB + 64;
    // two slots of the whole region (bond parity): the truncation sweep runs
    // the tail of bond i (V replay, Q V_r, swap of core i) on the side stream
    // while bond i - 1 is factored in the other slot
    const long long SLOT = (o_gq + gq_len + 31) / 32 * 32;
    size_t bytes = (size_t)(2 * SLOT) * sizeof(double) + 256;
    if ((rc = ptt_ws_reserve(c, bytes))) return rc;
    const size_t cnt_tree = (size_t)PMAX * 4 + 64;
    if ((rc = ptt_counters_reserve(c, cnt_tree + NGMAX + 2))) return rc;
    double* const ws0 = (double*)c->ws;
    // ints live after the doubles: qn [2P-1], pass [P], Info
    // Tree counters live alone in ctx->d_counters (zero between launches,
    // reset by the combining block); node ranks and pass flags in ws.
    double* wss[2] = {ws0, ws0 + SLOT};
    gq::GQ gqs[2] = {};
    for (int sl = 0; sl < 2 && use_gq; sl++) {
        gqs[sl].rec = wss[sl] + o_gq;
        gqs[sl].part = gqs[sl].rec + (gq::REC + 31) / 32 * 32;
        gqs[sl].gpart = gqs[sl].part + (long long)NBMAX * gq::UP;
        gqs[sl].qscr = gqs[sl].gpart + (long long)NGMAX * gq::UP;
        gqs[sl].cnt = c->d_counters + cnt_tree;  // main stream only
    }
    double* ws = ws0;
    Info* info = (Info*)(ws0 + base.o_info_d);
    gq::GQ* g = use_gq ? &gqs[0] : nullptr;

    auto mkplan = [&](long long mcap, int sl = 0) {
        Plan pl = base;
        Plan t;
        plan_bond(CT, mcap, KC, &t, pmax);
        int* ints = (int*)(wss[sl] + base.o_nodes);
        pl.L = t.L;
        pl.P = t.P;
        pl.KL = KLMAX;
        pl.cnt = c->d_counters;
        pl.qn = ints;
        pl.pass = ints + 2 * PMAX;
        pl.info = (Info*)(wss[sl] + base.o_info_d);
        pl.stats = c->d_stats;
        pl.work = (c->tkind == PTT_TIME_TSQR) ? c->d_work + PTT_TIME_TSQR : nullptr;
        return pl;
    };
    const DevDesc* dd = x->dd;

    if (phases & 4) {
        const int i = only;
        const long long mcap = (long long)rk[i] * x->n[i];
        Plan pl = mkplan(mcap);
        if ((rc = launch_factor<CT>(c, x, i, LEFT, pl, ws, g, mcap))) return rc;
        PTT_CUDA(ptt_launch(c, k_set_identity, dim3(32), dim3(256), 0, pl, ws));
        PTT_LAUNCHED(c);
        if ((rc = launch_apply<CT>(c, x, i, LEFT, pl, ws, &info->q, CT))) return rc;
        PTT_CUDA(ptt_launch(c, k_bond_finalize, dim3(1), dim3(32), 0, x->dd, i + 1, i, -1, (const int*)&info->q,
                            (const Info*)info));
        PTT_LAUNCHED(c);
        return PTT_OK;
    }
    // left-to-right orthogonalisation
    for (int i = 0; i < d - 1 && (phases & 1); i++) {
        const long long mcap = (long long)rk[i] * x->n[i];
        Plan pl = mkplan(mcap);
        if ((rc = launch_factor<CT>(c, x, i, LEFT, pl, ws, g, mcap))) return rc;
        {
            const long long ncap = (long long)x->n[i + 1] * rk[i + 2];
            int gy = (int)((ncap + GT - 1) / GT);
            if (gy > 4096) gy = 4096;
            if (c->ozaki && CT <= oz::KG)  // one wave, R split once per CTA
                PTT_CUDA(ptt_launch(c, k_gemm_rx_oz, dim3(1, gy < c->nsm ? gy : c->nsm), dim3(256), oz::SMEM_GEMM,
                                    x->dd, i + 1, pl, ws));
            else
                PTT_CUDA(ptt_launch(c, k_gemm_rx, dim3((CT + GT - 1) / GT, gy), dim3(256), 0, x->dd, i + 1, pl, ws,
                                    Fin{}));
            PTT_LAUNCHED(c);
        }
        PTT_CUDA(ptt_launch(c, k_set_identity, dim3(32), dim3(256), 0, pl, ws));
        PTT_LAUNCHED(c);
        if ((rc = launch_apply<CT>(c, x, i, LEFT, pl, ws, &info->q, CT))) return rc;
        PTT_CUDA(ptt_launch(c, k_bond_finalize, dim3(1), dim3(32), 0, x->dd, i + 1, i, i + 1, (const int*)&info->q,
                            (const Info*)info));
        PTT_LAUNCHED(c);
    }
    // right-to-left truncation.  The tail of bond i (V replay, Q V_r into
    // core i, swap of core i) is not needed by bond i - 1, which only reads
    // core i - 1 and the new rank r_i: it runs on the side stream from the
    // bond's slot (bond parity) while the main stream carries on; the main
    // stream waits for a slot's previous tail before reusing it, and for both
    // at the end.  Inside a caller's stream capture, and on the worker
    // contexts of a batch (which overlap whole roundings already: measured
    // 1.22 s against 0.98 s for 64 trains with the side stream), the sweep
    // stays serial.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    PTT_CUDA(cudaStreamIsCapturing(c->stream, &cap));
    const bool ovl = cap == cudaStreamCaptureStatusNone && !c->capturing && !c->lane;
    bool pending[2] = {false, false};
    for (int i = d - 1; i >= 1 && (phases & 2); i--) {
        const int sl = ovl ? (i & 1) : 0;
        if (pending[sl]) {
            PTT_CUDA(cudaStreamWaitEvent(c->stream, c->ev_tail[sl], 0));
            pending[sl] = false;
        }
        ws = wss[sl];
        info = (Info*)(ws + base.o_info_d);
        g = use_gq ? &gqs[sl] : nullptr;
        const long long mcap = (long long)x->n[i] * rk[i + 1];
        Plan pl = mkplan(mcap, sl);
        if ((rc = launch_factor<CT>(c, x, i, RIGHT_T, pl, ws, g, mcap))) return rc;
        const int mr = maxr ? maxr[i] : rk[i];
        ptt_time_begin(c, PTT_TIME_SVD);
        if (CT <= 64 && rk[i] > SVD_RING_MIN)  // columns in registers
            PTT_CUDA(ptt_launch(c, k_svd_ring<CT <= 64 ? CT : 64>, dim3(1), dim3(ring_nt<CT <= 64 ? CT : 64>()),
                                ring_smem<CT <= 64 ? CT : 64>(), pl, ws, delta, mr, i, c->d_status));
        else
            PTT_CUDA(ptt_launch(c, k_svd_jacobi<CT>, dim3(1), dim3(svd_nt<CT>()), svd_smem<CT>(), pl, ws, delta, mr,
                                i, c->d_status));
        ptt_time_end(c, PTT_TIME_SVD);
        PTT_LAUNCHED(c);
        // the tail: V_r, then Q V_r (Householder tree or grid Cholesky QR) into alt[i]
        auto tail = [&]() -> int {
            PTT_CUDA(ptt_launch(c, k_svd_replay, dim3((CT + 7) / 8), dim3(256), replay_smem<CT>(), pl, ws));
            PTT_LAUNCHED(c);
            int r2 = launch_apply<CT>(c, x, i, RIGHT_T, pl, ws, &info->rank, CT);
            if (r2) return r2;
            if (g) {  // Q V_r for a bond the grid Cholesky QR finished
                int gx = (int)((mcap + gq::WROWS - 1) / gq::WROWS);
                gx = gx < 1 ? 1 : (gx > 2 * c->nsm ? 2 * c->nsm : gx);
                PTT_CUDA(ptt_launch(c, gq::k_gq_write, dim3(gx), dim3(gq::NT), 0, dd, i, pl, *g, ws));
                PTT_LAUNCHED(c);
            }
            return PTT_OK;
        };
        if (ovl) {
            PTT_CUDA(cudaEventRecord(c->ev_svd[sl], c->stream));
            PTT_CUDA(cudaStreamWaitEvent(c->side, c->ev_svd[sl], 0));
            // the launch helpers issue on c->stream: point it at the side
            // stream; plain launches there (full stream order after the
            // event wait, no programmatic early start)
            cudaStream_t mainst = c->stream;
            const int pdl = c->no_pdl;
            c->stream = c->side;
            c->no_pdl = 1;
            rc = tail();
            if (!rc) {
                const cudaError_t e = ptt_launch(c, k_bond_finalize, dim3(1), dim3(32), 0, x->dd, i, i, -1,
                                                 (const int*)&info->rank, (const Info*)info);
                rc = e == cudaSuccess ? PTT_OK : ptt_set_error(PTT_ERR_CUDA, "CUDA: %s", cudaGetErrorString(e));
                PTT_LAUNCHED(c);
            }
            if (!rc) {
                const cudaError_t e = cudaEventRecord(c->ev_tail[sl], c->side);
                rc = e == cudaSuccess ? PTT_OK : ptt_set_error(PTT_ERR_CUDA, "CUDA: %s", cudaGetErrorString(e));
            }
            c->stream = mainst;
            c->no_pdl = pdl;
            if (rc) return rc;
            pending[sl] = true;
        } else if ((rc = tail())) {
            return rc;
        }
        {
            const long long mcap2 = (long long)rk[i - 1] * x->n[i - 1];
            int gx = (int)((mcap2 + GT - 1) / GT);
            if (gx > 4096) gx = 4096;
            if (c->ozaki && CT <= oz::KG)  // one wave, U_r S_r split once per CTA
                PTT_CUDA(ptt_launch(c, k_gemm_xm_oz, dim3(1, gx < c->nsm ? gx : c->nsm), dim3(256), oz::SMEM_GEMM,
                                    x->dd, i - 1, pl, ws));
            else
                PTT_CUDA(ptt_launch(c, k_gemm_xm, dim3(gx, (CT + GT - 1) / GT), dim3(256), 0, x->dd, i - 1, pl, ws,
                                    Fin{}));
            PTT_LAUNCHED(c);
        }
        // the new rank r_i and core i - 1 (core i too when the tail ran here)
        PTT_CUDA(ptt_launch(c, k_bond_finalize, dim3(1), dim3(32), 0, x->dd, i, ovl ? i - 1 : i, ovl ? -1 : i - 1,
                            (const int*)&info->rank, (const Info*)info));
        PTT_LAUNCHED(c);
    }
    for (int sl = 0; sl < 2; sl++)
        if (pending[sl]) PTT_CUDA(cudaStreamWaitEvent(c->stream, c->ev_tail[sl], 0));
    return PTT_OK;
}


// Rounding of a train whose ranks stay <= 32 on the warp-level TSQR.
// Per bond only the factorisation, the small product that moves R (or U S)
// into the neighbour core and the rank update run in sequence; Q (and V_r Q)
// is formed for all bonds of a sweep in one launch after the sweep, and the
// SVD rotations are replayed for all bonds in one launch.
// Every bond k has its own record region (ws + k * stride) so the deferred
// launches find each bond's reflectors.  Same phases as round_impl.
static bool wt_fits(const ptt_tt* x, const int* rk) {
    for (int i = 0; i < x->d; i++) {
        const long long ml = (long long)rk[i] * x->n[i], mr = (long long)x->n[i] * rk[i + 1];
        const long long mx = ml > mr ? ml : mr;
        if (mx > 32LL * wt::PMAX) return false;
    }
    return true;
}

static int g_cq_csmax[64];  // per device: cluster size it can schedule

// rows bucket of the autotuner's table: <= 512, 1024, ..., > 8192
static int cq_bucket(int mp) {
    int b = 0, lim = 512;
    while (b < 5 && mp > lim) {
        b++;
        lim <<= 1;
    }
    return b;
}

static int round_impl_w(ptt_tt* x, const int* rk, double delta, const int* maxr, int phases, int only) {
    using namespace wt;
    ptt_ctx* c = x->ctx;
    const int d = x->d;
    int rc = set_attrs<32>();
    if (rc) return rc;
    static std::atomic<unsigned long long> wattr{0};
    unsigned long long wbit;
    int dev = 0;
    cudaGetDevice(&dev);
    dev &= 63;
    if (!ptt_device_done(wattr, &wbit)) {
        g_cq_csmax[dev] = cq::CSMAX;
        PTT_CUDA(cudaFuncSetAttribute(k_wfactor<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wfactor_smem()));
        PTT_CUDA(cudaFuncSetAttribute(k_wfactor<24>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wfactor_smem()));
        PTT_CUDA(cudaFuncSetAttribute(k_wfactor<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wfactor_smem()));
        for (auto f : {(const void*)cq::k_cq_factor<16>, (const void*)cq::k_cq_factor<24>,
                       (const void*)cq::k_cq_factor<32>}) {
            PTT_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cq::SMEM_MAX));
            PTT_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        }
        // largest cluster the device can hold with one full-size CTA per SM
        cudaLaunchConfig_t qc = {};
        qc.gridDim = dim3(cq::CSMAX);
        qc.blockDim = dim3(cq::NT);
        qc.dynamicSmemBytes = cq::SMEM_MAX;
        cudaLaunchAttribute qa[1];
        qa[0].id = cudaLaunchAttributeClusterDimension;
        qa[0].val.clusterDim.x = cq::CSMAX;
        qa[0].val.clusterDim.y = 1;
        qa[0].val.clusterDim.z = 1;
        qc.attrs = qa;
        qc.numAttrs = 1;
        int ncl = 0;
        if (cudaOccupancyMaxActiveClusters(&ncl, (const void*)cq::k_cq_factor<32>, &qc) != cudaSuccess || ncl < 1) {
            cudaGetLastError();
            g_cq_csmax[dev] = 8;
        }
        wattr.fetch_or(wbit);
    }
    int Wl[PTT_MAX_DIM], Wr[PTT_MAX_DIM], Pcap = 1;
    for (int i = 0; i < d; i++) {
        const long long ml = (long long)rk[i] * x->n[i], mr = (long long)x->n[i] * rk[i + 1];
        Wl[i] = (int)((ml + 31) / 32);
        Wr[i] = (int)((mr + 31) / 32);
        const int pw = pow2_ge(Wl[i] > Wr[i] ? Wl[i] : Wr[i]);
        if (pw > Pcap) Pcap = pw;
    }
    Plan base;
    plan_bond(32, 1, 32, &base);
    base.NH = 1;
    long long o = carve(&base, 1, 1);
    WP wp;
    wp.o_R = o;
    o += (2LL * Pcap - 1) * SLOT;
    wp.o_tl = o;
    o += (long long)Pcap * 32;
    wp.o_tn = o;
    o += (long long)Pcap * 32;
    // Cholesky-QR record
    const int use_cq = c->no_cholqr ? 0 : 1;
    wp.o_cq = o;
    o += cq::REGION;
    wp.stride = (o + 31) / 32 * 32;
    wp.Pcap = Pcap;
    base.o_Rn = wp.o_R;  // root R = slot 0 (read by the SVD and the R product)
    if ((rc = ptt_ws_reserve(c, (size_t)wp.stride * d * sizeof(double) + 256))) return rc;
    if ((rc = ptt_counters_reserve(c, (size_t)Pcap * d + 64))) return rc;
    double* ws = (double*)c->ws;
    wp.cnt = c->d_counters;
    base.cnt = c->d_counters;
    int* fin_ticket = c->d_counters + (long long)Pcap * d;  // past the bonds' tree counters
    base.qn = nullptr;
    base.pass = nullptr;
    base.stats = c->d_stats;
    base.work = (c->tkind == PTT_TIME_TSQR) ? c->d_work + PTT_TIME_TSQR : nullptr;
    auto bond = [&](int i, double** wsb) {
        Plan pl = base;
        *wsb = ws + (long long)i * wp.stride;
        pl.info = (Info*)(*wsb + base.o_info_d);
        return pl;
    };
    // column bound of the unrolled Householder loops: the bond's rank bound
    auto cbound = [](int cols) { return cols <= 16 ? 16 : (cols <= 24 ? 24 : 32); };
    auto factor = [&](int i, int mode, int W, const Plan& pl, double* wsb) -> int {
        const int cb = cbound(mode == LEFT ? rk[i + 1] : rk[i]);
        const dim3 g((W + FPB - 1) / FPB), b(32 * FPB);
        const size_t sm = wfactor_smem();
        ptt_time_begin(c, PTT_TIME_TSQR);
        if (use_cq) {
            // Cholesky QR by one cluster; the TSQR below only runs for a bond
            // it did not finish
            const int mp = W * 32;  // bound on the unfolding's rows
            int cs = 1;
            if (c->cq_cs_force) {
                cs = c->cq_cs_force;
            } else if (c->cq_tuned && c->cq_cs[cb == 16 ? 0 : (cb == 24 ? 1 : 2)][cq_bucket(mp)]) {
                cs = c->cq_cs[cb == 16 ? 0 : (cb == 24 ? 1 : 2)][cq_bucket(mp)];
            } else {  // row-count rule: about RTARGET rows per CTA
                while (cs < g_cq_csmax[dev] && (long long)cs * cq::RTARGET < mp) cs <<= 1;
            }
            if (cs > g_cq_csmax[dev]) cs = g_cq_csmax[dev];
            const int rmax = cb == 16 ? cq::rpb_max<16>() : (cb == 24 ? cq::rpb_max<24>() : cq::rpb_max<32>());
            while (cs < g_cq_csmax[dev] && (mp + cs - 1) / cs > rmax) cs <<= 1;  // fit the rows
            int rpb = (mp + cs - 1) / cs;
            if (rpb > rmax) {  // too tall for the cluster's shared memory: falls back at once
                cs = 1;
                rpb = 1;
            }
            cudaLaunchConfig_t lc = {};
            lc.gridDim = dim3(cs);
            lc.blockDim = dim3(cq::NT);
            lc.dynamicSmemBytes = cb == 16 ? cq::smem<16>(rpb) : (cb == 24 ? cq::smem<24>(rpb) : cq::smem<32>(rpb));
            lc.stream = c->stream;
            cudaLaunchAttribute la[2];
            la[0].id = cudaLaunchAttributeClusterDimension;
            la[0].val.clusterDim.x = cs;
            la[0].val.clusterDim.y = 1;
            la[0].val.clusterDim.z = 1;
            la[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            la[1].val.programmaticStreamSerializationAllowed = 1;
            lc.attrs = la;
            lc.numAttrs = (c->no_pdl || c->capturing) ? 1 : 2;
            const DevDesc* dd = x->dd;
            if (cb == 16)
                PTT_CUDA(cudaLaunchKernelEx(&lc, cq::k_cq_factor<16>, dd, i, mode, pl, wp, wsb, rpb, c->d_qrstat));
            else if (cb == 24)
                PTT_CUDA(cudaLaunchKernelEx(&lc, cq::k_cq_factor<24>, dd, i, mode, pl, wp, wsb, rpb, c->d_qrstat));
            else
                PTT_CUDA(cudaLaunchKernelEx(&lc, cq::k_cq_factor<32>, dd, i, mode, pl, wp, wsb, rpb, c->d_qrstat));
            PTT_LAUNCHED(c);
        }
        if (cb == 16)
            PTT_CUDA(ptt_launch(c, k_wfactor<16>, dim3(g), dim3(b), sm, x->dd, i, mode, pl, wp, wsb, use_cq, c->d_status));
        else if (cb == 24)
            PTT_CUDA(ptt_launch(c, k_wfactor<24>, dim3(g), dim3(b), sm, x->dd, i, mode, pl, wp, wsb, use_cq, c->d_status));
        else
            PTT_CUDA(ptt_launch(c, k_wfactor<32>, dim3(g), dim3(b), sm, x->dd, i, mode, pl, wp, wsb, use_cq, c->d_status));
        ptt_time_end(c, PTT_TIME_TSQR);
        PTT_LAUNCHED(c);
        return PTT_OK;
    };
    auto apply = [&](int k0, int nb, int mode, int Wmax, int cmax, Fin fin = Fin{}) -> int {
        const int cb = cbound(cmax);
        const dim3 g((Wmax + WPB - 1) / WPB, nb), b(32 * WPB);
        if (cb == 16)
            PTT_CUDA(ptt_launch(c, k_wapply<16>, dim3(g), dim3(b), 0, x->dd, k0, mode, base, wp, ws, use_cq, fin));
        else if (cb == 24)
            PTT_CUDA(ptt_launch(c, k_wapply<24>, dim3(g), dim3(b), 0, x->dd, k0, mode, base, wp, ws, use_cq, fin));
        else
            PTT_CUDA(ptt_launch(c, k_wapply<32>, dim3(g), dim3(b), 0, x->dd, k0, mode, base, wp, ws, use_cq, fin));
        PTT_LAUNCHED(c);
        if (use_cq && mode == RIGHT_T) {  // LEFT: the cluster wrote Q already
            long long gx = ((long long)Wmax * 32 + cq::NT - 1) / cq::NT;
            gx = gx < 1 ? 1 : (gx > 4096 ? 4096 : gx);
            const dim3 gw((unsigned)gx, nb);
            if (cb == 16)
                PTT_CUDA(ptt_launch(c, cq::k_cq_write<16>, dim3(gw), dim3(cq::NT), 0, x->dd, k0, base, wp, ws));
            else if (cb == 24)
                PTT_CUDA(ptt_launch(c, cq::k_cq_write<24>, dim3(gw), dim3(cq::NT), 0, x->dd, k0, base, wp, ws));
            else
                PTT_CUDA(ptt_launch(c, cq::k_cq_write<32>, dim3(gw), dim3(cq::NT), 0, x->dd, k0, base, wp, ws));
            PTT_LAUNCHED(c);
        }
        return PTT_OK;
    };
    // the launches below, as one unit that can be captured and replayed;
    // the key holds every value they bake in
    struct Key {
        int tag, d, phases, only, use_cq, tuned;
        const void *dd, *ws, *cnt, *status, *stats;
        long long stride;
        int Pcap;
        double delta;
        int n[PTT_MAX_DIM], rk[PTT_MAX_DIM + 1], mr[PTT_MAX_DIM + 1];
    } key;
    memset(&key, 0, sizeof(key));
    key.tag = 1;
    key.d = d;
    key.phases = phases;
    key.only = only;
    key.use_cq = use_cq;
    key.tuned = c->cq_tuned;
    key.dd = x->dd;
    key.ws = ws;
    key.cnt = c->d_counters;
    key.status = c->d_status;
    key.stats = c->d_stats;
    key.stride = wp.stride;
    key.Pcap = wp.Pcap;
    key.delta = delta;
    for (int i = 0; i < d; i++) key.n[i] = x->n[i];
    for (int i = 0; i <= d; i++) {
        key.rk[i] = rk[i];
        key.mr[i] = maxr ? maxr[i] : -1;
    }
    auto issue = [&]() -> int {
        if (phases & 4) {
            const int i = only;
            double* wsb;
            Plan pl = bond(i, &wsb);
            if ((rc = factor(i, LEFT, Wl[i], pl, wsb))) return rc;
            // the apply's last block publishes the rank and swaps the core
            if ((rc = apply(i, 1, LEFT, Wl[i], rk[i + 1], Fin{fin_ticket, i + 1, i, &pl.info->q}))) return rc;
            return PTT_OK;
        }
        if (phases & 1) {
            int Wmax = 1, cmax = 1;
            for (int i = 0; i < d - 1; i++) {
                cmax = rk[i + 1] > cmax ? rk[i + 1] : cmax;
                double* wsb;
                Plan pl = bond(i, &wsb);
                if ((rc = factor(i, LEFT, Wl[i], pl, wsb))) return rc;
                Wmax = Wl[i] > Wmax ? Wl[i] : Wmax;
                const long long ncap = (long long)x->n[i + 1] * rk[i + 2];
                int gy = (int)((ncap + GT - 1) / GT);
                if (gy > 4096) gy = 4096;
                // the contraction's last block publishes the rank and swaps the core
                PTT_CUDA(ptt_launch(c, k_gemm_rx, dim3(dim3(1, gy)), dim3(256), 0, x->dd, i + 1, pl, wsb,
                                    Fin{fin_ticket, i + 1, i + 1, &pl.info->q}));
                PTT_LAUNCHED(c);
            }
            if (d > 1) {
                if ((rc = apply(0, d - 1, LEFT, Wmax, cmax))) return rc;
                PTT_CUDA(ptt_launch(c, k_wswap, dim3(1), dim3(64), 0, x->dd, 0, d - 1, c->d_status));
                PTT_LAUNCHED(c);
            }
        }
        if (phases & 2) {
            int Wmax = 1, cmax = 1;
            for (int i = d - 1; i >= 1; i--) {
                cmax = rk[i] > cmax ? rk[i] : cmax;
                double* wsb;
                Plan pl = bond(i, &wsb);
                if ((rc = factor(i, RIGHT_T, Wr[i], pl, wsb))) return rc;
                Wmax = Wr[i] > Wmax ? Wr[i] : Wmax;
                const int mr = maxr ? maxr[i] : rk[i];
                ptt_time_begin(c, PTT_TIME_SVD);
                PTT_CUDA(ptt_launch(c, k_svd_jacobi<32>, dim3(1), dim3(svd_nt<32>()), svd_smem<32>(), pl, wsb, delta, mr, i,
                                    c->d_status));
                ptt_time_end(c, PTT_TIME_SVD);
                PTT_LAUNCHED(c);
                const long long mcap = (long long)rk[i - 1] * x->n[i - 1];
                int gx = (int)((mcap + GT - 1) / GT);
                if (gx > 4096) gx = 4096;
                PTT_CUDA(ptt_launch(c, k_gemm_xm, dim3(dim3(gx, 1)), dim3(256), 0, x->dd, i - 1, pl, wsb,
                                    Fin{fin_ticket, i, i - 1, &pl.info->rank}));
                PTT_LAUNCHED(c);
            }
            if (d > 1) {
                PTT_CUDA(ptt_launch(c, k_svd_replay_b, dim3(dim3(4, d - 1)), dim3(256), replay_smem<32>(), base, ws, wp.stride, 1));
                PTT_LAUNCHED(c);
                if ((rc = apply(1, d - 1, RIGHT_T, Wmax, cmax))) return rc;
                PTT_CUDA(ptt_launch(c, k_wswap, dim3(1), dim3(64), 0, x->dd, 1, d, c->d_status));
                PTT_LAUNCHED(c);
            }
        }
        return PTT_OK;
    };
    return ptt_graph_run(c, &key, sizeof(key), issue);
}

}  // namespace

// Per-bond threshold of the reference applied to the unnormalised tensor.
double ptt_round_threshold(const ptt_tt* x, double tol) {
    const int d = x->d;
    if (d < 2) return INFINITY;
    double lg = 0.0;
    for (int k = 0; k < d; k++) lg += log((double)x->n[k]);
    return tol / sqrt(d - 1.0) * exp(0.5 * lg);
}

extern "C" int ptt_round_stats(ptt_ctx* c, int d, double* out) {
    if (!c || !out || d < 1 || d > PTT_MAX_DIM) return ptt_set_error(PTT_ERR_ARG, "ptt_round_stats: bad arguments");
    PTT_CUDA(cudaStreamSynchronize(c->stream));
    PTT_CUDA(cudaMemcpy(out, c->d_stats, sizeof(double) * PTT_STAT_LEN * (size_t)d, cudaMemcpyDeviceToHost));
    return PTT_OK;
}

int ptt_round_phases(ptt_tt* x, double tol, const int* maxrank, int phases, int only) {
    if (!x) return ptt_set_error(PTT_ERR_ARG, "ptt_round: null tt");
    if (x->d < 2) return PTT_OK;
    int rk[PTT_MAX_DIM + 1];
    cudaSetDevice(x->ctx->device);
    if (x->ctx->fixed_plans) {
        // capacity-sized plan: no host synchronisation (stream capture)
        for (int k = 0; k <= x->d; k++) rk[k] = x->rcap[k];
    } else {
        // plan from the actual ranks (one read-back): tiles, trees and grids
        // then match the tensor instead of its capacity
        int rc = ptt_tt_get_ranks(x, rk);
        if (rc) return rc;
    }
    return ptt_round_phases_rk(x, rk, tol, maxrank, phases, only);
}

// The same with upper bounds rk[0..d] of the ranks known to the caller (no
// read-back).
int ptt_round_phases_rk(ptt_tt* x, const int* rk, double tol, const int* maxrank, int phases, int only) {
    if (!x) return ptt_set_error(PTT_ERR_ARG, "ptt_round: null tt");
    if (x->d < 2) return PTT_OK;
    if (!(tol >= 0.0)) return ptt_set_error(PTT_ERR_ARG, "ptt_round: tol must be >= 0");
    cudaSetDevice(x->ctx->device);
    int rmax = 1;
    for (int k = 0; k <= x->d; k++) rmax = rk[k] > rmax ? rk[k] : rmax;
    const double delta = ptt_round_threshold(x, tol);
    if (rmax <= 32 && wt_fits(x, rk)) return round_impl_w(x, rk, delta, maxrank, phases, only);
    if (rmax <= 32) return round_impl<32>(x, rk, delta, maxrank, phases, only);
    if (rmax <= 64) return round_impl<64>(x, rk, delta, maxrank, phases, only);
    if (rmax <= 128) return round_impl<128>(x, rk, delta, maxrank, phases, only);
    return ptt_set_error(PTT_ERR_CAPACITY, "ptt_round: rank %d > 128 not supported", rmax);
}

extern "C" int ptt_ctx_fixed_plans(ptt_ctx* c, int on) {
    if (!c) return ptt_set_error(PTT_ERR_ARG, "null context");
    c->fixed_plans = on ? 1 : 0;
    return PTT_OK;
}

extern "C" int ptt_round(ptt_tt* x, double tol, const int* maxrank) {
    return ptt_round_phases(x, tol, maxrank, 3, 0);
}

extern "C" int ptt_ctx_ozaki(ptt_ctx* c, int on) {
    if (!c) return ptt_set_error(PTT_ERR_ARG, "null context");
    c->ozaki = on ? 1 : 0;
    for (int l = 0; l < c->nlanes; l++)
        if (c->lanes[l]) c->lanes[l]->ozaki = c->ozaki;
    return PTT_OK;
}

// G = A^T A of a device m x c column-major matrix (c <= 64): method 0 on the
// FP64 tensor cores, 1 by the Ozaki split on the fifth-generation tensor
// cores (the two Gram kernels of the grid Cholesky QR, ptt_gridqr.cuh and
// ptt_ozaki.cuh).
extern "C" int ptt_gram(ptt_ctx* c, const double* A, long long m, int cols, long long lda, double* G, int method) {
    if (!c || !A || !G || m < 1 || cols < 1 || cols > gq::CB || lda < m || (method != 0 && method != 1))
        return ptt_set_error(PTT_ERR_ARG, "ptt_gram: bad arguments");
    const long long nbl = (m + gq::RPB_MAX - 1) / gq::RPB_MAX;
    if (nbl > (1ll << 24)) return ptt_set_error(PTT_ERR_CAPACITY, "ptt_gram: %lld rows", m);
    cudaSetDevice(c->device);
    int rc;
    const int nb = (int)nbl, ng = (nb + gq::GROUP - 1) / gq::GROUP;
    if ((rc = ptt_ws_reserve(c, sizeof(double) * (size_t)(nb + ng) * gq::UP + 256))) return rc;
    if ((rc = ptt_counters_reserve(c, (size_t)ng + 1))) return rc;
    double* part = (double*)c->ws;
    double* gpart = part + (long long)nb * gq::UP;
    if (method == 1) {
        PTT_CUDA(cudaFuncSetAttribute(gq::k_gram<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)gq::SMEM_OZ));
        gq::k_gram<true><<<nb, gq::NT, gq::SMEM_OZ, c->stream>>>(A, m, cols, lda, part, gpart, c->d_counters, G);
    } else {
        PTT_CUDA(cudaFuncSetAttribute(gq::k_gram<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(sizeof(double) * gq::RPB_MAX * gq::XP)));
        gq::k_gram<false><<<nb, gq::NT, sizeof(double) * gq::RPB_MAX * gq::XP, c->stream>>>(A, m, cols, lda, part,
                                                                                          gpart, c->d_counters, G);
    }
    PTT_LAUNCHED(c);
    return PTT_OK;
}

// ---------------------------------------------------------------------------
// autotuner of the Cholesky-QR cluster size
// ---------------------------------------------------------------------------
namespace {
__global__ void k_tune_fill(double* p, long long cnt, unsigned long long seed) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cnt;
         e += (long long)gridDim.x * blockDim.x) {
        unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(e + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        p[e] = (double)(z >> 11) * 1.1102230246251565e-16 - 0.5;  // uniform in [-0.5, 0.5)
    }
}
}  // namespace

// For each column bound (16, 24, 32) and rows bucket (512 ... 16384), time the
// QR of one core (the single-core phase of a rounding, the path the sketch
// uses per core) of a random m x c unfolding with every cluster size the
// device can hold, and keep the fastest in the context's table.
extern "C" int ptt_ctx_autotune(ptt_ctx* c) {
    if (!c) return ptt_set_error(PTT_ERR_ARG, "null context");
    cudaSetDevice(c->device);
    const int graphs = c->graphs, tkind = c->tkind;
    c->graphs = 0;
    c->tkind = 0;
    int rc = PTT_OK;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ptt_tt *x = nullptr, *x0 = nullptr;
    PTT_CUDA(cudaEventCreate(&e0));
    PTT_CUDA(cudaEventCreate(&e1));
    static const int cbs[3] = {16, 24, 32};
    for (int ci = 0; ci < 3 && !rc; ci++) {
        for (int bi = 0; bi < 6 && !rc; bi++) {
            const int cb = cbs[ci], m = 512 << bi;
            int n[2] = {m, 1}, cap[3] = {1, cb, 1}, rk[3] = {1, cb, 1};
            x = ptt_tt_create(c, 2, n, cap);
            x0 = ptt_tt_create(c, 2, n, cap);
            if (!x || !x0) {
                rc = ptt_last_error() ? ptt_last_error() : PTT_ERR_CUDA;
                break;
            }
            if ((rc = ptt_pull_desc(x0))) break;
            k_tune_fill<<<148, 256, 0, c->stream>>>(x0->hd.core[0], (long long)m * cb, 1234567ull + 977ull * bi + ci);
            k_tune_fill<<<1, 32, 0, c->stream>>>(x0->hd.core[1], cb, 7654321ull + ci);
            if ((rc = ptt_cuda_check(cudaGetLastError(), "tune fill"))) break;
            float best = 1e30f, theur = 1e30f;
            int bestcs = 1;
            // the size the row-count heuristic would take
            int hcs = 1;
            {
                const int dev = c->device & 63;
                const int csmax = g_cq_csmax[dev] ? g_cq_csmax[dev] : cq::CSMAX;
                while (hcs < csmax && (long long)hcs * cq::RTARGET < m) hcs <<= 1;
            }
            for (int cs = 1; cs <= cq::CSMAX && !rc; cs <<= 1) {
                int dev = c->device & 63;
                if (g_cq_csmax[dev] && cs > g_cq_csmax[dev]) break;
                const int rmax = cb == 16 ? cq::rpb_max<16>() : (cb == 24 ? cq::rpb_max<24>() : cq::rpb_max<32>());
                if ((m + cs - 1) / cs > rmax) continue;
                c->cq_cs_force = cs;
                float tmin = 1e30f;
                for (int rep = 0; rep < 7 && !rc; rep++) {
                    if ((rc = ptt_tt_copy(x, x0))) break;
                    if ((rc = ptt_ctx_synchronize(c))) break;
                    PTT_CUDA(cudaEventRecord(e0, c->stream));
                    if ((rc = ptt_round_phases_rk(x, rk, 0.0, NULL, 4, 0))) break;
                    PTT_CUDA(cudaEventRecord(e1, c->stream));
                    PTT_CUDA(cudaEventSynchronize(e1));
                    float ms = 0.f;
                    PTT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                    if (rep > 0 && ms < tmin) tmin = ms;  // rep 0 warms up
                }
                if (tmin < best) {
                    best = tmin;
                    bestcs = cs;
                }
                if (cs == hcs) theur = tmin;
            }
            // a single timed QR is noisy: leave the heuristic's size unless
            // another one is clearly faster
            if (theur < 1e30f && !(best < 0.85f * theur)) bestcs = 0;  // 0: keep the row-count rule
            c->cq_cs[ci][bi] = (unsigned char)bestcs;
            ptt_tt_destroy(x);
            ptt_tt_destroy(x0);
            x = x0 = nullptr;
        }
    }
    if (x) ptt_tt_destroy(x);
    if (x0) ptt_tt_destroy(x0);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->cq_cs_force = 0;
    c->graphs = graphs;
    c->tkind = tkind;
    if (rc) return rc;
    c->cq_tuned++;
    if ((rc = ptt_gemm_autotune(c))) return rc;
    return ptt_ctx_synchronize(c);
}

extern "C" int ptt_ctx_autotune_table(const ptt_ctx* c, int* out) {
    if (!c || !out) return ptt_set_error(PTT_ERR_ARG, "ptt_ctx_autotune_table: bad arguments");
    for (int i = 0; i < 18; i++) out[i] = c->cq_tuned ? c->cq_cs[i / 6][i % 6] : 0;
    return PTT_OK;
}
