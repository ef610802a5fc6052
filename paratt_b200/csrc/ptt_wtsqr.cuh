// Warp-level TSQR for unfoldings with at most 32 columns (included by
// ptt_round.cu inside its anonymous namespace, after the block-level kernels).
//
// One warp owns one 32-row leaf of the m x c unfolding; lane l owns column l
// of the leaf tile, held in registers.  A Householder step then needs no
// barrier: the pivot lane's column norm and vector are broadcast with
// shuffles and every lane updates its own column.  The reflector loops are
// unrolled over the 32 rows, so every register index is a compile-time
// constant.
//
// Tree: leaves p = 0..W-1 (W = ceil(m / 32)) sit at heap slots P-1+p,
// P = next_pow2(W).  A node whose right subtree holds no leaf passes the left
// child's R up unchanged.  Otherwise the warp that arrives second (atomic
// ticket, nobody waits) combines [R_left; R_right] -- always left on top, so
// the result does not depend on which warp arrived first -- with Householder
// steps on the two triangles; the vectors replace R_right in its slot.  The
// last leaf may be short (h < 32 rows); it is never the upper triangle of a
// combination, and with m < c the single leaf gives a q = m row trapezoid.
//
// Pivot rows are always real rows of the unfolding (as in LAPACK), so Q has
// orthonormal columns also for rank-deficient unfoldings.
//
// Q is not formed while sweeping: k_wapply forms Q*B for all bonds of a sweep
// in one launch.  Each warp walks from the root to its leaf applying the node
// reflectors to B (c x qB, one column per lane), then its leaf's reflectors,
// and writes its 32 rows of Q*B.
#pragma once

namespace wt {

constexpr int WPB = 4;  // warps per block
constexpr unsigned FULL = 0xffffffffu;
constexpr int SLOT = 32 * 32;
constexpr int PMAX = 4096;  // leaves per bond (m <= 131072)
constexpr int CQ_DONE = 1;  // Cholesky-QR state: the bond is factored, skip it here

// Per-bond tree records.  Bond (core) k's region starts at ws + k * stride;
// offsets are in doubles within a region; counters of bond k at cnt + k * Pcap.
struct WP {
    long long o_R;   // (2 Pcap - 1) slots, R or vectors, row-major 32 x 32
    long long o_tl;  // leaf taus, Pcap x 32
    long long o_tn;  // node taus, Pcap x 32
    long long o_cq;  // Cholesky-QR record (ptt_cholqr.cuh); its first int is the bond's state
    long long stride;
    int Pcap;
    int* cnt;        // zero between launches; reset by the combining warp
};

__host__ __device__ __forceinline__ int pow2_ge(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// Rows [r0, r0 + h) x columns [0, c) of the view into X (lane = column),
// zero elsewhere.  Column-major views are read along rows and transposed
// through the warp's shared tile so every load is coalesced.
__device__ __forceinline__ void w_load(const double* p, long long rs, long long cs, int r0, int h, int c,
                                       double (&X)[32], double* sh) {
    const int lane = threadIdx.x & 31;
    if (rs == 1) {
        // lane = row: all column loads in flight at once, then transpose
#pragma unroll
        for (int l = 0; l < 32; l++) X[l] = (l < c && lane < h) ? p[(long long)(r0 + lane) + (long long)l * cs] : 0.0;
#pragma unroll
        for (int l = 0; l < 32; l++) sh[lane * 33 + l] = X[l];
        __syncwarp();
#pragma unroll
        for (int t = 0; t < 32; t++) X[t] = lane < c ? sh[t * 33 + lane] : 0.0;
        __syncwarp();
    } else {
#pragma unroll
        for (int t = 0; t < 32; t++)
            X[t] = (t < h && lane < c) ? p[(long long)(r0 + t) * rs + (long long)lane * cs] : 0.0;
    }
}

// Rows [r0, r0 + h) x columns [0, nc) of X (lane = column) into the view.
__device__ __forceinline__ void w_store(double* p, long long rs, long long cs, int r0, int h, int nc,
                                        const double (&X)[32], double* sh) {
    const int lane = threadIdx.x & 31;
    if (rs == 1) {
#pragma unroll
        for (int t = 0; t < 32; t++) sh[t * 33 + lane] = X[t];
        __syncwarp();
        if (lane < h)
#pragma unroll 8
            for (int l = 0; l < nc; l++) p[(long long)(r0 + lane) + (long long)l * cs] = sh[lane * 33 + l];
        __syncwarp();
    } else {
        if (lane < nc)
#pragma unroll
            for (int t = 0; t < 32; t++)
                if (t < h) p[(long long)(r0 + t) * rs + (long long)lane * cs] = X[t];
    }
}

// Householder QR of the h x c tile X (lane = column, rows >= h are zero).
// On exit rows t <= lane of X hold R and rows t > lane the vector of
// reflector `lane` (unit diagonal implied); returns that reflector's tau.
// Each step forms the dot products with the unscaled pivot column x (v = [1;
// sc x]), so they run while the reflector's scalars are computed:
//   w = tau (X_j + sc x.X),  X_j -= w,  X_t -= (w sc) x_t.
template <int CB>
__device__ __forceinline__ double w_geqrt(double (&X)[32], int c, int h) {
    const int lane = threadIdx.x & 31;
    const int nr = c < h ? c : h;
    double mytau = 0.0;
#pragma unroll
    for (int j = 0; j < CB; j++) {
        if (j >= nr) continue;
        double s[4] = {0.0, 0.0, 0.0, 0.0}, dd[4] = {0.0, 0.0, 0.0, 0.0};
        double xr[32];
#pragma unroll
        for (int t = j + 1; t < 32; t++) {
            xr[t] = __shfl_sync(FULL, X[t], j);
            s[t & 3] = fma(X[t], X[t], s[t & 3]);
            dd[t & 3] = fma(xr[t], X[t], dd[t & 3]);
        }
        const double alpha = __shfl_sync(FULL, X[j], j);
        const double s2 = __shfl_sync(FULL, (s[0] + s[1]) + (s[2] + s[3]), j);
        double beta, tau, sc;
        hh_params(alpha, s2, &beta, &tau, &sc);
        const double w = tau * fma(sc, (dd[0] + dd[1]) + (dd[2] + dd[3]), X[j]);
        if (lane > j) {
            const double ws = w * sc;
            X[j] -= w;
#pragma unroll
            for (int t = j + 1; t < 32; t++) X[t] = fma(-ws, xr[t], X[t]);
        } else if (lane == j) {
            X[j] = beta;
#pragma unroll
            for (int t = j + 1; t < 32; t++) X[t] = sc * xr[t];
            mytau = tau;
        }
    }
    return mytau;
}

// [T; B] with T, B upper triangular (lane = column): eliminate B into T.
// On exit T is the R of the pair and rows t <= lane of B hold the vector of
// reflector `lane` (its top part is e_lane); returns that reflector's tau.
// Same step structure as w_geqrt.
template <int CB>
__device__ __forceinline__ double w_ttqrt(double (&T)[32], double (&B)[32], int c) {
    const int lane = threadIdx.x & 31;
    double mytau = 0.0;
#pragma unroll
    for (int j = 0; j < CB; j++) {
        if (j >= c) continue;
        double s[4] = {0.0, 0.0, 0.0, 0.0}, dd[4] = {0.0, 0.0, 0.0, 0.0};
        double xr[32];
#pragma unroll
        for (int t = 0; t <= j; t++) {
            xr[t] = __shfl_sync(FULL, B[t], j);
            s[t & 3] = fma(B[t], B[t], s[t & 3]);
            dd[t & 3] = fma(xr[t], B[t], dd[t & 3]);
        }
        const double alpha = __shfl_sync(FULL, T[j], j);
        const double s2 = __shfl_sync(FULL, (s[0] + s[1]) + (s[2] + s[3]), j);
        double beta, tau, sc;
        hh_params(alpha, s2, &beta, &tau, &sc);
        const double w = tau * fma(sc, (dd[0] + dd[1]) + (dd[2] + dd[3]), T[j]);
        if (lane > j) {
            const double ws = w * sc;
            T[j] -= w;
#pragma unroll
            for (int t = 0; t <= j; t++) B[t] = fma(-ws, xr[t], B[t]);
        } else if (lane == j) {
            T[j] = beta;
#pragma unroll
            for (int t = 0; t <= j; t++) B[t] = sc * xr[t];
            mytau = tau;
        }
    }
    return mytau;
}

// Factor the unfolding (mode) of core k: leaf reflectors in place, taus and
// tree records in the bond's region wsb, R at slot 0, Info (m, c, q).
// A block holds FPB leaves; the lowest LB = log2(FPB) tree levels are
// combined inside the block through shared memory, the levels above by the
// warp 0 of each block through the global slots (last arriver combines).
constexpr int FLB = 3;         // tree levels combined inside a block
constexpr int FPB = 1 << FLB;  // warps (leaves) per factor block

__host__ __device__ constexpr size_t wfactor_smem() { return sizeof(double) * FPB * 32 * 33; }

template <int CB>
__global__ void __launch_bounds__(32 * FPB) k_wfactor(const DevDesc* D, int k, int mode, Plan pl, WP wp,
                                                      double* wsb, int use_cq, int* status) {
    PTT_PDL_ENTRY();
    extern __shared__ double fsm[];
    // a bond the Cholesky sequence finished needs no Householder factors
    if (use_cq && *(const int*)(wsb + wp.o_cq) == CQ_DONE) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int p = blockIdx.x * FPB + wid;
    const View A = make_view(D, k, mode, false);
    const int m = A.m, c = A.c;
    Info* info = (Info*)(wsb + pl.o_info_d);
    const int W = (m + 31) >> 5;
    const int P = pow2_ge(W);
    if (c > CB || c < 1 || m < 1 || P > wp.Pcap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            info->status = PTT_ERR_CAPACITY;
            PTT_STATUS_SET(status, PTT_ERR_CAPACITY);
        }
        return;  // uniform over the block
    }
    if (blockIdx.x * FPB >= W) return;  // uniform over the block
    if (pl.work && !use_cq && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(pl.work, 16.0 * (double)m * (double)c);
    double* sw = fsm + wid * (32 * 33);
    const bool valid = p < W;
    const int r0 = p * 32;
    const int h = valid ? ((m - r0) < 32 ? (m - r0) : 32) : 0;
    double* Rs = wsb + wp.o_R;
    double X[32];
    if (valid) {
        w_load(A.p, A.rs, A.cs, r0, h, c, X, sw);
        const double tl = w_geqrt<CB>(X, c, h);
        w_store(A.p, A.rs, A.cs, r0, h, c, X, sw);
        wsb[wp.o_tl + p * 32 + lane] = tl;
#pragma unroll
        for (int t = 0; t < 32; t++)
            if (t > lane) X[t] = 0.0;
    }
    // in-block levels: the left child's warp combines with its right sibling
    int lb = 0;
    while ((1 << lb) < P && lb < FLB) lb++;
    for (int lvl = 0; lvl < lb; lvl++) {
        const int span = 1 << lvl;
        const int mask = (2 << lvl) - 1;
        __syncthreads();
        if (valid && (wid & mask) == span) {
#pragma unroll
            for (int t = 0; t < 32; t++) sw[t * 32 + lane] = X[t];
        }
        __syncthreads();
        if (valid && (wid & mask) == 0 && p + span < W) {
            const double* Rr = fsm + (wid + span) * (32 * 33);
            double B[32];
#pragma unroll
            for (int t = 0; t < 32; t++) B[t] = t < CB ? Rr[t * 32 + lane] : 0.0;
            const double tn = w_ttqrt<CB>(X, B, c);
            const int node = ((P + p) >> (lvl + 1)) - 1;
            double* Vo = Rs + (long long)(2 * node + 2) * SLOT;
#pragma unroll
            for (int t = 0; t < CB; t++) Vo[t * 32 + lane] = B[t];
            wsb[wp.o_tn + node * 32 + lane] = tn;
        }
    }
    if (wid != 0) return;
    // global levels
    int* cnt = wp.cnt + (long long)k * wp.Pcap;
    int slot = ((P + p) >> lb) - 1, lvl = lb;
    while (slot > 0) {
        const int node = (slot - 1) >> 1;
        const int span = 1 << lvl;
        const int base = (p >> (lvl + 1)) << (lvl + 1);
        if (base + span >= W) {  // empty right subtree: pass R up
            slot = node;
            lvl++;
            continue;
        }
        double* Ro = Rs + (long long)slot * SLOT;
#pragma unroll
        for (int t = 0; t < CB; t++) Ro[t * 32 + lane] = X[t];
        __threadfence();
        int old = 0;
        if (lane == 0) old = atomicAdd(cnt + node, 1);
        old = __shfl_sync(FULL, old, 0);
        if (old == 0) return;  // the sibling's warp combines
        __threadfence();
        if (lane == 0) cnt[node] = 0;
        const double* Rl = Rs + (long long)(2 * node + 1) * SLOT;
        double* Rr = Rs + (long long)(2 * node + 2) * SLOT;
        double B[32];
#pragma unroll
        for (int t = 0; t < 32; t++) {
            X[t] = t < CB ? __ldcg(Rl + t * 32 + lane) : 0.0;
            B[t] = t < CB ? __ldcg(Rr + t * 32 + lane) : 0.0;
        }
        const double tn = w_ttqrt<CB>(X, B, c);
#pragma unroll
        for (int t = 0; t < CB; t++) Rr[t * 32 + lane] = B[t];
        wsb[wp.o_tn + node * 32 + lane] = tn;
        slot = node;
        lvl++;
    }
#pragma unroll
    for (int t = 0; t < 32; t++) Rs[t * 32 + lane] = t < CB ? X[t] : 0.0;
    if (lane == 0) {
        info->m = m;
        info->c = c;
        info->q = m < c ? m : c;
        info->rank = 0;
        info->status = 0;
    }
}

// out = Q * B for bonds (cores) k = k0 .. k0 + gridDim.y - 1 of one sweep,
// with the sizes recorded by k_wfactor (the descriptor's ranks have moved on).
//   LEFT:    B = I_q;                       out (m x q, column-major) -> alt[k]
//   RIGHT_T: B = V_r (Bn, row-major 32 x KC); out(row, col) -> alt[k][row * rank + col]
template <int CB>
__device__ __forceinline__ void wapply_body(const DevDesc* D, int k0, int mode, const Plan& pl, const WP& wp,
                                            double* ws, int use_cq) {
    __shared__ double sh[WPB][32 * 33];
    __shared__ double stau[WPB][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int k = k0 + blockIdx.y;
    double* wsb = ws + (long long)k * wp.stride;
    if (use_cq && *(const int*)(wsb + wp.o_cq) == CQ_DONE) return;  // k_cq_write forms this Q
    const Info* info = (const Info*)(wsb + pl.o_info_d);
    if (info->status) return;
    const int m = info->m, c = info->c, q = info->q;
    const int qB = (mode == LEFT) ? q : info->rank;
    const int W = (m + 31) >> 5, P = pow2_ge(W);
    const int p = blockIdx.x * WPB + wid;
    if (p >= W || c > CB) return;  // c <= CB: the factorisation used the same bound
    double* sw = sh[wid];
    volatile double* vs = sw;  // re-read in the updates instead of holding 32 values
    double* st = stau[wid];
    const double* Rs = wsb + wp.o_R;
    double X[32];
    if (mode == LEFT) {
#pragma unroll
        for (int t = 0; t < 32; t++) X[t] = (t == lane && lane < q) ? 1.0 : 0.0;
    } else {
        const double* Bn = wsb + pl.o_Bn;
#pragma unroll
        for (int t = 0; t < 32; t++) X[t] = lane < qB ? Bn[(long long)t * pl.KC + lane] : 0.0;
    }
    // root to leaf
    int s = 0, base = 0;
    for (int half = P >> 1; half >= 1; half >>= 1) {
        if (base + half >= W) {  // pass-through node
            s = 2 * s + 1;
            continue;
        }
        const bool right = p >= base + half;
        const double* V = Rs + (long long)(2 * s + 2) * SLOT;  // vector j: rows t <= j of column j
#pragma unroll 4
        for (int t = 0; t < 32; t++) sw[t * 33 + lane] = V[t * 32 + lane];
        st[lane] = wsb[wp.o_tn + s * 32 + lane];
        __syncwarp();
        double Bt[32];
#pragma unroll
        for (int t = 0; t < 32; t++) Bt[t] = 0.0;
#pragma unroll
        for (int j = CB - 1; j >= 0; j--) {
            if (j >= c) continue;
            const double tau = st[j];
            double d0 = 0.0, d1 = 0.0;
#pragma unroll
            for (int t = 0; t <= j; t++) {
                if (t & 1)
                    d0 = fma(sw[t * 33 + j], Bt[t], d0);
                else
                    d1 = fma(sw[t * 33 + j], Bt[t], d1);
            }
            const double w = tau * (X[j] + (d0 + d1));
            X[j] -= w;
#pragma unroll
            for (int t = 0; t <= j; t++) Bt[t] = fma(-w, vs[t * 33 + j], Bt[t]);
        }
        __syncwarp();
        if (right) {
#pragma unroll
            for (int t = 0; t < 32; t++) X[t] = Bt[t];
            base += half;
            s = 2 * s + 2;
        } else {
            s = 2 * s + 1;
        }
    }
    // leaf: reflectors stored in place in core k
    const double* Ap = D->core[k];
    const long long ars = (mode == LEFT) ? 1 : c, acs = (mode == LEFT) ? m : 1;
    const int r0 = p * 32;
    const int h = (m - r0) < 32 ? (m - r0) : 32;
    if (mode == LEFT) {
#pragma unroll 8
        for (int j = 0; j < c; j++) sw[lane * 33 + j] = lane < h ? Ap[(long long)(r0 + lane) + (long long)j * acs] : 0.0;
    } else {
#pragma unroll 4
        for (int t = 0; t < 32; t++) sw[t * 33 + lane] = (t < h && lane < c) ? Ap[(long long)(r0 + t) * ars + lane] : 0.0;
    }
    st[lane] = wsb[wp.o_tl + p * 32 + lane];
    __syncwarp();
    const int nr = c < h ? c : h;
#pragma unroll
    for (int j = CB - 1; j >= 0; j--) {
        if (j >= nr) continue;
        const double tau = st[j];
        double d0 = 0.0, d1 = 0.0;
#pragma unroll
        for (int t = j + 1; t < 32; t++) {
            if ((t - j) & 1)
                d0 = fma(sw[t * 33 + j], X[t], d0);
            else
                d1 = fma(sw[t * 33 + j], X[t], d1);
        }
        const double w = tau * (X[j] + (d0 + d1));
        X[j] -= w;
#pragma unroll
        for (int t = j + 1; t < 32; t++) X[t] = fma(-w, vs[t * 33 + j], X[t]);
    }
    __syncwarp();
    double* out = D->alt[k];
    if (mode == LEFT)
        w_store(out, 1, m, r0, h, qB, X, sw);
    else
        w_store(out, qB, 1, r0, h, qB, X, sw);
}

// With a ticket (fin.ticket) the last block also publishes the bond's rank
// and swaps its core, as k_bond_finalize would after it (one bond, k0).
template <int CB>
__global__ void __launch_bounds__(32 * WPB) k_wapply(DevDesc* D, int k0, int mode, Plan pl, WP wp, double* ws,
                                                     int use_cq, Fin fin) {
    PTT_PDL_ENTRY();
    wapply_body<CB>(D, k0, mode, pl, wp, ws, use_cq);
    fin_last_block(D, fin, (const Info*)(ws + (long long)k0 * wp.stride + pl.o_info_d));
}

// swap core and alt of cores [k0, k1) unless an error was recorded
__global__ void k_wswap(DevDesc* D, int k0, int k1, const int* status) {
    PTT_PDL_ENTRY();
    if (*status) return;
    for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
        double* t = D->core[k];
        D->core[k] = D->alt[k];
        D->alt[k] = t;
    }
}

}  // namespace wt
