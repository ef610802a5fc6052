// Tall-skinny QR (TSQR) of TT core unfoldings, FP64, as an in-kernel tree.
//
// Replaces the reference's MPI tree (tsqr_factorize tsqr.c:541-714,
// tsqr_make_q tsqr.c:716-1045, wflq_factorize tsqr.c:1048-1222,
// wflq_make_q tsqr.c:1225-1554) with one tree over thread blocks:
//
//  * leaf CTA p owns a contiguous row range of the m x c matrix.  It
//    Householder-factors its first c rows in shared memory (GEQRT), then
//    eliminates the remaining rows into that triangle H rows at a time
//    (TSQRT: pivot row from the triangle, vector from the chunk).  Vectors
//    are stored in place of the input rows, taus in the workspace.
//  * the leaf's R goes to the workspace; the CTA that arrives second at a
//    tree node (atomic counter, no spinning) eliminates its sibling's R into
//    its own (the same TSQRT on the sibling triangle's rows) and climbs on.
//  * Q (or Q*B for a small B) is produced top-down, one launch per tree
//    level, then one launch over the leaves, each block owning 32 columns
//    of B so the reflector loop needs no block-wide barrier.
//
// Pivot rows are always real rows, as in LAPACK, so Q has orthonormal
// columns also for rank-deficient unfoldings (x + x, formal sums).
#pragma once
#include "ptt_common.cuh"

namespace tsqr {

constexpr int H = 64;    // rows per elimination chunk
constexpr int NT = 256;  // threads per block
constexpr int KG = 32;   // columns of B per apply block

enum { LEFT = 0, RIGHT_T = 1 };

// Element (row, col) of the unfolding lives at p[row*rs + col*cs].
struct View {
    double* p;
    long long rs, cs;
    int m, c;
};

__device__ __forceinline__ View make_view(const DevDesc* D, int k, int mode, bool alt) {
    View v;
    const int r = D->r[k], n = D->n[k], r1 = D->r[k + 1];
    v.p = alt ? D->alt[k] : D->core[k];
    if (mode == LEFT) {
        v.m = r * n;
        v.c = r1;
        v.rs = 1;
        v.cs = v.m;
    } else {
        v.m = n * r1;
        v.c = r;
        v.rs = r;
        v.cs = 1;
    }
    return v;
}

// Per-call record written by the factor kernel, read by the later stages.
struct Info {
    int m, c, q;      // rows, columns, rank of the factorization
    int rank;         // truncation rank chosen by the SVD stage
    int sweeps;       // Jacobi sweeps
    int nsv;          // numerical rank kept by the SVD stage
    int status;
    int order;        // Jacobi pair order of the recorded rotations (0 circle, 1 stationary ring)
    double tail;      // retained tail sum (diagnostic)
};

// Workspace layout, computed on the host (identical formula in kernels).
struct Plan {
    int CT;          // column capacity (32, 64, 128)
    int L;           // rows per leaf (multiple of H, >= CT)
    int P;           // leaves (power of two)
    int KL;          // tau slots per leaf (1 GEQRT + TSQRT chunks)
    int NH;          // chunks per tree node (= ceil(CT / H))
    int KC;          // column capacity of B (multiple of KG)
    // offsets (in doubles) into the workspace
    long long o_tau_leaf, o_Rn, o_tau_node, o_Bn, o_US, o_rot, o_sig, o_info_d, o_nodes;
    long long total;  // doubles
    int* qn;          // device ints [2P-1]
    int* pass;        // device ints [P-1]
    int* cnt;         // device counters [P-1]
    Info* info;       // device
    double* stats;    // device, per-bond records of the rounding (may be null)
    double* work;     // device accumulator of algorithmic bytes (may be null)
    const int* gqstate;  // device state of the grid Cholesky QR of this bond (null: not used);
                         // the Householder kernels skip a bond it finished
};

// The grid Cholesky QR (ptt_gridqr.cuh) finished this bond: its state word
// is DONE (1) or FINISH (4).  Read from L2: it was written by an earlier
// launch of the same stream.
__device__ __forceinline__ bool gq_finished(const Plan& pl) {
    if (!pl.gqstate) return false;
    const int s = __ldcg(pl.gqstate);
    return s == 1 || s == 4;
}

// Leaf row range (identical on host and device).  The non-empty leaves are
// 0..Peff-1; the last one absorbs the tail so every non-empty leaf has at
// least min(m, L) >= min(m, c) rows.
__host__ __device__ __forceinline__ void leaf_range(int m, int L, int P, int p, int* r0, int* r1) {
    int peff = m / L;
    if (peff < 1) peff = 1;
    if (peff > P) peff = P;
    if (p >= peff) {
        *r0 = *r1 = 0;
        return;
    }
    *r0 = p * L;
    *r1 = (p == peff - 1) ? m : (p + 1) * L;
}

}  // namespace tsqr
