// Ozaki split-precision Gram matrix of a CTA's rows on the fifth-generation
// tensor cores: tcgen05.mma with BF16 operands from shared memory and FP32
// accumulators in tensor memory, recombined to double precision.  Included by
// ptt_gridqr.cuh (inside ptt_round.cu's anonymous namespace).
//
// Splitting (error-free transformation of Ozaki, Ogita, Oishi, Rump, Numer.
// Algorithms 59 (2012), in the integer-digit form of Ootomo, Ozaki, Yokota,
// IJHPCA 38 (2024)): column j of the CTA's rows x (h <= KMAX of them) is
// scaled by 2^(56 - e_j), e_j the exponent with max_k |x_kj| < 2^e_j, and
// rounded to the integer N = rint(x 2^(56 - e_j)), |N| < 2^56; with the
// offset C = 128 (1 + 256 + ... + 256^5), M = N + C splits into its top
// T = M >> 48 and six bytes b_k, and
//
//     N = T 256^6 + sum_{k<6} (b_k - 128) 256^k:
//
// seven balanced digits d_0 = T in [-256, 256], d_s = b_{6-s} - 128 in
// [-128, 127] (s >= 1), x = 2^(e_j - 8) sum_s d_s 256^-s up to the rounding
// of N (2^(e_j - 57)).  Each digit is an integer of at most 8 significant
// bits, exact in BF16 (made from its byte by a float with a fixed exponent,
// no conversion instruction).  With D_s the h x c matrix of digits s,
//
//     G_ij = 2^(e_i + e_j - 16) sum_{s + t <= 6} 256^-(s+t) (D_s^T D_t)_ij
//
// summed in double precision in a fixed order; the terms left out (s + t >=
// 7 and the rounding of N) are below 2^-52 max|x_i| max|x_j| per row: the
// partial matches an FP64 Gram to the rounding of the double sums (the FP64
// path's own error is of the same order).
//
// Shared memory (K-major, no swizzle: 8 x 16-byte core matrices): digit s of
// element (k, j) at byte
//     s SL + (j / 8) SBO + (k / 8) 128 + (j % 8) 16 + (k % 8) 2,
// SBO = KMAX 16, SL = 8 SBO.  Slices are contiguous, so M = 128 rows of an
// operand are two consecutive slices and N = 64 nb columns nb consecutive
// ones; one mma step takes K = 16 (two core matrices 128 bytes apart: LBO).
// An eighth slice stays zero (the second half of the M = 128 tile of digit 6).
//
// Tensor memory: 448 of 512 columns x 128 lanes of FP32.  For s = 0, 2, 4, 6
// the product of A = slices (s, s+1) (M = 128) and B = slices 0 .. 6 - s
// (N = 64 (7 - s), in pieces of at most 256) accumulates into columns
// 64 s .. 447, so column block c (64 c .. 64 c + 63) holds in lanes 0-63
// sum_{s even} D_s^T D_{c-s} (weight 256^-c) and in lanes 64-127
// sum_{s even} D_{s+1}^T D_{c-s} (weight 256^-(c+1); block 6 of these lanes
// is weight 7 and never read).  A block adds at most four digit products per
// row, at most two of them with d_0: |sum| <= 112 (2 2^15 + 2 2^14) < 2^24,
// so the FP32 accumulation is exact whatever the order of the tensor core's
// additions.  One round: 42 mma steps, one commit, then every warp reads its
// lanes' blocks (warps w and w + 4 share lanes 32 (w % 4) .. + 31 and split
// the 64 j's), the even- and odd-digit rows sum their blocks with their
// weights, and the two halves are added through shared memory.
//
// Waits: the completion of the products is signalled by tcgen05.commit on an
// mbarrier; every thread gives up after OZ_WAIT_NS (globaltimer).  If the wait
// runs out the CTA waits once more (bounded) for the products in flight, frees
// its tensor memory and writes NaN for its partial, so the decision that
// reads it falls back to the Householder factorisation; nothing spins without
// a limit.
#pragma once

namespace oz {

constexpr int S = 7;                  // digits
constexpr int NSL = 8;                // slices stored (the last stays zero)
constexpr int KMAX = 112;             // rows per CTA (K of the products), a multiple of 16
constexpr int SBO = KMAX * 16;        // bytes between 8-column groups of a slice
constexpr int SL = 8 * SBO;           // bytes of one slice of 64 columns
constexpr size_t SMEM = (size_t)NSL * SL;
constexpr int TCOLS = 512;            // tensor-memory columns held
constexpr unsigned long long OZ_WAIT_NS = 2000000000ull;  // an mbarrier wait gives up after 2 s
static_assert(KMAX % 16 == 0, "K steps of 16");
static_assert(KMAX * (2 * 32768 + 2 * 16384) < (1 << 24), "a tensor-memory block's sums exact in FP32");

struct Piece {
    int s, t0, nb;  // A = slices s, s + 1; B = slices t0 .. t0 + nb - 1; columns from 64 (s + t0)
};
constexpr int NPIECE = 6;
__host__ __device__ constexpr Piece piece(int q) {
    return q == 0 ? Piece{0, 0, 4} : q == 1 ? Piece{0, 4, 3} : q == 2 ? Piece{2, 0, 4}
         : q == 3 ? Piece{2, 4, 1} : q == 4 ? Piece{4, 0, 3} : Piece{6, 0, 1};
}

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start, LBO = 128 B (the two K halves of a
// step), SBO (8-row groups), version 1 (bit 46), no swizzle
__device__ __forceinline__ unsigned long long sdesc(unsigned saddr) {
    return (unsigned long long)((saddr >> 4) & 0x3FFFu) | ((unsigned long long)(128 >> 4) << 16) |
           ((unsigned long long)(SBO >> 4) << 32) | (1ull << 46);
}
// instruction descriptor of kind::f16: FP32 accumulator (bit 4), A and B BF16
// (bits 7, 10), both K-major, N / 8 at bit 17, M / 16 at bit 24 (M = 128)
__device__ __forceinline__ unsigned idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(n >> 3) << 17) | ((unsigned)(128 >> 4) << 24);
}
__device__ __forceinline__ void mma(unsigned tmem_d, unsigned long long a, unsigned long long b, unsigned id,
                                    int accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(id), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void commit(unsigned mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
__device__ __forceinline__ unsigned long long gtime() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool mbar_wait(unsigned mbar, unsigned parity) {
    const unsigned long long t0 = gtime();
    for (;;) {
        unsigned ok;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (gtime() - t0 > OZ_WAIT_NS) return false;
    }
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive FP32 columns of this warp's 32 lanes
__device__ __forceinline__ void ld32(unsigned taddr, float* v) {
    unsigned r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 32; q++) v[q] = __uint_as_float(r[q]);
}

// BF16 bits of the digits b0 - 128 and b1 - 128 (bytes in [0, 255]) packed
// low | high: the float 2^23 + b minus 2^23 + 128 is b - 128 exactly, and its
// top half is its BF16 value (the low half is zero)
__device__ __forceinline__ unsigned bf16_pair(unsigned b0, unsigned b1) {
    const float f0 = __uint_as_float(0x4B000000u | b0) - 8388736.0f;
    const float f1 = __uint_as_float(0x4B000000u | b1) - 8388736.0f;
    return __byte_perm(__float_as_uint(f0), __float_as_uint(f1), 0x7632);
}
// the same for the leading digits t0, t1 in [-256, 256]
__device__ __forceinline__ unsigned bf16_pair_top(int t0, int t1) {
    const float f0 = __uint_as_float(0x4B000000u | (unsigned)(t0 + 256)) - 8388864.0f;
    const float f1 = __uint_as_float(0x4B000000u | (unsigned)(t1 + 256)) - 8388864.0f;
    return __byte_perm(__float_as_uint(f0), __float_as_uint(f1), 0x7632);
}
// 2^k as a double, |k| <= 1022
__device__ __forceinline__ double pow2(int k) { return __longlong_as_double((long long)(1023 + k) << 52); }

// Partial Gram matrix of X (h x c rows of pitch xp, zero beyond c and h up to
// a multiple of 8) written to P as the 36 upper 8 x 8 tiles (tile q at P + 64
// q, row-major).  All NT = 256 threads; `sl` = SMEM bytes of shared memory,
// 16-byte aligned; `xtmp` = 64 x 65 doubles of shared memory, may alias X.
// A non-finite element, a misaligned buffer or a wait that runs out gives a
// NaN partial.
template <int NT>
__device__ void gram_partial(const double* X, int xp, int h, int c, unsigned char* sl, double* xtmp, double* P) {
    static_assert(NT == 256, "eight warps: two per tensor-memory lane quarter");
    __shared__ __align__(8) unsigned long long s_mbar;
    __shared__ unsigned s_tmem;
    __shared__ int s_e[64];
    __shared__ double s_sc[64];  // 2^(e_j - 8)
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 32) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // column exponents: max over the rows in four phases
    {
        double* red = (double*)sl;  // 4 x 64
        const int j = tid & 63, q = tid >> 6;
        double mx = 0.0;
        if (j < c)
            for (int r = q; r < h; r += 4) mx = fmax(mx, fabs(X[r * xp + j]));
        red[q * 64 + j] = mx;
        __syncthreads();
        if (tid < 64) {
            const double a = fmax(fmax(red[tid], red[64 + tid]), fmax(red[128 + tid], red[192 + tid]));
            int e = 0;
            if (a > 0.0 && a <= 1.7976931348623157e308) frexp(a, &e);
            s_e[tid] = e;
            s_sc[tid] = ldexp(1.0, e - 8);
        }
        __syncthreads();
    }
    // digits: item = (column j, 8-row block kb) -> one 16-byte row of a core
    // matrix in every slice
    bool nonfinite = false;
    for (int it = tid; it < 64 * (KMAX / 8); it += NT) {
        const int j = it & 63, kb = it >> 6;
        const int sh = 56 - s_e[j], sa = sh / 2;
        const double fa = pow2(sa), fb = pow2(sh - sa);
        unsigned lo[8], hi[8];
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const int k = kb * 8 + r;
            const double x = (k < h && j < c) ? X[k * xp + j] : 0.0;
            nonfinite |= !(fabs(x) <= 1.7976931348623157e308);
            const long long M = __double2ll_rn((x * fa) * fb) + 0x0000808080808080ll;
            lo[r] = (unsigned)M;
            hi[r] = (unsigned)(M >> 32);
        }
        unsigned char* dst = sl + (j >> 3) * SBO + kb * 128 + (j & 7) * 16;
        unsigned w[4];
#pragma unroll
        for (int p = 0; p < 4; p++)
            w[p] = bf16_pair_top((int)hi[2 * p] >> 16, (int)hi[2 * p + 1] >> 16);
        *(uint4*)dst = make_uint4(w[0], w[1], w[2], w[3]);
#pragma unroll
        for (int s = 1; s < S; s++) {  // digit s = byte 6 - s of M
            const int k = 6 - s;
#pragma unroll
            for (int p = 0; p < 4; p++) {
                const unsigned a = k >= 4 ? hi[2 * p] >> (8 * (k - 4)) : lo[2 * p] >> (8 * k);
                const unsigned b = k >= 4 ? hi[2 * p + 1] >> (8 * (k - 4)) : lo[2 * p + 1] >> (8 * k);
                w[p] = bf16_pair(a & 0xFFu, b & 0xFFu);
            }
            *(uint4*)(dst + s * SL) = make_uint4(w[0], w[1], w[2], w[3]);
        }
        *(uint4*)(dst + S * SL) = make_uint4(0u, 0u, 0u, 0u);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // digits visible to the tensor cores
    fence_before();
    nonfinite = __syncthreads_or(nonfinite) != 0;
    fence_after();
    const unsigned tbase = s_tmem;
    const unsigned mbar = smem_u32(&s_mbar);
    const unsigned sbase = smem_u32(sl);
    const int ksteps = h > 0 ? (h + 15) / 16 : 1;
    const int q4 = warp & 3, half = q4 >> 1, jh = warp >> 2;
    const int i = (q4 & 1) * 32 + lane;
    const unsigned taddr = tbase + ((unsigned)(q4 * 32) << 16);
    double acc[32];
#pragma unroll
    for (int q = 0; q < 32; q++) acc[q] = 0.0;
    // a descriptor addresses 16-byte units: a misaligned buffer takes the NaN
    // path without issuing a product (uniform over the CTA)
    bool bad = nonfinite || (sbase & 15u) != 0u;
    if (!bad) {
        if (tid == 0) {
#pragma unroll
            for (int q = 0; q < NPIECE; q++) {
                const Piece T = piece(q);
                const unsigned id = idesc(64 * T.nb);
                const unsigned long long da = sdesc(sbase + (unsigned)(T.s * SL));
                const unsigned long long db = sdesc(sbase + (unsigned)(T.t0 * SL));
#pragma unroll 1
                for (int kk = 0; kk < ksteps; kk++)  // a K step is 256 bytes: 16 in the address field
                    mma(tbase + (unsigned)(64 * (T.s + T.t0)), da + 16ull * kk, db + 16ull * kk, id,
                        (T.s > 0 || kk > 0) ? 1 : 0);
            }
            commit(mbar);
        }
        const bool ok = mbar_wait(mbar, 0u);
        bad = __syncthreads_or(!ok) != 0;
        if (bad) {
            mbar_wait(mbar, 0u);  // let the products in flight finish (bounded)
        } else {
            fence_after();
#pragma unroll
            for (int cb = 0; cb < S; cb++) {
                if (cb + half <= S - 1) {  // uniform over the warp
                    float v[32];
                    ld32(taddr + (unsigned)(64 * cb + 32 * jh), v);
                    const double w = pow2(-8 * (cb + half));
#pragma unroll
                    for (int q = 0; q < 32; q++) acc[q] = fma((double)v[q], w, acc[q]);
                }
            }
            fence_before();
            __syncthreads();  // every read done before the tensor memory is freed
            fence_after();
        }
    }
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TCOLS) : "memory");
    // odd digits (lanes 64-127) through shared memory, added to the even ones
    // and scaled; the sums written out in tile order (coalesced)
    if (half == 1)
#pragma unroll
        for (int q = 0; q < 32; q++) xtmp[i * 65 + 32 * jh + q] = acc[q];
    __syncthreads();
    if (half == 0) {
        const double si = s_sc[i];
#pragma unroll
        for (int q = 0; q < 32; q++) {  // times 2^(e_i + e_j - 16): two exact power-of-two products
            const int j = 32 * jh + q;
            xtmp[i * 65 + j] = bad ? __longlong_as_double(0x7ff8000000000000ll)
                                   : (acc[q] + xtmp[i * 65 + j]) * si * s_sc[j];
        }
    }
    __syncthreads();
    for (int u = tid; u < 36 * 64; u += NT) {
        int q = u >> 6, ti = 0;
        while (q >= 8 - ti) {
            q -= 8 - ti;
            ti++;
        }
        P[u] = xtmp[(ti * 8 + ((u >> 3) & 7)) * 65 + (ti + q) * 8 + (u & 7)];
    }
}

}  // namespace oz
