// Ozaki split-precision products on the fifth-generation tensor cores:
// tcgen05.mma with BF16 operands from shared memory and FP32 accumulators in
// tensor memory, recombined to double precision -- the Gram partial of a
// CTA's rows (gram_partial, the grid Cholesky QR's Gram stages) and a small
// factor times 64-column tiles of a core (gemm_tiles, the R X and X U_r S_r
// contractions of the block-level sweeps).  Included by ptt_round.cu inside
// its anonymous namespace.  Described below for the Gram; the tile products
// split both operands the same way (per-row scales for the factor, per-column
// for the tile) with K = the bond rank <= KG = 64.
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
// SBO = 16 x the K bound (KMAX; KG for the tile products), SL = 8 SBO.
// Slices are contiguous, so M = 128 rows of an
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
__device__ __forceinline__ unsigned long long sdesc(unsigned saddr, unsigned sbo) {
    return (unsigned long long)((saddr >> 4) & 0x3FFFu) | ((unsigned long long)(128 >> 4) << 16) |
           ((unsigned long long)(sbo >> 4) << 32) | (1ull << 46);
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

// Tensor memory and the mbarrier of one CTA's products (tensor memory
// allocated by warp 0 of the CTA, the permit to allocate again given up).
struct Tm {
    unsigned long long mbar;
    unsigned addr;
};
template <int NT>
__device__ __forceinline__ void tm_open(Tm* t) {
    if ((threadIdx.x >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&t->addr)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 32) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&t->mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
}
__device__ __forceinline__ void tm_close(const Tm* t) {
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(t->addr), "r"(TCOLS) : "memory");
}

// Digits of a block of up to KM x 64 doubles, element (k, j) at src[k sk + j
// sj] for k < h, j < w (zero elsewhere): per-column exponents and scales
// 2^(e_j - 8) in s_e / s_sc, the eight slices (the last zero) at `sl`
// (slice stride 8 KM 16 bytes, 8-column groups KM 16 bytes apart).  All NT
// threads; returns (uniformly) whether an element was not finite.
template <int NT, int KM>
__device__ bool split(const double* src, long long sk, long long sj, int h, int w, unsigned char* sl, int* s_e,
                      double* s_sc) {
    static_assert(NT == 256 && KM % 16 == 0, "");
    constexpr int SB = KM * 16, SLB = 8 * SB;
    __shared__ double red[4 * 64];
    const int tid = threadIdx.x;
    {  // column exponents: max over the rows in four phases
        const int j = tid & 63, q = tid >> 6;
        double mx = 0.0;
        if (j < w)
            for (int r = q; r < h; r += 4) mx = fmax(mx, fabs(src[r * sk + j * sj]));
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
    // item = (column j, 8-row block kb) -> one 16-byte row of a core matrix
    // in every slice
    bool nonfinite = false;
    for (int it = tid; it < 64 * (KM / 8); it += NT) {
        const int j = it & 63, kb = it >> 6;
        const int sh = 56 - s_e[j], sa = sh / 2;
        const double fa = pow2(sa), fb = pow2(sh - sa);
        unsigned lo[8], hi[8];
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const int k = kb * 8 + r;
            const double x = (k < h && j < w) ? src[k * sk + j * sj] : 0.0;
            nonfinite |= !(fabs(x) <= 1.7976931348623157e308);
            const long long M = __double2ll_rn((x * fa) * fb) + 0x0000808080808080ll;
            lo[r] = (unsigned)M;
            hi[r] = (unsigned)(M >> 32);
        }
        unsigned char* dst = sl + (j >> 3) * SB + kb * 128 + (j & 7) * 16;
        unsigned v[4];
#pragma unroll
        for (int p = 0; p < 4; p++) v[p] = bf16_pair_top((int)hi[2 * p] >> 16, (int)hi[2 * p + 1] >> 16);
        *(uint4*)dst = make_uint4(v[0], v[1], v[2], v[3]);
#pragma unroll
        for (int s = 1; s < S; s++) {  // digit s = byte 6 - s of M
            const int k = 6 - s;
#pragma unroll
            for (int p = 0; p < 4; p++) {
                const unsigned a = k >= 4 ? hi[2 * p] >> (8 * (k - 4)) : lo[2 * p] >> (8 * k);
                const unsigned b = k >= 4 ? hi[2 * p + 1] >> (8 * (k - 4)) : lo[2 * p + 1] >> (8 * k);
                v[p] = bf16_pair(a & 0xFFu, b & 0xFFu);
            }
            *(uint4*)(dst + s * SLB) = make_uint4(v[0], v[1], v[2], v[3]);
        }
        *(uint4*)(dst + S * SLB) = make_uint4(0u, 0u, 0u, 0u);
    }
    return __syncthreads_or(nonfinite) != 0;
}

// The slice products of A digits (slices at sla) and B digits (at slb), both
// KM deep, K = 16 ksteps used, weighted sums of this thread's 32 outputs in
// acc: the thread is lane i = 32 (warp & 1) + lane of the even- (warps 0, 1,
// 4, 5) or odd-digit (2, 3, 6, 7) half, columns j = 32 (warp >> 2) + 0..31.
// Callers make the digits visible first (fence.proxy.async, a barrier);
// parity = the number of earlier products of this Tm, mod 2.  Returns false (uniformly) if the wait ran out; the products in flight have
// then been waited for once more, and acc is not to be used.
template <int NT, int KM>
__device__ bool products(const Tm* t, unsigned char* sla, unsigned char* slb, int ksteps, double* acc,
                         unsigned parity) {
    constexpr unsigned SB = KM * 16, SLB = 8 * SB;
    const int tid = threadIdx.x, warp = tid >> 5;
#pragma unroll
    for (int q = 0; q < 32; q++) acc[q] = 0.0;
    fence_after();
    const unsigned tbase = t->addr;
    const unsigned mbar = smem_u32(&t->mbar);
    const unsigned sa = smem_u32(sla), sb = smem_u32(slb);
    if (((sa | sb) & 15u) != 0u) return false;  // uniform: no product issued
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < NPIECE; q++) {
            const Piece T = piece(q);
            const unsigned id = idesc(64 * T.nb);
            const unsigned long long da = sdesc(sa + T.s * SLB, SB);
            const unsigned long long db = sdesc(sb + T.t0 * SLB, SB);
#pragma unroll 1
            for (int kk = 0; kk < ksteps; kk++)  // a K step is 256 bytes: 16 in the address field
                mma(tbase + (unsigned)(64 * (T.s + T.t0)), da + 16ull * kk, db + 16ull * kk, id,
                    (T.s > 0 || kk > 0) ? 1 : 0);
        }
        commit(mbar);
    }
    const bool ok = mbar_wait(mbar, parity);
    if (__syncthreads_or(!ok)) {
        mbar_wait(mbar, parity);  // let the products in flight finish (bounded)
        return false;
    }
    fence_after();
    const int q4 = warp & 3, half = q4 >> 1, jh = warp >> 2;
    const unsigned taddr = tbase + ((unsigned)(q4 * 32) << 16);
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
    __syncthreads();  // every read done before the tensor memory is freed or reused
    return true;
}

// The odd-digit half's sums added to the even half's through xtmp (64 x 65
// doubles of shared memory) and scaled by sa[i] sb[j]: on return xtmp[i *
// 65 + j] holds output (i, j) (NaN everywhere if !ok).
template <int NT>
__device__ void combine(const double* acc, bool ok, const double* sa, const double* sb, double* xtmp) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q4 = warp & 3, half = q4 >> 1, jh = warp >> 2;
    const int i = (q4 & 1) * 32 + lane;
    if (half == 1)
#pragma unroll
        for (int q = 0; q < 32; q++) xtmp[i * 65 + 32 * jh + q] = acc[q];
    __syncthreads();
    if (half == 0) {
        const double si = sa[i];
#pragma unroll
        for (int q = 0; q < 32; q++) {  // times 2^(e_i + e_j - 16): two exact power-of-two products
            const int j = 32 * jh + q;
            xtmp[i * 65 + j] = ok ? (acc[q] + xtmp[i * 65 + j]) * si * sb[j] : __longlong_as_double(0x7ff8000000000000ll);
        }
    }
    __syncthreads();
}

// Partial Gram matrix of X (h x c rows of pitch xp, zero beyond c and h up to
// a multiple of 8) written to P as the 36 upper 8 x 8 tiles (tile q at P + 64
// q, row-major).  All NT = 256 threads; `sl` = SMEM bytes of shared memory,
// 16-byte aligned; `xtmp` = 64 x 65 doubles of shared memory, may alias X.
// A non-finite element, a misaligned buffer or a wait that runs out gives a
// NaN partial.
template <int NT>
__device__ void gram_partial(const double* X, int xp, int h, int c, unsigned char* sl, double* xtmp, double* P) {
    __shared__ Tm tm;
    __shared__ int s_e[64];
    __shared__ double s_sc[64];
    const int tid = threadIdx.x;
    tm_open<NT>(&tm);
    const bool nonfinite = split<NT, KMAX>(X, xp, 1, h, c, sl, s_e, s_sc);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // digits visible to the tensor cores
    fence_before();
    __syncthreads();
    double acc[32];
#pragma unroll
    for (int q = 0; q < 32; q++) acc[q] = 0.0;
    const bool ok = !nonfinite && products<NT, KMAX>(&tm, sl, sl, h > 0 ? (h + 15) / 16 : 1, acc, 0u);
    tm_close(&tm);
    combine<NT>(acc, ok, s_sc, s_sc, xtmp);
    for (int u = tid; u < 36 * 64; u += NT) {  // tile order (coalesced)
        int q = u >> 6, ti = 0;
        while (q >= 8 - ti) {
            q -= 8 - ti;
            ti++;
        }
        P[u] = xtmp[(ti * 8 + ((u >> 3) & 7)) * 65 + (ti + q) * 8 + (u & 7)];
    }
}

// C = A B for A (m x kd, element (i, l) at A[i ars + l acs]) and B (kd x n,
// element (l, j) at B[l brs + j bcs]), m, kd <= 64, C column-major with
// leading dimension ldc (ct: C^T stored, element (i, j) at C[j + i ldc]):
// CTA y forms the column tiles [64 t, 64 t + 64),
// t = y, y + gridDim.y, ..., each as the Ozaki product of A's digits
// (per-row scales, split once) and the tile's digits (per-column scales), K
// = kd <= 64 (every tensor-memory block sum below 64 (2 2^15 + 2 2^14) <
// 2^24: exact).  A non-finite element gives NaN outputs for the tile, as it
// propagates in FP64.  Shared memory: SMEM_GEMM bytes.
// A 64 x 64 block (element (k, j) at src[k sk + j sj], zero for k >= h or
// j >= w) copied to dst (pitch 65) with coalesced loads, along k when sk ==
// 1, else along j (sj == 1); each thread's 16 loads are all in flight before
// the first store
template <int NT>
__device__ void stage(const double* src, long long sk, long long sj, int h, int w, double* dst) {
    static_assert(64 * 64 % NT == 0, "");
    constexpr int PT = 64 * 64 / NT;
    const bool kfast = sk == 1;
    double v[PT];
#pragma unroll
    for (int t = 0; t < PT; t++) {
        const int e = threadIdx.x + t * NT;
        const int k = kfast ? (e & 63) : (e >> 6), j = kfast ? (e >> 6) : (e & 63);
        v[t] = (k < h && j < w) ? src[(long long)k * sk + (long long)j * sj] : 0.0;
    }
#pragma unroll
    for (int t = 0; t < PT; t++) {
        const int e = threadIdx.x + t * NT;
        const int k = kfast ? (e & 63) : (e >> 6), j = kfast ? (e >> 6) : (e & 63);
        dst[k * 65 + j] = v[t];
    }
    __syncthreads();
}

constexpr int KG = 64;                          // K bound of the products
constexpr int SLK = 8 * 8 * KG * 16;            // eight slices of 64 x KG digits
constexpr size_t SMEM_GEMM = 2 * (size_t)SLK + sizeof(double) * 64 * 65;
template <int NT>
__device__ void gemm_tiles(const double* A, long long ars, long long acs, const double* B, long long brs,
                           long long bcs, double* C, long long ldc, int m, int n, int kd, unsigned char* smem,
                           bool ct) {
    __shared__ Tm tm;
    __shared__ int s_ea[64], s_eb[64];
    __shared__ double s_sa[64], s_sb[64];
    unsigned char* sla = smem;
    unsigned char* slb = smem + SLK;
    double* xtmp = (double*)(smem + 2 * SLK);
    const int tid = threadIdx.x;
    const int ksteps = kd > 0 ? (kd + 15) / 16 : 1;
    tm_open<NT>(&tm);
    // A's digits: the M index is A's row i, the K index its column l
    stage<NT>(A, acs, ars, kd, m, xtmp);  // xtmp: the staging buffer until the products are summed
    const bool bad_a = split<NT, KG>(xtmp, 65, 1, kd, m, sla, s_ea, s_sa);
    const bool aligned = ((smem_u32(sla) | smem_u32(slb)) & 15u) == 0u;  // else no product is issued
    unsigned parity = 0;  // completed phases of the mbarrier, mod 2
    for (int y = blockIdx.y; 64 * y < n; y += gridDim.y) {
        const int j0 = 64 * y, w = (n - j0) < 64 ? (n - j0) : 64;
        stage<NT>(B + (long long)j0 * bcs, brs, bcs, kd, w, xtmp);
        const bool bad_b = split<NT, KG>(xtmp, 65, 1, kd, w, slb, s_eb, s_sb);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // digits visible to the tensor cores
        fence_before();
        __syncthreads();
        double acc[32];
        bool ok = false;
        if (aligned && !bad_a && !bad_b) {  // uniform
            ok = products<NT, KG>(&tm, sla, slb, ksteps, acc, parity);
            parity ^= 1u;
        } else {
#pragma unroll
            for (int q = 0; q < 32; q++) acc[q] = 0.0;
        }
        combine<NT>(acc, ok, s_sa, s_sb, xtmp);
        if (ct) {
            for (int e = tid; e < 64 * 64; e += NT) {  // C^T: the tile's columns contiguous
                const int i = e >> 6, jj = e & 63;
                if (i < m && jj < w) C[(long long)(j0 + jj) + (long long)i * ldc] = xtmp[i * 65 + jj];
            }
        } else {
            for (int e = tid; e < 64 * w; e += NT) {  // column-major C: rows contiguous
                const int jj = e >> 6, i = e & 63;
                if (i < m) C[(long long)i + (long long)(j0 + jj) * ldc] = xtmp[i * 65 + jj];
            }
        }
        __syncthreads();  // xtmp and the slices free for the next tile
    }
    tm_close(&tm);
}

}  // namespace oz
