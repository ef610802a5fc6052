/*
 * paratt_b200 -- device-resident tensor-train hot path for NVIDIA B200 (sm_100a).
 *
 * This is the native C ABI underneath the reference-compatible API in
 * paratt.h / paratt_ode.h.  A ptt_tt is one tensor train whose cores live in
 * HBM at a fixed rank capacity; its actual ranks live in device memory too,
 * so every operation below is a fixed sequence of kernel launches on the
 * context's stream (no host synchronisation, CUDA-graph capturable) unless
 * its comment says it reads results back.
 *
 * Core layout is the reference's (source/paratt.h:36-42): core k is
 * r_k x n_k x r_{k+1}, column-major, element (i, j, l) at
 * i + r_k*(j + n_k*l).
 *
 * All functions return PTT_OK (0) or a PTT_ERR_* code; ptt_last_error()
 * and ptt_last_error_message() describe the most recent failure.
 */
#ifndef PARATT_B200_H
#define PARATT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define PTT_MAX_DIM 128

#if defined(__GNUC__)
#define PTT_API __attribute__((visibility("default")))
#else
#define PTT_API
#endif

enum {
    PTT_OK = 0,
    PTT_ERR_ARG = 1,       /* invalid argument / shape mismatch            */
    PTT_ERR_CUDA = 2,      /* CUDA runtime error (message has the details) */
    PTT_ERR_CAPACITY = 3,  /* ranks exceed the allocated rank capacity      */
    PTT_ERR_NUMERIC = 4,   /* non-finite values or a solver did not converge */
    PTT_ERR_NOGPU = 5,     /* no CUDA device: this library has no CPU path  */
    PTT_ERR_TIMEOUT = 6    /* a bounded device-side wait expired            */
};

typedef struct ptt_ctx ptt_ctx; /* device, stream, workspace, status word */
typedef struct ptt_tt ptt_tt;   /* one device-resident tensor train      */

PTT_API int ptt_last_error(void);
PTT_API const char* ptt_last_error_message(void);

/* ---- context ---------------------------------------------------------- */
PTT_API ptt_ctx* ptt_ctx_create(int device);
PTT_API void ptt_ctx_destroy(ptt_ctx* ctx);
/* Blocks until the stream drains; returns the first device-side status
 * (PTT_ERR_NUMERIC / PTT_ERR_TIMEOUT) raised since the last call, or a CUDA
 * error.  The status word is cleared. */
PTT_API int ptt_ctx_synchronize(ptt_ctx* ctx);
PTT_API void* ptt_ctx_stream(ptt_ctx* ctx); /* the cudaStream_t, as void* */
/* Launch counter: number of kernels this context has launched. */
PTT_API long long ptt_ctx_launch_count(const ptt_ctx* ctx);
/* Measurement: record event `slot` (0..63) on the context's stream; elapsed
 * milliseconds between two recorded slots (waits for the second). */
PTT_API int ptt_ctx_mark(ptt_ctx* ctx, int slot);
PTT_API int ptt_ctx_elapsed(ptt_ctx* ctx, int a, int b, double* ms);
/* Time every launch of one kernel class with an event pair (adds a few us
 * per launch): PTT_TIME_TSQR (TSQR factor tree), PTT_TIME_SVD (bond SVD),
 * PTT_TIME_GEMM (sketch contractions); 0 stops.  ptt_ctx_kernel_time
 * resolves the pairs (synchronises) and returns total ms and launch count. */
#define PTT_TIME_TSQR 1
#define PTT_TIME_SVD 2
#define PTT_TIME_GEMM 3
PTT_API int ptt_ctx_time_kernels(ptt_ctx* ctx, int kind);
PTT_API int ptt_ctx_kernel_time(ptt_ctx* ctx, double* ms, long long* count);
/* Algorithmic work of the timed launches: bytes for PTT_TIME_TSQR (16 m c
 * per factorisation of an m x c unfolding), flops for PTT_TIME_GEMM. */
PTT_API int ptt_ctx_kernel_work(ptt_ctx* ctx, double* work);
/* Replay roundings from CUDA graphs (no counterpart in the reference): with
 * on != 0, each rounding's launch sequence is captured once per distinct
 * (train, ranks, threshold, workspace) and replayed from then on; results are
 * identical.  Off by default; bypassed while kernels are timed and inside a
 * capture the caller makes.  The cache holds device pointers: a train
 * destroyed and recreated at the same address reuses its graph, which is
 * correct because the graph reads the descriptor at run time. */
PTT_API int ptt_ctx_graphs(ptt_ctx* ctx, int on);
/* Factorisation used for unfoldings with at most 64 columns (no counterpart
 * in the reference, whose TSQR is Householder throughout): with on != 0 (the
 * default) a shifted/repeated Cholesky-QR sequence -- by one thread-block
 * cluster up to 32 columns, by all SMs (one launch per Gram stage) for 33 to
 * 64 -- which falls back to the Householder TSQR for a bond it cannot make
 * orthonormal; with on == 0 the Householder TSQR only.  ptt_ctx_qr_counts returns, summed over the context
 * and its batch workers: [0] factorisations finished by Cholesky QR, [1] fell
 * back, [2] Gram stages of the finished ones (synchronises). */
PTT_API int ptt_ctx_cholqr(ptt_ctx* ctx, int on);
/* Precision of the contractions of the rounding's 33- to 64-column bonds
 * (no counterpart in the reference): with on != 0 the Gram matrices of the
 * Cholesky-QR stages and the R x core products of the left-to-right sweep are
 * Ozaki split-precision products -- each operand split into seven BF16 digit
 * slices of 8 bits with a power-of-two scale per row or column, the slice
 * products on the fifth-generation tensor cores (tcgen05.mma, FP32
 * accumulation, exact for the <= 112-term sums each accumulator takes),
 * recombined in double precision; with on == 0 (the default) FP64 mma.  The
 * digits drop less than 2^-52 max|a_i| max|b_j| per term, so both give the
 * products to double precision; the triangular solves, the factors and the
 * SVD stay FP64. */
PTT_API int ptt_ctx_ozaki(ptt_ctx* ctx, int on);
/* G = A^T A of a device m x c column-major matrix A (1 <= c <= 64, leading
 * dimension lda >= m) into the device array G (c x c, column-major), on the
 * context's stream (no counterpart in the reference: the Gram kernels of the
 * factorisation on their own).  method 0: FP64 mma; 1: the Ozaki split of
 * ptt_ctx_ozaki.  Deterministic; uses the context's workspace. */
PTT_API int ptt_gram(ptt_ctx* ctx, const double* A, long long m, int c, long long lda, double* G, int method);
/* Programmatic dependent launch of the rounding's kernel chain (no counterpart
 * in the reference): with on != 0 (the default) each kernel of a rounding may
 * be scheduled while its predecessor finishes and waits on the device for it
 * before touching memory, which hides most of the launch gap; on == 0 launches
 * them plainly.  Results are identical.  The library's own graph captures
 * launch plainly; inside a capture the caller makes, the launches become
 * programmatic edges of the caller's graph -- call ptt_ctx_pdl(ctx, 0) first
 * where that is not wanted. */
PTT_API int ptt_ctx_pdl(ptt_ctx* ctx, int on);
/* Autotuner (no counterpart in the reference): times the single-core QR of
 * random m x c unfoldings (c = 16, 24, 32; m = 512 ... 16384) with every
 * Cholesky-QR cluster size the device holds and keeps the fastest per
 * (c, m) bucket in the context; roundings then use that table (results
 * differ from the untuned sizes only by rounding order).  Takes well under a
 * second; synchronises.  A size replaces the built-in rule (about 384 rows
 * per CTA) only when it timed at least 15 % faster.  ptt_ctx_autotune_table
 * writes the 18 entries (row-major [c bucket][m bucket]): the chosen size,
 * or 0 where the rule is kept (all 0 if not tuned). */
PTT_API int ptt_ctx_autotune(ptt_ctx* ctx);
PTT_API int ptt_ctx_autotune_table(const ptt_ctx* ctx, int* out18);
/* The autotuner also times the sketch contractions: a batch of 48 x 48 x 48
 * products with 64- or 32-wide tiles, and one 40 x 40 product over K = 8192
 * split to fill 1, 2 or 4 times the SM count; a setting replaces the built-in
 * one (64-wide tiles from M, N >= 48; split-K up to 2 x SMs tiles) only when
 * it timed at least 10 % faster.  out2: [0] the smallest M, N of 64-wide
 * tiles, [1] the split-K tile target in force. */
PTT_API int ptt_ctx_autotune_gemm(const ptt_ctx* ctx, int* out2);
PTT_API int ptt_ctx_qr_counts(ptt_ctx* ctx, long long* out3);
/* Device memory held by the context's grow-on-demand workspaces (bytes), and
 * cudaMemGetInfo for the context's device (the caller's current device is
 * kept).  For checking that a call allocated nothing. */
PTT_API int ptt_ctx_workspace_bytes(const ptt_ctx* ctx, unsigned long long* bytes);
PTT_API int ptt_ctx_mem_info(const ptt_ctx* ctx, unsigned long long* free_bytes, unsigned long long* total_bytes);
/* Overwrite a device buffer of twice the L2 size on the context's stream. */
PTT_API int ptt_ctx_flush_l2(ptt_ctx* ctx);
/* Page-lock / release host memory for fast transfers (cudaHostRegister). */
PTT_API int ptt_host_pin(void* ptr, unsigned long long bytes);
PTT_API int ptt_host_unpin(void* ptr);

/* ---- tensor trains ----------------------------------------------------- */
/* rank_cap has d+1 entries (rank_cap[0] = rank_cap[d] = 1). */
PTT_API ptt_tt* ptt_tt_create(ptt_ctx* ctx, int d, const int* n, const int* rank_cap);
PTT_API void ptt_tt_destroy(ptt_tt* t);
PTT_API int ptt_tt_shape(const ptt_tt* t, int* d, int* n, int* rank_cap);
/* Grow the rank capacity (never shrinks); contents are kept. Allocates. */
PTT_API int ptt_tt_reserve(ptt_tt* t, const int* rank_cap);
/* Copy host cores in (ranks has d+1 entries; cores[k] holds
 * ranks[k]*n[k]*ranks[k+1] doubles).  Synchronous w.r.t. the host buffers. */
PTT_API int ptt_tt_set(ptt_tt* t, const int* ranks, const double* const* cores);
/* Read ranks (d+1 ints) and, if cores != NULL, the cores (each cores[k]
 * must hold ranks[k]*n[k]*ranks[k+1] doubles).  Synchronises the stream;
 * with cores != NULL it also returns (and clears), like ptt_ctx_synchronize,
 * a device-side error raised by the context's earlier work. */
PTT_API int ptt_tt_get(ptt_tt* t, int* ranks, double* const* cores);
PTT_API int ptt_tt_get_ranks(ptt_tt* t, int* ranks);
/* dst <- src (shapes must agree, capacity of dst must cover src). */
PTT_API int ptt_tt_copy(ptt_tt* dst, const ptt_tt* src);
/* Raw device addresses of the current core buffers (valid until the next
 * operation on t) and of the device rank array. */
PTT_API int ptt_tt_device_cores(const ptt_tt* t, double** cores, int** ranks);
/* The context a train belongs to. */
PTT_API ptt_ctx* ptt_tt_context(const ptt_tt* t);

/* ---- checkpoint / resume (the reference's .cr core files) -------------- */
/* Snapshot of a train into <folder>/core_<k+1>.cr, the format of
 * pattac_write_tt_folder (paratt.c:1621-1706): header "r_l,N,r_r", values
 * "%+1.16e" column-major, which round-trips every double.  The cores are
 * copied to page-locked host memory in stream order and a background thread
 * writes the files (write-behind): the call returns at once (after reading
 * the ranks), later work on the train does not change the snapshot, and
 * ptt_checkpoint_wait blocks until the files are written, returns the
 * outcome and releases the handle.  NULL on a bad argument or a failed
 * allocation. */
typedef struct ptt_checkpoint ptt_checkpoint;
PTT_API ptt_checkpoint* ptt_checkpoint_begin(ptt_tt* t, const char* folder);
PTT_API int ptt_checkpoint_wait(ptt_checkpoint* cp);
/* Resume: load a folder of .cr files (from either library, d files matching
 * t's mode sizes, ranks continuing from 1 to 1) into t, growing its rank
 * capacity if needed (pattac_load_tt_folder, paratt.c:1744-1892). */
PTT_API int ptt_tt_load_folder(ptt_tt* t, const char* folder);

/* ---- hot path ---------------------------------------------------------- */
/* paratt_truncate semantics (paratt.c:316-342, pattac.c:590-675): tol is
 * absolute on the grid-normalised norm ||X||_F / sqrt(prod n_k); per-bond
 * threshold tol/sqrt(d-1); maxrank has d+1 entries (NULL = capacity). */
PTT_API int ptt_round(ptt_tt* x, double tol, const int* maxrank);
/* By default ptt_round reads the actual ranks back (one synchronisation) and
 * sizes its tiles and trees from them.  With fixed plans on, it sizes them
 * from the rank capacity instead and never synchronises (for stream capture
 * of a whole step).  Results are identical either way. */
PTT_API int ptt_ctx_fixed_plans(ptt_ctx* ctx, int on);
/* Per-bond record of the context's last ptt_round (bond i = 1..d-1, record i;
 * PTT_STAT_LEN doubles each): rank, numerical rank, Jacobi sweeps, q, r_i,
 * dropped tail sum of squares, threshold, 0, then the top PTT_STAT_NSIG
 * singular values of the bond (of the unnormalised tensor).  Synchronises. */
#define PTT_STAT_NSIG 16
#define PTT_STAT_LEN (8 + PTT_STAT_NSIG)
PTT_API int ptt_round_stats(ptt_ctx* ctx, int d, double* out);
/* z = a*x + b*y in formal form (attacFormalAXPBY, attac.c:81-112). */
PTT_API int ptt_axpby(double a, const ptt_tt* x, double b, const ptt_tt* y, ptt_tt* z);
/* z = x (.) y in formal form (attacHadamard, attac.c:128-136). */
PTT_API int ptt_hadamard(const ptt_tt* x, const ptt_tt* y, ptt_tt* z);
/* z = x (.) x as an exact TT of ranks r_k (r_k + 1) / 2 instead of r_k^2:
 * the formal product restricted to the symmetric subspace of R^r (x) R^r.
 * No counterpart in the reference (which forms the rank r^2 product); the
 * tensor is the same, so its rounding matches to rounding error. */
PTT_API int ptt_square_sym(const ptt_tt* x, ptt_tt* z);
PTT_API int ptt_scale(double a, ptt_tt* x);                          /* paratt.c:271 */
PTT_API int ptt_mult_diag(ptt_tt* x, int mode, const double* vec);   /* paratt.c:571 */
/* Centred periodic stencil along one mode (paratt.c:584-661); an even slen
 * is decremented.  slen <= 15. */
PTT_API int ptt_stencil(ptt_tt* x, int mode, const double* sten, int slen);
/* y = sum_i S_i x + shift*x where S_i applies the centred periodic stencil
 * to mode i: an exact TT of rank 2 r_x (the formal sum of the d single-mode
 * stencil applications has rank d r_x). */
PTT_API int ptt_op_sum(const ptt_tt* x, const double* sten, int slen, double shift, ptt_tt* y);
/* z = round(x (.) y) through a Gaussian TT sketch of ranks ell[k] (d+1
 * entries, NULL = 72) without forming the rank r_x r_y product, then the
 * deterministic truncation of ptt_round (tol, maxrank).  Reads the input
 * ranks (synchronises).  Randomised: error ~ tail beyond ell, seeded. */
PTT_API int ptt_round_hadamard(const ptt_tt* x, const ptt_tt* y, ptt_tt* z, const int* ell,
                               unsigned long long seed, double tol, const int* maxrank);

/* Randomised rounding of x (y == NULL) or of x (.) y, as ptt_round_hadamard,
 * plus the acceptance check of the sketch: *accepted = 1 when every bond's
 * truncated rank stayed at least `pad` below its sketch rank (or the sketch
 * spanned the whole bond), else 0 -- the caller then falls back to the
 * deterministic rounding.  Reads ranks (synchronises). */
PTT_API int ptt_round_sketch(const ptt_tt* x, const ptt_tt* y, ptt_tt* z, const int* ell,
                             unsigned long long seed, double tol, const int* maxrank, int pad, int* accepted);

/* Round count independent trains (distinct, one context), train i with
 * tol[i] and rank caps maxrank[i] (d_i + 1 ints, or maxrank == NULL / a NULL
 * entry for no cap): the same result as ptt_round on each.  The trains are
 * rounded concurrently on up to `lanes` worker streams (<= 16) of the
 * context; reads every train's ranks once (synchronises) and returns with
 * the context's stream ordered after all of them.  No counterpart in the
 * reference. */
PTT_API int ptt_round_batch(ptt_tt* const* xs, int count, const double* tol, const int* const* maxrank, int lanes);

/* ---- reaction-Burgers step-truncation RK2 ------------------------------- */
typedef struct {
    double dt;        /* time step                                            */
    double tol;       /* absolute rounding tolerance (paratt_truncate meaning)  */
    double nu;        /* diffusion coefficient                                */
    double L;         /* box length, grid x_j = -L/2 + j L/n (periodic)         */
    int maxrank;      /* rank cap of every rounding (<= 64)                   */
    int sketch_pad;   /* product sketch rank = maxrank + sketch_pad            */
    unsigned long long seed;
} ptt_rxn_params;
typedef struct ptt_rxn_ws ptt_rxn_ws;
PTT_API ptt_rxn_ws* ptt_rxn_ws_create(ptt_ctx* ctx, int d, const int* n, int maxrank);
PTT_API void ptt_rxn_ws_destroy(ptt_rxn_ws* ws);
PTT_API int ptt_rxn_ws_counts(const ptt_rxn_ws* ws, long long* formal, long long* sketch);
/* F = nu sum d2_i u - (1/d) sum d1_i (u^2/2) + u - u^2, rounded (see
 * paratt_b200/csrc/host/rxn_burgers.c for the composition). */
PTT_API int ptt_rxn_burgers_F(ptt_tt* u, ptt_tt* F, ptt_rxn_ws* ws, const ptt_rxn_params* p);
/* u <- one step-truncation midpoint step of the reaction-Burgers equation. */
PTT_API int ptt_rxn_burgers_rk2_step(ptt_tt* u, ptt_rxn_ws* ws, const ptt_rxn_params* p);

/* The same step with every rounding done by a Gaussian TT sketch of per-bond
 * ranks ell[k] (d+1 entries) plus the deterministic truncation, F taken as one
 * sketch of the formal sum a + b; a rounding whose sketch fails the check of
 * ptt_round_sketch (margin `pad`) is redone deterministically. */
PTT_API int ptt_rxn_burgers_rk2_step_sketch(ptt_tt* u, ptt_rxn_ws* ws, const ptt_rxn_params* p, const int* ell,
                                            int pad);
/* Rounding kinds of a step: the product u.u, the field F, the two stage
 * roundings (u_s and u+). */
#define PTT_RXN_KIND_PRODUCT 0
#define PTT_RXN_KIND_FIELD 1
#define PTT_RXN_KIND_STAGE 2
#define PTT_RXN_KINDS 3
/* The sketch step with sketch ranks per kind: ell holds PTT_RXN_KINDS blocks
 * of d+1 entries, block t for the roundings of kind t. */
PTT_API int ptt_rxn_burgers_rk2_step_sketch_kinds(ptt_tt* u, ptt_rxn_ws* ws, const ptt_rxn_params* p,
                                                  const int* ell, int pad);
PTT_API int ptt_rxn_ws_sketch_counts(const ptt_rxn_ws* ws, long long* calls, long long* fallbacks);
/* Logging (reads each rounding's statistics back): per step the largest kept
 * rank of every bond over the step's roundings, and the top PTT_STAT_NSIG
 * singular values of every bond of the last rounding with its threshold. */
PTT_API int ptt_rxn_ws_log(ptt_rxn_ws* ws, int on);
PTT_API int ptt_rxn_ws_last_step(const ptt_rxn_ws* ws, int* ranks, double* sig, double* delta);
/* The same restricted to the roundings of one kind (PTT_RXN_KIND_*): their
 * largest kept rank per bond in the last step, and the spectra and threshold
 * of the last rounding of that kind. */
PTT_API int ptt_rxn_ws_last_step_kind(const ptt_rxn_ws* ws, int kind, int* ranks, double* sig, double* delta);

/* ---- sketch-rank proposer: MLP nin -> width -> width -> 1 (ReLU), BF16
 * weights, FP32 accumulation, trained with hand-written kernels (Adam) ---- */
typedef struct ptt_mlp ptt_mlp;
PTT_API ptt_mlp* ptt_mlp_create(ptt_ctx* ctx, int nin, int width, unsigned long long seed);
PTT_API void ptt_mlp_destroy(ptt_mlp* m);
PTT_API long long ptt_mlp_num_params(const ptt_mlp* m);
/* parameter vector (FP32 master copy): W1[w x nin] b1[w] W2[w x w] b2[w] W3[w] b3 */
PTT_API int ptt_mlp_get_params(ptt_mlp* m, float* out);
PTT_API int ptt_mlp_set_params(ptt_mlp* m, const float* in);
/* host buffers: x[B x nin] row-major, y[B], t[B] */
PTT_API int ptt_mlp_forward(ptt_mlp* m, const float* x, int B, float* y);
/* loss = mean(a (y - t)^2), a = under-weight if y < t else 1; gradients of
 * the BF16-weight network with respect to the parameters */
PTT_API int ptt_mlp_grads(ptt_mlp* m, const float* x, const float* t, int B, float* grads, float* loss);
PTT_API int ptt_mlp_train_step(ptt_mlp* m, const float* x, const float* t, int B, float lr, float* loss);
PTT_API int ptt_mlp_set_under_weight(ptt_mlp* m, float w);

/* ---- CDF-problem stencils and marginals (one process) ------------------
 * The reference's post-processing for its Burgers-Hopf CDF driver, each in
 * place on core `mode` (the ghost cells of the reference's MPI exchange are
 * rows of the same core with one process):
 *   ptt_cdf_stencil      pattac_apply_cdf_stencil (paratt.c:772-923): centred
 *                        stencil (even slen drops its last tap, slen <= 15);
 *                        below the grid the reference reads f[a - j - 1], above
 *                        it f[2n - 1 - j] (mirrored rows)
 *   ptt_cdf_lf_flux      pattac_apply_cdf_lf_flux (paratt.c:926-1093):
 *                        wave_speed[n], gc_wave_speed[2], source_coef[n]
 *   ptt_cdf_lw_rhs       pattac_apply_cdf_lw_rhs (paratt.c:1096-1250): adds
 *                        bdry_wave_speed[n + 1]
 *   ptt_marginal_cusum   pattac_marginal_cusum (paratt.c:1393-1445)
 *   ptt_marginal_trap    pattac_marginal_trap (paratt.c:1448-1524)
 *   ptt_scale_weight_sum pattac_scale_weight_sum (paratt.c:1527-1618)
 *   ptt_apply_marginal   pattac_apply_marginal (paratt.c:1252-1390): z (d - 1
 *                        modes, capacity for x's ranks without r_{mode+1}, or
 *                        with r_{d-1} -> 1 when mode = d - 1) = x contracted
 *                        along `mode` with the row vector w[n_mode]
 * Host vectors are copied in before the call returns. */
PTT_API int ptt_cdf_stencil(ptt_tt* x, int mode, const double* sten, int slen);
PTT_API int ptt_cdf_lf_flux(ptt_tt* x, int mode, const double* wave_speed, const double* gc_wave_speed,
                            const double* source_coef, double dt, double dx);
PTT_API int ptt_cdf_lw_rhs(ptt_tt* x, int mode, const double* wave_speed, const double* gc_wave_speed,
                           const double* bdry_wave_speed, const double* source_coef, double dt, double dx);
PTT_API int ptt_marginal_cusum(ptt_tt* x, int mode, const double* w);
PTT_API int ptt_marginal_trap(ptt_tt* x, int mode, const double* w);
PTT_API int ptt_scale_weight_sum(ptt_tt* x, int mode, const double* scale, const double* sum_w);
PTT_API int ptt_apply_marginal(const ptt_tt* x, int mode, const double* w, ptt_tt* z);

/* Reductions (these read a scalar back, so they synchronise). */
PTT_API int ptt_dot(const ptt_tt* x, const ptt_tt* y, double* out);  /* <X,Y>/prod n */
PTT_API int ptt_norm(const ptt_tt* x, double* out);                  /* RMS norm     */
PTT_API int ptt_entry(const ptt_tt* x, const int* idx, double* out);

/* ptt_dot without any device allocation.  No counterpart in the reference:
 * for callers that must not have a library call cudaMalloc (a framework that
 * owns the GPU's memory pool, a loop that cannot afford cudaMalloc's implicit
 * synchronisation, an embedding that forbids allocation after start-up).
 * Scratch lives in a fixed device array of PTT_DOT_NOALLOC_MAX_DOUBLES
 * doubles (4 MiB, held by every GPU that loads the library until exit); a
 * call needs 2*max_k(rx_k ry_k) + max_k(rx_k n_k ry_{k+1}) doubles and fails
 * with PTT_ERR_CAPACITY beyond that.  ptt_ctx_create loads the array and looks
 * up its address on the context's device, so the array is reserved when the
 * context is created (create it before another allocator takes the GPU's
 * memory) and no call loads or allocates anything later.  All calls share the
 * array, so calls that overlap on the GPU race.  Reads the ranks and the
 * result back (synchronises). */
#define PTT_DOT_NOALLOC_MAX_DOUBLES (1 << 19)
PTT_API int ptt_dot_noalloc(const ptt_tt* x, const ptt_tt* y, double* out);

#ifdef __cplusplus
}
#endif
#endif
