/*
 * paratt.h -- reference-compatible C API of the paratt tensor-train library,
 * implemented on one B200 by libparatt_b200.so.
 *
 * The structs and signatures are the reference's (source/paratt.h:25-345) so
 * a driver written against the reference compiles and links unchanged.  Cores
 * stay in host memory, allocated and grown by this library exactly as in the
 * reference (callers may read and write coreList[k] between calls and must
 * not cache core pointers across calls that can reallocate them); each call
 * stages the cores it needs through HBM and runs on the GPU.  For device-
 * resident work without host copies use paratt_b200.h.
 *
 * Single-process semantics: mpi_sz == 1, mpi_rk == 0.  Include <mpi.h> from
 * a real MPI or from include/mpi_compat/.
 */
#ifndef PARATT_PARALLEL_TT_H
#define PARATT_PARALLEL_TT_H

#include <stdlib.h>
#include <mpi.h>

#ifdef __cplusplus
extern "C" {
#endif

/* opaque in this implementation: holds the HBM mirror of the tensor */
typedef struct tsqr_tree tsqr_tree;

#if defined(__GNUC__)
#define PARATT_API __attribute__((visibility("default")))
#else
#define PARATT_API
#endif

/* source/paratt.h:25-54 */
typedef struct {
    int numDim;
    int* dim;
    int* ttRank;        /* numDim+1 entries, first and last are 1 */
    double** coreList;  /* core k: ttRank[k] x dim[k] x ttRank[k+1], column-major */
    int* coreMem;       /* doubles allocated per core */
    double* wk;
    int wksz;
} attac_tt;

/* source/paratt.h:56-65 */
typedef struct {
    attac_tt* x;
    int mpi_rk;
    int mpi_sz;
    int* distrib_dim_mat;
    int* dim;
    int numDim;
    int* iwk;
    int iwksz;
    tsqr_tree* orthog_wk;
} paratt;

/* ---- allocation (paratt.c:73-189) ---------------------------------------- */
attac_tt* alloc_tt(int ndims, int* d, int* ttR);
paratt* alloc_ptt(int ndims, int* d, int* ttR);
attac_tt* rank_change_tt(attac_tt* x_tt, int* ttR);
void copy_rank_change_tt(attac_tt* dest_tt, attac_tt* src_tt);
void free_tt(attac_tt* x_tt);
void free_ptt(paratt* x_ptt);

/* ---- halo exchange helpers (paratt.c:192-234): no peers in one process ---- */
void send_recv_below(void* send_buff, void* recv_buff, int msg_sz, MPI_Datatype dat_t,
                     MPI_Request* sendReq, MPI_Request* recvReq);
void send_recv_above(void* send_buff, void* recv_buff, int msg_sz, MPI_Datatype dat_t,
                     MPI_Request* sendReq, MPI_Request* recvReq);

/* ---- arithmetic (paratt.c:237-581) --------------------------------------- */
void attac_tt_axpby(double a, attac_tt* x_tt, double b, attac_tt* y_tt, attac_tt* z_tt);
void attac_tt_scale(double a, attac_tt* x_tt);
/* The reference's serial truncation reads singular values that are never
 * computed (attac.c:341ff); here it is the same rounding as paratt_truncate. */
void attac_tt_truncate(attac_tt* x_tt, double tol, int* maxRank);
void paratt_truncate(paratt* x_ptt, double tol, int* maxRank);
double attac_tt_norm(attac_tt* x_tt);         /* ||X||_F                      */
double paratt_norm(paratt* x_ptt);             /* ||X||_F / sqrt(prod dim)     */
double paratt_dotprod(paratt* x_ptt, paratt* y_ptt); /* <X,Y> / prod dim      */
double paratt_entry(paratt* x_ptt, int* mIdx);
void attac_set_rank1(attac_tt** x_tt_ptr, double** vec, int ndims, int* d);
attac_tt* attac_sum_of_product(double*** vec, int ndims, int* d, int all_ttR);
void attac_mult_diag_mat(attac_tt* f_tt, int mode, double* vec);
void attac_apply_periodic_stencil(attac_tt* f_tt, int mode, double* sten, int slen);
void pattac_apply_periodic_stencil(paratt* f_ptt, int mode, double* sten, int slen);

/* ---- CDF-problem operators and marginals (paratt.c:772-1618): outside the
 * accelerated path; these print a message and abort. ------------------------ */
void pattac_apply_cdf_stencil(paratt* f_ptt, int mode, double* sten, int slen);
void pattac_apply_cdf_lf_flux(paratt* f_ptt, int mode, double* wave_speed, double* gc_wave_speed,
                              double* source_coef, double dt, double dx);
void pattac_apply_cdf_lw_rhs(paratt* f_ptt, int mode, double* wave_speed, double* gc_wave_speed,
                             double* bdry_wave_speed, double* source_coef, double dt, double dx);
void pattac_apply_marginal(paratt* f_ptt, paratt** marginal_ptt_ptr, int mode, double* row_vector);
void pattac_marginal_cusum(paratt* f_ptt, int mode, double* row_vector);
void pattac_marginal_trap(paratt* f_ptt, int mode, double* row_vector);
void pattac_scale_weight_sum(paratt* f_ptt, int mode, double* scale, double* sum_w);

/* ---- .cr core files (paratt.c:1621-1892) ---------------------------------- */
void pattac_write_tt_folder(char* folder_name, paratt* f_ptt);
paratt* pattac_load_tt_folder(char* folder_name, int ndims);
void read_core_size(char* fname, int* rl, int* N, int* rr);
void load_core_slice(char* fname, double** cr, int* cr_sz, int* rl, int* N, int* rr, int N_beg, int N_end);

/* ---- extensions ----------------------------------------------------------- */
/* z = x (.) y in formal form (attacHadamard, attac.c:128-136; ranks multiply).
 * The reference exposes it only as pattacHadamard on raw arrays. */
void attac_tt_hadamard(attac_tt* x_tt, attac_tt* y_tt, attac_tt* z_tt);
/* 0 if the last call succeeded, else a PTT_ERR_* code (paratt_b200.h).  The
 * reference has no return codes: it exits on LAPACK failure. */
int paratt_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
