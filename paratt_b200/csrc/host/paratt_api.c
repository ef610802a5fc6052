/*
 * Reference-compatible paratt API (source/paratt.h) in C over the device
 * library (paratt_b200.h).
 *
 * Ownership follows the reference: the library mallocs structs and host
 * cores, grows cores with realloc (paratt.c:133-147, 253-257), and callers
 * may touch coreList[k] between calls.  Each tensor train gets an HBM mirror
 * (kept in a registry keyed by the attac_tt pointer, released by free_tt);
 * a call uploads the cores it reads, runs the kernels and downloads what it
 * wrote.  There is no CPU arithmetic path: without a GPU every call fails
 * with a message and exit(1), like the reference on a LAPACK error.
 */
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <sys/types.h>

#include "../../../include/paratt.h"
#include "../../../include/paratt_b200.h"

/* ------------------------------------------------------------------------ */
/* context and mirrors                                                      */
/* ------------------------------------------------------------------------ */
static ptt_ctx* g_ctx = NULL;
static int g_err = 0;

typedef struct {
    const attac_tt* key;
    ptt_tt* dev;
} mirror_t;

static mirror_t* g_mir = NULL;
static int g_nmir = 0, g_capmir = 0;

/* host allocation that stops with a message instead of returning NULL (the
   reference dereferences its unchecked malloc results) */
static void* xmalloc(size_t bytes) {
    void* p = malloc(bytes ? bytes : 1);
    if (!p) {
        fprintf(stderr, "paratt_b200: out of host memory (%zu bytes)\n", bytes);
        exit(1);
    }
    return p;
}

static void fail(const char* where) {
    fprintf(stderr, "paratt_b200: %s: %s\n", where, ptt_last_error_message());
    exit(1);
}

static int check(int rc, const char* where) {
    g_err = rc;
    if (rc == PTT_ERR_NOGPU || rc == PTT_ERR_CUDA) fail(where);
    if (rc) fprintf(stderr, "paratt_b200: %s: %s\n", where, ptt_last_error_message());
    return rc;
}

static ptt_ctx* ctx(void) {
    if (!g_ctx) {
        const char* e = getenv("PARATT_DEVICE");
        g_ctx = ptt_ctx_create(e ? atoi(e) : 0);
        if (!g_ctx) fail("context");
    }
    return g_ctx;
}

int paratt_last_error(void) { return g_err; }

static ptt_tt* find_mirror(const attac_tt* x) {
    for (int i = 0; i < g_nmir; i++)
        if (g_mir[i].key == x) return g_mir[i].dev;
    return NULL;
}

static void drop_mirror(const attac_tt* x) {
    for (int i = 0; i < g_nmir; i++)
        if (g_mir[i].key == x) {
            ptt_tt_destroy(g_mir[i].dev);
            g_mir[i] = g_mir[--g_nmir];
            return;
        }
}

/* Mirror with capacity at least `ranks` (NULL: the tensor's own ranks). */
static ptt_tt* mirror(const attac_tt* x, const int* ranks) {
    const int* r = ranks ? ranks : x->ttRank;
    ptt_tt* m = find_mirror(x);
    if (!m) {
        m = ptt_tt_create(ctx(), x->numDim, x->dim, r);
        if (!m) fail("mirror allocation");
        if (g_nmir == g_capmir) {
            g_capmir = g_capmir ? 2 * g_capmir : 16;
            g_mir = (mirror_t*)realloc(g_mir, sizeof(mirror_t) * g_capmir);
        }
        g_mir[g_nmir].key = x;
        g_mir[g_nmir].dev = m;
        g_nmir++;
    } else if (check(ptt_tt_reserve(m, r), "reserve")) {
        fail("reserve");
    }
    return m;
}

static ptt_tt* upload(const attac_tt* x) {
    ptt_tt* m = mirror(x, NULL);
    if (check(ptt_tt_set(m, x->ttRank, (const double* const*)x->coreList), "upload")) fail("upload");
    return m;
}

/* Grow host cores to hold `ranks` (grow-only realloc, paratt.c:133-147). */
static void host_fit(attac_tt* x, const int* ranks) {
    for (int k = 0; k < x->numDim; k++) {
        int need = x->dim[k] * ranks[k] * ranks[k + 1];
        if (x->coreMem[k] < need) {
            double* p = (double*)realloc(x->coreList[k], sizeof(double) * (size_t)need);
            if (!p) {  /* the reference would crash on the NULL core; stop with a message */
                fprintf(stderr, "paratt_b200: out of host memory growing core %d\n", k);
                exit(1);
            }
            x->coreList[k] = p;
            x->coreMem[k] = need;
        }
    }
    for (int k = 0; k <= x->numDim; k++) x->ttRank[k] = ranks[k];
}

static void download(attac_tt* x, ptt_tt* m) {
    int r[PTT_MAX_DIM + 1];
    if (check(ptt_ctx_synchronize(ctx()), "device")) return;
    if (check(ptt_tt_get_ranks(m, r), "ranks")) fail("download");
    host_fit(x, r);
    if (check(ptt_tt_get(m, r, x->coreList), "download")) fail("download");
}

/* ------------------------------------------------------------------------ */
/* allocation                                                               */
/* ------------------------------------------------------------------------ */
attac_tt* alloc_tt(int ndims, int* d, int* ttR) {
    attac_tt* t = (attac_tt*)xmalloc(sizeof(attac_tt));
    t->numDim = ndims;
    t->dim = (int*)xmalloc(sizeof(int) * ndims);
    t->ttRank = (int*)xmalloc(sizeof(int) * (ndims + 1));
    t->coreList = (double**)xmalloc(sizeof(double*) * ndims);
    t->coreMem = (int*)xmalloc(sizeof(int) * ndims);
    for (int k = 0; k < ndims; k++) {
        t->dim[k] = d[k];
        t->ttRank[k] = ttR[k];
        int sz = d[k] * (k == 0 ? 1 : ttR[k]) * ttR[k + 1];
        t->coreList[k] = (double*)xmalloc(sizeof(double) * (size_t)sz);
        t->coreMem[k] = sz;
    }
    t->ttRank[ndims] = ttR[ndims];
    t->wk = NULL;
    t->wksz = 0;
    return t;
}

paratt* alloc_ptt(int ndims, int* d, int* ttR) {
    paratt* p = (paratt*)xmalloc(sizeof(paratt));
    p->mpi_rk = 0;
    p->mpi_sz = 1;
    p->numDim = ndims;
    p->dim = (int*)xmalloc(sizeof(int) * ndims);
    p->distrib_dim_mat = (int*)xmalloc(sizeof(int) * ndims);
    for (int k = 0; k < ndims; k++) p->dim[k] = p->distrib_dim_mat[k] = d[k];
    p->iwk = (int*)xmalloc(sizeof(int) * (ndims + 1));
    p->iwksz = ndims + 1;
    p->orthog_wk = NULL;
    p->x = alloc_tt(ndims, d, ttR);
    return p;
}

attac_tt* rank_change_tt(attac_tt* x, int* ttR) {
    host_fit(x, ttR);
    return x;
}

void copy_rank_change_tt(attac_tt* dest, attac_tt* src) {
    host_fit(dest, src->ttRank);
    for (int k = 0; k < dest->numDim; k++)
        memcpy(dest->coreList[k], src->coreList[k],
               sizeof(double) * (size_t)src->ttRank[k] * src->dim[k] * src->ttRank[k + 1]);
}

void free_tt(attac_tt* x) {
    if (!x) return;
    drop_mirror(x);
    for (int k = 0; k < x->numDim; k++) free(x->coreList[k]);
    free(x->coreList);
    free(x->coreMem);
    free(x->dim);
    free(x->ttRank);
    free(x->wk);
    free(x);
}

void free_ptt(paratt* p) {
    if (!p) return;
    free_tt(p->x);
    free(p->distrib_dim_mat);
    free(p->iwk);
    free(p->dim);
    free(p);
}

void send_recv_below(void* s, void* r, int n, MPI_Datatype t, MPI_Request* sq, MPI_Request* rq) {
    (void)s; (void)r; (void)n; (void)t; (void)sq; (void)rq;
    fprintf(stderr, "paratt_b200: send_recv_below: one process per GPU, no ring peers\n");
    exit(1);
}

void send_recv_above(void* s, void* r, int n, MPI_Datatype t, MPI_Request* sq, MPI_Request* rq) {
    (void)s; (void)r; (void)n; (void)t; (void)sq; (void)rq;
    fprintf(stderr, "paratt_b200: send_recv_above: one process per GPU, no ring peers\n");
    exit(1);
}

/* ------------------------------------------------------------------------ */
/* arithmetic                                                               */
/* ------------------------------------------------------------------------ */
void attac_tt_axpby(double a, attac_tt* x, double b, attac_tt* y, attac_tt* z) {
    ptt_tt* mx = upload(x);
    ptt_tt* my = (y == x) ? mx : upload(y);
    int need[PTT_MAX_DIM + 1];
    need[0] = need[x->numDim] = 1;
    for (int k = 1; k < x->numDim; k++) need[k] = x->ttRank[k] + y->ttRank[k];
    ptt_tt* mz = mirror(z, need);
    if (check(ptt_axpby(a, mx, b, my, mz), "attac_tt_axpby")) return;
    download(z, mz);
}

void attac_tt_hadamard(attac_tt* x, attac_tt* y, attac_tt* z) {
    ptt_tt* mx = upload(x);
    ptt_tt* my = (y == x) ? mx : upload(y);
    int need[PTT_MAX_DIM + 1];
    for (int k = 0; k <= x->numDim; k++) need[k] = x->ttRank[k] * y->ttRank[k];
    ptt_tt* mz = mirror(z, need);
    if (check(ptt_hadamard(mx, my, mz), "attac_tt_hadamard")) return;
    download(z, mz);
}

void attac_tt_scale(double a, attac_tt* x) {
    ptt_tt* m = upload(x);
    if (check(ptt_scale(a, m), "attac_tt_scale")) return;
    download(x, m);
}

void paratt_truncate(paratt* p, double tol, int* maxRank) {
    ptt_tt* m = upload(p->x);
    if (check(ptt_round(m, tol, maxRank), "paratt_truncate")) return;
    download(p->x, m);
}

void attac_tt_truncate(attac_tt* x, double tol, int* maxRank) {
    ptt_tt* m = upload(x);
    if (check(ptt_round(m, tol, maxRank), "attac_tt_truncate")) return;
    download(x, m);
}

double paratt_dotprod(paratt* x, paratt* y) {
    ptt_tt* mx = upload(x->x);
    ptt_tt* my = (y == x) ? mx : upload(y->x);
    double v = 0.0;
    check(ptt_dot(mx, my, &v), "paratt_dotprod");
    return v;
}

double paratt_norm(paratt* x) {
    ptt_tt* m = upload(x->x);
    double v = 0.0;
    check(ptt_norm(m, &v), "paratt_norm");
    return v;
}

double attac_tt_norm(attac_tt* x) {
    ptt_tt* m = upload(x);
    double v = 0.0;
    check(ptt_norm(m, &v), "attac_tt_norm");
    double lg = 0.0;
    for (int k = 0; k < x->numDim; k++) lg += log((double)x->dim[k]);
    return v * exp(0.5 * lg);
}

double paratt_entry(paratt* x, int* mIdx) {
    ptt_tt* m = upload(x->x);
    double v = 0.0;
    check(ptt_entry(m, mIdx, &v), "paratt_entry");
    return v;
}

void attac_mult_diag_mat(attac_tt* f, int mode, double* vec) {
    ptt_tt* m = upload(f);
    if (check(ptt_mult_diag(m, mode, vec), "attac_mult_diag_mat")) return;
    download(f, m);
}

void attac_apply_periodic_stencil(attac_tt* f, int mode, double* sten, int slen) {
    ptt_tt* m = upload(f);
    if (check(ptt_stencil(m, mode, sten, slen), "attac_apply_periodic_stencil")) return;
    download(f, m);
}

/* With one process the distributed stencil is the serial one.  (The
 * reference's P=1 branch, paratt.c:721-769, agrees with it for 3-point
 * stencils; for 5 or more taps it reads the wrap-around ghost rows out of
 * order at 0 < a < h -- this implementation is periodic for every length.) */
void pattac_apply_periodic_stencil(paratt* f, int mode, double* sten, int slen) {
    attac_apply_periodic_stencil(f->x, mode, sten, slen);
}

void attac_set_rank1(attac_tt** x_ptr, double** vec, int ndims, int* d) {
    int* r = (int*)xmalloc(sizeof(int) * (ndims + 1));
    for (int i = 0; i <= ndims; i++) r[i] = 1;
    attac_tt* x = alloc_tt(ndims, d, r);
    for (int i = 0; i < ndims; i++) memcpy(x->coreList[i], vec[i], sizeof(double) * d[i]);
    free(r);
    *x_ptr = x;
}

/* Sum of rank-1 terms, paratt.c:517-568: the formal sums of the reference
 * give core 0 = [v_0 | v_1 | ...], diagonal interior cores and a stacked
 * last core, which is what is built here directly. */
attac_tt* attac_sum_of_product(double*** vec, int ndims, int* d, int R) {
    if (R == 1) {
        attac_tt* x;
        attac_set_rank1(&x, vec[0], ndims, d);
        return x;
    }
    int* r = (int*)xmalloc(sizeof(int) * (ndims + 1));
    r[0] = r[ndims] = 1;
    for (int i = 1; i < ndims; i++) r[i] = R;
    attac_tt* x = alloc_tt(ndims, d, r);
    for (int k = 0; k < ndims; k++) {
        int rl = r[k], rr = r[k + 1], n = d[k];
        double* c = x->coreList[k];
        memset(c, 0, sizeof(double) * (size_t)rl * n * rr);
        for (int t = 0; t < R; t++)
            for (int j = 0; j < n; j++) {
                int i = (k == 0) ? 0 : t, l = (k == ndims - 1) ? 0 : t;
                c[i + rl * (j + n * l)] = vec[t][k][j];
            }
    }
    free(r);
    return x;
}

/* ------------------------------------------------------------------------ */
/* CDF-problem stencils and marginals (paratt.c:772-1618), one process       */
/* ------------------------------------------------------------------------ */
void pattac_apply_cdf_stencil(paratt* f, int mode, double* sten, int slen) {
    ptt_tt* m = upload(f->x);
    if (check(ptt_cdf_stencil(m, mode, sten, slen), "pattac_apply_cdf_stencil")) return;
    download(f->x, m);
}

void pattac_apply_cdf_lf_flux(paratt* f, int mode, double* wave_speed, double* gc_wave_speed, double* source_coef,
                              double dt, double dx) {
    ptt_tt* m = upload(f->x);
    if (check(ptt_cdf_lf_flux(m, mode, wave_speed, gc_wave_speed, source_coef, dt, dx), "pattac_apply_cdf_lf_flux"))
        return;
    download(f->x, m);
}

void pattac_apply_cdf_lw_rhs(paratt* f, int mode, double* wave_speed, double* gc_wave_speed, double* bdry_wave_speed,
                             double* source_coef, double dt, double dx) {
    ptt_tt* m = upload(f->x);
    if (check(ptt_cdf_lw_rhs(m, mode, wave_speed, gc_wave_speed, bdry_wave_speed, source_coef, dt, dx),
              "pattac_apply_cdf_lw_rhs"))
        return;
    download(f->x, m);
}

void pattac_marginal_cusum(paratt* f, int mode, double* row_vector) {
    ptt_tt* m = upload(f->x);
    if (check(ptt_marginal_cusum(m, mode, row_vector), "pattac_marginal_cusum")) return;
    download(f->x, m);
}

void pattac_marginal_trap(paratt* f, int mode, double* row_vector) {
    ptt_tt* m = upload(f->x);
    if (check(ptt_marginal_trap(m, mode, row_vector), "pattac_marginal_trap")) return;
    download(f->x, m);
}

void pattac_scale_weight_sum(paratt* f, int mode, double* scale, double* sum_w) {
    ptt_tt* m = upload(f->x);
    if (check(ptt_scale_weight_sum(m, mode, scale, sum_w), "pattac_scale_weight_sum")) return;
    download(f->x, m);
}

/* The marginal with one mode fewer is allocated here, as the reference does
 * (paratt.c:1258-1282); *marginal must be NULL on entry. */
void pattac_apply_marginal(paratt* f, paratt** marginal, int mode, double* row_vector) {
    if (*marginal != NULL) {
        fprintf(stderr, "pattac_apply_marginal: Error.\nInput marginal_tt_ptr was not NULL.\n");
        exit(1);
    }
    const int d = f->numDim;
    if (d < 2 || mode < 0 || mode >= d) {
        fprintf(stderr, "paratt_b200: pattac_apply_marginal: mode %d of a %d-mode train\n", mode, d);
        exit(1);
    }
    int dims[PTT_MAX_DIM], ranks[PTT_MAX_DIM + 1];
    for (int k = 0, t = 0; k < d; k++)
        if (k != mode) dims[t++] = f->dim[k];
    for (int t = 0; t < d; t++) {
        if (mode < d - 1)
            ranks[t] = t <= mode ? f->x->ttRank[t] : f->x->ttRank[t + 1];
        else
            ranks[t] = t < d - 1 ? f->x->ttRank[t] : 1;
    }
    *marginal = alloc_ptt(d - 1, dims, ranks);
    ptt_tt* mx = upload(f->x);
    ptt_tt* mz = mirror((*marginal)->x, ranks);
    if (check(ptt_apply_marginal(mx, mode, row_vector, mz), "pattac_apply_marginal")) return;
    download((*marginal)->x, mz);
}

/* ------------------------------------------------------------------------ */
/* .cr files: header "r_l,N,r_r\n", then r_l*N*r_r values "%+1.16e\n" in    */
/* column-major order (paratt.c:1621-1892).                                 */
/* ------------------------------------------------------------------------ */
void pattac_write_tt_folder(char* folder, paratt* f) {
    struct stat st;
    if (stat(folder, &st) == -1) mkdir(folder, 0777);
    char name[4096];
    attac_tt* x = f->x;
    for (int k = 0; k < x->numDim; k++) {
        snprintf(name, sizeof(name), "%s/core_%d.cr", folder, k + 1);
        FILE* fp = fopen(name, "w");
        if (!fp) {
            fprintf(stderr, "\nTT write error: can't open %s\n", name);
            exit(1);
        }
        size_t cnt = (size_t)x->ttRank[k] * x->dim[k] * x->ttRank[k + 1];
        fprintf(fp, "%d,%d,%d\n", x->ttRank[k], f->dim[k], x->ttRank[k + 1]);
        for (size_t e = 0; e < cnt; e++) fprintf(fp, "%+1.16e\n", x->coreList[k][e]);
        fclose(fp);
    }
}

static int read_header(FILE* fp, int* sz) {
    char line[256];
    if (!fgets(line, sizeof(line), fp)) return -1;
    if (!strchr(line, '\n')) return -1;
    char* p = line;
    for (int i = 0; i < 3; i++) {
        char* end;
        errno = 0;
        long v = strtol(p, &end, 10);
        if (end == p || errno) return -1;
        sz[i] = (int)v;
        p = end;
        if (i < 2) {
            if (*p != ',') return -1;
            p++;
        }
    }
    return 0;
}

void read_core_size(char* fname, int* rl, int* N, int* rr) {
    FILE* fp = fopen(fname, "r");
    if (!fp) {
        fprintf(stderr, "\nread_core_size error: can't open %s\n", fname);
        return;
    }
    int sz[3];
    if (read_header(fp, sz)) {
        fprintf(stderr, "\nread_core_size error: can't read line 1.\n");
        fclose(fp);
        return;
    }
    *rl = sz[0];
    *N = sz[1];
    *rr = sz[2];
    fclose(fp);
}

void load_core_slice(char* fname, double** cr, int* cr_sz, int* rl, int* N, int* rr, int N_beg, int N_end) {
    FILE* fp = fopen(fname, "r");
    if (!fp) {
        fprintf(stderr, "\nload_core_slice error: can't open %s\n", fname);
        return;
    }
    int sz[3];
    if (read_header(fp, sz)) {
        fprintf(stderr, "\nload_core_slice error: can't read line 1.\n");
        fclose(fp);
        return;
    }
    if (N_end > sz[1] || N_beg < 0) {
        fclose(fp);
        fprintf(stderr,
                "\nload_core_slice error: slice indexes out of bounds.\nN_beg = %d, N_end = %d, core_sz[1] = %d\n",
                N_beg, N_end, sz[1]);
        return;
    }
    int need = sz[0] * (N_end - N_beg) * sz[2];
    if (*cr_sz < need) {
        double* p = (double*)realloc(*cr, sizeof(double) * (size_t)(need ? need : 1));
        if (!p) {
            fclose(fp);
            fprintf(stderr, "\nload_core_slice error: out of host memory.\n");
            exit(1);
        }
        *cr = p;
        *cr_sz = need;
    }
    *rl = sz[0];
    *N = N_end - N_beg;
    *rr = sz[2];
    int idx = 0, line = 1;
    char buf[256];
    for (int l = 0; l < sz[2]; l++)
        for (int j = 0; j < sz[1]; j++)
            for (int i = 0; i < sz[0]; i++) {
                if (!fgets(buf, sizeof(buf), fp)) {
                    fprintf(stderr, "\nload_core_slice error: can't read line %d.\n", line);
                    fclose(fp);
                    return;
                }
                if (N_beg <= j && j < N_end) (*cr)[idx++] = strtod(buf, NULL);
                line++;
            }
    fclose(fp);
}

paratt* pattac_load_tt_folder(char* folder, int ndims) {
    char name[4096];
    int* dim = (int*)xmalloc(sizeof(int) * ndims);
    int* r = (int*)xmalloc(sizeof(int) * (ndims + 1));
    int rl = 0, rr = 0, prev = 1;
    for (int k = 0; k < ndims; k++) {
        snprintf(name, sizeof(name), "%s/core_%d.cr", folder, k + 1);
        rl = rr = -1;
        read_core_size(name, &rl, &dim[k], &rr);
        if (rl != prev)
            fprintf(stderr, "%s:Line %d %s::pattac_load_tt_folder:: Bad left TT rank in file %d.\n", __FILE__,
                    __LINE__, __func__, k);
        r[k] = rl;
        prev = rr;
    }
    if (rr != 1)
        fprintf(stderr, "%s:Line %d %s::pattac_load_tt_folder:: Bad right TT rank in file %d.\n", __FILE__,
                __LINE__, __func__, ndims);
    r[0] = 1;
    r[ndims] = rr;
    paratt* p = alloc_ptt(ndims, dim, r);
    for (int k = 0; k < ndims; k++) {
        snprintf(name, sizeof(name), "%s/core_%d.cr", folder, k + 1);
        load_core_slice(name, &p->x->coreList[k], &p->x->coreMem[k], &p->x->ttRank[k], &p->x->dim[k],
                        &p->x->ttRank[k + 1], 0, dim[k]);
    }
    free(dim);
    free(r);
    return p;
}

/* ------------------------------------------------------------------------ */
/* reaction-Burgers midpoint step on host cores (extension)                 */
/* ------------------------------------------------------------------------ */
static ptt_rxn_ws* g_rxn = NULL;
static int g_rxn_d = 0, g_rxn_n = 0, g_rxn_maxr = 0;

void pattac_rxn_burgers_midpoint_st(paratt* f, double dt, double tol, int maxrank) {
    attac_tt* x = f->x;
    for (int k = 1; k < x->numDim; k++)
        if (x->dim[k] != x->dim[0]) {
            fprintf(stderr, "paratt_b200: rxn-burgers step needs one grid size for every mode\n");
            g_err = PTT_ERR_ARG;
            return;
        }
    if (!g_rxn || g_rxn_d != x->numDim || g_rxn_n != x->dim[0] || g_rxn_maxr != maxrank) {
        ptt_rxn_ws_destroy(g_rxn);
        g_rxn = ptt_rxn_ws_create(ctx(), x->numDim, x->dim, maxrank);
        if (!g_rxn) fail("rxn workspace");
        g_rxn_d = x->numDim;
        g_rxn_n = x->dim[0];
        g_rxn_maxr = maxrank;
    }
    int cap[PTT_MAX_DIM + 1];
    for (int k = 0; k <= x->numDim; k++) cap[k] = (k == 0 || k == x->numDim) ? 1 : 2 * maxrank;
    ptt_tt* m = mirror(x, cap);
    if (check(ptt_tt_set(m, x->ttRank, (const double* const*)x->coreList), "upload")) fail("upload");
    ptt_rxn_params p;
    p.dt = dt;
    p.tol = tol;
    p.nu = 0.05;
    p.L = 10.0;
    p.maxrank = maxrank;
    p.sketch_pad = 8;
    p.seed = 0x5eed;
    if (check(ptt_rxn_burgers_rk2_step(m, g_rxn, &p), "rxn-burgers step")) return;
    download(x, m);
}
