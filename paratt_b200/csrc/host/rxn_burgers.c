/*
 * Reaction-Burgers vector field and step-truncation midpoint (RK2) step on
 * device-resident tensor trains.
 *
 *   u_t = nu sum_i d2_i u - (1/d) sum_i d1_i (u^2 / 2) + u (1 - u)
 *
 * on the periodic box [-L/2, L/2)^d with second-order central differences
 * (h = L/n).  The reference has no such solver (its only driver is a
 * Burgers-Hopf CDF problem, mpi_pattac_rxn_burgers_rank_max_read_file.c);
 * the step is composed from the reference's primitives exactly as the CPU
 * oracle composes them (oracle/tt_oracle.py rxn_burgers_F / _rk2_step):
 *
 *   w = T(u . u)
 *   a = T(nu sum_i D2_i u + u)             structured rank-2r operator TT
 *   b = T(-(1/2d) sum_i D1_i w - w)
 *   F = T(a + b)
 *   midpoint (paratt_ode.h:77-112, stage rounded as well):
 *   u_s = T(u + dt/2 F(u)),  u+ = T(u + dt F(u_s))
 *
 * T = paratt_truncate semantics with an absolute tolerance.  The product
 * u . u is formed exactly at rank r_u (r_u + 1) / 2 (ptt_square_sym: the
 * same tensor as the reference's rank r_u^2 attacHadamard, restricted to
 * its symmetric subspace) while that fits the rounding kernels (<= 128),
 * and is otherwise rounded through a Gaussian TT sketch of rank
 * min(r_u^2, maxrank + sketch_pad) without forming it.
 *
 * Sketch step (ptt_rxn_burgers_rk2_step_sketch): the same step with every
 * rounding done by a Gaussian TT sketch of per-bond ranks ell[k] followed by
 * the deterministic truncation, and F = T(a + b) taken in one sketch of the
 * formal sum (no separate roundings of a and b).  A sketch is accepted when
 * each bond's truncated rank stays `pad` below its sketch rank; otherwise
 * that rounding is redone deterministically (the plain composition), and
 * the fallback is counted.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../../include/paratt_b200.h"

struct ptt_rxn_ws {
    ptt_ctx* ctx;
    int d, maxrank;
    ptt_tt *w, *a, *b, *k, *us, *s, *t;
    long long hadamard_formal, hadamard_sketch, sketch_calls, sketch_fallbacks;
    int log;
    int step_rank[PTT_MAX_DIM + 1];                   /* max kept rank per bond in this step */
    double sig[(PTT_MAX_DIM + 1) * PTT_STAT_NSIG];   /* top spectra of the last rounding */
    double delta;                                     /* its per-bond threshold */
    double stats[(PTT_MAX_DIM + 1) * PTT_STAT_LEN];
    /* the same per rounding kind (PTT_RXN_KIND_*) */
    int kind_rank[PTT_RXN_KINDS][PTT_MAX_DIM + 1];
    double kind_sig[PTT_RXN_KINDS][(PTT_MAX_DIM + 1) * PTT_STAT_NSIG];
    double kind_delta[PTT_RXN_KINDS];
};

#define KIND_NONE (-1) /* intermediate roundings of the plain F (a, b): step maximum only */

#define FORMAL_MAX 128

static ptt_tt* mk(ptt_ctx* c, int d, const int* n, int inner) {
    int cap[PTT_MAX_DIM + 1];
    for (int k = 0; k <= d; k++) cap[k] = (k == 0 || k == d) ? 1 : inner;
    return ptt_tt_create(c, d, n, cap);
}

ptt_rxn_ws* ptt_rxn_ws_create(ptt_ctx* c, int d, const int* n, int maxrank) {
    if (!c || d < 1 || d > PTT_MAX_DIM || maxrank < 1 || 2 * maxrank > 128) return NULL;
    ptt_rxn_ws* ws = (ptt_rxn_ws*)calloc(1, sizeof(ptt_rxn_ws));
    ws->ctx = c;
    ws->d = d;
    ws->maxrank = maxrank;
    ws->w = mk(c, d, n, FORMAL_MAX);
    ws->a = mk(c, d, n, 2 * maxrank);
    ws->b = mk(c, d, n, 2 * maxrank);
    ws->k = mk(c, d, n, 2 * maxrank);
    ws->us = mk(c, d, n, 2 * maxrank);
    ws->s = mk(c, d, n, 4 * maxrank);
    ws->t = mk(c, d, n, 2 * maxrank);
    if (!ws->w || !ws->a || !ws->b || !ws->k || !ws->us || !ws->s || !ws->t) {
        ptt_rxn_ws_destroy(ws);
        return NULL;
    }
    return ws;
}

void ptt_rxn_ws_destroy(ptt_rxn_ws* ws) {
    if (!ws) return;
    ptt_tt_destroy(ws->w);
    ptt_tt_destroy(ws->a);
    ptt_tt_destroy(ws->b);
    ptt_tt_destroy(ws->k);
    ptt_tt_destroy(ws->us);
    ptt_tt_destroy(ws->s);
    ptt_tt_destroy(ws->t);
    free(ws);
}

int ptt_rxn_ws_counts(const ptt_rxn_ws* ws, long long* formal, long long* sketch) {
    if (!ws) return PTT_ERR_ARG;
    if (formal) *formal = ws->hadamard_formal;
    if (sketch) *sketch = ws->hadamard_sketch;
    return PTT_OK;
}

int ptt_rxn_ws_sketch_counts(const ptt_rxn_ws* ws, long long* calls, long long* fallbacks) {
    if (!ws) return PTT_ERR_ARG;
    if (calls) *calls = ws->sketch_calls;
    if (fallbacks) *fallbacks = ws->sketch_fallbacks;
    return PTT_OK;
}

int ptt_rxn_ws_log(ptt_rxn_ws* ws, int on) {
    if (!ws) return PTT_ERR_ARG;
    ws->log = on ? 1 : 0;
    return PTT_OK;
}

int ptt_rxn_ws_last_step(const ptt_rxn_ws* ws, int* ranks, double* sig, double* delta) {
    if (!ws) return PTT_ERR_ARG;
    if (ranks) memcpy(ranks, ws->step_rank, sizeof(int) * (ws->d + 1));
    if (sig) memcpy(sig, ws->sig, sizeof(double) * (ws->d + 1) * PTT_STAT_NSIG);
    if (delta) *delta = ws->delta;
    return PTT_OK;
}

int ptt_rxn_ws_last_step_kind(const ptt_rxn_ws* ws, int kind, int* ranks, double* sig, double* delta) {
    if (!ws || kind < 0 || kind >= PTT_RXN_KINDS) return PTT_ERR_ARG;
    if (ranks) memcpy(ranks, ws->kind_rank[kind], sizeof(int) * (ws->d + 1));
    if (sig) memcpy(sig, ws->kind_sig[kind], sizeof(double) * (ws->d + 1) * PTT_STAT_NSIG);
    if (delta) *delta = ws->kind_delta[kind];
    return PTT_OK;
}

/* After a rounding of the given kind: fold its per-bond ranks into the step
 * maximum (and the kind's maximum) and keep its spectra (logging mode only:
 * reads the statistics back). */
static int logged_kind(ptt_rxn_ws* ws, int rc, int kind) {
    if (rc || !ws->log) return rc;
    const int d = ws->d;
    if ((rc = ptt_round_stats(ws->ctx, d, ws->stats))) return rc;
    for (int k = 1; k < d; k++) {
        const double* st = ws->stats + (size_t)k * PTT_STAT_LEN;
        const int r = (int)st[0];
        if (r > ws->step_rank[k]) ws->step_rank[k] = r;
        memcpy(ws->sig + (size_t)k * PTT_STAT_NSIG, st + 8, sizeof(double) * PTT_STAT_NSIG);
        ws->delta = st[6];
        if (kind >= 0) {
            if (r > ws->kind_rank[kind][k]) ws->kind_rank[kind][k] = r;
            memcpy(ws->kind_sig[kind] + (size_t)k * PTT_STAT_NSIG, st + 8, sizeof(double) * PTT_STAT_NSIG);
            ws->kind_delta[kind] = st[6];
        }
    }
    return PTT_OK;
}

static void step_begin(ptt_rxn_ws* ws) {
    for (int k = 0; k <= ws->d; k++) {
        ws->step_rank[k] = 0;
        for (int t = 0; t < PTT_RXN_KINDS; t++) ws->kind_rank[t][k] = 0;
    }
}

static void stencils(const ptt_rxn_params* p, int d, int n, double* d2, double* d1) {
    const double h = p->L / n;
    d2[0] = p->nu / (h * h);
    d2[1] = -2.0 * p->nu / (h * h);
    d2[2] = p->nu / (h * h);
    /* -(1/d) d1(u^2/2) = -(1/(2d)) d1(u*u); d1 = [-1, 0, 1]/(2h) */
    d1[0] = 1.0 / (4.0 * d * h);
    d1[1] = 0.0;
    d1[2] = -1.0 / (4.0 * d * h);
}

static int shape(ptt_tt* u, int* d, int* n) {
    int rc = ptt_tt_shape(u, d, n, NULL);
    if (rc) return rc;
    for (int k = 1; k < *d; k++)
        if (n[k] != n[0]) return PTT_ERR_ARG; /* one grid for every mode */
    return PTT_OK;
}

/* w = T(u . u): exact symmetric square while r(r+1)/2 fits, else through a sketch of rank ell. */
static int product(ptt_tt* u, ptt_rxn_ws* ws, const ptt_rxn_params* p, const int* mr, const int* ell_sketch) {
    int rc, r[PTT_MAX_DIM + 1], d = ws->d;
    if ((rc = ptt_tt_get_ranks(u, r))) return rc;
    int rmax = 1;
    for (int k = 0; k <= d; k++) rmax = r[k] > rmax ? r[k] : rmax;
    if (!ell_sketch && rmax * (rmax + 1) / 2 <= FORMAL_MAX) {
        if ((rc = ptt_square_sym(u, ws->w))) return rc;
        ws->hadamard_formal++;
        return logged_kind(ws, ptt_round(ws->w, p->tol, mr), PTT_RXN_KIND_PRODUCT);
    }
    int ell[PTT_MAX_DIM + 1];
    for (int k = 0; k <= d; k++) ell[k] = ell_sketch ? ell_sketch[k] : p->maxrank + p->sketch_pad;
    ws->hadamard_sketch++;
    return logged_kind(ws, ptt_round_hadamard(u, u, ws->w, ell, p->seed, p->tol, mr), PTT_RXN_KIND_PRODUCT);
}

int ptt_rxn_burgers_F(ptt_tt* u, ptt_tt* F, ptt_rxn_ws* ws, const ptt_rxn_params* p) {
    int rc, d, n[PTT_MAX_DIM], mr[PTT_MAX_DIM + 1];
    if (!u || !F || !ws || !p) return PTT_ERR_ARG;
    if ((rc = shape(u, &d, n))) return rc;
    for (int k = 0; k <= d; k++) mr[k] = p->maxrank;
    double d2[3], d1[3];
    stencils(p, d, n[0], d2, d1);
    if ((rc = product(u, ws, p, mr, NULL))) return rc;
    if ((rc = ptt_op_sum(u, d2, 3, 1.0, ws->a))) return rc;
    if ((rc = logged_kind(ws, ptt_round(ws->a, p->tol, mr), KIND_NONE))) return rc;
    if ((rc = ptt_op_sum(ws->w, d1, 3, -1.0, ws->b))) return rc;
    if ((rc = logged_kind(ws, ptt_round(ws->b, p->tol, mr), KIND_NONE))) return rc;
    if ((rc = ptt_axpby(1.0, ws->a, 1.0, ws->b, F))) return rc;
    return logged_kind(ws, ptt_round(F, p->tol, mr), PTT_RXN_KIND_FIELD);
}

int ptt_rxn_burgers_rk2_step(ptt_tt* u, ptt_rxn_ws* ws, const ptt_rxn_params* p) {
    int rc, d, mr[PTT_MAX_DIM + 1];
    if (!u || !ws || !p) return PTT_ERR_ARG;
    if ((rc = ptt_tt_shape(u, &d, NULL, NULL))) return rc;
    for (int k = 0; k <= d; k++) mr[k] = p->maxrank;
    step_begin(ws);
    if ((rc = ptt_rxn_burgers_F(u, ws->k, ws, p))) return rc;
    if ((rc = ptt_axpby(1.0, u, 0.5 * p->dt, ws->k, ws->us))) return rc;
    if ((rc = logged_kind(ws, ptt_round(ws->us, p->tol, mr), PTT_RXN_KIND_STAGE))) return rc;
    if ((rc = ptt_rxn_burgers_F(ws->us, ws->k, ws, p))) return rc;
    if ((rc = ptt_axpby(1.0, u, p->dt, ws->k, u))) return rc;
    return logged_kind(ws, ptt_round(u, p->tol, mr), PTT_RXN_KIND_STAGE);
}

/* ------------------------------------------------------------------------ */
/* sketch step                                                              */
/* ------------------------------------------------------------------------ */

/* dst <- T(src) by a sketch of ranks ell (src != dst); on rejection
 * deterministic rounding of src in place and copy.  src must fit the
 * deterministic kernels (rank <= 128) for the fallback. */
static int sketch_or_round(ptt_tt* src, ptt_tt* dst, ptt_rxn_ws* ws, const ptt_rxn_params* p, const int* mr,
                           const int* ell, int pad, unsigned long long salt) {
    int ok = 0, rc;
    ws->sketch_calls++;
    rc = logged_kind(ws, ptt_round_sketch(src, NULL, dst, ell, p->seed ^ salt, p->tol, mr, pad, &ok),
                     PTT_RXN_KIND_STAGE);
    if (rc) return rc;
    if (ok) return PTT_OK;
    ws->sketch_fallbacks++;
    if ((rc = logged_kind(ws, ptt_round(src, p->tol, mr), PTT_RXN_KIND_STAGE))) return rc;
    return ptt_tt_copy(dst, src);
}

static int F_sketch(ptt_tt* u, ptt_tt* F, ptt_rxn_ws* ws, const ptt_rxn_params* p, const int* ell_prod,
                    const int* ell_field, int pad, unsigned long long salt) {
    int rc, d, n[PTT_MAX_DIM], mr[PTT_MAX_DIM + 1];
    if ((rc = shape(u, &d, n))) return rc;
    for (int k = 0; k <= d; k++) mr[k] = p->maxrank;
    double d2[3], d1[3];
    stencils(p, d, n[0], d2, d1);
    /* product: sketch of rank ell, with the fixed-rank sketch as fallback */
    {
        int ok = 0, r[PTT_MAX_DIM + 1], full[PTT_MAX_DIM + 1];
        if ((rc = ptt_tt_get_ranks(u, r))) return rc;
        for (int k = 0; k <= d; k++) full[k] = r[k] * r[k];
        ws->sketch_calls++;
        ws->hadamard_sketch++;
        rc = logged_kind(ws, ptt_round_sketch(u, u, ws->w, ell_prod, p->seed ^ (salt * 7 + 1), p->tol, mr, pad, &ok),
                         PTT_RXN_KIND_PRODUCT);
        if (rc) return rc;
        if (!ok) {
            ws->sketch_fallbacks++;
            if ((rc = product(u, ws, p, mr, NULL))) return rc;
        }
        (void)full;
    }
    if ((rc = ptt_op_sum(u, d2, 3, 1.0, ws->a))) return rc;
    if ((rc = ptt_op_sum(ws->w, d1, 3, -1.0, ws->b))) return rc;
    if ((rc = ptt_axpby(1.0, ws->a, 1.0, ws->b, ws->s))) return rc;
    int ok = 0;
    ws->sketch_calls++;
    rc = logged_kind(ws, ptt_round_sketch(ws->s, NULL, F, ell_field, p->seed ^ (salt * 7 + 2), p->tol, mr, pad, &ok),
                     PTT_RXN_KIND_FIELD);
    if (rc) return rc;
    if (ok) return PTT_OK;
    /* fallback: the deterministic composition T(T(a) + T(b)) */
    ws->sketch_fallbacks++;
    if ((rc = logged_kind(ws, ptt_round(ws->a, p->tol, mr), KIND_NONE))) return rc;
    if ((rc = logged_kind(ws, ptt_round(ws->b, p->tol, mr), KIND_NONE))) return rc;
    if ((rc = ptt_axpby(1.0, ws->a, 1.0, ws->b, F))) return rc;
    return logged_kind(ws, ptt_round(F, p->tol, mr), PTT_RXN_KIND_FIELD);
}

int ptt_rxn_burgers_rk2_step_sketch_kinds(ptt_tt* u, ptt_rxn_ws* ws, const ptt_rxn_params* p, const int* ell,
                                          int pad) {
    int rc, d, mr[PTT_MAX_DIM + 1];
    if (!u || !ws || !p || !ell) return PTT_ERR_ARG;
    if ((rc = ptt_tt_shape(u, &d, NULL, NULL))) return rc;
    for (int k = 0; k <= d; k++) mr[k] = p->maxrank;
    const int* ep = ell + (size_t)PTT_RXN_KIND_PRODUCT * (d + 1);
    const int* ef = ell + (size_t)PTT_RXN_KIND_FIELD * (d + 1);
    const int* es = ell + (size_t)PTT_RXN_KIND_STAGE * (d + 1);
    step_begin(ws);
    if ((rc = F_sketch(u, ws->k, ws, p, ep, ef, pad, 1))) return rc;
    if ((rc = ptt_axpby(1.0, u, 0.5 * p->dt, ws->k, ws->t))) return rc;
    if ((rc = sketch_or_round(ws->t, ws->us, ws, p, mr, es, pad, 3))) return rc;
    if ((rc = F_sketch(ws->us, ws->k, ws, p, ep, ef, pad, 4))) return rc;
    if ((rc = ptt_axpby(1.0, u, p->dt, ws->k, ws->t))) return rc;
    return sketch_or_round(ws->t, u, ws, p, mr, es, pad, 5);
}

int ptt_rxn_burgers_rk2_step_sketch(ptt_tt* u, ptt_rxn_ws* ws, const ptt_rxn_params* p, const int* ell, int pad) {
    int d, rc;
    if (!u || !ws || !p || !ell) return PTT_ERR_ARG;
    if ((rc = ptt_tt_shape(u, &d, NULL, NULL))) return rc;
    int all[PTT_RXN_KINDS * (PTT_MAX_DIM + 1)];
    for (int t = 0; t < PTT_RXN_KINDS; t++) memcpy(all + (size_t)t * (d + 1), ell, sizeof(int) * (d + 1));
    return ptt_rxn_burgers_rk2_step_sketch_kinds(u, ws, p, all, pad);
}
