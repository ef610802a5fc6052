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
 * u . u is formed formally (attacHadamard) while r_u^2 fits the rounding
 * kernels (<= 128) and is otherwise rounded through a Gaussian TT sketch of
 * rank min(r_u^2, maxrank + sketch_pad) without forming it.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../../include/paratt_b200.h"

struct ptt_rxn_ws {
    ptt_ctx* ctx;
    int d;
    ptt_tt *w, *a, *b, *k, *us;
    long long hadamard_formal, hadamard_sketch;
};

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
    ws->w = mk(c, d, n, FORMAL_MAX);
    ws->a = mk(c, d, n, 2 * maxrank);
    ws->b = mk(c, d, n, 2 * maxrank);
    ws->k = mk(c, d, n, 2 * maxrank);
    ws->us = mk(c, d, n, 2 * maxrank);
    if (!ws->w || !ws->a || !ws->b || !ws->k || !ws->us) {
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
    free(ws);
}

int ptt_rxn_ws_counts(const ptt_rxn_ws* ws, long long* formal, long long* sketch) {
    if (!ws) return PTT_ERR_ARG;
    if (formal) *formal = ws->hadamard_formal;
    if (sketch) *sketch = ws->hadamard_sketch;
    return PTT_OK;
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

int ptt_rxn_burgers_F(ptt_tt* u, ptt_tt* F, ptt_rxn_ws* ws, const ptt_rxn_params* p) {
    int rc, d, n[PTT_MAX_DIM], r[PTT_MAX_DIM + 1], mr[PTT_MAX_DIM + 1];
    if (!u || !F || !ws || !p) return PTT_ERR_ARG;
    if ((rc = ptt_tt_shape(u, &d, n, NULL))) return rc;
    for (int k = 1; k < d; k++)
        if (n[k] != n[0]) return PTT_ERR_ARG; /* one grid for every mode */
    for (int k = 0; k <= d; k++) mr[k] = p->maxrank;
    double d2[3], d1[3];
    stencils(p, d, n[0], d2, d1);
    if ((rc = ptt_tt_get_ranks(u, r))) return rc;
    int rmax = 1;
    for (int k = 0; k <= d; k++) rmax = r[k] > rmax ? r[k] : rmax;
    if (rmax * rmax <= FORMAL_MAX) {
        if ((rc = ptt_hadamard(u, u, ws->w))) return rc;
        if ((rc = ptt_round(ws->w, p->tol, mr))) return rc;
        ws->hadamard_formal++;
    } else {
        int ell[PTT_MAX_DIM + 1];
        for (int k = 0; k <= d; k++) ell[k] = p->maxrank + p->sketch_pad;
        if ((rc = ptt_round_hadamard(u, u, ws->w, ell, p->seed, p->tol, mr))) return rc;
        ws->hadamard_sketch++;
    }
    if ((rc = ptt_op_sum(u, d2, 3, 1.0, ws->a))) return rc;
    if ((rc = ptt_round(ws->a, p->tol, mr))) return rc;
    if ((rc = ptt_op_sum(ws->w, d1, 3, -1.0, ws->b))) return rc;
    if ((rc = ptt_round(ws->b, p->tol, mr))) return rc;
    if ((rc = ptt_axpby(1.0, ws->a, 1.0, ws->b, F))) return rc;
    return ptt_round(F, p->tol, mr);
}

int ptt_rxn_burgers_rk2_step(ptt_tt* u, ptt_rxn_ws* ws, const ptt_rxn_params* p) {
    int rc, d, mr[PTT_MAX_DIM + 1];
    if (!u || !ws || !p) return PTT_ERR_ARG;
    if ((rc = ptt_tt_shape(u, &d, NULL, NULL))) return rc;
    for (int k = 0; k <= d; k++) mr[k] = p->maxrank;
    if ((rc = ptt_rxn_burgers_F(u, ws->k, ws, p))) return rc;
    if ((rc = ptt_axpby(1.0, u, 0.5 * p->dt, ws->k, ws->us))) return rc;
    if ((rc = ptt_round(ws->us, p->tol, mr))) return rc;
    if ((rc = ptt_rxn_burgers_F(ws->us, ws->k, ws, p))) return rc;
    if ((rc = ptt_axpby(1.0, u, p->dt, ws->k, u))) return rc;
    return ptt_round(u, p->tol, mr);
}
