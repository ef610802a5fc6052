/*
 * Step-truncation integrators of paratt_ode.h.
 *
 *  euler     pattac_exp_euler_st (paratt_ode.c:25-36), attac twin (12-23)
 *  midpoint  attac_exp_midpoint_st, documented at paratt_ode.h:77-112 and
 *            never defined by the reference; composed here from the same
 *            primitives.
 */
#include "../../../include/paratt_ode.h"

void attac_exp_euler_st(attac_tt* f_old, attac_tt* f_new, attac_tt* work,
                        void (*vecField)(attac_tt*, attac_tt*, int, ...), double dt, double eps_1, double eps_2) {
    vecField(f_old, work, 0);
    attac_tt_truncate(work, eps_1, work->ttRank);
    attac_tt_axpby(1.0, f_old, dt, work, f_new);
    attac_tt_truncate(f_new, eps_2, f_new->ttRank);
}

void pattac_exp_euler_st(paratt* f_old, paratt* f_new, paratt* work, void (*vecField)(paratt*, paratt*, int, ...),
                         double dt, double eps_1, double eps_2) {
    vecField(f_old, work, 0);
    paratt_truncate(work, eps_1, work->x->ttRank);
    attac_tt_axpby(1.0, f_old->x, dt, work->x, f_new->x);
    paratt_truncate(f_new, eps_2, f_new->x->ttRank);
}

/* f_s   = T1(f_old + dt/2 * T1(F(f_old)))   (stage kept in f_new)
 * f_new = T3(f_old + dt * T2(F(f_s)))                                    */
void attac_exp_midpoint_st(attac_tt* f_old, attac_tt* f_new, attac_tt* work,
                           void (*vecField)(attac_tt*, attac_tt*, int, ...), double dt, double eps_1, double eps_2,
                           double eps_3) {
    vecField(f_old, work, 0);
    attac_tt_truncate(work, eps_1, work->ttRank);
    attac_tt_axpby(1.0, f_old, 0.5 * dt, work, f_new);
    attac_tt_truncate(f_new, eps_1, f_new->ttRank);
    vecField(f_new, work, 0);
    attac_tt_truncate(work, eps_2, work->ttRank);
    attac_tt_axpby(1.0, f_old, dt, work, f_new);
    attac_tt_truncate(f_new, eps_3, f_new->ttRank);
}

void pattac_exp_midpoint_st(paratt* f_old, paratt* f_new, paratt* work, void (*vecField)(paratt*, paratt*, int, ...),
                            double dt, double eps_1, double eps_2, double eps_3) {
    vecField(f_old, work, 0);
    paratt_truncate(work, eps_1, work->x->ttRank);
    attac_tt_axpby(1.0, f_old->x, 0.5 * dt, work->x, f_new->x);
    paratt_truncate(f_new, eps_1, f_new->x->ttRank);
    vecField(f_new, work, 0);
    paratt_truncate(work, eps_2, work->x->ttRank);
    attac_tt_axpby(1.0, f_old->x, dt, work->x, f_new->x);
    paratt_truncate(f_new, eps_3, f_new->x->ttRank);
}
