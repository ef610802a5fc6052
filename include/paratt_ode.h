/*
 * paratt_ode.h -- step-truncation ODE integrators (source/paratt_ode.h:61-120).
 *
 *   euler:    f_new = T2( f_old + dt * T1( F(f_old) ) )
 *   midpoint: f_s   = T1'( f_old + dt/2 * T1( F(f_old) ) )
 *             f_new = T3( f_old + dt * T2( F(f_s) ) )
 * where Tk rounds with tolerance eps_k (paratt_truncate semantics).
 *
 * The reference declares the midpoint integrator but never defines it
 * (paratt_ode.h:113-120 vs paratt_ode.c:1-37); it is defined here from its
 * documentation, with one addition: the stage f_s is rounded with eps_1
 * (T1') so the vector field, whose nonlinear term squares the rank, is never
 * evaluated on an unrounded sum.
 */
#ifndef PARATT_ODE_SOLVE_H
#define PARATT_ODE_SOLVE_H

#include <stdarg.h>
#include <stdlib.h>

#include "paratt.h"

#ifdef __cplusplus
extern "C" {
#endif

void attac_exp_euler_st(attac_tt* f_old_tt, attac_tt* f_new_tt, attac_tt* work_tt,
                        void (*vecField)(attac_tt*, attac_tt*, int, ...), double dt, double eps_1,
                        double eps_2);

void pattac_exp_euler_st(paratt* f_old_ptt, paratt* f_new_ptt, paratt* work_ptt,
                         void (*vecField)(paratt*, paratt*, int, ...), double dt, double eps_1,
                         double eps_2);

void attac_exp_midpoint_st(attac_tt* f_old_tt, attac_tt* f_new_tt, attac_tt* work_tt,
                           void (*vecField)(attac_tt*, attac_tt*, int, ...), double dt, double eps_1,
                           double eps_2, double eps_3);

void pattac_exp_midpoint_st(paratt* f_old_ptt, paratt* f_new_ptt, paratt* work_ptt,
                            void (*vecField)(paratt*, paratt*, int, ...), double dt, double eps_1,
                            double eps_2, double eps_3);

/* Extension: one step-truncation midpoint step of the reaction-Burgers
 * equation u_t = 0.05 lap u - (1/d) sum_i d_i(u^2/2) + u(1-u) on the periodic
 * box [-5,5)^d (second-order central differences), in place on f's host
 * cores; tol is absolute (paratt_truncate semantics) for every rounding.
 * The vector field and step are listed in paratt_b200/csrc/host/rxn_burgers.c. */
void pattac_rxn_burgers_midpoint_st(paratt* f, double dt, double tol, int maxrank);

#ifdef __cplusplus
}
#endif
#endif
