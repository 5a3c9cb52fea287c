/*
 * pdhg_oracle.h - TEST INFRASTRUCTURE. The CPU checker of the B200 PDHG
 * engine: a plain-C restatement of the reference's FP64 first-order LP path
 * (anukulan src/anukulan/pdhg.cpp, scaling.cpp, sparse.cpp, backend.cpp).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library, and only to check or to time the reference algorithm on the
 * host. The engine never links, loads or calls it.
 *
 * Pinning: the restatement reproduces the reference's operation order (serial
 * left-to-right sums, the same fmin/fmax/sqrt/log/exp calls, no FMA
 * contraction), so on identical inputs its iterates, iteration and restart
 * counts and objectives are bit-identical to the reference built from its own
 * sources (oracle/_ref); tests/test_oracle_pin.py checks that.
 */
#ifndef PDHG_ORACLE_H
#define PDHG_ORACLE_H

#include "../include/anu_pdhg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* solve_pdhg (pdhg.cpp:377-1285) with cpu_backend() semantics. */
int oracle_pdhg_solve(const anu_lp* lp, const anu_pdhg_options* options,
                      const double* warm_x, const double* warm_y, double* x,
                      double* y, anu_pdhg_result* result);

/* evaluate_residual (pdhg.cpp:112-174). */
void oracle_evaluate_residual(const anu_lp* lp, const double* x, const double* y,
                              anu_pdhg_residual* out);

/* estimate_matrix_norm (pdhg.cpp:223-282); scaled != 0 applies scale_lp with
 * default options first (what solve_pdhg measures). */
double oracle_estimate_matrix_norm(const anu_lp* lp, int iterations,
                                   double tolerance, int scaled);

/* scale_lp (scaling.cpp:75-100). Outputs as in ref_scale_lp. */
int oracle_scale_lp(const anu_lp* lp, int ruiz_iterations, int pock_chambolle,
                    double* k_value, double* c, double* q, double* lower,
                    double* upper, double* row_scale, double* col_scale,
                    double* spreads);

/* Runs the same solve on `count` independent LPs with `threads` worker
 * threads (one LP per thread at a time), for the CPU baseline of a case
 * stack. x and y are concatenated per LP. */
int oracle_pdhg_solve_many(int count, const anu_lp* lps,
                           const anu_pdhg_options* options, int threads,
                           double* const* xs, double* const* ys,
                           anu_pdhg_result* results);

#ifdef __cplusplus
}
#endif

#endif
