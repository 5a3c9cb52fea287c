/*
 * pdhg_oracle.c - TEST INFRASTRUCTURE: the CPU checker of the B200 PDHG
 * engine. A restatement in C of the reference's FP64 first-order LP path:
 *
 *   CSR product / transpose / norms  src/anukulan/sparse.cpp:72-146
 *   diagonal scaling                 src/anukulan/scaling.cpp:32-100
 *   cpu_backend operations           src/anukulan/backend.cpp:9-202
 *   evaluate_residual                src/anukulan/pdhg.cpp:112-174
 *   is_infeasibility_certificate     src/anukulan/pdhg.cpp:191-221
 *   estimate_matrix_norm             src/anukulan/pdhg.cpp:223-282
 *   weighted_kkt_error               src/anukulan/pdhg.cpp:295-340
 *   polishing sub-problems           src/anukulan/pdhg.cpp:350-368
 *   solve_pdhg                       src/anukulan/pdhg.cpp:377-1285
 *
 * Every sum is serial and left to right and every comparison is the
 * reference's, so the results are bit-identical to the reference compiled
 * without FMA contraction (this file is built with -ffp-contract=off).
 * Only the tests and the CPU leg of the benchmark use this file.
 */
#define _POSIX_C_SOURCE 200809L
#include "pdhg_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ------------------------------------------------------------------ CSR */

typedef struct {
  int32_t rows, cols, nnz;
  int32_t* start;
  int32_t* index;
  double* value;
} ocsr;

typedef struct {
  ocsr k, kt;
  double *c, *q, *lower, *upper;
  int32_t num_eq;
  double obj_scale, obj_offset;
} olp;

static double* vzero(int64_t n) { return (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }
static double* vdup(const double* a, int64_t n) {
  double* p = vzero(n);
  if (n > 0) memcpy(p, a, (size_t)n * sizeof(double));
  return p;
}

static void csr_free(ocsr* a) {
  free(a->start);
  free(a->index);
  free(a->value);
  memset(a, 0, sizeof(*a));
}

static void csr_copy(const ocsr* a, ocsr* out) {
  out->rows = a->rows;
  out->cols = a->cols;
  out->nnz = a->nnz;
  out->start = (int32_t*)malloc(sizeof(int32_t) * (size_t)(a->rows + 1));
  memcpy(out->start, a->start, sizeof(int32_t) * (size_t)(a->rows + 1));
  out->index = (int32_t*)malloc(sizeof(int32_t) * (size_t)(a->nnz > 0 ? a->nnz : 1));
  out->value = vzero(a->nnz);
  if (a->nnz > 0) {
    memcpy(out->index, a->index, sizeof(int32_t) * (size_t)a->nnz);
    memcpy(out->value, a->value, sizeof(double) * (size_t)a->nnz);
  }
}

/* y = A x, each row summed left to right (sparse.cpp:72-80). */
static void csr_multiply(const ocsr* a, const double* x, double* y) {
  for (int32_t r = 0; r < a->rows; ++r) {
    double sum = 0.0;
    for (int32_t k = a->start[r]; k < a->start[r + 1]; ++k) sum += a->value[k] * x[a->index[k]];
    y[r] = sum;
  }
}

/* Counting-sort transpose (sparse.cpp:93-117): rows visited in increasing
 * order, so every transposed row comes out sorted. */
static void csr_transpose(const ocsr* a, ocsr* t) {
  t->rows = a->cols;
  t->cols = a->rows;
  t->nnz = a->nnz;
  t->start = (int32_t*)calloc((size_t)a->cols + 1, sizeof(int32_t));
  t->index = (int32_t*)malloc(sizeof(int32_t) * (size_t)(a->nnz > 0 ? a->nnz : 1));
  t->value = vzero(a->nnz);
  for (int32_t k = 0; k < a->nnz; ++k) t->start[a->index[k] + 1]++;
  for (int32_t i = 1; i <= a->cols; ++i) t->start[i] += t->start[i - 1];
  int32_t* cursor = (int32_t*)malloc(sizeof(int32_t) * (size_t)(a->cols > 0 ? a->cols : 1));
  if (a->cols > 0) memcpy(cursor, t->start, sizeof(int32_t) * (size_t)a->cols);
  for (int32_t r = 0; r < a->rows; ++r) {
    for (int32_t k = a->start[r]; k < a->start[r + 1]; ++k) {
      const int32_t dest = cursor[a->index[k]]++;
      t->index[dest] = r;
      t->value[dest] = a->value[k];
    }
  }
  free(cursor);
}

/* row_norms / col_norms (sparse.cpp:119-138): infinity norm or 1-norm. */
static void csr_row_norms(const ocsr* a, int one_norm, double* out) {
  for (int32_t r = 0; r < a->rows; ++r) {
    double acc = 0.0;
    for (int32_t k = a->start[r]; k < a->start[r + 1]; ++k) {
      const double v = fabs(a->value[k]);
      acc = one_norm ? acc + v : fmax(acc, v);
    }
    out[r] = acc;
  }
}

static void csr_col_norms(const ocsr* a, int one_norm, double* out) {
  for (int32_t c = 0; c < a->cols; ++c) out[c] = 0.0;
  for (int32_t k = 0; k < a->nnz; ++k) {
    const double v = fabs(a->value[k]);
    double* acc = &out[a->index[k]];
    *acc = one_norm ? *acc + v : fmax(*acc, v);
  }
}

static void olp_from_anu(const anu_lp* in, olp* lp) {
  memset(lp, 0, sizeof(*lp));
  lp->k.rows = in->k.rows;
  lp->k.cols = in->k.cols;
  lp->k.nnz = in->k.nnz;
  lp->k.start = (int32_t*)malloc(sizeof(int32_t) * (size_t)(in->k.rows + 1));
  memcpy(lp->k.start, in->k.start, sizeof(int32_t) * (size_t)(in->k.rows + 1));
  lp->k.index = (int32_t*)malloc(sizeof(int32_t) * (size_t)(in->k.nnz > 0 ? in->k.nnz : 1));
  lp->k.value = vzero(in->k.nnz);
  if (in->k.nnz > 0) {
    memcpy(lp->k.index, in->k.index, sizeof(int32_t) * (size_t)in->k.nnz);
    memcpy(lp->k.value, in->k.value, sizeof(double) * (size_t)in->k.nnz);
  }
  csr_transpose(&lp->k, &lp->kt);
  lp->c = vdup(in->c, in->k.cols);
  lp->q = vdup(in->q, in->k.rows);
  lp->lower = vdup(in->lower, in->k.cols);
  lp->upper = vdup(in->upper, in->k.cols);
  lp->num_eq = in->num_equalities;
  lp->obj_scale = in->objective_scale;
  lp->obj_offset = in->objective_offset;
}

static void olp_copy(const olp* a, olp* out) {
  memset(out, 0, sizeof(*out));
  csr_copy(&a->k, &out->k);
  csr_copy(&a->kt, &out->kt);
  out->c = vdup(a->c, a->k.cols);
  out->q = vdup(a->q, a->k.rows);
  out->lower = vdup(a->lower, a->k.cols);
  out->upper = vdup(a->upper, a->k.cols);
  out->num_eq = a->num_eq;
  out->obj_scale = a->obj_scale;
  out->obj_offset = a->obj_offset;
}

static void olp_free(olp* lp) {
  csr_free(&lp->k);
  csr_free(&lp->kt);
  free(lp->c);
  free(lp->q);
  free(lp->lower);
  free(lp->upper);
  memset(lp, 0, sizeof(*lp));
}

/* --------------------------------------------------- vector arithmetic */

static double vdot(const double* a, const double* b, int64_t n) {
  double s = 0.0;
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}
static double vnorm2(const double* a, int64_t n) { return sqrt(vdot(a, a, n)); }
static double vnorminf(const double* a, int64_t n) {
  double m = 0.0;
  for (int64_t i = 0; i < n; ++i) m = fmax(m, fabs(a[i]));
  return m;
}

static double standard_objective(const olp* lp, const double* x) {
  double s = 0.0;
  for (int32_t j = 0; j < lp->k.cols; ++j) s += lp->c[j] * x[j];
  return s;
}
static double model_objective(const olp* lp, const double* x) {
  return lp->obj_scale * standard_objective(lp, x) + lp->obj_offset;
}

/* --------------------------------------------------------- scaling */

typedef struct {
  double* row_scale;
  double* col_scale;
  double spreads[4];
} oscaling;

static double spread_of(const double* v, int64_t n) {
  double lo = INFINITY, hi = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    if (v[i] <= 0.0) continue;
    lo = fmin(lo, v[i]);
    hi = fmax(hi, v[i]);
  }
  if (hi == 0.0) return 1.0;
  return hi / lo;
}

/* One equilibration sweep (scaling.cpp:32-59). */
static void equilibrate(olp* lp, int one_norm, oscaling* acc) {
  const int32_t m = lp->k.rows, n = lp->k.cols;
  double* rn = vzero(m);
  double* cn = vzero(n);
  csr_row_norms(&lp->k, one_norm, rn);
  csr_col_norms(&lp->k, one_norm, cn);
  double* d1 = vzero(m);
  double* d2 = vzero(n);
  for (int32_t i = 0; i < m; ++i) d1[i] = (rn[i] > 0.0) ? 1.0 / sqrt(rn[i]) : 1.0;
  for (int32_t j = 0; j < n; ++j) d2[j] = (cn[j] > 0.0) ? 1.0 / sqrt(cn[j]) : 1.0;
  for (int32_t r = 0; r < m; ++r)
    for (int32_t k = lp->k.start[r]; k < lp->k.start[r + 1]; ++k) lp->k.value[k] *= d1[r];
  for (int32_t k = 0; k < lp->k.nnz; ++k) lp->k.value[k] *= d2[lp->k.index[k]];
  for (int32_t i = 0; i < m; ++i) {
    lp->q[i] *= d1[i];
    acc->row_scale[i] *= d1[i];
  }
  for (int32_t j = 0; j < n; ++j) {
    lp->c[j] *= d2[j];
    lp->lower[j] /= d2[j];
    lp->upper[j] /= d2[j];
    acc->col_scale[j] *= d2[j];
  }
  free(rn);
  free(cn);
  free(d1);
  free(d2);
}

/* scale_lp (scaling.cpp:75-100); rebuilds kt afterwards. */
static void scale_lp(olp* lp, int ruiz, int pc, oscaling* s) {
  const int32_t m = lp->k.rows, n = lp->k.cols;
  s->row_scale = vzero(m);
  s->col_scale = vzero(n);
  for (int32_t i = 0; i < m; ++i) s->row_scale[i] = 1.0;
  for (int32_t j = 0; j < n; ++j) s->col_scale[j] = 1.0;
  double* rn = vzero(m);
  double* cn = vzero(n);
  csr_row_norms(&lp->k, 0, rn);
  csr_col_norms(&lp->k, 0, cn);
  s->spreads[0] = spread_of(rn, m);
  s->spreads[2] = spread_of(cn, n);
  for (int it = 0; it < ruiz; ++it) equilibrate(lp, 0, s);
  if (pc) equilibrate(lp, 1, s);
  csr_row_norms(&lp->k, 0, rn);
  csr_col_norms(&lp->k, 0, cn);
  s->spreads[1] = spread_of(rn, m);
  s->spreads[3] = spread_of(cn, n);
  free(rn);
  free(cn);
  csr_free(&lp->kt);
  csr_transpose(&lp->k, &lp->kt);
}

static void scaling_free(oscaling* s) {
  free(s->row_scale);
  free(s->col_scale);
}

/* ------------------------------------------------ residual evaluation */

static void residual_terms_to(anu_pdhg_residual* r, double q_two, double c_two, double q_inf,
                              double c_inf) {
  r->relative_primal = r->primal_residual / (1.0 + q_two);
  r->relative_dual = r->dual_residual / (1.0 + c_two);
  r->relative_primal_inf = r->primal_residual_inf / (1.0 + q_inf);
  r->relative_dual_inf = r->dual_residual_inf / (1.0 + c_inf);
  r->relative_gap = r->absolute_gap / (1.0 + fabs(r->primal_objective) + fabs(r->dual_objective));
}

/* evaluate_residual (pdhg.cpp:112-174) with both products computed here. */
static void evaluate_residual(const olp* lp, const double* x, const double* y,
                              anu_pdhg_residual* r) {
  const int32_t m = lp->k.rows, n = lp->k.cols;
  memset(r, 0, sizeof(*r));
  double* kx = vzero(m);
  csr_multiply(&lp->k, x, kx);
  double sum_sq = 0.0, worst = 0.0;
  for (int32_t i = 0; i < m; ++i) {
    const double row = kx[i];
    const double violation = (i < lp->num_eq) ? (row - lp->q[i]) : fmin(row - lp->q[i], 0.0);
    sum_sq += violation * violation;
    worst = fmax(worst, fabs(violation));
  }
  r->primal_residual = sqrt(sum_sq);
  r->primal_residual_inf = worst;
  double* kty = vzero(n);
  csr_multiply(&lp->kt, y, kty);
  double dual_sq = 0.0, bound_term = 0.0;
  for (int32_t j = 0; j < n; ++j) {
    const int has_lo = lp->lower[j] > -INFINITY;
    const int has_hi = lp->upper[j] < INFINITY;
    const double l = lp->c[j] - kty[j];
    double leftover = 0.0;
    if (has_lo && has_hi) leftover = 0.0;
    else if (has_lo) leftover = fmin(l, 0.0);
    else if (has_hi) leftover = fmax(l, 0.0);
    else leftover = l;
    dual_sq += leftover * leftover;
    r->dual_residual_inf = fmax(r->dual_residual_inf, fabs(leftover));
    const double absorbed = l - leftover;
    if (absorbed > 0.0) bound_term += absorbed * lp->lower[j];
    else if (absorbed < 0.0) bound_term += absorbed * lp->upper[j];
  }
  r->dual_residual = sqrt(dual_sq);
  r->primal_objective = standard_objective(lp, x);
  r->dual_objective = vdot(lp->q, y, m) + bound_term;
  r->absolute_gap = fabs(r->primal_objective - r->dual_objective);
  residual_terms_to(r, vnorm2(lp->q, m), vnorm2(lp->c, n), vnorminf(lp->q, m),
                    vnorminf(lp->c, n));
  free(kx);
  free(kty);
}

static int residual_primal_ok(const anu_pdhg_residual* r, double tol, double abs_tol, int inf) {
  int ok = r->relative_primal <= tol;
  if (inf) ok = ok && r->relative_primal_inf <= tol;
  if (abs_tol > 0.0) ok = ok && r->primal_residual_inf <= abs_tol;
  return ok;
}
static int residual_dual_ok(const anu_pdhg_residual* r, double tol, double abs_tol, int inf) {
  int ok = r->relative_dual <= tol;
  if (inf) ok = ok && r->relative_dual_inf <= tol;
  if (abs_tol > 0.0) ok = ok && r->dual_residual_inf <= abs_tol;
  return ok;
}
static int residual_converged(const anu_pdhg_residual* r, double tol, double abs_tol, int inf,
                              double gap_tol) {
  return residual_primal_ok(r, tol, abs_tol, inf) && residual_dual_ok(r, tol, abs_tol, inf) &&
         r->relative_gap <= (gap_tol > 0.0 ? gap_tol : tol);
}

/* Farkas test on the dual iterate difference (pdhg.cpp:191-221). */
static int is_infeasibility_certificate(const olp* lp, const double* dy, double tol,
                                        double* work) {
  double scale = 0.0;
  for (int32_t i = 0; i < lp->k.rows; ++i) {
    if (i >= lp->num_eq && dy[i] < 0.0) return 0;
    scale = fmax(scale, fabs(dy[i]));
  }
  if (scale <= 0.0) return 0;
  csr_multiply(&lp->kt, dy, work);
  double support = 0.0;
  for (int32_t j = 0; j < lp->k.cols; ++j) {
    const double lambda = work[j];
    if (lambda > 0.0) {
      if (lp->upper[j] >= INFINITY) return 0;
      support += lambda * lp->upper[j];
    } else if (lambda < 0.0) {
      if (lp->lower[j] <= -INFINITY) return 0;
      support += lambda * lp->lower[j];
    }
  }
  double rhs = 0.0;
  for (int32_t i = 0; i < lp->k.rows; ++i) rhs += lp->q[i] * dy[i];
  return (rhs - support) / scale > tol;
}

/* Power iteration on K'K (pdhg.cpp:223-282). */
static double estimate_matrix_norm(const olp* lp, int iterations, double tolerance) {
  const int32_t n = lp->k.cols, m = lp->k.rows;
  if (n == 0 || m == 0 || lp->k.nnz == 0) return 0.0;
  double* v = vzero(n);
  for (int32_t j = 0; j < n; ++j) v[j] = 1.0 + 0.1 * (double)(j % 7);
  const double norm = vnorm2(v, n);
  if (norm == 0.0) {
    free(v);
    return 0.0;
  }
  for (int32_t j = 0; j < n; ++j) v[j] /= norm;
  double* kv = vzero(m);
  double* ktkv = vzero(n);
  double sigma = 0.0;
  for (int it = 0; it < iterations; ++it) {
    csr_multiply(&lp->k, v, kv);
    csr_multiply(&lp->kt, kv, ktkv);
    const double next = vnorm2(ktkv, n);
    if (next == 0.0) {
      sigma = 0.0;
      break;
    }
    for (int32_t j = 0; j < n; ++j) v[j] = ktkv[j] / next;
    const double estimate = sqrt(next);
    if (it > 0 && fabs(estimate - sigma) <= tolerance * estimate) {
      sigma = estimate;
      break;
    }
    sigma = estimate;
  }
  free(v);
  free(kv);
  free(ktkv);
  return sigma;
}

/* cuPDLP restart metric (pdhg.cpp:295-340), on the scaled problem. */
static double weighted_kkt_error(const olp* lp, const double* x, const double* y, double omega) {
  const int32_t m = lp->k.rows, n = lp->k.cols;
  double* kx = vzero(m);
  double* kty = vzero(n);
  csr_multiply(&lp->k, x, kx);
  csr_multiply(&lp->kt, y, kty);
  double primal_sq = 0.0;
  for (int32_t i = 0; i < m; ++i) {
    const double v = (i < lp->num_eq) ? (kx[i] - lp->q[i]) : fmin(kx[i] - lp->q[i], 0.0);
    primal_sq += v * v;
  }
  double dual_sq = 0.0, bound_term = 0.0;
  for (int32_t j = 0; j < n; ++j) {
    const double lambda = lp->c[j] - kty[j];
    const int has_lo = lp->lower[j] > -INFINITY;
    const int has_hi = lp->upper[j] < INFINITY;
    double leftover = 0.0;
    if (has_lo && has_hi) leftover = 0.0;
    else if (has_lo) leftover = fmin(lambda, 0.0);
    else if (has_hi) leftover = fmax(lambda, 0.0);
    else leftover = lambda;
    dual_sq += leftover * leftover;
    const double absorbed = lambda - leftover;
    if (absorbed > 0.0) bound_term += absorbed * lp->lower[j];
    else if (absorbed < 0.0) bound_term += absorbed * lp->upper[j];
  }
  const double gap = standard_objective(lp, x) - (vdot(lp->q, y, m) + bound_term);
  const double value = omega * omega * primal_sq + dual_sq / (omega * omega) + gap * gap;
  free(kx);
  free(kty);
  return sqrt(value);
}

/* ------------------------------------------------ backend operations */

/* cpu_backend primal_update (backend.cpp:60-79). */
static void primal_update(int32_t n, double tau, double gamma, double halpern, const double* x,
                          const double* c, const double* kt_y, const double* lower,
                          const double* upper, const double* anchor, double* x_out, double* dx,
                          double* x_bar) {
  for (int32_t j = 0; j < n; ++j) {
    const double x_j = x[j];
    double v = x_j - tau * (c[j] - kt_y[j]);
    if (v < lower[j]) v = lower[j];
    if (v > upper[j]) v = upper[j];
    const double d = v - x_j;
    dx[j] = d;
    x_bar[j] = v + d;
    double next = v;
    if (gamma != 0.0) next += gamma * d;
    if (anchor != NULL) next = halpern * next + (1.0 - halpern) * anchor[j];
    x_out[j] = next;
  }
}

/* cpu_backend dual_update (backend.cpp:81-111). */
static void dual_update(int32_t m, int32_t num_eq, double sigma, double gamma, double halpern,
                        const double* y, const double* q, const double* k_x_bar,
                        const double* k_x, const double* anchor_y, const double* anchor_kx,
                        double* y_out, double* dy, double* k_out, double* k_dx) {
  for (int32_t i = 0; i < m; ++i) {
    const double y_i = y[i];
    const double bar = k_x_bar[i];
    const double kx = k_x[i];
    double v = y_i + sigma * (q[i] - bar);
    if (i >= num_eq && v < 0.0) v = 0.0;
    const double d = v - y_i;
    dy[i] = d;
    const double kd = 0.5 * (bar - kx);
    k_dx[i] = kd;
    double next_y = v;
    double next_k = 0.5 * (bar + kx);
    if (gamma != 0.0) {
      next_y += gamma * d;
      next_k += gamma * kd;
    }
    if (anchor_y != NULL) {
      next_y = halpern * next_y + (1.0 - halpern) * anchor_y[i];
      next_k = halpern * next_k + (1.0 - halpern) * anchor_kx[i];
    }
    y_out[i] = next_y;
    k_out[i] = next_k;
  }
}

static double weighted_norm_squared(int32_t n, int32_t m, const double* dx, const double* dy,
                                    double omega) {
  return omega * vdot(dx, dx, n) + vdot(dy, dy, m) / omega;
}

typedef struct {
  double primal_sq, primal_inf, q_dot_y, dual_sq, dual_inf, bound_term, c_dot_x;
} oterms;

/* LinAlgBackend::convergence_terms (backend.cpp:143-202): the unscaled check
 * from the scaled iterate and its products. */
static void convergence_terms(const olp* orig, const double* row_scale, const double* col_scale,
                              const double* x, const double* k_x, const double* y,
                              const double* kt_y, oterms* t) {
  memset(t, 0, sizeof(*t));
  const int32_t m = orig->k.rows, n = orig->k.cols;
  for (int32_t i = 0; i < m; ++i) {
    const double scale = row_scale[i];
    const double row = scale != 0.0 ? k_x[i] / scale : k_x[i];
    const double violation =
        (i < orig->num_eq) ? (row - orig->q[i]) : fmin(row - orig->q[i], 0.0);
    t->primal_sq += violation * violation;
    t->primal_inf = fmax(t->primal_inf, fabs(violation));
    t->q_dot_y += orig->q[i] * (scale * y[i]);
  }
  for (int32_t j = 0; j < n; ++j) {
    const double scale = col_scale[j];
    const double product = scale != 0.0 ? kt_y[j] / scale : kt_y[j];
    const double lambda = orig->c[j] - product;
    const int has_lo = orig->lower[j] > -INFINITY;
    const int has_hi = orig->upper[j] < INFINITY;
    double leftover = 0.0;
    if (has_lo && has_hi) leftover = 0.0;
    else if (has_lo) leftover = fmin(lambda, 0.0);
    else if (has_hi) leftover = fmax(lambda, 0.0);
    else leftover = lambda;
    t->dual_sq += leftover * leftover;
    t->dual_inf = fmax(t->dual_inf, fabs(leftover));
    const double absorbed = lambda - leftover;
    if (absorbed > 0.0) t->bound_term += absorbed * orig->lower[j];
    else if (absorbed < 0.0) t->bound_term += absorbed * orig->upper[j];
    t->c_dot_x += orig->c[j] * (scale * x[j]);
  }
}

/* residual_from_terms (pdhg.cpp:70-87). */
static void residual_from_terms(const oterms* t, double q_two, double c_two, double q_inf,
                                double c_inf, anu_pdhg_residual* r) {
  memset(r, 0, sizeof(*r));
  r->primal_residual = sqrt(t->primal_sq);
  r->primal_residual_inf = t->primal_inf;
  r->dual_residual = sqrt(t->dual_sq);
  r->dual_residual_inf = t->dual_inf;
  r->primal_objective = t->c_dot_x;
  r->dual_objective = t->q_dot_y + t->bound_term;
  r->absolute_gap = fabs(r->primal_objective - r->dual_objective);
  residual_terms_to(r, q_two, c_two, q_inf, c_inf);
}

/* ------------------------------------------------------------ solve */

static double now_seconds(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void set_message(anu_pdhg_result* r, const char* text) {
  snprintf(r->message, sizeof(r->message), "%s", text);
}

/* Output of one solve: owned x (n) and y (m). */
typedef struct {
  anu_pdhg_result res;
  double* x;
  double* y;
} osolve;

static void solve(const olp* original, const anu_pdhg_options* options, const double* warm_x,
                  const double* warm_y, osolve* out);

/* make_primal_feasibility / make_dual_feasibility (pdhg.cpp:350-368). */
static void make_primal_feasibility(olp* lp) {
  for (int32_t j = 0; j < lp->k.cols; ++j) lp->c[j] = 0.0;
  lp->obj_offset = 0.0;
}
static void make_dual_feasibility(olp* lp) {
  for (int32_t i = 0; i < lp->k.rows; ++i) lp->q[i] = 0.0;
  for (int32_t j = 0; j < lp->k.cols; ++j) {
    if (lp->lower[j] > -INFINITY) lp->lower[j] = 0.0;
    if (lp->upper[j] < INFINITY) lp->upper[j] = 0.0;
  }
  lp->obj_offset = 0.0;
}

typedef struct {
  const olp* original;
  const olp* lp; /* scaled */
  const oscaling* scaling;
  const anu_pdhg_options* options;
  double matrix_norm;
  double start_time;
  int built;
  olp primal_lp, dual_lp;
} polish_ctx;

/* run_polish (pdhg.cpp:666-751): two one-sided sub-solves from a scaled
 * seed; returns the unscaled polished pair, its residual and the cost. */
static void run_polish(polish_ctx* p, const double* seed_x, const double* seed_y, int32_t budget,
                       double eta, double omega, double* out_x, double* out_y,
                       anu_pdhg_residual* out_r, int32_t* spent) {
  const int32_t n = p->lp->k.cols, m = p->lp->k.rows;
  if (!p->built) {
    olp_copy(p->lp, &p->primal_lp);
    make_primal_feasibility(&p->primal_lp);
    olp_copy(p->lp, &p->dual_lp);
    make_dual_feasibility(&p->dual_lp);
    p->built = 1;
  }
  anu_pdhg_options sub = *p->options;
  sub.polish_feasibility = 0;
  sub.polish_on_exit = 0;
  sub.detect_infeasibility = 0;
  sub.verbose = 0;
  sub.known_matrix_norm = p->matrix_norm;
  sub.ruiz_iterations = 0;
  sub.pock_chambolle = 0;
  sub.max_iterations = budget;
  {
    int32_t freq = p->options->termination_check_frequency;
    int32_t quarter = budget / 4;
    int32_t inner = freq < quarter ? freq : quarter;
    sub.termination_check_frequency = inner > 10 ? inner : 10;
  }
  sub.time_limit_seconds = fmax(0.0, p->options->time_limit_seconds - (now_seconds() - p->start_time));
  sub.initial_step_size = eta;
  sub.initial_primal_weight = omega;
  double* zero_x = vzero(n);
  double* zero_y = vzero(m);
  osolve primal, dual;
  sub.termination = ANU_TERMINATION_PRIMAL_FEASIBILITY;
  solve(&p->primal_lp, &sub, seed_x, zero_y, &primal);
  sub.termination = ANU_TERMINATION_DUAL_FEASIBILITY;
  solve(&p->dual_lp, &sub, zero_x, seed_y, &dual);
  *spent = primal.res.iterations + dual.res.iterations;
  for (int32_t j = 0; j < n; ++j) out_x[j] = p->scaling->col_scale[j] * primal.x[j];
  for (int32_t i = 0; i < m; ++i) out_y[i] = p->scaling->row_scale[i] * dual.y[i];
  evaluate_residual(p->original, out_x, out_y, out_r);
  free(primal.x);
  free(primal.y);
  free(dual.x);
  free(dual.y);
  free(zero_x);
  free(zero_y);
}

static int32_t polish_budget(const anu_pdhg_options* o, int32_t at_iteration) {
  int32_t budget = (int32_t)(o->polish_iteration_factor * (double)(at_iteration + 1));
  if (budget < o->polish_minimum_iterations) budget = o->polish_minimum_iterations;
  if (budget > o->polish_maximum_iterations) budget = o->polish_maximum_iterations;
  return budget;
}

static int passes(const anu_pdhg_options* o, const anu_pdhg_residual* r, double gap_tol) {
  const int inf = o->require_inf_norm_termination != 0;
  switch (o->termination) {
    case ANU_TERMINATION_PRIMAL_FEASIBILITY:
      return residual_primal_ok(r, o->tolerance, o->absolute_tolerance, inf);
    case ANU_TERMINATION_DUAL_FEASIBILITY:
      return residual_dual_ok(r, o->tolerance, o->absolute_tolerance, inf);
    default:
      return residual_converged(r, o->tolerance, o->absolute_tolerance, inf, gap_tol);
  }
}

#define SWAP(a, b)  \
  do {              \
    double* t_ = a; \
    a = b;          \
    b = t_;         \
  } while (0)

/* solve_pdhg (pdhg.cpp:377-1285). */
static void solve(const olp* original, const anu_pdhg_options* options, const double* warm_x,
                  const double* warm_y, osolve* out) {
  const double start_time = now_seconds();
  double phase_mark = start_time;
#define PHASE_END() (__extension__({ const double now_ = now_seconds(); const double s_ = now_ - phase_mark; phase_mark = now_; s_; }))
  anu_pdhg_result* result = &out->res;
  memset(result, 0, sizeof(*result));
  result->status = ANU_PDHG_NUMERICAL_ERROR;
  const int32_t n = original->k.cols;
  const int32_t m = original->k.rows;
  out->x = vzero(n);
  out->y = vzero(m);

  olp lp;
  olp_copy(original, &lp);
  oscaling sc;
  scale_lp(&lp, options->ruiz_iterations, options->pock_chambolle != 0, &sc);
  result->row_spread_before = sc.spreads[0];
  result->row_spread_after = sc.spreads[1];
  result->col_spread_before = sc.spreads[2];
  result->col_spread_after = sc.spreads[3];
  result->phases.scaling = PHASE_END();

  const double matrix_norm = options->known_matrix_norm > 0.0
                                 ? options->known_matrix_norm
                                 : estimate_matrix_norm(&lp, 200, 1e-8);
  result->phases.matrix_norm = PHASE_END();
  result->matrix_norm_estimate = matrix_norm;
  if (matrix_norm <= 0.0) {
    for (int32_t j = 0; j < n; ++j) {
      const double lo = original->lower[j], hi = original->upper[j], cj = original->c[j];
      double value = 0.0;
      if (cj > 0.0) value = lo;
      else if (cj < 0.0) value = hi;
      else value = isfinite(lo) ? lo : (isfinite(hi) ? hi : 0.0);
      out->x[j] = isfinite(value) ? value : 0.0;
    }
    evaluate_residual(original, out->x, out->y, &result->residual);
    result->objective = model_objective(original, out->x);
    result->status = residual_converged(&result->residual, options->tolerance,
                                        options->absolute_tolerance,
                                        options->require_inf_norm_termination != 0, 0.0)
                         ? ANU_PDHG_OPTIMAL
                         : ANU_PDHG_NUMERICAL_ERROR;
    set_message(result, "no constraint matrix content");
    result->solve_seconds = now_seconds() - start_time;
    olp_free(&lp);
    scaling_free(&sc);
    return;
  }

  double eta = 0.9 / matrix_norm;
  const int adaptive = options->adaptive_step_size && !options->constant_step_size;
  if (options->constant_step_size) eta = options->constant_step_scale / matrix_norm;
  double omega = 1.0;
  if (options->primal_weight_updates) {
    const double c_norm = vnorm2(lp.c, n);
    const double q_norm = vnorm2(lp.q, m);
    if (c_norm > 1e-12 && q_norm > 1e-12) omega = c_norm / q_norm;
  }
  if (options->initial_step_size > 0.0) eta = options->initial_step_size;
  if (options->initial_primal_weight > 0.0) omega = options->initial_primal_weight;

  double* x = vzero(n);
  double* y = vzero(m);
  const int warm = warm_x != NULL && warm_y != NULL;
  if (warm) {
    memcpy(x, warm_x, sizeof(double) * (size_t)n);
    memcpy(y, warm_y, sizeof(double) * (size_t)m);
    for (int32_t i = lp.num_eq; i < m; ++i)
      if (!(y[i] > 0.0)) y[i] = 0.0;
  }
  for (int32_t j = 0; j < n; ++j) {
    const double lo = lp.lower[j], hi = lp.upper[j];
    double v = warm ? x[j] : 0.0;
    if (!isfinite(v)) v = 0.0;
    if (v < lo) v = isfinite(lo) ? lo : 0.0;
    if (v > hi) v = isfinite(hi) ? hi : 0.0;
    x[j] = v;
  }

  double* host_x = vdup(x, n);
  double* host_y = vdup(y, m);
  double* host_dy = vzero(m);
  double* host_avg_x = vzero(n);
  double* host_avg_y = vzero(m);

  double* d_x = vdup(host_x, n);
  double* x_next = vzero(n);
  double* kt_y = vzero(n);
  double* x_bar = vzero(n);
  double* dx = vzero(n);
  double* sum_x = vzero(n);
  double* avg_x = vzero(n);
  double* d_y = vdup(host_y, m);
  double* y_next = vzero(m);
  double* k_x_bar = vzero(m);
  double* k_x = vzero(m);
  double* dy = vzero(m);
  double* k_dx = vzero(m);
  double* k_next = vzero(m);
  double* sum_y = vzero(m);
  double* avg_y = vzero(m);

  const double res_q_two = vnorm2(original->q, m);
  const double res_c_two = vnorm2(original->c, n);
  const double res_q_inf = vnorminf(original->q, m);
  const double res_c_inf = vnorminf(original->c, n);

  csr_multiply(&lp.k, d_x, k_x);

  double sum_weight = 0.0;
  double* anchor_x = vzero(n);
  double* anchor_y = vzero(m);
  double* anchor_kx = vzero(m);
  int anchor_needs_reset = 1;
  int32_t halpern_k = 0;
  double movement = 0.0;
  double epoch_start_movement = 0.0;

  double* restart_x = vdup(host_x, n);
  double* restart_y = vdup(host_y, m);
  double* previous_restart_x = vdup(host_x, n);
  double* previous_restart_y = vdup(host_y, m);
  int have_previous_restart = 0;

  double kkt_at_restart = weighted_kkt_error(&lp, x, y, omega);
  double last_candidate_kkt = INFINITY;
  double residual_at_restart = INFINITY;
  double last_residual = INFINITY;
  double weight_error_sum = 0.0;
  double weight_error_previous = 0.0;

  double* unscaled_x = vzero(n);
  double* unscaled_y = vzero(m);
  double* infeasibility_work = vzero(n);

  const double tolerance = options->tolerance;
  const double gap_tolerance = options->gap_tolerance > 0.0 ? options->gap_tolerance : tolerance;
  const int halpern = options->halpern && options->restarts;
  const double reflection = halpern ? options->reflection : 0.0;
  const int inf_norm = options->require_inf_norm_termination != 0;

  polish_ctx pctx;
  memset(&pctx, 0, sizeof(pctx));
  pctx.original = original;
  pctx.lp = &lp;
  pctx.scaling = &sc;
  pctx.options = options;
  pctx.matrix_norm = matrix_norm;
  pctx.start_time = start_time;
  double* polished_x = NULL;
  double* polished_y = NULL;
  anu_pdhg_residual polished_residual;
  memset(&polished_residual, 0, sizeof(polished_residual));
  int have_polished = 0;
  int32_t next_polish_iteration = options->polish_first_iteration;

  int32_t iteration = 0;
  int32_t iterations_since_restart = 0;
  int32_t status = ANU_PDHG_ITERATION_LIMIT;
  result->phases.setup = PHASE_END();

  for (; iteration < options->max_iterations; ++iteration) {
    const int check = ((iteration + 1) % options->termination_check_frequency == 0);
    const int blend = halpern && !anchor_needs_reset;
    const double halpern_weight =
        blend ? (double)(halpern_k + 1) / (double)(halpern_k + 2) : 1.0;
    const int need_movement = adaptive || options->halpern_restart || check;

    csr_multiply(&lp.kt, d_y, kt_y);

    for (int attempt = 0;; ++attempt) {
      const double tau = eta / omega;
      const double sigma = eta * omega;
      primal_update(n, tau, reflection, halpern_weight, d_x, lp.c, kt_y, lp.lower, lp.upper,
                    blend ? anchor_x : NULL, x_next, dx, x_bar);
      csr_multiply(&lp.k, x_bar, k_x_bar);
      dual_update(m, lp.num_eq, sigma, reflection, halpern_weight, d_y, lp.q, k_x_bar, k_x,
                  blend ? anchor_y : NULL, blend ? anchor_kx : NULL, y_next, dy, k_next, k_dx);
      if (!adaptive) {
        if (need_movement) movement = weighted_norm_squared(n, m, dx, dy, omega);
        break;
      }
      const double interaction = fabs(vdot(dy, k_dx, m));
      movement = weighted_norm_squared(n, m, dx, dy, omega);
      double eta_bar = INFINITY;
      if (interaction > 0.0) eta_bar = movement / (2.0 * interaction);
      const double k1 = (double)(iteration + 1);
      double eta_next = eta;
      if (isfinite(eta_bar)) {
        eta_next = fmin((1.0 - pow(k1, -0.3)) * eta_bar, (1.0 + pow(k1, -0.6)) * eta);
      } else {
        eta_next = (1.0 + pow(k1, -0.6)) * eta;
      }
      if (!(eta_next > 0.0) || !isfinite(eta_next)) eta_next = eta;
      const int accept = (eta <= eta_bar);
      eta = eta_next;
      if (accept) break;
      if (attempt > 60) break;
    }

    SWAP(d_x, x_next);
    SWAP(d_y, y_next);
    SWAP(k_x, k_next);
    ++iterations_since_restart;

    if (halpern) {
      if (anchor_needs_reset) {
        memcpy(anchor_x, d_x, sizeof(double) * (size_t)n);
        memcpy(anchor_y, d_y, sizeof(double) * (size_t)m);
        memcpy(anchor_kx, k_x, sizeof(double) * (size_t)m);
        anchor_needs_reset = 0;
        halpern_k = 0;
        epoch_start_movement = movement;
      } else {
        ++halpern_k;
      }
    }
    if (options->restarts && !halpern) {
      for (int32_t j = 0; j < n; ++j) sum_x[j] += eta * d_x[j];
      for (int32_t i = 0; i < m; ++i) sum_y[i] += eta * d_y[i];
      sum_weight += eta;
    }
    if (halpern && options->halpern_restart && !anchor_needs_reset &&
        epoch_start_movement > 0.0 && halpern_k >= options->halpern_minimum_epoch) {
      if (movement <= epoch_start_movement / 7.389056098930650) {
        anchor_needs_reset = 1;
        ++result->restarts;
      }
    }

    if (!check) continue;
    result->phases.iterating += PHASE_END();
    const double check_start = phase_mark;

    int host_iterate_valid = 0;
#define PULL_ITERATE()                                                        \
  (host_iterate_valid ? (void)0                                               \
                      : (void)(memcpy(host_x, d_x, sizeof(double) * (size_t)n), \
                               memcpy(host_y, d_y, sizeof(double) * (size_t)m), \
                               host_iterate_valid = 1))

    int stop_loop = 0;
    if (options->detect_infeasibility) {
      memcpy(host_dy, dy, sizeof(double) * (size_t)m);
      if (is_infeasibility_certificate(&lp, host_dy, options->infeasibility_tolerance,
                                       infeasibility_work)) {
        status = ANU_PDHG_PRIMAL_INFEASIBLE;
        set_message(result, "Farkas certificate found in the dual iterate difference");
        ++iteration;
        stop_loop = 1;
      }
    }
    if (stop_loop) {
      result->phases.checks += now_seconds() - check_start;
      phase_mark = now_seconds();
      break;
    }

    const int need_kkt = (options->restarts && !halpern) ||
                         (options->restarts && !options->restart_on_fixed_point) ||
                         options->verbose;
    const int need_average = options->restarts && !halpern && sum_weight > 0.0;
    if (need_kkt || need_average) PULL_ITERATE();
    const double current_kkt = need_kkt ? weighted_kkt_error(&lp, host_x, host_y, omega) : 0.0;
    int use_average = 0;
    double candidate_kkt = current_kkt;
    if (need_average) {
      for (int32_t j = 0; j < n; ++j) avg_x[j] = sum_x[j] / sum_weight;
      for (int32_t i = 0; i < m; ++i) avg_y[i] = sum_y[i] / sum_weight;
      memcpy(host_avg_x, avg_x, sizeof(double) * (size_t)n);
      memcpy(host_avg_y, avg_y, sizeof(double) * (size_t)m);
      const double average_kkt = weighted_kkt_error(&lp, host_avg_x, host_avg_y, omega);
      if (average_kkt < current_kkt) {
        use_average = 1;
        candidate_kkt = average_kkt;
      }
    }
#define CANDIDATE_X() (PULL_ITERATE(), (use_average ? host_avg_x : host_x))
#define CANDIDATE_Y() (PULL_ITERATE(), (use_average ? host_avg_y : host_y))
#define ADOPT_CANDIDATE()                                          \
  do {                                                             \
    if (use_average) {                                             \
      memcpy(d_x, avg_x, sizeof(double) * (size_t)n);              \
      memcpy(d_y, avg_y, sizeof(double) * (size_t)m);              \
      memcpy(host_x, host_avg_x, sizeof(double) * (size_t)n);      \
      memcpy(host_y, host_avg_y, sizeof(double) * (size_t)m);      \
    }                                                              \
  } while (0)

    anu_pdhg_residual r;
    if (options->reuse_products && !use_average) {
      csr_multiply(&lp.kt, d_y, kt_y);
      oterms terms;
      convergence_terms(original, sc.row_scale, sc.col_scale, d_x, k_x, d_y, kt_y, &terms);
      residual_from_terms(&terms, res_q_two, res_c_two, res_q_inf, res_c_inf, &r);
    } else {
      const double* cx = CANDIDATE_X();
      const double* cy = CANDIDATE_Y();
      for (int32_t j = 0; j < n; ++j) unscaled_x[j] = sc.col_scale[j] * cx[j];
      for (int32_t i = 0; i < m; ++i) unscaled_y[i] = sc.row_scale[i] * cy[i];
      evaluate_residual(original, unscaled_x, unscaled_y, &r);
    }

    if (!isfinite(r.primal_residual) || !isfinite(r.dual_residual)) {
      status = ANU_PDHG_NUMERICAL_ERROR;
      set_message(result, "iterates stopped being finite");
      ++iteration;
      ADOPT_CANDIDATE();
      stop_loop = 1;
    } else if (passes(options, &r, gap_tolerance)) {
      status = ANU_PDHG_OPTIMAL;
      ++iteration;
      ADOPT_CANDIDATE();
      stop_loop = 1;
    }
    if (stop_loop) {
      result->phases.checks += PHASE_END();
      break;
    }

    if (options->polish_feasibility && options->termination == ANU_TERMINATION_FULL &&
        iteration + 1 >= next_polish_iteration) {
      while (next_polish_iteration <= iteration + 1) next_polish_iteration *= 2;
      const int32_t budget = polish_budget(options, iteration);
      if (r.relative_gap <= gap_tolerance && budget > 0) {
        double* try_x = vzero(n);
        double* try_y = vzero(m);
        anu_pdhg_residual try_r;
        int32_t spent = 0;
        const double* from_x = CANDIDATE_X();
        const double* from_y = CANDIDATE_Y();
        result->phases.checks += PHASE_END();
        run_polish(&pctx, from_x, from_y, budget, eta, omega, try_x, try_y, &try_r, &spent);
        result->phases.polishing += PHASE_END();
        ++result->polish_attempts;
        result->polish_iterations += spent;
        if (residual_converged(&try_r, tolerance, options->absolute_tolerance, inf_norm,
                               gap_tolerance)) {
          polished_x = try_x;
          polished_y = try_y;
          polished_residual = try_r;
          have_polished = 1;
          result->polished = 1;
          status = ANU_PDHG_OPTIMAL;
          set_message(result, "converged after feasibility polishing");
          ++iteration;
          break;
        }
        free(try_x);
        free(try_y);
      }
    }
    if (options->verbose && options->log_frequency > 0 &&
        (iteration + 1) % options->log_frequency == 0) {
      printf("  iter %7d  primal %.3e  dual %.3e  gap %.3e  kkt %.3e  eta %.3e  w %.3e\n",
             iteration + 1, r.relative_primal, r.relative_dual, r.relative_gap, candidate_kkt,
             eta, omega);
    }
    if (now_seconds() - start_time > options->time_limit_seconds ||
        (options->stop != NULL && __atomic_load_n(options->stop, __ATOMIC_ACQUIRE) != 0)) {
      status = ANU_PDHG_TIME_LIMIT;
      ++iteration;
      ADOPT_CANDIDATE();
      result->phases.checks += PHASE_END();
      break;
    }

    if (!options->restarts) {
      result->phases.checks += PHASE_END();
      continue;
    }

    const double residual = sqrt(fmax(movement, 0.0));
    const int by_residual = options->restart_on_fixed_point != 0;
    if (by_residual && !isfinite(residual_at_restart)) residual_at_restart = residual;
    const double measure = by_residual ? residual : candidate_kkt;
    const double at_restart = by_residual ? residual_at_restart : kkt_at_restart;
    const double previous = by_residual ? last_residual : last_candidate_kkt;
    const int sufficient = measure <= 0.2 * at_restart;
    const int necessary = measure <= 0.8 * at_restart && measure > previous;
    const int too_long =
        (double)iterations_since_restart >= 0.36 * (double)(iteration + 1);
    last_candidate_kkt = candidate_kkt;
    last_residual = residual;
    if (!(sufficient || necessary || too_long)) {
      result->phases.checks += PHASE_END();
      continue;
    }

    ADOPT_CANDIDATE();
    csr_multiply(&lp.k, d_x, k_x);
    PULL_ITERATE();
    if (options->primal_weight_updates && have_previous_restart) {
      const double* base_x = options->pid_primal_weight ? restart_x : previous_restart_x;
      const double* base_y = options->pid_primal_weight ? restart_y : previous_restart_y;
      double delta_x_sq = 0.0, delta_y_sq = 0.0;
      for (int32_t j = 0; j < n; ++j) {
        const double d = host_x[j] - base_x[j];
        delta_x_sq += d * d;
      }
      for (int32_t i = 0; i < m; ++i) {
        const double d = host_y[i] - base_y[i];
        delta_y_sq += d * d;
      }
      const double delta_x = sqrt(delta_x_sq);
      const double delta_y = sqrt(delta_y_sq);
      if (delta_x > 1e-12 && delta_y > 1e-12) {
        double candidate = 0.0;
        if (options->pid_primal_weight) {
          const double e = log(omega * delta_x / delta_y);
          weight_error_sum += e;
          const double correction = options->primal_weight_kp * e +
                                    options->primal_weight_ki * weight_error_sum +
                                    options->primal_weight_kd * (e - weight_error_previous);
          weight_error_previous = e;
          candidate = exp(log(omega) - correction);
        } else {
          candidate = exp(0.5 * log(delta_y / delta_x) + 0.5 * log(omega));
        }
        if (isfinite(candidate) && candidate > 1e-12 && candidate < 1e12) omega = candidate;
      }
    }
    memcpy(previous_restart_x, restart_x, sizeof(double) * (size_t)n);
    memcpy(previous_restart_y, restart_y, sizeof(double) * (size_t)m);
    have_previous_restart = 1;
    memcpy(restart_x, host_x, sizeof(double) * (size_t)n);
    memcpy(restart_y, host_y, sizeof(double) * (size_t)m);
    memset(sum_x, 0, sizeof(double) * (size_t)n);
    memset(sum_y, 0, sizeof(double) * (size_t)m);
    sum_weight = 0.0;
    anchor_needs_reset = 1;
    iterations_since_restart = 0;
    last_candidate_kkt = INFINITY;
    last_residual = INFINITY;
    residual_at_restart = sqrt(fmax(movement, 0.0));
    if (!options->restart_on_fixed_point)
      kkt_at_restart = weighted_kkt_error(&lp, host_x, host_y, omega);
    ++result->restarts;
    result->phases.checks += PHASE_END();
  }

  if (!have_polished) {
    memcpy(host_x, d_x, sizeof(double) * (size_t)n);
    memcpy(host_y, d_y, sizeof(double) * (size_t)m);
    for (int32_t j = 0; j < n; ++j) out->x[j] = sc.col_scale[j] * host_x[j];
    for (int32_t i = 0; i < m; ++i) out->y[i] = sc.row_scale[i] * host_y[i];
    evaluate_residual(original, out->x, out->y, &result->residual);
    const int worth_trying =
        options->polish_feasibility && options->polish_on_exit &&
        options->termination == ANU_TERMINATION_FULL && status != ANU_PDHG_OPTIMAL &&
        status != ANU_PDHG_PRIMAL_INFEASIBLE && status != ANU_PDHG_NUMERICAL_ERROR &&
        isfinite(result->residual.primal_residual) && isfinite(result->residual.dual_residual) &&
        now_seconds() - start_time < options->time_limit_seconds;
    const int32_t exit_budget = worth_trying ? polish_budget(options, iteration) : 0;
    if (exit_budget > 0) {
      double* try_x = vzero(n);
      double* try_y = vzero(m);
      anu_pdhg_residual try_r;
      int32_t spent = 0;
      run_polish(&pctx, host_x, host_y, exit_budget, eta, omega, try_x, try_y, &try_r, &spent);
      ++result->polish_attempts;
      result->polish_iterations += spent;
      const double gap_ceiling = fmax(gap_tolerance, result->residual.relative_gap);
      const anu_pdhg_residual* cur = &result->residual;
      const int improved = try_r.relative_primal <= cur->relative_primal &&
                           try_r.relative_dual <= cur->relative_dual &&
                           (try_r.relative_primal < cur->relative_primal ||
                            try_r.relative_dual < cur->relative_dual);
      if (improved && try_r.relative_gap <= gap_ceiling) {
        memcpy(out->x, try_x, sizeof(double) * (size_t)n);
        memcpy(out->y, try_y, sizeof(double) * (size_t)m);
        result->residual = try_r;
        result->polished = 1;
        if (residual_converged(&try_r, tolerance, options->absolute_tolerance, inf_norm,
                               gap_tolerance)) {
          status = ANU_PDHG_OPTIMAL;
          set_message(result, "converged after feasibility polishing");
        } else if (result->message[0] == '\0') {
          set_message(result, "feasibility polished");
        } else {
          char buf[sizeof(result->message)];
          snprintf(buf, sizeof(buf), "%.130s, feasibility polished", result->message);
          set_message(result, buf);
        }
      }
      free(try_x);
      free(try_y);
    }
  } else {
    memcpy(out->x, polished_x, sizeof(double) * (size_t)n);
    memcpy(out->y, polished_y, sizeof(double) * (size_t)m);
    result->residual = polished_residual;
    free(polished_x);
    free(polished_y);
  }
  result->objective = model_objective(original, out->x);
  result->iterations = iteration;
  result->status = status;
  result->final_step_size = eta;
  result->final_primal_weight = omega;
  result->solve_seconds = now_seconds() - start_time;

  double* owned[] = {x, y, host_x, host_y, host_dy, host_avg_x, host_avg_y, d_x, x_next, kt_y,
                     x_bar, dx, sum_x, avg_x, d_y, y_next, k_x_bar, k_x, dy, k_dx, k_next,
                     sum_y, avg_y, anchor_x, anchor_y, anchor_kx, restart_x, restart_y,
                     previous_restart_x, previous_restart_y, unscaled_x, unscaled_y,
                     infeasibility_work};
  for (size_t i = 0; i < sizeof(owned) / sizeof(owned[0]); ++i) free(owned[i]);
  if (pctx.built) {
    olp_free(&pctx.primal_lp);
    olp_free(&pctx.dual_lp);
  }
  olp_free(&lp);
  scaling_free(&sc);
#undef PHASE_END
}

/* ------------------------------------------------------------ API */

int oracle_pdhg_solve(const anu_lp* lp_in, const anu_pdhg_options* options,
                      const double* warm_x, const double* warm_y, double* x, double* y,
                      anu_pdhg_result* result) {
  olp lp;
  olp_from_anu(lp_in, &lp);
  osolve s;
  solve(&lp, options, warm_x, warm_y, &s);
  memcpy(x, s.x, sizeof(double) * (size_t)lp.k.cols);
  memcpy(y, s.y, sizeof(double) * (size_t)lp.k.rows);
  *result = s.res;
  free(s.x);
  free(s.y);
  olp_free(&lp);
  return 0;
}

void oracle_evaluate_residual(const anu_lp* lp_in, const double* x, const double* y,
                              anu_pdhg_residual* out) {
  olp lp;
  olp_from_anu(lp_in, &lp);
  evaluate_residual(&lp, x, y, out);
  olp_free(&lp);
}

double oracle_estimate_matrix_norm(const anu_lp* lp_in, int iterations, double tolerance,
                                   int scaled) {
  olp lp;
  olp_from_anu(lp_in, &lp);
  if (scaled) {
    oscaling sc;
    scale_lp(&lp, 10, 1, &sc);
    scaling_free(&sc);
  }
  const double v = estimate_matrix_norm(&lp, iterations, tolerance);
  olp_free(&lp);
  return v;
}

int oracle_scale_lp(const anu_lp* lp_in, int ruiz_iterations, int pock_chambolle,
                    double* k_value, double* c, double* q, double* lower, double* upper,
                    double* row_scale, double* col_scale, double* spreads) {
  olp lp;
  olp_from_anu(lp_in, &lp);
  oscaling sc;
  scale_lp(&lp, ruiz_iterations, pock_chambolle, &sc);
  memcpy(k_value, lp.k.value, sizeof(double) * (size_t)lp.k.nnz);
  memcpy(c, lp.c, sizeof(double) * (size_t)lp.k.cols);
  memcpy(lower, lp.lower, sizeof(double) * (size_t)lp.k.cols);
  memcpy(upper, lp.upper, sizeof(double) * (size_t)lp.k.cols);
  memcpy(col_scale, sc.col_scale, sizeof(double) * (size_t)lp.k.cols);
  memcpy(q, lp.q, sizeof(double) * (size_t)lp.k.rows);
  memcpy(row_scale, sc.row_scale, sizeof(double) * (size_t)lp.k.rows);
  memcpy(spreads, sc.spreads, sizeof(double) * 4);
  scaling_free(&sc);
  olp_free(&lp);
  return 0;
}

typedef struct {
  int count;
  const anu_lp* lps;
  const anu_pdhg_options* options;
  double* const* xs;
  double* const* ys;
  anu_pdhg_result* results;
  int next;
  pthread_mutex_t lock;
} many_ctx;

static void* many_worker(void* arg) {
  many_ctx* ctx = (many_ctx*)arg;
  for (;;) {
    pthread_mutex_lock(&ctx->lock);
    const int i = ctx->next++;
    pthread_mutex_unlock(&ctx->lock);
    if (i >= ctx->count) break;
    oracle_pdhg_solve(&ctx->lps[i], ctx->options, NULL, NULL, ctx->xs[i], ctx->ys[i],
                      &ctx->results[i]);
  }
  return NULL;
}

int oracle_pdhg_solve_many(int count, const anu_lp* lps, const anu_pdhg_options* options,
                           int threads, double* const* xs, double* const* ys,
                           anu_pdhg_result* results) {
  many_ctx ctx;
  ctx.count = count;
  ctx.lps = lps;
  ctx.options = options;
  ctx.xs = xs;
  ctx.ys = ys;
  ctx.results = results;
  ctx.next = 0;
  pthread_mutex_init(&ctx.lock, NULL);
  if (threads < 1) threads = 1;
  pthread_t* tid = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
  for (int t = 0; t < threads; ++t) pthread_create(&tid[t], NULL, many_worker, &ctx);
  for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
  free(tid);
  pthread_mutex_destroy(&ctx.lock);
  return 0;
}
