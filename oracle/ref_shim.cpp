// Test infrastructure, not product code: a C shim over the reference's own
// PDHG path (anukulan, src/anukulan/*.cpp compiled unmodified from the
// reference tree by oracle/Makefile into oracle/_ref/). The tests and the CPU
// leg of bench.py load oracle/_ref/libanuref.so through ctypes to pin the
// oracle restatement (oracle/pdhg_oracle.c) and the CUDA engine against the
// reference itself. Nothing in the engine links or loads this.
//
// Options and results use the engine's own C structs (include/anu_pdhg.h),
// which mirror PdhgOptions / PdhgResult field for field, so one options
// object drives the reference, the oracle and the engine identically.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "anu_pdhg.h"
#include "shim_lp.hpp"
#include "anukulan/backend.hpp"
#include "anukulan/model.hpp"
#include "anukulan/pdhg.hpp"
#include "anukulan/scaling.hpp"
#include "anukulan/simplex.hpp"
#include "anukulan/sparse.hpp"
#include "anukulan/standard_form.hpp"
#include "anukulan/threading.hpp"

namespace {

using anukulan::Int;

using shim::csr_to_matrix;
using shim::to_lp;
using shim::to_options;

void copy_residual(const anukulan::PdhgResidual& r, anu_pdhg_residual* out) {
  out->primal_residual = r.primal_residual;
  out->dual_residual = r.dual_residual;
  out->primal_residual_inf = r.primal_residual_inf;
  out->dual_residual_inf = r.dual_residual_inf;
  out->primal_objective = r.primal_objective;
  out->dual_objective = r.dual_objective;
  out->absolute_gap = r.absolute_gap;
  out->relative_primal = r.relative_primal;
  out->relative_dual = r.relative_dual;
  out->relative_gap = r.relative_gap;
  out->relative_primal_inf = r.relative_primal_inf;
  out->relative_dual_inf = r.relative_dual_inf;
}

}  // namespace

extern "C" {

// The reference's solve_pdhg on cpu_backend() (threads <= 1) or
// threaded_cpu_backend(threads). threads < 0 means default_thread_count().
int ref_pdhg_solve(const anu_lp* lp_in, const anu_pdhg_options* opt_in,
                   int threads, const double* warm_x, const double* warm_y,
                   double* x, double* y, anu_pdhg_result* out) {
  try {
    const anukulan::StandardLp lp = to_lp(*lp_in);
    anukulan::PdhgOptions options = to_options(*opt_in);
    if (threads == -2) {
#ifdef ANUKULAN_WITH_CUDA
      // The reference's own GPU backend (src/anukulan/cuda_backend.cu).
      options.backend = &anukulan::cuda_backend();
#else
      throw std::runtime_error("this build of the reference has no CUDA backend");
#endif
    } else {
      if (threads < 0) threads = anukulan::default_thread_count();
      options.backend = threads <= 1 ? &anukulan::cpu_backend()
                                     : &anukulan::threaded_cpu_backend(threads);
    }
    std::vector<double> wx, wy;
    if (warm_x != nullptr && warm_y != nullptr) {
      wx.assign(warm_x, warm_x + lp_in->k.cols);
      wy.assign(warm_y, warm_y + lp_in->k.rows);
      options.warm_x = &wx;
      options.warm_y = &wy;
    }
    const anukulan::PdhgResult r = anukulan::solve_pdhg(lp, options);
    std::memset(out, 0, sizeof(*out));
    out->status = static_cast<int32_t>(r.status);
    out->objective = r.objective;
    out->iterations = r.iterations;
    out->restarts = r.restarts;
    out->polish_attempts = r.polish_attempts;
    out->polish_iterations = r.polish_iterations;
    out->polished = r.polished ? 1 : 0;
    out->solve_seconds = r.solve_seconds;
    out->matrix_norm_estimate = r.matrix_norm_estimate;
    out->final_step_size = r.final_step_size;
    out->final_primal_weight = r.final_primal_weight;
    out->phases.scaling = r.phases.scaling;
    out->phases.matrix_norm = r.phases.matrix_norm;
    out->phases.setup = r.phases.setup;
    out->phases.iterating = r.phases.iterating;
    out->phases.checks = r.phases.checks;
    out->phases.polishing = r.phases.polishing;
    copy_residual(r.residual, &out->residual);
    out->row_spread_before = r.scaling.row_spread_before;
    out->row_spread_after = r.scaling.row_spread_after;
    out->col_spread_before = r.scaling.col_spread_before;
    out->col_spread_after = r.scaling.col_spread_after;
    std::snprintf(out->message, sizeof(out->message), "%s", r.message.c_str());
    for (std::size_t j = 0; j < r.x.size(); ++j) x[j] = r.x[j];
    for (std::size_t i = 0; i < r.y.size(); ++i) y[i] = r.y[i];
    return 0;
  } catch (const std::exception& e) {
    std::snprintf(out->message, sizeof(out->message), "exception: %s", e.what());
    return 1;
  }
}

int ref_evaluate_residual(const anu_lp* lp_in, const double* x, const double* y,
                          anu_pdhg_residual* out) {
  const anukulan::StandardLp lp = to_lp(*lp_in);
  std::vector<double> vx(x, x + lp_in->k.cols), vy(y, y + lp_in->k.rows);
  copy_residual(anukulan::evaluate_residual(lp, vx, vy), out);
  return 0;
}

double ref_estimate_matrix_norm(const anu_lp* lp_in, int iterations, double tolerance,
                                int scaled) {
  anukulan::StandardLp lp = to_lp(*lp_in);
  if (scaled) anukulan::scale_lp(&lp);
  return anukulan::estimate_matrix_norm(lp, iterations, tolerance, nullptr);
}

// scale_lp (src/anukulan/scaling.cpp:75-100) with its default options: writes
// the scaled K values in CSR order of the input (the input must already be in
// from_triplets order: sorted unique columns, no zeros), the scaled c, q,
// bounds and the two diagonals.
int ref_scale_lp(const anu_lp* lp_in, int ruiz_iterations, int pock_chambolle,
                 double* k_value, double* c, double* q, double* lower, double* upper,
                 double* row_scale, double* col_scale, double* spreads) {
  anukulan::StandardLp lp = to_lp(*lp_in);
  if (lp.k.nnz() != lp_in->k.nnz) return 1;
  anukulan::ScalingOptions so;
  so.ruiz_iterations = ruiz_iterations;
  so.pock_chambolle = pock_chambolle != 0;
  const anukulan::ScalingReport rep = anukulan::scale_lp(&lp, so);
  for (Int k = 0; k < lp.k.nnz(); ++k) k_value[k] = lp.k.value()[static_cast<std::size_t>(k)];
  for (std::size_t j = 0; j < lp.c.size(); ++j) {
    c[j] = lp.c[j];
    lower[j] = lp.lower[j];
    upper[j] = lp.upper[j];
    col_scale[j] = rep.scaling.col_scale[j];
  }
  for (std::size_t i = 0; i < lp.q.size(); ++i) {
    q[i] = lp.q[i];
    row_scale[i] = rep.scaling.row_scale[i];
  }
  spreads[0] = rep.row_spread_before;
  spreads[1] = rep.row_spread_after;
  spreads[2] = rep.col_spread_before;
  spreads[3] = rep.col_spread_after;
  return 0;
}

// The reference dual simplex (src/anukulan/simplex.hpp:452) through solve_lp,
// which falls back to the primal when the start cannot be made dual feasible.
// Returns the SimplexStatus as an int; x (n) and y (m) receive the solution.
int ref_simplex_solve(const anu_lp* lp_in, double time_limit, double* x, double* y,
                      double* objective, int* iterations) {
  const anukulan::StandardLp lp = to_lp(*lp_in);
  anukulan::SimplexOptions so;
  so.time_limit_seconds = time_limit;
  const anukulan::SimplexResult r = anukulan::solve_lp(lp, so);
  for (std::size_t j = 0; j < r.x.size() && j < static_cast<std::size_t>(lp_in->k.cols); ++j)
    x[j] = r.x[j];
  for (std::size_t i = 0; i < r.y.size() && i < static_cast<std::size_t>(lp_in->k.rows); ++i)
    y[i] = r.y[i];
  *objective = r.objective;
  *iterations = r.iterations;
  return static_cast<int>(r.status);
}

int ref_default_thread_count(void) { return anukulan::default_thread_count(); }

// LinAlgBackend::name() of the backend solve_pdhg gets when it names none
// (default_backend(), backend.cpp:209-221): "cpu" without a device, "cuda"
// in the reference's own CUDA build, "b200" where cuda_backend() is the
// adapter over the engine. Returns the length written.
int ref_default_backend_name(char* buf, int size) {
  const std::string name = anukulan::default_backend().name();
  return std::snprintf(buf, static_cast<std::size_t>(size), "%s", name.c_str());
}

// PdhgOptions{} (src/anukulan/pdhg.hpp:19-415) written into the engine's
// options struct, so the tests can check both carry the same defaults.
void ref_default_options(anu_pdhg_options* o) {
  const anukulan::PdhgOptions p;
  std::memset(o, 0, sizeof(*o));
  o->tolerance = p.tolerance;
  o->gap_tolerance = p.gap_tolerance;
  o->max_iterations = p.max_iterations;
  o->time_limit_seconds = p.time_limit_seconds;
  o->termination_check_frequency = p.termination_check_frequency;
  o->absolute_tolerance = p.absolute_tolerance;
  o->require_inf_norm_termination = p.require_inf_norm_termination;
  o->adaptive_step_size = p.adaptive_step_size;
  o->primal_weight_updates = p.primal_weight_updates;
  o->restarts = p.restarts;
  o->halpern = p.halpern;
  o->halpern_restart = p.halpern_restart;
  o->halpern_minimum_epoch = p.halpern_minimum_epoch;
  o->polish_feasibility = p.polish_feasibility;
  o->polish_first_iteration = p.polish_first_iteration;
  o->polish_iteration_factor = p.polish_iteration_factor;
  o->polish_minimum_iterations = p.polish_minimum_iterations;
  o->polish_maximum_iterations = p.polish_maximum_iterations;
  o->polish_on_exit = p.polish_on_exit;
  o->reflection = p.reflection;
  o->constant_step_size = p.constant_step_size;
  o->constant_step_scale = p.constant_step_scale;
  o->restart_on_fixed_point = p.restart_on_fixed_point;
  o->pid_primal_weight = p.pid_primal_weight;
  o->primal_weight_kp = p.primal_weight_kp;
  o->primal_weight_ki = p.primal_weight_ki;
  o->primal_weight_kd = p.primal_weight_kd;
  o->ruiz_iterations = p.scaling.ruiz_iterations;
  o->pock_chambolle = p.scaling.pock_chambolle;
  o->reuse_products = p.reuse_products;
  o->detect_infeasibility = p.detect_infeasibility;
  o->infeasibility_tolerance = p.infeasibility_tolerance;
  o->termination = static_cast<int32_t>(p.termination);
  o->known_matrix_norm = p.known_matrix_norm;
  o->initial_step_size = p.initial_step_size;
  o->initial_primal_weight = p.initial_primal_weight;
  o->verbose = p.verbose;
  o->log_frequency = p.log_frequency;
}

// to_standard_form (src/anukulan/standard_form.cpp:72-165) of a model given
// as CSR rows with row and column bounds. Output capacity: 2*rows rows and
// 2*nnz nonzeros. Returns the standard-form row count, or -1 on failure;
// sizes[0] = num_equalities, sizes[1] = nnz.
int ref_to_standard_form(int32_t rows, int32_t cols, int32_t nnz, const int32_t* start,
                         const int32_t* index, const double* value, const double* objective,
                         const double* row_lower, const double* row_upper,
                         const double* col_lower, const double* col_upper, int maximize,
                         double offset, int32_t* out_start, int32_t* out_index,
                         double* out_value, double* out_c, double* out_q,
                         int32_t* out_origin_row, double* out_origin_sign,
                         double* out_scale_offset, int32_t* sizes) {
  anukulan::Model model;
  anu_csr a{rows, cols, nnz, start, index, value};
  model.constraints = csr_to_matrix(a);
  model.objective.assign(objective, objective + cols);
  model.row_lower.assign(row_lower, row_lower + rows);
  model.row_upper.assign(row_upper, row_upper + rows);
  model.col_lower.assign(col_lower, col_lower + cols);
  model.col_upper.assign(col_upper, col_upper + cols);
  model.col_type.assign(static_cast<std::size_t>(cols), anukulan::VarType::kContinuous);
  model.sense = maximize ? anukulan::ObjSense::kMaximize : anukulan::ObjSense::kMinimize;
  model.objective_offset = offset;
  const anukulan::StandardFormResult sf = anukulan::to_standard_form(model);
  if (!sf.ok) return -1;
  const anukulan::StandardLp& lp = sf.lp;
  for (Int i = 0; i <= lp.k.rows(); ++i) out_start[i] = lp.k.start()[static_cast<std::size_t>(i)];
  for (Int k = 0; k < lp.k.nnz(); ++k) {
    out_index[k] = lp.k.index()[static_cast<std::size_t>(k)];
    out_value[k] = lp.k.value()[static_cast<std::size_t>(k)];
  }
  for (std::size_t j = 0; j < lp.c.size(); ++j) out_c[j] = lp.c[j];
  for (std::size_t i = 0; i < lp.q.size(); ++i) {
    out_q[i] = lp.q[i];
    out_origin_row[i] = lp.row_origin[i].model_row;
    out_origin_sign[i] = lp.row_origin[i].sign;
  }
  out_scale_offset[0] = lp.objective_scale;
  out_scale_offset[1] = lp.objective_offset;
  sizes[0] = lp.num_equalities;
  sizes[1] = lp.k.nnz();
  return lp.k.rows();
}

}  // extern "C"
