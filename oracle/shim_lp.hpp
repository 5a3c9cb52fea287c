// Test infrastructure, not product code: conversions from the engine's C
// structs (include/anu_pdhg.h) to the reference's types, shared by the shims
// that oracle/Makefile compiles with the reference's own sources.
#pragma once

#include <cstddef>
#include <utility>
#include <vector>

#include "anu_pdhg.h"
#include "anukulan/pdhg.hpp"
#include "anukulan/sparse.hpp"
#include "anukulan/standard_form.hpp"

namespace shim {

using anukulan::Int;

inline anukulan::SparseMatrix csr_to_matrix(const anu_csr& a) {
  std::vector<anukulan::Triplet> t;
  t.reserve(static_cast<std::size_t>(a.nnz));
  for (Int r = 0; r < a.rows; ++r) {
    for (Int k = a.start[r]; k < a.start[r + 1]; ++k) {
      t.push_back(anukulan::Triplet{r, a.index[k], a.value[k]});
    }
  }
  return anukulan::SparseMatrix::from_triplets(a.rows, a.cols, std::move(t));
}

inline anukulan::StandardLp to_lp(const anu_lp& in) {
  anukulan::StandardLp lp;
  lp.k = csr_to_matrix(in.k);
  lp.kt = lp.k.transpose();
  const std::size_t n = static_cast<std::size_t>(in.k.cols);
  const std::size_t m = static_cast<std::size_t>(in.k.rows);
  lp.c.assign(in.c, in.c + n);
  lp.q.assign(in.q, in.q + m);
  lp.lower.assign(in.lower, in.lower + n);
  lp.upper.assign(in.upper, in.upper + n);
  lp.num_equalities = in.num_equalities;
  lp.objective_scale = in.objective_scale;
  lp.objective_offset = in.objective_offset;
  lp.row_origin.resize(m);
  for (std::size_t i = 0; i < m; ++i) {
    lp.row_origin[i] = anukulan::StandardLp::RowOrigin{static_cast<Int>(i), 1.0};
  }
  return lp;
}

inline anukulan::PdhgOptions to_options(const anu_pdhg_options& o) {
  anukulan::PdhgOptions p;
  p.tolerance = o.tolerance;
  p.gap_tolerance = o.gap_tolerance;
  p.max_iterations = o.max_iterations;
  p.time_limit_seconds = o.time_limit_seconds;
  p.termination_check_frequency = o.termination_check_frequency;
  p.absolute_tolerance = o.absolute_tolerance;
  p.require_inf_norm_termination = o.require_inf_norm_termination != 0;
  p.adaptive_step_size = o.adaptive_step_size != 0;
  p.primal_weight_updates = o.primal_weight_updates != 0;
  p.restarts = o.restarts != 0;
  p.halpern = o.halpern != 0;
  p.halpern_restart = o.halpern_restart != 0;
  p.halpern_minimum_epoch = o.halpern_minimum_epoch;
  p.polish_feasibility = o.polish_feasibility != 0;
  p.polish_first_iteration = o.polish_first_iteration;
  p.polish_iteration_factor = o.polish_iteration_factor;
  p.polish_minimum_iterations = o.polish_minimum_iterations;
  p.polish_maximum_iterations = o.polish_maximum_iterations;
  p.polish_on_exit = o.polish_on_exit != 0;
  p.reflection = o.reflection;
  p.constant_step_size = o.constant_step_size != 0;
  p.constant_step_scale = o.constant_step_scale;
  p.restart_on_fixed_point = o.restart_on_fixed_point != 0;
  p.pid_primal_weight = o.pid_primal_weight != 0;
  p.primal_weight_kp = o.primal_weight_kp;
  p.primal_weight_ki = o.primal_weight_ki;
  p.primal_weight_kd = o.primal_weight_kd;
  p.scaling.ruiz_iterations = o.ruiz_iterations;
  p.scaling.pock_chambolle = o.pock_chambolle != 0;
  p.reuse_products = o.reuse_products != 0;
  p.detect_infeasibility = o.detect_infeasibility != 0;
  p.infeasibility_tolerance = o.infeasibility_tolerance;
  switch (o.termination) {
    case ANU_TERMINATION_PRIMAL_FEASIBILITY:
      p.termination = anukulan::PdhgOptions::Termination::kPrimalFeasibility;
      break;
    case ANU_TERMINATION_DUAL_FEASIBILITY:
      p.termination = anukulan::PdhgOptions::Termination::kDualFeasibility;
      break;
    default:
      p.termination = anukulan::PdhgOptions::Termination::kFull;
  }
  p.known_matrix_norm = o.known_matrix_norm;
  p.initial_step_size = o.initial_step_size;
  p.initial_primal_weight = o.initial_primal_weight;
  p.verbose = o.verbose != 0;
  p.log_frequency = o.log_frequency;
  return p;
}

}  // namespace shim
