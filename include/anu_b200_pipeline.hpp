// anu_b200_pipeline.hpp - anukulan's first-order LP pipeline (presolve ->
// standard form -> PDHG -> postsolve) as one library call, with the PDHG step
// on this engine's kernels.
//
// anukulan assembles this pipeline in its command-line tool
// (app/anukulan_cli.cpp:1398-1500) and has no library function for it. This
// header restates those steps, in that order, over anukulan's own presolve,
// standard form and postsolve, and its solve_pdhg with the LinAlgBackend
// adapter of anu_b200_backend.hpp (or any backend the options name):
//
//   1. presolve (skipped on request); a status other than kReduced ends the
//      pipeline with that status and no solve, as the CLI does;
//   2. to_standard_form of the (reduced) model;
//   3. solve_pdhg on it;
//   4. x mapped back through the postsolve stack;
//   5. y folded from standard-form rows onto model rows (each row's sign and
//      model row, since a two-sided row becomes two), then recovered through
//      the postsolve stack with the reduced model's reduced costs;
//   6. the original model's violation measured at x; with presolve, a PDHG
//      optimum that misses the caller's tolerance on the original model is
//      reported as a numerical error, by the CLI's rule (absolute violation
//      against absolute_tolerance when one is set, else the relative row
//      violation against tolerance).
//
// Compiled with anukulan's headers and sources, like anu_b200_backend.hpp.
#pragma once

#include <string>
#include <vector>

#include "anu_b200_backend.hpp"
#include "anukulan/model.hpp"
#include "anukulan/pdhg.hpp"
#include "anukulan/presolve.hpp"
#include "anukulan/standard_form.hpp"

namespace anu_b200 {

struct PipelineResult {
  // kReduced when the model went on to PDHG; otherwise presolve decided it.
  anukulan::PresolveStatus presolve_status = anukulan::PresolveStatus::kReduced;
  std::string message;
  anukulan::PdhgResult pdhg;        // the solve of the standard-form LP
  std::vector<double> x;            // the original model's columns
  std::vector<double> y;            // the original model's rows
  bool dual_exact = true;           // PostsolveStack::dual_is_exact()
  anukulan::ModelViolation violation;  // measure_violation(original, x)
  bool ok = false;                  // the steps ran (a standard form existed)
};

// `options.backend` null means this engine (anu_b200::backend()), which
// throws without a CUDA device; name another backend to run the same
// pipeline elsewhere.
inline PipelineResult solve_model_pdhg(const anukulan::Model& model,
                                       anukulan::PdhgOptions options,
                                       bool use_presolve = true,
                                       const anukulan::PresolveOptions& presolve_options = {}) {
  using anukulan::Int;
  using anukulan::sz;
  PipelineResult out;
  if (options.backend == nullptr) options.backend = &backend();

  anukulan::PresolveResult pre;
  anukulan::Model solved_model = model;
  if (use_presolve) {
    pre = anukulan::presolve(model, presolve_options);
    out.presolve_status = pre.status;
    if (pre.status != anukulan::PresolveStatus::kReduced) {
      out.message = pre.message;
      return out;
    }
    solved_model = pre.reduced;
  }

  const anukulan::StandardFormResult sf = anukulan::to_standard_form(solved_model);
  if (!sf.ok) {
    out.message = sf.error;
    return out;
  }
  out.pdhg = anukulan::solve_pdhg(sf.lp, options);
  out.x = use_presolve ? pre.postsolve.apply(out.pdhg.x) : out.pdhg.x;

  std::vector<double> model_dual(sz(solved_model.num_rows()), 0.0);
  for (Int i = 0; i < sf.lp.num_rows(); ++i) {
    const auto& origin = sf.lp.row_origin[sz(i)];
    model_dual[sz(origin.model_row)] += origin.sign * out.pdhg.y[sz(i)];
  }
  out.y = model_dual;
  if (use_presolve) {
    std::vector<double> reduced_costs = solved_model.objective;
    for (Int i = 0; i < solved_model.num_rows(); ++i) {
      const double yi = model_dual[sz(i)];
      if (yi == 0.0) continue;
      for (Int e = solved_model.constraints.row_begin(i);
           e < solved_model.constraints.row_end(i); ++e) {
        reduced_costs[sz(solved_model.constraints.index()[sz(e)])] -=
            yi * solved_model.constraints.value()[sz(e)];
      }
    }
    out.y = pre.postsolve.apply_dual(model_dual, reduced_costs, model.objective);
    out.dual_exact = pre.postsolve.dual_is_exact();
  }

  out.violation = anukulan::measure_violation(model, out.x);
  if (use_presolve && out.pdhg.status == anukulan::PdhgStatus::kOptimal) {
    const bool absolute = options.absolute_tolerance > 0.0;
    const double measured =
        absolute ? out.violation.worst() : out.violation.relative_row_violation;
    const double cap = absolute ? options.absolute_tolerance : options.tolerance;
    if (measured > cap) {
      out.pdhg.status = anukulan::PdhgStatus::kNumericalError;
      out.pdhg.message =
          "the reduced model met the tolerance and the original does not; tighten the "
          "tolerance or set an absolute one";
    }
  }
  out.ok = true;
  return out;
}

}  // namespace anu_b200
