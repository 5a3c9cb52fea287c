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
// solve_model_crossover runs the CLI's `simplex --crossover` path
// (app/anukulan_cli.cpp:574-636) the same way: presolve and standard form, a
// PDHG seed on this engine at the crossover tolerance, crossover_basis at the
// seed, the simplex from that basis with the cold solve when the seeded one
// misses the optimum, and x through the postsolve stack. finish_with_simplex
// is its crossover-and-simplex step alone, for a point the caller already
// has, such as each case of a case stack.
//
// Compiled with anukulan's headers and sources, like anu_b200_backend.hpp.
#pragma once

#include <algorithm>
#include <string>
#include <vector>

#include "anu_b200_backend.hpp"
#include "anukulan/crossover.hpp"
#include "anukulan/model.hpp"
#include "anukulan/pdhg.hpp"
#include "anukulan/presolve.hpp"
#include "anukulan/simplex.hpp"
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

// The seed the CLI asks of PDHG before crossover, with its defaults
// (app/anukulan_cli.cpp:430-482 and 597-611).
struct CrossoverSettings {
  bool enabled = true;                 // false: no seed, the simplex starts cold
  double tolerance = 1e-4;             // PDHG tolerance and gap tolerance of the seed
  anukulan::Int max_iterations = 5000; // iteration budget, at least this
  double iterations_per_row = 10.0;    // ... and at least this many per row (0: off)
  anukulan::CrossoverOptions crossover;
};

struct SimplexFinish {
  anukulan::CrossoverResult crossover;
  anukulan::SimplexResult simplex;   // the answer: seeded, or cold after a miss
  anukulan::Int seeded_iterations = 0;  // pivots of the seeded solve, when there was one
  bool seeded = false;     // the crossover gave a basis and the simplex started from it
  bool fell_back = false;  // the seeded solve missed the optimum; the cold one answered
};

// crossover_basis at (x, y), then solve_lp from the basis it gives; when that
// basis exists and the seeded solve does not end optimal, the cold solve is
// run and kept if it is optimal (app/anukulan_cli.cpp:607-631). Without a
// basis the simplex starts cold. seeded_pivot_limit > 0 caps the seeded
// solve's pivots (the CLI has no cap): a basis that would take longer than a
// cold start ends there and the cold solve answers instead.
inline SimplexFinish finish_with_simplex(const anukulan::StandardLp& lp,
                                         const std::vector<double>& x,
                                         const std::vector<double>& y,
                                         const anukulan::SimplexOptions& simplex_options = {},
                                         const anukulan::CrossoverOptions& crossover_options = {},
                                         anukulan::Int seeded_pivot_limit = 0) {
  SimplexFinish out;
  out.crossover = anukulan::crossover_basis(lp, x, y, crossover_options);
  anukulan::SimplexOptions options = simplex_options;
  if (out.crossover.ok) {
    options.start_basic = &out.crossover.basic;
    options.start_status = &out.crossover.status;
    if (seeded_pivot_limit > 0)
      options.max_iterations = std::min(options.max_iterations, seeded_pivot_limit);
    out.seeded = true;
  }
  out.simplex = anukulan::solve_lp(lp, options);
  if (out.seeded) out.seeded_iterations = out.simplex.iterations;
  if (out.seeded && out.simplex.status != anukulan::SimplexStatus::kOptimal) {
    anukulan::SimplexOptions cold = simplex_options;
    cold.start_basic = nullptr;
    cold.start_status = nullptr;
    anukulan::SimplexResult again = anukulan::solve_lp(lp, cold);
    if (again.status == anukulan::SimplexStatus::kOptimal) {
      out.simplex = std::move(again);
      out.fell_back = true;
    }
  }
  return out;
}

struct CrossoverPipelineResult {
  anukulan::PresolveStatus presolve_status = anukulan::PresolveStatus::kReduced;
  std::string message;
  anukulan::PdhgResult seed;        // the PDHG seed on the standard-form LP
  SimplexFinish finish;             // crossover and simplex from the seed
  std::vector<double> x;            // the original model's columns
  double objective = 0.0;           // the original model's objective at x
  anukulan::ModelViolation violation;  // measure_violation(original, x)
  bool ok = false;                  // the steps ran (a standard form existed)
};

// The CLI's `simplex --crossover` with the seed on this engine: `options`
// supplies the backend (null: this engine) and every PDHG setting except the
// tolerance, gap tolerance and budget, which `settings` fixes as the CLI does.
inline CrossoverPipelineResult solve_model_crossover(
    const anukulan::Model& model, anukulan::PdhgOptions options,
    const anukulan::SimplexOptions& simplex_options = {}, const CrossoverSettings& settings = {},
    bool use_presolve = true, const anukulan::PresolveOptions& presolve_options = {}) {
  using anukulan::sz;
  CrossoverPipelineResult out;
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

  if (!settings.enabled) {
    out.finish.simplex = anukulan::solve_lp(sf.lp, simplex_options);
  } else {
    options.tolerance = settings.tolerance;
    options.gap_tolerance = settings.tolerance;
    anukulan::Int budget = settings.max_iterations;
    if (settings.iterations_per_row > 0.0)
      budget = std::max<anukulan::Int>(
          budget, static_cast<anukulan::Int>(settings.iterations_per_row * sf.lp.num_rows()));
    if (budget > 0) options.max_iterations = budget;
    out.seed = anukulan::solve_pdhg(sf.lp, options);
    out.finish = finish_with_simplex(sf.lp, out.seed.x, out.seed.y, simplex_options,
                                     settings.crossover);
  }

  out.x = out.finish.simplex.x;
  if (use_presolve && !out.x.empty()) out.x = pre.postsolve.apply(out.x);
  if (out.x.size() == sz(model.num_cols())) {
    double obj = model.objective_offset;
    for (std::size_t j = 0; j < out.x.size(); ++j) obj += model.objective[j] * out.x[j];
    out.objective = obj;
    out.violation = anukulan::measure_violation(model, out.x);
  }
  out.ok = true;
  return out;
}

struct CaseFinish {
  anukulan::PresolveStatus presolve_status = anukulan::PresolveStatus::kReduced;
  std::string message;
  SimplexFinish finish;             // crossover and simplex on the (reduced) model
  std::vector<double> x;            // the model's columns
  double objective = 0.0;           // the model's objective at x
  anukulan::ModelViolation violation;  // measure_violation(model, x)
  bool ok = false;                  // the steps ran
};

// Finishes one case exactly from a first-order point of its unpresolved
// standard form (x: its columns, y: its rows), as a case stack's cases come
// back from this engine. y is folded onto the model's rows (row_origin); with
// presolve both are carried onto the reduced model's surviving columns and
// rows (reduced_to_original, reduced_row_to_original) and onto its standard
// form, whose rows take the sign of their origin. There crossover_basis and
// the simplex run (finish_with_simplex), and x goes back through the
// postsolve stack. Crossover gets a basis from an approximate point, so
// nothing here needs the point to be exact: a reduction that rewrites a
// column only makes the guess worse, never the answer.
//
// Presolve is off by default. On the refinery-shaped case stack a first-order
// point of the full model, carried onto the presolved model, gives crossover
// a basis that needs about 11,000 pivots there, against about 300 on the full
// model from the same point and about 1,500 for a cold start; the crossover
// on a reduced model pays off when the seed is computed on that model
// (solve_model_crossover).
inline CaseFinish finish_model_with_simplex(
    const anukulan::Model& model, const std::vector<double>& x, const std::vector<double>& y,
    bool use_presolve = false, const anukulan::SimplexOptions& simplex_options = {},
    const anukulan::CrossoverOptions& crossover_options = {},
    const anukulan::PresolveOptions& presolve_options = {},
    anukulan::Int seeded_pivot_limit = 0) {
  using anukulan::Int;
  using anukulan::sz;
  CaseFinish out;
  const anukulan::StandardFormResult full = anukulan::to_standard_form(model);
  if (!full.ok) {
    out.message = full.error;
    return out;
  }
  if (x.size() != sz(full.lp.num_cols()) || y.size() != sz(full.lp.num_rows())) {
    out.message = "the point does not match the model's standard form";
    return out;
  }
  std::vector<double> model_y(sz(model.num_rows()), 0.0);
  for (Int i = 0; i < full.lp.num_rows(); ++i) {
    const auto& origin = full.lp.row_origin[sz(i)];
    model_y[sz(origin.model_row)] += origin.sign * y[sz(i)];
  }

  anukulan::PresolveResult pre;
  const anukulan::Model* solved = &model;
  std::vector<double> solved_x = x, solved_y = model_y;
  if (use_presolve) {
    pre = anukulan::presolve(model, presolve_options);
    out.presolve_status = pre.status;
    if (pre.status != anukulan::PresolveStatus::kReduced) {
      out.message = pre.message;
      return out;
    }
    solved = &pre.reduced;
    const std::vector<Int>& cols = pre.postsolve.reduced_to_original();
    const std::vector<Int>& rows = pre.postsolve.reduced_row_to_original();
    solved_x.assign(cols.size(), 0.0);
    for (std::size_t j = 0; j < cols.size(); ++j) solved_x[j] = x[sz(cols[j])];
    solved_y.assign(rows.size(), 0.0);
    for (std::size_t i = 0; i < rows.size(); ++i) solved_y[i] = model_y[sz(rows[i])];
  }
  const anukulan::StandardFormResult sf = anukulan::to_standard_form(*solved);
  if (!sf.ok) {
    out.message = sf.error;
    return out;
  }
  std::vector<double> sf_y(sz(sf.lp.num_rows()), 0.0);
  for (Int i = 0; i < sf.lp.num_rows(); ++i) {
    const auto& origin = sf.lp.row_origin[sz(i)];
    const double v = origin.sign * solved_y[sz(origin.model_row)];
    sf_y[sz(i)] = i < sf.lp.num_equalities ? v : std::max(v, 0.0);
  }
  solved_x.resize(sz(sf.lp.num_cols()), 0.0);
  out.finish = finish_with_simplex(sf.lp, solved_x, sf_y, simplex_options, crossover_options,
                                   seeded_pivot_limit);
  out.x = out.finish.simplex.x;
  if (use_presolve && !out.x.empty()) out.x = pre.postsolve.apply(out.x);
  if (out.x.size() == sz(model.num_cols())) {
    double obj = model.objective_offset;
    for (std::size_t j = 0; j < out.x.size(); ++j) obj += model.objective[j] * out.x[j];
    out.objective = obj;
    out.violation = anukulan::measure_violation(model, out.x);
  }
  out.ok = true;
  return out;
}

}  // namespace anu_b200
