// Test infrastructure: a C entry over anu_b200::solve_model_pdhg
// (include/anu_b200_pipeline.hpp), the reference's first-order pipeline
// (presolve -> standard form -> solve_pdhg -> postsolve, app/anukulan_cli.cpp:
// 1398-1500) with its PDHG step on a chosen backend. Built only into
// oracle/_ref/libanuref_b200.so, with the reference's unmodified sources.

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

#include <chrono>

#include "anu_b200_pipeline.hpp"
#include "anu_pdhg.h"
#include "anukulan/backend.hpp"
#include "shim_lp.hpp"

namespace {

anukulan::Model to_model(int32_t rows, int32_t cols, int32_t nnz, const int32_t* start,
                         const int32_t* index, const double* value, const double* objective,
                         const double* row_lower, const double* row_upper,
                         const double* col_lower, const double* col_upper, int maximize,
                         double offset) {
  std::vector<anukulan::Triplet> t;
  t.reserve(static_cast<std::size_t>(nnz));
  for (int32_t r = 0; r < rows; ++r)
    for (int32_t k = start[r]; k < start[r + 1]; ++k)
      t.push_back(anukulan::Triplet{r, index[k], value[k]});
  anukulan::Model model;
  model.constraints = anukulan::SparseMatrix::from_triplets(rows, cols, std::move(t));
  model.objective.assign(objective, objective + cols);
  model.row_lower.assign(row_lower, row_lower + rows);
  model.row_upper.assign(row_upper, row_upper + rows);
  model.col_lower.assign(col_lower, col_lower + cols);
  model.col_upper.assign(col_upper, col_upper + cols);
  model.col_type.assign(static_cast<std::size_t>(cols), anukulan::VarType::kContinuous);
  model.sense = maximize ? anukulan::ObjSense::kMaximize : anukulan::ObjSense::kMinimize;
  model.objective_offset = offset;
  return model;
}

}  // namespace

extern "C" {

// backend: 1 = the reference's cpu_backend(), 0 = the engine (the adapter).
// Returns 0 when the pipeline ran, 1 when presolve decided the model or no
// standard form exists (presolve_status and out->message say why), 2 on an
// exception. out->objective is the original model's objective at x, in its
// sense; out->status is the PDHG status after the original-model check.
// info[0] = worst violation, info[1] = relative row violation,
// info[2] = 1 if the dual is exact, info[3] = presolve status.
int ref_pipeline_solve(int32_t rows, int32_t cols, int32_t nnz, const int32_t* start,
                       const int32_t* index, const double* value, const double* objective,
                       const double* row_lower, const double* row_upper,
                       const double* col_lower, const double* col_upper, int maximize,
                       double offset, const anu_pdhg_options* opt, int use_presolve,
                       int backend, double* x, double* y, anu_pdhg_result* out, double* info) {
  std::memset(out, 0, sizeof(*out));
  try {
    const anukulan::Model model = to_model(rows, cols, nnz, start, index, value, objective,
                                           row_lower, row_upper, col_lower, col_upper,
                                           maximize, offset);
    anukulan::PdhgOptions options;
    options.tolerance = opt->tolerance;
    options.gap_tolerance = opt->gap_tolerance;
    options.max_iterations = opt->max_iterations;
    options.absolute_tolerance = opt->absolute_tolerance;
    options.backend = backend == 1 ? &anukulan::cpu_backend() : nullptr;
    const anu_b200::PipelineResult r = anu_b200::solve_model_pdhg(model, options, use_presolve != 0);
    info[3] = static_cast<double>(static_cast<int>(r.presolve_status));
    if (!r.ok) {
      std::snprintf(out->message, sizeof(out->message), "%s", r.message.c_str());
      return 1;
    }
    double obj = model.objective_offset;
    for (int32_t j = 0; j < cols; ++j) obj += model.objective[static_cast<std::size_t>(j)] * r.x[static_cast<std::size_t>(j)];
    out->status = static_cast<int32_t>(r.pdhg.status);
    out->objective = obj;
    out->iterations = r.pdhg.iterations;
    out->restarts = r.pdhg.restarts;
    std::snprintf(out->message, sizeof(out->message), "%s", r.pdhg.message.c_str());
    for (int32_t j = 0; j < cols; ++j) x[j] = r.x[static_cast<std::size_t>(j)];
    for (int32_t i = 0; i < rows; ++i) y[i] = r.y[static_cast<std::size_t>(i)];
    info[0] = r.violation.worst();
    info[1] = r.violation.relative_row_violation;
    info[2] = r.dual_exact ? 1.0 : 0.0;
    return 0;
  } catch (const std::exception& e) {
    std::snprintf(out->message, sizeof(out->message), "exception: %s", e.what());
    return 2;
  }
}

// anu_b200::solve_model_crossover: the CLI's `simplex --crossover` with the
// PDHG seed on a chosen backend (1 = cpu_backend(), 0 = the engine). opt
// gives the seed's other PDHG settings; crossover_tolerance its tolerance
// (0: no seed, the simplex starts cold, as the CLI without --crossover).
// Returns 0 when the steps ran, 1 when presolve decided the model or no
// standard form exists, 2 on an exception. x (cols) receives the original
// model's columns. info[0] simplex status, [1] simplex pivots of the answer,
// [2] 1 if seeded, [3] 1 if it fell back to the cold solve, [4] pivots of the
// seeded solve, [5] seed PDHG iterations, [6] seed PDHG status, [7] relative
// row violation, [8] objective, [9] crossover candidates, [10] pushed,
// [11] presolve status.
int ref_pipeline_crossover(int32_t rows, int32_t cols, int32_t nnz, const int32_t* start,
                           const int32_t* index, const double* value, const double* objective,
                           const double* row_lower, const double* row_upper,
                           const double* col_lower, const double* col_upper, int maximize,
                           double offset, const anu_pdhg_options* opt, int use_presolve,
                           int backend, double crossover_tolerance, double* x, double* info) {
  try {
    const anukulan::Model model = to_model(rows, cols, nnz, start, index, value, objective,
                                           row_lower, row_upper, col_lower, col_upper,
                                           maximize, offset);
    anukulan::PdhgOptions options = shim::to_options(*opt);
    options.backend = backend == 1 ? &anukulan::cpu_backend() : nullptr;
    anu_b200::CrossoverSettings settings;
    settings.enabled = crossover_tolerance > 0.0;
    if (settings.enabled) settings.tolerance = crossover_tolerance;
    const anu_b200::CrossoverPipelineResult r =
        anu_b200::solve_model_crossover(model, options, {}, settings, use_presolve != 0);
    info[11] = static_cast<double>(static_cast<int>(r.presolve_status));
    if (!r.ok) return 1;
    info[0] = static_cast<double>(static_cast<int>(r.finish.simplex.status));
    info[1] = r.finish.simplex.iterations;
    info[2] = r.finish.seeded ? 1.0 : 0.0;
    info[3] = r.finish.fell_back ? 1.0 : 0.0;
    info[4] = r.finish.seeded_iterations;
    info[5] = r.seed.iterations;
    info[6] = static_cast<double>(static_cast<int>(r.seed.status));
    info[7] = r.violation.relative_row_violation;
    info[8] = r.objective;
    info[9] = r.finish.crossover.candidates;
    info[10] = r.finish.crossover.pushed;
    for (std::size_t j = 0; j < r.x.size() && j < static_cast<std::size_t>(cols); ++j) x[j] = r.x[j];
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_pipeline_crossover: %s\n", e.what());
    return 2;
  }
}

// anu_b200::finish_with_simplex on a standard-form LP at a given point
// (x: n, y: m): crossover_basis, the simplex from its basis, the cold solve
// after a miss; dual = 1 runs the dual simplex (SimplexOptions::Algorithm),
// 0 the default. x_out (n) and y_out (m) receive the simplex answer.
// info[0] simplex status, [1] pivots of the answer, [2] seeded, [3] fell
// back, [4] pivots of the seeded solve, [5] objective (standard form, with
// its scale and offset), [6] seconds, [7] crossover candidates, [8] pushed.
// When basic_out is given the simplex's final basis is written as by
// ref_simplex_basis. Returns 0, 1 when a basis capacity is too small, or 2 on
// an exception.
int ref_finish_simplex(const anu_lp* lp_in, const double* x, const double* y, int dual,
                       double* x_out, double* y_out, double* info, int32_t* basic_out,
                       int32_t* nb_out, int32_t* status_out, int32_t* ns_out) {
  try {
    const auto t0 = std::chrono::steady_clock::now();
    const anukulan::StandardLp lp = shim::to_lp(*lp_in);
    const std::size_t n = static_cast<std::size_t>(lp_in->k.cols);
    const std::size_t m = static_cast<std::size_t>(lp_in->k.rows);
    anukulan::SimplexOptions so;
    if (dual) so.algorithm = anukulan::SimplexOptions::Algorithm::kDual;
    const anu_b200::SimplexFinish f = anu_b200::finish_with_simplex(
        lp, std::vector<double>(x, x + n), std::vector<double>(y, y + m), so);
    const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    info[0] = static_cast<double>(static_cast<int>(f.simplex.status));
    info[1] = f.simplex.iterations;
    info[2] = f.seeded ? 1.0 : 0.0;
    info[3] = f.fell_back ? 1.0 : 0.0;
    info[4] = f.seeded_iterations;
    info[5] = f.simplex.objective;
    info[6] = dt;
    info[7] = f.crossover.candidates;
    info[8] = f.crossover.pushed;
    for (std::size_t j = 0; j < f.simplex.x.size() && j < n; ++j) x_out[j] = f.simplex.x[j];
    for (std::size_t i = 0; i < f.simplex.y.size() && i < m; ++i) y_out[i] = f.simplex.y[i];
    if (basic_out != nullptr) {
      if (static_cast<int32_t>(f.simplex.final_basic.size()) > *nb_out ||
          static_cast<int32_t>(f.simplex.final_status.size()) > *ns_out)
        return 1;
      for (std::size_t i = 0; i < f.simplex.final_basic.size(); ++i)
        basic_out[i] = f.simplex.final_basic[i];
      for (std::size_t i = 0; i < f.simplex.final_status.size(); ++i)
        status_out[i] = static_cast<int32_t>(f.simplex.final_status[i]);
      *nb_out = static_cast<int32_t>(f.simplex.final_basic.size());
      *ns_out = static_cast<int32_t>(f.simplex.final_status.size());
    }
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_finish_simplex: %s\n", e.what());
    return 2;
  }
}

// anu_b200::finish_model_with_simplex: one case finished exactly from a
// point (x: cols, y: the rows of the model's standard form, sf_rows of
// them). dual = 1 runs the dual simplex. x_out (cols) receives the model's
// columns; seeded_pivot_limit > 0 caps the seeded solve's pivots. info[0]
// simplex status, [1] pivots of the answer, [2] seeded,
// [3] fell back, [4] pivots of the seeded solve, [5] objective (model),
// [6] seconds, [7] crossover candidates, [8] pushed, [9] relative row
// violation, [10] presolve status. Returns 0 when the steps ran, 1 when
// presolve decided the model or the point does not fit, 2 on an exception.
int ref_finish_model(int32_t rows, int32_t cols, int32_t nnz, const int32_t* start,
                     const int32_t* index, const double* value, const double* objective,
                     const double* row_lower, const double* row_upper, const double* col_lower,
                     const double* col_upper, int maximize, double offset, const double* x,
                     const double* y, int32_t sf_rows, int use_presolve, int dual,
                     int32_t seeded_pivot_limit, double* x_out, double* info) {
  try {
    const auto t0 = std::chrono::steady_clock::now();
    const anukulan::Model model = to_model(rows, cols, nnz, start, index, value, objective,
                                           row_lower, row_upper, col_lower, col_upper,
                                           maximize, offset);
    anukulan::SimplexOptions so;
    if (dual) so.algorithm = anukulan::SimplexOptions::Algorithm::kDual;
    const anu_b200::CaseFinish f = anu_b200::finish_model_with_simplex(
        model, std::vector<double>(x, x + cols), std::vector<double>(y, y + sf_rows),
        use_presolve != 0, so, {}, {}, seeded_pivot_limit);
    info[10] = static_cast<double>(static_cast<int>(f.presolve_status));
    if (!f.ok) {
      std::fprintf(stderr, "ref_finish_model: %s\n", f.message.c_str());
      return 1;
    }
    info[0] = static_cast<double>(static_cast<int>(f.finish.simplex.status));
    info[1] = f.finish.simplex.iterations;
    info[2] = f.finish.seeded ? 1.0 : 0.0;
    info[3] = f.finish.fell_back ? 1.0 : 0.0;
    info[4] = f.finish.seeded_iterations;
    info[5] = f.objective;
    info[7] = f.finish.crossover.candidates;
    info[8] = f.finish.crossover.pushed;
    info[9] = f.violation.relative_row_violation;
    for (std::size_t j = 0; j < f.x.size() && j < static_cast<std::size_t>(cols); ++j)
      x_out[j] = f.x[j];
    info[6] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_finish_model: %s\n", e.what());
    return 2;
  }
}

// The reference's `family --from-first` step (app/anukulan_cli.cpp:1065-1230)
// for one member: solve_lp started from a remembered basis, or cold (and
// remembering its basis) when basic is NULL. basic holds nb entries, status
// ns (VarStatus as int). When basic_out is given the final basis is written
// to basic_out (capacity *nb_out) and status_out (capacity *ns_out), and
// *nb_out / *ns_out receive the lengths. info[0] status, [1] pivots,
// [2] objective, [3] seconds. Returns 0, 1 when a capacity is too small, 2 on
// an exception.
int ref_simplex_basis(const anu_lp* lp_in, const int32_t* basic, int32_t nb,
                      const int32_t* status, int32_t ns, int32_t* basic_out, int32_t* nb_out,
                      int32_t* status_out, int32_t* ns_out, double* info) {
  try {
    const anukulan::StandardLp lp = shim::to_lp(*lp_in);
    anukulan::SimplexOptions so;
    so.algorithm = anukulan::SimplexOptions::Algorithm::kDual;
    std::vector<anukulan::Int> b;
    std::vector<anukulan::VarStatus> st;
    if (basic != nullptr) {
      b.assign(basic, basic + nb);
      st.reserve(static_cast<std::size_t>(ns));
      for (int32_t i = 0; i < ns; ++i) st.push_back(static_cast<anukulan::VarStatus>(status[i]));
      so.start_basic = &b;
      so.start_status = &st;
    }
    const anukulan::SimplexResult r = anukulan::solve_lp(lp, so);
    info[0] = static_cast<double>(static_cast<int>(r.status));
    info[1] = r.iterations;
    info[2] = r.objective;
    info[3] = r.solve_seconds;
    if (basic_out != nullptr) {
      if (static_cast<int32_t>(r.final_basic.size()) > *nb_out ||
          static_cast<int32_t>(r.final_status.size()) > *ns_out)
        return 1;
      for (std::size_t i = 0; i < r.final_basic.size(); ++i) basic_out[i] = r.final_basic[i];
      for (std::size_t i = 0; i < r.final_status.size(); ++i)
        status_out[i] = static_cast<int32_t>(r.final_status[i]);
      *nb_out = static_cast<int32_t>(r.final_basic.size());
      *ns_out = static_cast<int32_t>(r.final_status.size());
    }
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_simplex_basis: %s\n", e.what());
    return 2;
  }
}

}  // extern "C"
