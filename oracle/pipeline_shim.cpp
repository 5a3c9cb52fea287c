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

#include "anu_b200_pipeline.hpp"
#include "anu_pdhg.h"
#include "anukulan/backend.hpp"

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

}  // extern "C"
