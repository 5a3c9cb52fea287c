// anu_b200_backend.hpp - anukulan's LinAlgBackend implemented over this
// library's C ABI (anu_backend_*, include/anu_pdhg.h).
//
// This header is the C++ side of the seam. It is compiled together with
// anukulan's own sources (it includes "anukulan/backend.hpp" from the
// anukulan tree), and it lets anukulan's solve_pdhg, unchanged, run its
// arithmetic on these sm_100a kernels:
//
//   anukulan::PdhgOptions options;
//   options.backend = &anu_b200::backend();
//   anukulan::PdhgResult r = anukulan::solve_pdhg(lp, options);
//
// anukulan_b200/integration/cuda_backend_b200.cpp goes one step further: built in place of anukulan's src/anukulan/cuda_backend.cu, it
// makes anukulan::cuda_backend() and therefore default_backend() return this
// adapter, so every caller of solve_pdhg and every test built with
// ANUKULAN_WITH_CUDA runs on these kernels with no source change.
//
// Mapping (src/anukulan/backend.hpp:24-215): one virtual, one anu_backend_*
// call, same argument order. Matrices are uploaded once per
// SparseMatrix::id() (sparse.hpp:51), never keyed by address, and a product
// on a matrix that was not prepared prepares it first, as the reference's
// CUDA backend does (cuda_backend.cu:832-834). Calls run in order on one
// library stream; those that return a value or take a host buffer are
// complete when they return, the pure device operations once queued, as with
// the reference's CUDA backend. A failed call throws std::runtime_error with
// the library's message, the reference's error convention
// (cuda_backend.cu:32-37); a failure inside queued work surfaces at the next
// call that waits.
//
// This route runs one launch per seam call, in FP64. It is the compatibility
// path; anu_pdhg_solve is the fused fast path.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "anu_pdhg.h"
#include "anukulan/backend.hpp"
#include "anukulan/sparse.hpp"

namespace anu_b200 {

class Backend final : public anukulan::LinAlgBackend {
 public:
  using Int = anukulan::Int;
  using SparseMatrix = anukulan::SparseMatrix;

  // Throws when the library sees no usable CUDA device, so that
  // default_backend() falls back to the CPU as it does for the reference's
  // own CUDA backend (backend.cpp:209-221).
  Backend() {
    if (anu_device_count() < 1) throw std::runtime_error("anu_pdhg: no CUDA device");
  }

  std::string name() const override { return "b200"; }

  void prepare(const SparseMatrix& a) const override {
    const anu_csr csr{a.rows(), a.cols(), a.nnz(), a.start().data(), a.index().data(),
                      a.value().data()};
    check(anu_backend_prepare(a.id(), &csr));
  }
  void release() const override { check(anu_backend_release()); }

  double* allocate(Int n) const override {
    double* p = nullptr;
    check(anu_backend_allocate(n, &p));
    return p;
  }
  void deallocate(double* p) const override { check(anu_backend_deallocate(p)); }
  void upload(const double* host, double* target, Int n) const override {
    check(anu_backend_upload(host, target, n));
  }
  void download(const double* source, double* host, Int n) const override {
    check(anu_backend_download(source, host, n));
  }
  void fill(double* target, Int n, double value) const override {
    check(anu_backend_fill(target, n, value));
  }
  void copy(const double* source, double* target, Int n) const override {
    check(anu_backend_copy(source, target, n));
  }

  void multiply(const SparseMatrix& a, const double* x, double* y) const override {
    prepare(a);
    check(anu_backend_multiply(a.id(), x, y));
  }
  // A^T is stored explicitly by the caller, so the transpose product is the
  // plain product of that matrix.
  void multiply_transpose(const SparseMatrix& at, const double* y, double* x) const override {
    prepare(at);
    check(anu_backend_multiply(at.id(), y, x));
  }

  double dot(const double* a, const double* b, Int n) const override {
    double out = 0.0;
    check(anu_backend_dot(a, b, n, &out));
    return out;
  }
  double two_norm(const double* a, Int n) const override {
    double out = 0.0;
    check(anu_backend_two_norm(a, n, &out));
    return out;
  }
  double inf_norm(const double* a, Int n) const override {
    double out = 0.0;
    check(anu_backend_inf_norm(a, n, &out));
    return out;
  }

  void primal_update(Int n, double tau, double gamma, double halpern, const double* x,
                     const double* c, const double* kt_y, const double* lower,
                     const double* upper, const double* anchor, double* x_out, double* dx,
                     double* x_bar) const override {
    check(anu_backend_primal_update(n, tau, gamma, halpern, x, c, kt_y, lower, upper, anchor,
                                    x_out, dx, x_bar));
  }
  void dual_update(Int m, Int num_equalities, double sigma, double gamma, double halpern,
                   const double* y, const double* q, const double* k_x_bar, const double* k_x,
                   const double* anchor_y, const double* anchor_kx, double* y_out, double* dy,
                   double* k_out, double* k_dx) const override {
    check(anu_backend_dual_update(m, num_equalities, sigma, gamma, halpern, y, q, k_x_bar, k_x,
                                  anchor_y, anchor_kx, y_out, dy, k_out, k_dx));
  }

  void accumulate(Int n, double weight, const double* v, double* sum) const override {
    check(anu_backend_accumulate(n, weight, v, sum));
  }
  void scale_into(Int n, double weight, const double* sum, double* out) const override {
    check(anu_backend_scale_into(n, weight, sum, out));
  }

  double weighted_norm_squared(Int n, Int m, const double* dx, const double* dy,
                               double omega) const override {
    double out = 0.0;
    check(anu_backend_weighted_norm_squared(n, m, dx, dy, omega, &out));
    return out;
  }
  void step_size_terms(Int n, Int m, const double* dx, const double* dy, const double* k_dx,
                       double omega, double* interaction, double* movement) const override {
    check(anu_backend_step_size_terms(n, m, dx, dy, k_dx, omega, interaction, movement));
  }

  void convergence_terms(Int n, Int m, const ConvergenceProblem& lp, const double* x,
                         const double* k_x, const double* y, const double* kt_y,
                         ConvergenceTerms* out) const override {
    double t[7] = {0, 0, 0, 0, 0, 0, 0};
    check(anu_backend_convergence_terms(n, m, lp.c, lp.lower, lp.upper, lp.q, lp.row_scale,
                                        lp.col_scale, lp.num_equalities, x, k_x, y, kt_y, t));
    out->primal_sq = t[0];
    out->primal_inf = t[1];
    out->q_dot_y = t[2];
    out->dual_sq = t[3];
    out->dual_inf = t[4];
    out->bound_term = t[5];
    out->c_dot_x = t[6];
  }

  // backend.hpp:213-214: the library times each seam operation's device work
  // with CUDA events while profiling is on (anu_backend_set_profiling) and
  // reports the table the CLI's --profile prints.
  void set_profiling(bool on) const override { check(anu_backend_set_profiling(on ? 1 : 0)); }
  std::string profile_report() const override {
    int32_t length = 0;
    check(anu_backend_profile_report(nullptr, 0, &length));
    std::vector<char> buf(static_cast<std::size_t>(length) + 1, '\0');
    check(anu_backend_profile_report(buf.data(), static_cast<int32_t>(buf.size()), &length));
    return std::string(buf.data());
  }

 private:
  static void check(int rc) {
    if (rc == ANU_OK) return;
    char msg[512];
    anu_last_error(msg, static_cast<int32_t>(sizeof msg));
    throw std::runtime_error(std::string("anu_pdhg: ") + msg);
  }
};

// One process-wide instance, like the reference's backends (cuda_backend.cu:
// 894-897). Its first use throws when there is no device, and a later call
// tries again.
inline const anukulan::LinAlgBackend& backend() {
  static const Backend instance;
  return instance;
}

}  // namespace anu_b200
