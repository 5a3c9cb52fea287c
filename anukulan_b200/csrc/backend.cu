// The LinAlgBackend seam (src/anukulan/backend.hpp:24-215) on device memory.
//
// Each anu_backend_* entry point is one coarse operation of the reference's
// backend interface, so a thin C++ adapter class can implement LinAlgBackend
// over this library and run the reference's own solve_pdhg on these kernels.
// Matrices are cached under the caller's identity key (SparseMatrix::id(),
// src/anukulan/sparse.hpp:51), never by address. Operations run in order on
// one library stream. Those that hand the host a value or take a host buffer
// (upload, download, the reductions, allocate) return when done; the pure
// device operations (fill, copy, the products, the updates, accumulate,
// scale_into) return once queued, as the reference's CUDA backend's kernel
// launches do (cuda_backend.cu:530-559, 832-858).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "engine.hpp"

namespace anu {
namespace {

struct Timing {
  double seconds = 0.0;
  long long calls = 0;
};

struct BackendState {
  std::mutex lock;
  Exec exec;
  std::map<uint64_t, std::unique_ptr<DevCsr>> matrices;
  DevBuf<double> partial;
  DevBuf<double> out;
  bool ready = false;
  // Profiling (LinAlgBackend::set_profiling, backend.hpp:213): per seam
  // operation, the device time of the work it queued and how often it ran.
  bool profiling = false;
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  std::map<std::string, Timing> timings;
  // Matrices prepared while profiling was on, described when prepared: the
  // reference's solve_pdhg releases its matrices before it returns, which is
  // before a caller asks for the report.
  std::map<uint64_t, std::string> profiled_matrices;
};

BackendState& state() {
  static BackendState s;
  return s;
}

void ensure(BackendState& s) {
  if (s.ready) return;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    throw Error(ANU_ERR_NO_DEVICE, "no CUDA device is available; this engine has no CPU fallback");
  }
  // A blocking stream: ordered with the legacy default stream, so work a
  // caller queues there (anu_backend_convergence_terms_noalloc among it)
  // runs after the seam operations queued before it.
  ANU_CUDA(cudaStreamCreateWithFlags(&s.exec.stream, cudaStreamDefault));
  s.out.alloc(16);
  s.ready = true;
}

// Times the device work one seam operation queues on the library stream:
// an event before it, an event after it and a wait for the second. With
// profiling off it does nothing, so the ordinary path pays one branch. The
// wait serialises the stream, so a profiled run is slower than a plain one;
// the shares are what it is for.
class Timed {
 public:
  Timed(BackendState& s, const char* name) : s_(s), name_(name) {
    if (s_.profiling) on_ = cudaEventRecord(s_.ev_start, s_.exec.stream) == cudaSuccess;
  }
  Timed(const Timed&) = delete;
  Timed& operator=(const Timed&) = delete;
  ~Timed() {
    if (!on_) return;
    float ms = 0.0f;
    if (cudaEventRecord(s_.ev_stop, s_.exec.stream) != cudaSuccess ||
        cudaEventSynchronize(s_.ev_stop) != cudaSuccess ||
        cudaEventElapsedTime(&ms, s_.ev_start, s_.ev_stop) != cudaSuccess)
      return;  // a failure in the queued work surfaces at the next waiting call
    Timing& t = s_.timings[name_];
    t.seconds += static_cast<double>(ms) * 1e-3;
    t.calls += 1;
  }

 private:
  BackendState& s_;
  std::string name_;
  bool on_ = false;
};

std::string profile_report(const BackendState& s) {
  if (s.timings.empty()) return {};
  std::vector<std::pair<std::string, Timing>> rows(s.timings.begin(), s.timings.end());
  std::sort(rows.begin(), rows.end(),
            [](const auto& a, const auto& b) { return a.second.seconds > b.second.seconds; });
  double total = 0.0;
  long long calls = 0;
  for (const auto& r : rows) {
    total += r.second.seconds;
    calls += r.second.calls;
  }
  std::string out;
  char line[256];
  std::snprintf(line, sizeof(line), "%-26s %12s %9s %12s %10s\n", "operation", "seconds",
                "share", "calls", "us each");
  out += line;
  for (const auto& [name, t] : rows) {
    std::snprintf(line, sizeof(line), "%-26s %12.6f %8.1f%% %12lld %10.2f\n", name.c_str(),
                  t.seconds, total > 0.0 ? 100.0 * t.seconds / total : 0.0, t.calls,
                  t.calls > 0 ? 1e6 * t.seconds / static_cast<double>(t.calls) : 0.0);
    out += line;
  }
  std::snprintf(line, sizeof(line), "%-26s %12.6f %8.1f%% %12lld\n", "total on the device",
                total, 100.0, calls);
  out += line;
  if (!s.profiled_matrices.empty()) {
    out += "\nmatrices prepared while profiling (schedule of the product kernel):\n";
    for (const auto& m : s.profiled_matrices) out += m.second;
  }
  return out;
}

std::string describe_matrix(uint64_t id, const DevCsr& d) {
  char line[256];
  if (d.uniform_len > 0)
    std::snprintf(line, sizeof(line), "  id %-12llu %9d rows %10d nonzeros %7.2f per row  ell, %d per row\n",
                  static_cast<unsigned long long>(id), d.rows, d.nnz,
                  d.rows > 0 ? static_cast<double>(d.nnz) / d.rows : 0.0, d.uniform_len);
  else
    std::snprintf(line, sizeof(line), "  id %-12llu %9d rows %10d nonzeros %7.2f per row  %d row blocks\n",
                  static_cast<unsigned long long>(id), d.rows, d.nnz,
                  d.rows > 0 ? static_cast<double>(d.nnz) / d.rows : 0.0, d.num_blocks);
  return line;
}

template <class F>
int guard(F&& body) {
  try {
    clear_last_error();
    BackendState& s = state();
    std::lock_guard<std::mutex> g(s.lock);
    ensure(s);
    body(s);
    return ANU_OK;
  } catch (const Error& e) {
    set_last_error(e.code, e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(ANU_ERR_INTERNAL, e.what());
    return ANU_ERR_INTERNAL;
  }
}

// backend.cpp:60-79, one thread per entry, no FMA contraction.
__global__ void primal_update_kernel(int64_t n, double tau, double gamma, double halpern,
                                     const double* x, const double* __restrict__ c,
                                     const double* __restrict__ kt_y,
                                     const double* __restrict__ lower,
                                     const double* __restrict__ upper, const double* anchor,
                                     double* x_out, double* dx, double* x_bar) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    const double xj = x[j];
    double v = sub(xj, mul(tau, sub(c[j], kt_y[j])));
    if (v < lower[j]) v = lower[j];
    if (v > upper[j]) v = upper[j];
    const double d = sub(v, xj);
    const double next0 = v;
    double next = next0;
    if (gamma != 0.0) next = add(next, mul(gamma, d));
    if (anchor != nullptr) next = add(mul(halpern, next), mul(sub(1.0, halpern), anchor[j]));
    dx[j] = d;
    x_bar[j] = add(v, d);
    x_out[j] = next;
  }
}

// backend.cpp:81-111.
__global__ void dual_update_kernel(int64_t m, int64_t num_eq, double sigma, double gamma,
                                   double halpern, const double* y, const double* __restrict__ q,
                                   const double* k_x_bar, const double* k_x,
                                   const double* anchor_y, const double* anchor_kx, double* y_out,
                                   double* dy, double* k_out, double* k_dx) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double yi = y[i];
    const double bar = k_x_bar[i];
    const double kx = k_x[i];
    double v = add(yi, mul(sigma, sub(q[i], bar)));
    if (i >= num_eq && v < 0.0) v = 0.0;
    const double d = sub(v, yi);
    const double kd = mul(0.5, sub(bar, kx));
    double next_y = v;
    double next_k = mul(0.5, add(bar, kx));
    if (gamma != 0.0) {
      next_y = add(next_y, mul(gamma, d));
      next_k = add(next_k, mul(gamma, kd));
    }
    if (anchor_y != nullptr) {
      next_y = add(mul(halpern, next_y), mul(sub(1.0, halpern), anchor_y[i]));
      next_k = add(mul(halpern, next_k), mul(sub(1.0, halpern), anchor_kx[i]));
    }
    dy[i] = d;
    k_dx[i] = kd;
    y_out[i] = next_y;
    k_out[i] = next_k;
  }
}

__global__ void fill_kernel(int64_t n, double value, double* __restrict__ t) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    t[i] = value;
}

__global__ void accumulate64_kernel(int64_t n, double w, const double* __restrict__ v,
                                    double* __restrict__ sum) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    sum[i] = add(sum[i], mul(w, v[i]));
}

__global__ void divide_kernel(int64_t n, double w, const double* __restrict__ sum,
                              double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = sum[i] / w;
}

struct DotTerms {
  static constexpr int NT = 1;
  const double* __restrict__ a;
  const double* __restrict__ b;
  __device__ static void init(double* s) { s[0] = 0.0; }
  __device__ static double identity(int) { return 0.0; }
  __device__ static double combine(int, double x, double y) { return anu::add(x, y); }
  __device__ void add(double* s, int32_t i, int32_t) const { s[0] = anu::add(s[0], mul(a[i], b[i])); }
};

struct MaxAbsTerms {
  static constexpr int NT = 1;
  const double* __restrict__ a;
  __device__ static void init(double* s) { s[0] = 0.0; }
  __device__ static double identity(int) { return 0.0; }
  __device__ static double combine(int, double x, double y) { return fmax(x, y); }
  __device__ void add(double* s, int32_t i, int32_t) const { s[0] = fmax(s[0], fabs(a[i])); }
};

int grid_n(int64_t n) { return grid_for(n, 256, 148 * 8); }

void check_len(int64_t n) {
  if (n < 0 || n > INT32_MAX) throw Error(ANU_ERR_INVALID, "vector length out of range");
}

double reduce_scalar_dot(BackendState& s, const double* a, const double* b, int64_t n) {
  check_len(n);
  if (n == 0) return 0.0;
  reduce_terms(s.exec, static_cast<int32_t>(n), 1, DotTerms{a, b}, s.partial, s.out.p, 1, 0);
  double h = 0.0;
  ANU_CUDA(cudaMemcpyAsync(&h, s.out.p, sizeof(double), cudaMemcpyDeviceToHost, s.exec.stream));
  ANU_CUDA(cudaStreamSynchronize(s.exec.stream));
  return h;
}

}  // namespace
}  // namespace anu

using anu::BackendState;
using anu::Error;

extern "C" {

int anu_backend_allocate(int64_t n, double** device_ptr) {
  return anu::guard([&](BackendState& s) {
    if (device_ptr == nullptr || n < 0) throw Error(ANU_ERR_INVALID, "bad allocation request");
    *device_ptr = nullptr;
    if (n == 0) return;
    ANU_CUDA(cudaMalloc(reinterpret_cast<void**>(device_ptr), sizeof(double) * n));
    ANU_CUDA(cudaMemsetAsync(*device_ptr, 0, sizeof(double) * n, s.exec.stream));
    ANU_CUDA(cudaStreamSynchronize(s.exec.stream));
  });
}

int anu_backend_deallocate(double* p) {
  return anu::guard([&](BackendState&) {
    if (p) ANU_CUDA(cudaFree(p));
  });
}

int anu_backend_upload(const double* host, double* dev, int64_t n) {
  return anu::guard([&](BackendState& s) {
    if (n <= 0) return;
    ANU_CUDA(cudaMemcpyAsync(dev, host, sizeof(double) * n, cudaMemcpyHostToDevice, s.exec.stream));
    ANU_CUDA(cudaStreamSynchronize(s.exec.stream));
  });
}

int anu_backend_download(const double* dev, double* host, int64_t n) {
  return anu::guard([&](BackendState& s) {
    if (n <= 0) return;
    ANU_CUDA(cudaMemcpyAsync(host, dev, sizeof(double) * n, cudaMemcpyDeviceToHost, s.exec.stream));
    ANU_CUDA(cudaStreamSynchronize(s.exec.stream));
  });
}

int anu_backend_fill(double* dev, int64_t n, double value) {
  return anu::guard([&](BackendState& s) {
    if (n <= 0) return;
    anu::Timed t(s, "fill");
    anu::fill_kernel<<<anu::grid_n(n), 256, 0, s.exec.stream>>>(n, value, dev);
    ANU_CUDA(cudaGetLastError());
  });
}

int anu_backend_copy(const double* source, double* target, int64_t n) {
  return anu::guard([&](BackendState& s) {
    if (n <= 0) return;
    anu::Timed t(s, "copy");
    ANU_CUDA(cudaMemcpyAsync(target, source, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                             s.exec.stream));
  });
}

int anu_backend_prepare(uint64_t id, const anu_csr* a) {
  return anu::guard([&](BackendState& s) {
    if (a == nullptr) throw Error(ANU_ERR_INVALID, "null matrix");
    if (s.matrices.count(id)) return;
    const std::string e = anu::validate_csr(a->rows, a->cols, a->nnz, a->start, a->index);
    if (!e.empty()) throw Error(ANU_ERR_INVALID, "invalid matrix: " + e);
    const anu::HostCsr h = anu::copy_csr(a->rows, a->cols, a->nnz, a->start, a->index, a->value);
    auto d = std::make_unique<anu::DevCsr>();
    d->upload(h, false, s.exec.stream);
    if (s.profiling) s.profiled_matrices[id] = anu::describe_matrix(id, *d);
    s.matrices[id] = std::move(d);
  });
}

int anu_backend_release(void) {
  return anu::guard([&](BackendState& s) { s.matrices.clear(); });
}

int anu_backend_multiply(uint64_t id, const double* x, double* y) {
  return anu::guard([&](BackendState& s) {
    auto it = s.matrices.find(id);
    if (it == s.matrices.end()) throw Error(ANU_ERR_INVALID, "matrix was not prepared");
    anu::Timed t(s, "multiply");
    anu::product<double, double, double>(s.exec, *it->second, x, 1, anu::StoreEpi<double>{1, y});
  });
}

int anu_backend_dot(const double* a, const double* b, int64_t n, double* out) {
  return anu::guard([&](BackendState& s) {
    anu::Timed t(s, "dot");
    *out = anu::reduce_scalar_dot(s, a, b, n);
  });
}

int anu_backend_two_norm(const double* a, int64_t n, double* out) {
  return anu::guard([&](BackendState& s) {
    anu::Timed t(s, "two norm");
    *out = std::sqrt(anu::reduce_scalar_dot(s, a, a, n));
  });
}

int anu_backend_inf_norm(const double* a, int64_t n, double* out) {
  return anu::guard([&](BackendState& s) {
    anu::check_len(n);
    *out = 0.0;
    if (n == 0) return;
    anu::Timed t(s, "inf norm");
    anu::reduce_terms(s.exec, static_cast<int32_t>(n), 1, anu::MaxAbsTerms{a}, s.partial, s.out.p, 1, 0);
    ANU_CUDA(cudaMemcpyAsync(out, s.out.p, sizeof(double), cudaMemcpyDeviceToHost, s.exec.stream));
    ANU_CUDA(cudaStreamSynchronize(s.exec.stream));
  });
}

int anu_backend_primal_update(int64_t n, double tau, double gamma, double halpern, const double* x,
                              const double* c, const double* kt_y, const double* lower,
                              const double* upper, const double* anchor, double* x_out,
                              double* dx, double* x_bar) {
  return anu::guard([&](BackendState& s) {
    if (n <= 0) return;
    anu::Timed t(s, "primal update");
    anu::primal_update_kernel<<<anu::grid_n(n), 256, 0, s.exec.stream>>>(
        n, tau, gamma, halpern, x, c, kt_y, lower, upper, anchor, x_out, dx, x_bar);
    ANU_CUDA(cudaGetLastError());
  });
}

int anu_backend_dual_update(int64_t m, int64_t num_equalities, double sigma, double gamma,
                            double halpern, const double* y, const double* q,
                            const double* k_x_bar, const double* k_x, const double* anchor_y,
                            const double* anchor_kx, double* y_out, double* dy, double* k_out,
                            double* k_dx) {
  return anu::guard([&](BackendState& s) {
    if (m <= 0) return;
    anu::Timed t(s, "dual update");
    anu::dual_update_kernel<<<anu::grid_n(m), 256, 0, s.exec.stream>>>(
        m, num_equalities, sigma, gamma, halpern, y, q, k_x_bar, k_x, anchor_y, anchor_kx, y_out,
        dy, k_out, k_dx);
    ANU_CUDA(cudaGetLastError());
  });
}

int anu_backend_accumulate(int64_t n, double weight, const double* v, double* sum) {
  return anu::guard([&](BackendState& s) {
    if (n <= 0) return;
    anu::Timed t(s, "accumulate");
    anu::accumulate64_kernel<<<anu::grid_n(n), 256, 0, s.exec.stream>>>(n, weight, v, sum);
    ANU_CUDA(cudaGetLastError());
  });
}

int anu_backend_scale_into(int64_t n, double weight, const double* sum, double* out) {
  return anu::guard([&](BackendState& s) {
    if (n <= 0) return;
    anu::Timed t(s, "scale into");
    anu::divide_kernel<<<anu::grid_n(n), 256, 0, s.exec.stream>>>(n, weight, sum, out);
    ANU_CUDA(cudaGetLastError());
  });
}

int anu_backend_weighted_norm_squared(int64_t n, int64_t m, const double* dx, const double* dy,
                                      double omega, double* out) {
  return anu::guard([&](BackendState& s) {
    anu::Timed t(s, "weighted norm");
    const double a = anu::reduce_scalar_dot(s, dx, dx, n);
    const double b = anu::reduce_scalar_dot(s, dy, dy, m);
    *out = omega * a + b / omega;
  });
}

int anu_backend_step_size_terms(int64_t n, int64_t m, const double* dx, const double* dy,
                                const double* k_dx, double omega, double* interaction,
                                double* movement) {
  return anu::guard([&](BackendState& s) {
    anu::Timed t(s, "step-size terms");
    *interaction = std::fabs(anu::reduce_scalar_dot(s, dy, k_dx, m));
    const double a = anu::reduce_scalar_dot(s, dx, dx, n);
    const double b = anu::reduce_scalar_dot(s, dy, dy, m);
    *movement = omega * a + b / omega;
  });
}

int anu_backend_convergence_terms(int64_t n, int64_t m, const double* c, const double* lower,
                                  const double* upper, const double* q, const double* row_scale,
                                  const double* col_scale, int64_t num_equalities,
                                  const double* x, const double* k_x, const double* y,
                                  const double* kt_y, double* out) {
  return anu::guard([&](BackendState& s) {
    anu::check_len(n);
    anu::check_len(m);
    if (s.out.n < 18) s.out.alloc(18);
    anu::Timed t(s, "convergence terms");
    anu::RowCheckTerms<double, double, double> rt{1, static_cast<int32_t>(num_equalities), k_x,
                                                  y, nullptr, nullptr, nullptr, nullptr, q,
                                                  nullptr, row_scale};
    anu::ColCheckTerms<double, double> ct{1, kt_y, x, nullptr, nullptr, nullptr, nullptr, c,
                                          lower, upper, col_scale, nullptr, nullptr, nullptr};
    anu::reduce_terms(s.exec, static_cast<int32_t>(m), 1, rt, s.partial, s.out.p, 18, 0);
    anu::reduce_terms(s.exec, static_cast<int32_t>(n), 1, ct, s.partial, s.out.p, 18, 9);
    double h[18];
    ANU_CUDA(cudaMemcpyAsync(h, s.out.p, sizeof(h), cudaMemcpyDeviceToHost, s.exec.stream));
    ANU_CUDA(cudaStreamSynchronize(s.exec.stream));
    // ConvergenceTerms order: primal_sq, primal_inf, q_dot_y, dual_sq,
    // dual_inf, bound_term, c_dot_x.
    out[0] = h[0];
    out[1] = h[1];
    out[2] = h[2];
    out[3] = h[9];
    out[4] = h[10];
    out[5] = h[11];
    out[6] = h[12];
  });
}

int anu_backend_set_profiling(int32_t on) {
  return anu::guard([&](BackendState& s) {
    if (on && s.ev_start == nullptr) {
      ANU_CUDA(cudaEventCreate(&s.ev_start));
      ANU_CUDA(cudaEventCreate(&s.ev_stop));
    }
    s.profiling = on != 0;
    if (!s.profiling) {
      s.timings.clear();
      s.profiled_matrices.clear();
    }
  });
}

int anu_backend_profile_report(char* buf, int32_t size, int32_t* length) {
  return anu::guard([&](BackendState& s) {
    const std::string r = anu::profile_report(s);
    if (length != nullptr) *length = static_cast<int32_t>(r.size());
    if (buf != nullptr && size > 0) {
      const size_t k = std::min(r.size(), static_cast<size_t>(size - 1));
      std::memcpy(buf, r.data(), k);
      buf[k] = '\0';
    }
  });
}

}  // extern "C"
