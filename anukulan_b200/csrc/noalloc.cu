// anu_backend_convergence_terms_noalloc: the convergence-terms reduction of
// the LinAlgBackend seam, for callers that cannot allocate device memory.
//
// Who needs this: a host that runs inside a memory manager it does not own.
// Examples are a process whose CUDA allocations all go through a pool owned by
// another runtime, a plugin loaded into an application that has reserved the
// whole device for itself, and code that must not call cudaMalloc while that
// application has a stream capture open. Such a host can pass its own input
// and output arrays. It cannot let this library call cudaMalloc behind its
// back. The regular entry point, anu_backend_convergence_terms, keeps its
// partial sums in buffers it allocates on first use, and it creates a stream.
//
// This variant keeps the partial sums in a fixed array in the library's own
// device image (`g_noalloc_scratch` below). Every GPU that loads the library
// holds the array until the process exits. It runs on the legacy default
// stream, so it creates nothing either.
#include <climits>
#include <mutex>

#include "engine.hpp"

namespace anu {
namespace {

// The reduction runs in two stages. The row side and the column side each
// write one partial per block and term, and stage 2 folds them into the 18
// totals. The block count never exceeds kNoAllocBlocks, whatever the vector
// lengths are. So the scratch has a fixed size:
//   rows:    kNoAllocBlocks * 9 doubles
//   columns: kNoAllocBlocks * 9 doubles
//   totals:  18 doubles
// That is 5,346 doubles, or 42,768 bytes.
constexpr int kNoAllocBlocks = 296;
constexpr int kNoAllocTerms = 9;
constexpr size_t kNoAllocPartial = static_cast<size_t>(kNoAllocBlocks) * kNoAllocTerms;
constexpr size_t kNoAllocWords = 2 * kNoAllocPartial + 18;

__device__ __align__(256) double g_noalloc_scratch[kNoAllocWords];

// In host code, g_noalloc_scratch names a host-side stand-in, not device
// memory. The device address comes from cudaGetSymbolAddress, once per
// device, with that device current.
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_lock;
double* g_noalloc_address[kNoAllocMaxDevices] = {};

double* scratch_on_current_device() {
  int device = -1;
  cuda_check(cudaGetDevice(&device), "cudaGetDevice");
  if (device < 0 || device >= kNoAllocMaxDevices)
    throw Error(ANU_ERR_INVALID, "device ordinal beyond the 64 devices this entry point tracks");
  std::lock_guard<std::mutex> g(g_noalloc_lock);
  if (g_noalloc_address[device] == nullptr) {
    double* ptr = nullptr;
    cuda_check(cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), g_noalloc_scratch),
               "cudaGetSymbolAddress(g_noalloc_scratch)");
    if (ptr == nullptr) throw Error(ANU_ERR_CUDA, "cudaGetSymbolAddress returned a null address");
    g_noalloc_address[device] = ptr;
  }
  return g_noalloc_address[device];
}

template <class Terms>
void reduce_into_scratch(int32_t len, const Terms& t, double* partial, double* totals,
                         int offset) {
  const int blocks = grid_for(len, kThreads, kNoAllocBlocks);
  if (static_cast<size_t>(blocks) * Terms::NT > kNoAllocPartial)
    throw Error(ANU_ERR_INTERNAL, "no-alloc reduction grid exceeds its scratch");
  terms_stage1<Terms, 1, 1><<<blocks, kThreads, 0, 0>>>(len, 1, t, partial);
  cuda_check(cudaGetLastError(), "kernel launch");
  terms_stage2<Terms><<<(Terms::NT * 32 + 255) / 256, 256, 0, 0>>>(blocks, 1, partial, totals,
                                                                   18, offset);
  cuda_check(cudaGetLastError(), "kernel launch");
}

}  // namespace
}  // namespace anu

extern "C" {

int anu_backend_convergence_terms_noalloc(int64_t n, int64_t m, const double* c,
                                          const double* lower, const double* upper,
                                          const double* q, const double* row_scale,
                                          const double* col_scale, int64_t num_equalities,
                                          const double* x, const double* k_x, const double* y,
                                          const double* kt_y, double* out) {
  try {
    anu::clear_last_error();
    if (n < 0 || m < 0 || n > INT32_MAX || m > INT32_MAX)
      throw anu::Error(ANU_ERR_INVALID,
                       "vector length outside 0..2147483647, the most this entry point takes");
    if (num_equalities < 0 || num_equalities > m)
      throw anu::Error(ANU_ERR_INVALID, "num_equalities outside 0..m");
    if (out == nullptr) throw anu::Error(ANU_ERR_INVALID, "null output array");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      cudaGetLastError();
      throw anu::Error(ANU_ERR_NO_DEVICE,
                       "no CUDA device is available; this engine has no CPU fallback");
    }
    double* scratch = anu::scratch_on_current_device();
    double* rows = scratch;
    double* cols = scratch + anu::kNoAllocPartial;
    double* totals = scratch + 2 * anu::kNoAllocPartial;
    // Stage 1 writes every partial that stage 2 reads, and stage 2 writes
    // every total that is copied out, so no word of the scratch is read
    // before this call has written it, and nothing needs clearing.
    anu::RowCheckTerms<double, double, double> rt{1, static_cast<int32_t>(num_equalities), k_x,
                                                  y, nullptr, nullptr, nullptr, nullptr, q,
                                                  nullptr, row_scale};
    anu::ColCheckTerms<double, double> ct{1, kt_y, x, nullptr, nullptr, nullptr, nullptr, c,
                                          lower, upper, col_scale, nullptr, nullptr, nullptr};
    anu::reduce_into_scratch(static_cast<int32_t>(m), rt, rows, totals, 0);
    anu::reduce_into_scratch(static_cast<int32_t>(n), ct, cols, totals, 9);
    double h[18];
    ANU_CUDA(cudaMemcpyAsync(h, totals, sizeof(h), cudaMemcpyDeviceToHost, 0));
    ANU_CUDA(cudaStreamSynchronize(0));
    // ConvergenceTerms order: primal_sq, primal_inf, q_dot_y, dual_sq,
    // dual_inf, bound_term, c_dot_x.
    out[0] = h[0];
    out[1] = h[1];
    out[2] = h[2];
    out[3] = h[9];
    out[4] = h[10];
    out[5] = h[11];
    out[6] = h[12];
    return ANU_OK;
  } catch (const anu::Error& e) {
    anu::set_last_error(e.code, e.what());
    return e.code;
  } catch (const std::exception& e) {
    anu::set_last_error(ANU_ERR_INTERNAL, e.what());
    return ANU_ERR_INTERNAL;
  }
}

}  // extern "C"
