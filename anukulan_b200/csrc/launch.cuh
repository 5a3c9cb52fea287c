// Launch helpers shared by the solver and the backend seam: the sparse
// product in its single-case and case-stack shapes, the two-stage per-case
// reductions, and masked per-case copies.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>

#include "cluster.cuh"
#include "kernels.cuh"

namespace anu {

void cuda_check(cudaError_t status, const char* what);

// A stream and a count of the kernels launched on it.
struct Exec {
  cudaStream_t stream = nullptr;
  int64_t launches = 0;
};


inline int grid_for(int64_t items, int per_block, int cap) {
  int64_t g = (items + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return static_cast<int>(g);
}


// Shared-memory carveout for rows_kernel. Its residency is set by registers:
// in FP32 12 CTAs of 128 threads at 40 registers, which need about 75 KB of
// shared memory, while the driver by default sizes the carveout for the
// shared-memory limit alone (21 CTAs, 132 KB) and leaves the rest to L1. The
// hint asks for what the register-bound CTAs need, so every CTA stays
// resident and the gathered vectors get the remaining L1. Set once per
// instantiation; it is only a hint, and a failure to set it is ignored.
template <class F>
void prefer_register_bound_carveout(F kernel, int threads) {
  int dev = 0;
  cudaFuncAttributes fa{};
  int smem_sm = 0, regs_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaFuncGetAttributes(&fa, kernel) != cudaSuccess ||
      cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) !=
          cudaSuccess ||
      cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) !=
          cudaSuccess ||
      fa.numRegs <= 0 || smem_sm <= 0) {
    cudaGetLastError();
    return;
  }
  const int by_regs = regs_sm / (fa.numRegs * threads);
  const int by_warps = 64 / ((threads + 31) / 32);
  const int blocks = std::max(1, std::min(by_regs, by_warps));
  const size_t need = static_cast<size_t>(blocks) * (fa.sharedSizeBytes + 1024);
  const int percent = static_cast<int>(std::min<size_t>(100, (need * 100 + smem_sm - 1) / smem_sm));
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, percent) !=
      cudaSuccess)
    cudaGetLastError();
}

// Applied at the first launch of each instantiation that is not being
// captured into a graph (no attribute calls inside a capture).
template <class V, class X, class Acc, class Epi, int kThreads = kRowThreads>
void rows_kernel_setup(cudaStream_t s) {
  static std::atomic<bool> done{false};
  if (done.load(std::memory_order_acquire)) return;
  cudaStreamCaptureStatus status = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &status) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  if (status != cudaStreamCaptureStatusNone) return;
  prefer_register_bound_carveout(rows_kernel<V, X, Acc, Epi, kThreads>, kThreads);
  done.store(true, std::memory_order_release);
}

// The carveout hint for the single-LP iteration kernels of precision T, at
// every tile size. Their first launches are usually inside a graph capture,
// where rows_kernel_setup leaves them alone, so the problem set-up applies
// it beforehand.
template <class T>
void prepare_iteration_kernels(cudaStream_t s) {
  rows_kernel_setup<T, T, T, PrimalEpi<T>, kTileThreads[0]>(s);
  rows_kernel_setup<T, T, T, DualEpi<T>, kTileThreads[0]>(s);
  rows_kernel_setup<T, T, T, PrimalEpi<T>, kTileThreads[1]>(s);
  rows_kernel_setup<T, T, T, DualEpi<T>, kTileThreads[1]>(s);
}

// One single-LP product launch at tile size kThreads: ell_kernel for a
// matrix of uniform 8-nonzero rows, rows_kernel on the row-block schedule
// otherwise.
template <int kThreads, class V, class X, class Acc, class Epi, class Mat>
void single_product(cudaStream_t s, const Mat& a, const X* x, const Epi& epi, bool pdl) {
  cudaLaunchConfig_t cfg = {};
  cfg.blockDim = dim3(kThreads);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  if (a.uniform_len == kEllWidth) {
    cfg.gridDim = dim3((a.rows + kThreads - 1) / kThreads);
    cuda_check(cudaLaunchKernelEx(&cfg, ell_kernel<V, X, Acc, Epi, kThreads>,
                                  a.template view<V>(), x, epi),
               "ell_kernel launch");
  } else {
    rows_kernel_setup<V, X, Acc, Epi, kThreads>(s);
    cfg.gridDim = dim3(a.num_blocks);
    cuda_check(cudaLaunchKernelEx(&cfg, rows_kernel<V, X, Acc, Epi, kThreads>,
                                  a.template view<V>(), x, epi),
               "rows_kernel launch");
  }
}

// y = A x (any epilogue) for K cases.
template <class V, class X, class Acc, class Epi, class Mat>
void product(Exec& p, const Mat& a, const X* x, int K, const Epi& epi, bool pdl = false) {
  if (a.rows == 0) return;
  cudaStream_t s = p.stream;
  if (K == 1) {
    if (a.tile_threads == kTileThreads[1])
      single_product<kTileThreads[1], V, X, Acc>(s, a, x, epi, pdl);
    else
      single_product<kTileThreads[0], V, X, Acc>(s, a, x, epi, pdl);
  } else {
#define ANU_CASES(L_, CPL_)                                                              \
  do {                                                                                   \
    cudaLaunchConfig_t cfg = {};                                                         \
    cfg.gridDim = dim3(a.num_ctas);                                                      \
    cfg.blockDim = dim3(32 * a.seg_per_cta);                                             \
    cfg.dynamicSmemBytes = sizeof(Acc) * a.seg_per_cta * kMaxCaseLanes;                  \
    cfg.stream = s;                                                                      \
    cudaLaunchAttribute attr[1];                                                         \
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;                     \
    attr[0].val.programmaticStreamSerializationAllowed = 1;                              \
    cfg.attrs = attr;                                                                    \
    cfg.numAttrs = pdl ? 1 : 0;                                                          \
    /* The default shape has its own instantiation, compiled for its CTA size. */     \
    auto kernel = a.seg_per_cta <= kSegPerCta                                            \
                      ? seg_kernel<V, X, Acc, Epi, L_, CPL_, kSegThreads>                \
                      : seg_kernel<V, X, Acc, Epi, L_, CPL_, 32 * kSegPerCtaMax>;        \
    cuda_check(cudaLaunchKernelEx(&cfg, kernel, a.template view<V>(), x, K, epi),        \
               "seg_kernel launch");                                                     \
  } while (0)
    if (K <= 4) ANU_CASES(4, 1);
    else if (K <= 8) ANU_CASES(8, 1);
    else if (K <= 16) ANU_CASES(16, 1);
    else if (K <= 32) ANU_CASES(32, 1);
    else ANU_CASES(32, 2);
#undef ANU_CASES
  }
  cuda_check(cudaGetLastError(), "kernel launch");
  ++p.launches;
}

// Most CTAs of chunk_kernel<T, CPL> resident at once on the current device.
template <class T, int CPL>
int chunk_capacity() {
  int dev = 0, sms = 0, per_sm = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev),
             "cudaDeviceGetAttribute");
  cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, chunk_kernel<T, CPL>,
                                                           kSegThreads, 0),
             "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  return sms * per_sm;
}

// Whether a stack of K cases over (kt, k) can run as chunk_kernel: 17 to
// 64 cases, and one CTA per schedule slice of the larger product, all of
// them resident at once.
template <class T, class Mat>
bool chunk_fits(const Mat& kt, const Mat& k, int K) {
  if (K < 17 || K > 2 * 32) return false;
  if (kt.rows == 0 || k.rows == 0) return false;
  // The chunk kernel is built for the default segment shape.
  if (kt.seg_per_cta != kSegPerCta || k.seg_per_cta != kSegPerCta) return false;
  const int grid = kt.num_ctas > k.num_ctas ? kt.num_ctas : k.num_ctas;
  const int cap = K <= 32 ? chunk_capacity<T, 1>() : chunk_capacity<T, 2>();
  return grid >= 1 && grid <= cap;
}

// `len` iterations of the stack in one cooperative launch; sync.arrived
// must be zero on the stream when the kernel starts.
template <class T, class Mat>
void launch_chunk(Exec& p, const Mat& kt, const Mat& k, const T* y, const T* x_bar, int K,
                  int len, uint32_t flags, uint32_t last_flags, const PrimalEpi<T>& pe,
                  const DualEpi<T>& de, GridSync sync) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kt.num_ctas > k.num_ctas ? kt.num_ctas : k.num_ctas);
  cfg.blockDim = dim3(kSegThreads);
  cfg.stream = p.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const CsrView<T> vt = kt.template view<T>();
  const CsrView<T> vk = k.template view<T>();
  if (K <= 32)
    cuda_check(cudaLaunchKernelEx(&cfg, chunk_kernel<T, 1>, vt, vk, y, x_bar, K, len, flags,
                                  last_flags, pe, de, sync),
               "chunk_kernel launch");
  else
    cuda_check(cudaLaunchKernelEx(&cfg, chunk_kernel<T, 2>, vt, vk, y, x_bar, K, len, flags,
                                  last_flags, pe, de, sync),
               "chunk_kernel launch");
  ++p.launches;
}

// ------------------------------------------ cluster-resident single-LP chunks

// The most dynamic shared memory cluster_chunk_kernel asks for: its copies of
// y and x_bar and its slices of the two matrices (ClusterLayout).
constexpr size_t kClusterSmemMax = 200 * 1024;

// The CTAs per cluster the device runs cluster_chunk_kernel<., T> with: 16
// where a 16-CTA cluster with smem16 bytes of dynamic shared memory per CTA
// fits (a non-portable size), else 8 with smem8 bytes, else 0.
template <class T>
int cluster_ctas_for(size_t smem16, size_t smem8) {
  auto fits = [&](auto kernel, int ctas, size_t smem) {
    if (smem > kClusterSmemMax) return false;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kClusterSmemMax)) != cudaSuccess ||
        (ctas > 8 &&
         cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
             cudaSuccess)) {
      cudaGetLastError();
      return false;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ctas);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = ctas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, kernel, &cfg) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    return clusters >= 1;
  };
  if (fits(cluster_chunk_kernel<16, T>, 16, smem16)) return 16;
  if (fits(cluster_chunk_kernel<8, T>, 8, smem8)) return 8;
  return 0;
}

// `len` iterations of one LP as one launch of one cluster of `ctas` CTAs
// (from cluster_ctas_for); the schedules must be the ones for that size.
template <class T>
void launch_cluster_chunk(Exec& p, int ctas, const CsrView<T>& kt, const ClusterRows& ktr,
                          const CsrView<T>& k, const ClusterRows& kr, const PrimalEpi<T>& pe,
                          const DualEpi<T>& de, int len, uint32_t flags, uint32_t last_flags) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ctas);
  cfg.blockDim = dim3(kClusterThreads);
  cfg.dynamicSmemBytes = ClusterLayout::of<T>(k.rows, kt.rows, ktr, kr).total;
  cfg.stream = p.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = ctas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (ctas == 16)
    cuda_check(cudaLaunchKernelEx(&cfg, cluster_chunk_kernel<16, T>, kt, ktr, k, kr, pe, de, len,
                                  flags, last_flags),
               "cluster_chunk_kernel launch");
  else
    cuda_check(cudaLaunchKernelEx(&cfg, cluster_chunk_kernel<8, T>, kt, ktr, k, kr, pe, de, len,
                                  flags, last_flags),
               "cluster_chunk_kernel launch");
  ++p.launches;
}

// Two-stage per-case reduction of `t` over len rows; results land in
// out[case*stride + offset + term] (device).
template <class Terms, class Buf>
void reduce_terms(Exec& p, int32_t len, int K, const Terms& t, Buf& partial,
                  double* out, int stride, int offset) {
  constexpr int NT = Terms::NT;
  cudaStream_t s = p.stream;
  int blocks = 0;
#define ANU_TERMS(L_, CPL_)                                                           \
  do {                                                                                \
    blocks = grid_for(len, kThreads / L_, 296);                                       \
    if (partial.n < static_cast<size_t>(blocks) * K * NT)                             \
      partial.alloc(static_cast<size_t>(blocks) * K * NT);                            \
    terms_stage1<Terms, L_, CPL_><<<blocks, kThreads, 0, s>>>(len, K, t, partial.p);  \
  } while (0)
  if (K == 1) ANU_TERMS(1, 1);
  else if (K <= 4) ANU_TERMS(4, 1);
  else if (K <= 8) ANU_TERMS(8, 1);
  else if (K <= 16) ANU_TERMS(16, 1);
  else if (K <= 32) ANU_TERMS(32, 1);
  else ANU_TERMS(32, 2);
#undef ANU_TERMS
  cuda_check(cudaGetLastError(), "kernel launch");
  terms_stage2<Terms><<<(K * NT * 32 + 255) / 256, 256, 0, s>>>(blocks, K, partial.p, out,
                                                                 stride, offset);
  cuda_check(cudaGetLastError(), "kernel launch");
  p.launches += 2;
}

template <class D, class S>
void masked_copy(Exec& p, int64_t len, int K, const int32_t* mask, const S* src, D* dst) {
  const int64_t total = len * K;
  if (total == 0) return;
  masked_copy_kernel<D, S><<<grid_for(total, 256, 148 * 8), 256, 0, p.stream>>>(total, K, mask,
                                                                              src, dst);
  cuda_check(cudaGetLastError(), "kernel launch");
  ++p.launches;
}

template <class D>
void masked_fill(Exec& p, int64_t len, int K, const int32_t* mask, D value, D* dst) {
  const int64_t total = len * K;
  if (total == 0) return;
  masked_fill_kernel<D><<<grid_for(total, 256, 148 * 8), 256, 0, p.stream>>>(total, K, mask,
                                                                           value, dst);
  cuda_check(cudaGetLastError(), "kernel launch");
  ++p.launches;
}


}  // namespace anu
