// cluster_chunk_kernel: a whole check period of ONE small LP in one launch of
// one thread-block cluster.
//
// A small LP's two product kernels per iteration are latency-bound: each
// launch has a few dozen CTAs on 148 SMs, and an iteration costs two launch
// and dependency latencies however little work it holds. Here the cluster's
// CTAs stay resident for the `len` iterations of a chunk. Each CTA owns a
// contiguous range of the rows of K~' (the primal side) and of K~ (the dual
// side), cut by nonzeros (ClusterSchedule), and keeps in its shared memory a
// full copy of y and of x_bar. An iteration is two phases:
//
//   primal: for its columns j, (K~'y)_j from the local y copy, then the
//           primal step (PrimalEpi); the new x_bar_j is stored into every
//           CTA's x_bar copy (distributed shared memory);
//   cluster barrier;
//   dual:   for its rows i, (K~ x_bar)_i from the local x_bar copy, then the
//           dual step (DualEpi); the new y_i goes into every CTA's y copy;
//   cluster barrier.
//
// A phase reads one copy and the peers write the other, so one barrier per
// phase orders everything. The barrier is the hardware cluster barrier:
// every thread of every CTA arrives at each of the 1 + 2 len barriers, with
// no early exit, so it cannot wait on a thread that never comes.
//
// Every row is summed exactly as rows_kernel sums it: a row of at most
// kSerialRow nonzeros by one thread, left to right from zero, with each
// product and each sum rounded on its own; a longer row (up to kLongRow) by
// one warp, lane-strided partial sums and then the same shuffle tree. The
// epilogues are the same functors. So the iterates are the ones the two
// launches per iteration give, bit for bit. Rows longer than kLongRow are
// not taken here (cluster_shape).
//
// Each CTA also holds its slices of both matrices and the step vectors of
// its own rows and columns in shared memory for the chunk, so an iteration
// touches global memory only for the per-case parameters and Halpern
// weights. Measured on a 2,760 x 3,840 refinery case it is still slower than
// the two launches per iteration (7.7 against 5.7 us per iteration in FP32;
// 6.9 with the broadcast stores left out, so the per-row chains of a
// 256-thread CTA, two warps per scheduler, and the barriers cost more than
// two launch latencies), and at parity on a 1,000-row LP. It is therefore
// opt-in (options.cluster_chunks).
#pragma once

#include <cooperative_groups.h>

#include "kernels.cuh"

namespace anu {

// CTAs per cluster: 16 (the non-portable maximum) where the device takes a
// cluster of that size with this shared memory, else 8. Threads per CTA.
constexpr int kClusterThreads = 256;
// The longest chunk the kernel takes: its Halpern weights sit in shared
// memory.
constexpr int kClusterMaxLen = 1024;

// One matrix's share of the cluster: row bounds per CTA and each CTA's
// warp-summed rows.
struct ClusterRows {
  const int32_t* __restrict__ bounds;      // CTAs + 1
  const int32_t* __restrict__ warp_start;  // CTAs + 1
  const int32_t* __restrict__ warp_rows;
  int32_t max_rows;  // most rows, and most nonzeros, one CTA holds
  int32_t max_nnz;
};

// Byte offsets of a CTA's dynamic shared memory: the copies of y (m) and
// x_bar (n), then the CTA's slices of K~' and K~ (values, then local row
// starts and column indices), each section 16-byte aligned.
struct ClusterLayout {
  // ep, ed: the step vectors of the CTA's own columns and rows, kStepVectors
  // arrays of max_rows entries each (StepSlice).
  static constexpr int kStepVectors = 8;
  size_t ys, xbs, wt, vt, vk, ep, ed, st, it, sk, ik, total;
  template <class T>
  __host__ __device__ static ClusterLayout of(int32_t m, int32_t n, const ClusterRows& ktr,
                                              const ClusterRows& kr) {
    auto up = [](size_t b) { return (b + 15) & ~size_t(15); };
    ClusterLayout l{};
    l.ys = 0;
    l.xbs = up(l.ys + sizeof(T) * m);
    l.wt = up(l.xbs + sizeof(T) * n);
    l.vt = up(l.wt + sizeof(double) * kClusterMaxLen);
    l.vk = up(l.vt + sizeof(T) * ktr.max_nnz);
    l.ep = up(l.vk + sizeof(T) * kr.max_nnz);
    l.ed = up(l.ep + sizeof(T) * kStepVectors * ktr.max_rows);
    l.st = up(l.ed + sizeof(T) * kStepVectors * kr.max_rows);
    l.it = up(l.st + sizeof(int32_t) * (ktr.max_rows + 1));
    l.sk = up(l.it + sizeof(int32_t) * ktr.max_nnz);
    l.ik = up(l.sk + sizeof(int32_t) * (kr.max_rows + 1));
    l.total = up(l.ik + sizeof(int32_t) * kr.max_nnz);
    return l;
  }
};

// A CTA's rows [rb, re) of a matrix, copied to shared memory: local row
// starts (from 0), column indices and values.
template <class T>
struct RowSlice {
  int32_t rb, re;
  const int32_t* start;
  const int32_t* idx;
  const T* val;
};

// Copies rows [rb, re) of `a` into the CTA's shared arrays.
template <class T>
__device__ __forceinline__ RowSlice<T> load_slice(const CsrView<T>& a, int32_t rb, int32_t re,
                                                  int32_t* start, int32_t* idx, T* val) {
  const int32_t nz0 = a.start[rb];
  const int32_t nz = a.start[re] - nz0;
  for (int32_t i = threadIdx.x; i <= re - rb; i += blockDim.x) start[i] = a.start[rb + i] - nz0;
  for (int32_t q = threadIdx.x; q < nz; q += blockDim.x) {
    idx[q] = a.index[nz0 + q];
    val[q] = a.value[nz0 + q];
  }
  return {rb, re, start, idx, val};
}

__device__ __forceinline__ void cluster_barrier() {
  // Non-.aligned forms: correct whether or not the warp has reconverged.
  __syncwarp();
  asm volatile("barrier.cluster.arrive.release;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire;\n" ::: "memory");
}

// Stores v at the address of `local` in the shared memory of the cluster's
// CTA `rank`.
__device__ __forceinline__ void st_cluster(const float* local, int rank, float v) {
  const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(local));
  uint32_t ra;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(a), "r"(rank));
  asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(ra), "f"(v) : "memory");
}
__device__ __forceinline__ void st_cluster(const double* local, int rank, double v) {
  const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(local));
  uint32_t ra;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(a), "r"(rank));
  asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(ra), "d"(v) : "memory");
}

// The sum of slice row r against the local copy `xs`, in rows_kernel's
// serial order (the row has at most kSerialRow nonzeros); four nonzeros'
// loads are issued before their products are added, in order.
template <class T>
__device__ __forceinline__ T serial_row_sum(const RowSlice<T>& a, const T* xs, int32_t r) {
  const int32_t b = a.start[r - a.rb], e = a.start[r - a.rb + 1];
  T s = 0;
  int32_t k = b;
  for (; k + 4 <= e; k += 4) {
    T v[4], x[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      v[u] = a.val[k + u];
      x[u] = xs[a.idx[k + u]];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) s = strict_add(s, strict_mul(v[u], x[u]));
  }
  for (; k < e; ++k) s = strict_add(s, strict_mul(a.val[k], xs[a.idx[k]]));
  return s;
}

// The warp sum of slice row r (lane-strided partials, then the shuffle
// tree), as rows_kernel's warp path; the result is valid in lane 0.
template <class T>
__device__ __forceinline__ T warp_row_sum(const RowSlice<T>& a, const T* xs, int32_t r, int lane) {
  const int32_t b = a.start[r - a.rb], e = a.start[r - a.rb + 1];
  T s = 0;
  for (int32_t k = b + lane; k < e; k += 32) s = strict_add(s, strict_mul(a.val[k], xs[a.idx[k]]));
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s = strict_add(s, __shfl_down_sync(0xffffffffu, s, off));
  return s;
}

// The slice's rows, their sums against `xs` fed to `epi`; the value each
// finish() returns (the entry the other phase gathers) is stored at the same
// index of every CTA's copy `copy`.
template <int C, class T, class Epi>
__device__ __forceinline__ void cluster_phase(const RowSlice<T>& a, const ClusterRows& cr,
                                              int rank, const T* xs, const Epi& epi,
                                              const T* copy) {
  const int t = threadIdx.x;
  for (int32_t r = a.rb + t; r < a.re; r += kClusterThreads) {
    if (a.start[r - a.rb + 1] - a.start[r - a.rb] > kSerialRow) continue;
    const typename Epi::Pre pre = epi.prefetch(r, 0);
    const T v = epi.finish(r, 0, serial_row_sum(a, xs, r), pre);
#pragma unroll
    for (int q = 0; q < C; ++q) st_cluster(copy + r, q, v);
  }
  const int warp = t / 32, lane = t % 32;
  const int32_t w0 = cr.warp_start[rank], w1 = cr.warp_start[rank + 1];
  for (int32_t i = w0 + warp; i < w1; i += kClusterThreads / 32) {
    const int32_t r = cr.warp_rows[i];
    typename Epi::Pre pre{};
    if (lane == 0) pre = epi.prefetch(r, 0);
    const T s = warp_row_sum(a, xs, r, lane);
    if (lane == 0) {
      const T v = epi.finish(r, 0, s, pre);
#pragma unroll
      for (int q = 0; q < C; ++q) st_cluster(copy + r, q, v);
    }
  }
}

// The step vectors of a CTA's own columns [b, e) (primal) or rows (dual),
// held in shared memory for the chunk: a copy of the epilogue whose pointers
// address those arrays at the global indices (each array shifted down by b,
// and only ever indexed in [b, e)), filled at the chunk's start and written
// back at its end. The epilogue's per-case parameters and Halpern weights
// stay in global memory (read-only, L1-resident).
template <class T>
__device__ __forceinline__ T* shifted(T* base, int32_t b) {
  return base - b;
}

template <class T>
__device__ __forceinline__ PrimalEpi<T> primal_in_smem(const PrimalEpi<T>& g, T* s, int32_t stride,
                                                      int32_t b, int32_t e, bool accumulate) {
  T* x = s;
  T* c = s + stride;
  T* lo = s + 2 * stride;
  T* hi = s + 3 * stride;
  T* xb = s + 4 * stride;
  T* an = s + 5 * stride;
  T* dx = s + 6 * stride;
  T* su = s + 7 * stride;
  for (int32_t i = threadIdx.x; i < e - b; i += blockDim.x) {
    x[i] = g.x_in[b + i];
    c[i] = g.c[b + i];
    lo[i] = g.lo[b + i];
    hi[i] = g.hi[b + i];
    xb[i] = g.x_bar[b + i];
    an[i] = g.anchor[b + i];
    dx[i] = g.dx[b + i];
    if (accumulate) su[i] = g.sum_x[b + i];
  }
  PrimalEpi<T> l = g;
  l.x_in = shifted(x, b);
  l.x_out = shifted(x, b);
  l.c = shifted(c, b);
  l.lo = shifted(lo, b);
  l.hi = shifted(hi, b);
  l.x_bar = shifted(xb, b);
  l.anchor = shifted(an, b);
  l.dx = shifted(dx, b);
  l.sum_x = shifted(su, b);
  return l;
}

template <class T>
__device__ __forceinline__ void primal_out(const PrimalEpi<T>& g, const T* s, int32_t stride,
                                           int32_t b, int32_t e, bool accumulate, bool delta) {
  for (int32_t i = threadIdx.x; i < e - b; i += blockDim.x) {
    g.x_out[b + i] = s[i];
    g.x_bar[b + i] = s[4 * stride + i];
    g.anchor[b + i] = s[5 * stride + i];
    if (delta) g.dx[b + i] = s[6 * stride + i];
    if (accumulate) g.sum_x[b + i] = s[7 * stride + i];
  }
}

template <class T>
__device__ __forceinline__ DualEpi<T> dual_in_smem(const DualEpi<T>& g, T* s, int32_t stride,
                                                  int32_t b, int32_t e, bool accumulate) {
  T* y = s;
  T* q = s + stride;
  T* kx = s + 2 * stride;
  T* ay = s + 3 * stride;
  T* ak = s + 4 * stride;
  T* dy = s + 5 * stride;
  T* su = s + 6 * stride;
  T* fl = s + 7 * stride;
  for (int32_t i = threadIdx.x; i < e - b; i += blockDim.x) {
    y[i] = g.y_in[b + i];
    q[i] = g.q[b + i];
    kx[i] = g.kx_in[b + i];
    ay[i] = g.anchor_y[b + i];
    ak[i] = g.anchor_kx[b + i];
    dy[i] = g.dy[b + i];
    if (accumulate) su[i] = g.sum_y[b + i];
    if (g.ylo) fl[i] = g.ylo[b + i];
  }
  DualEpi<T> l = g;
  l.y_in = shifted(y, b);
  l.y_out = shifted(y, b);
  l.q = shifted(q, b);
  l.kx_in = shifted(kx, b);
  l.kx_out = shifted(kx, b);
  l.anchor_y = shifted(ay, b);
  l.anchor_kx = shifted(ak, b);
  l.dy = shifted(dy, b);
  l.sum_y = shifted(su, b);
  l.ylo = g.ylo ? shifted(fl, b) : nullptr;
  return l;
}

template <class T>
__device__ __forceinline__ void dual_out(const DualEpi<T>& g, const T* s, int32_t stride,
                                         int32_t b, int32_t e, bool accumulate, bool delta) {
  for (int32_t i = threadIdx.x; i < e - b; i += blockDim.x) {
    g.y_out[b + i] = s[i];
    g.kx_out[b + i] = s[2 * stride + i];
    g.anchor_y[b + i] = s[3 * stride + i];
    g.anchor_kx[b + i] = s[4 * stride + i];
    if (delta) g.dy[b + i] = s[5 * stride + i];
    if (accumulate) g.sum_y[b + i] = s[6 * stride + i];
  }
}

// `len` (at most kClusterMaxLen) iterations of one LP: K~'y with the primal
// step, then K~ x_bar with
// the dual step, on one cluster of C CTAs (the launch sets the cluster
// shape). pe and de carry the chunk's first iteration; `flags` is every
// iteration's epilogue flags, `last_flags` the last one's. Dynamic shared
// memory: ClusterLayout::of<T>(m, n, ktr, kr).total bytes.
template <int C, class T>
__global__ void __launch_bounds__(kClusterThreads)
    cluster_chunk_kernel(CsrView<T> kt, ClusterRows ktr, CsrView<T> k, ClusterRows kr,
                         PrimalEpi<T> pe, DualEpi<T> de, int32_t len, uint32_t flags,
                         uint32_t last_flags) {
  extern __shared__ __align__(16) unsigned char cluster_smem[];
  const int rank = static_cast<int>(cooperative_groups::this_cluster().block_rank());
  const int32_t m = k.rows, n = kt.rows;
  const ClusterLayout l = ClusterLayout::of<T>(m, n, ktr, kr);
  T* ys = reinterpret_cast<T*>(cluster_smem + l.ys);
  T* xbs = reinterpret_cast<T*>(cluster_smem + l.xbs);
  const RowSlice<T> st = load_slice(kt, ktr.bounds[rank], ktr.bounds[rank + 1],
                                    reinterpret_cast<int32_t*>(cluster_smem + l.st),
                                    reinterpret_cast<int32_t*>(cluster_smem + l.it),
                                    reinterpret_cast<T*>(cluster_smem + l.vt));
  const RowSlice<T> sk = load_slice(k, kr.bounds[rank], kr.bounds[rank + 1],
                                    reinterpret_cast<int32_t*>(cluster_smem + l.sk),
                                    reinterpret_cast<int32_t*>(cluster_smem + l.ik),
                                    reinterpret_cast<T*>(cluster_smem + l.vk));
  for (int32_t i = threadIdx.x; i < m; i += kClusterThreads) ys[i] = de.y_in[i];
  const bool accumulate = (flags & kAccumulate) != 0;
  T* ep = reinterpret_cast<T*>(cluster_smem + l.ep);
  T* ed = reinterpret_cast<T*>(cluster_smem + l.ed);
  PrimalEpi<T> lpe = primal_in_smem(pe, ep, ktr.max_rows, st.rb, st.re, accumulate);
  DualEpi<T> lde = dual_in_smem(de, ed, kr.max_rows, sk.rb, sk.re, accumulate);
  // The chunk's Halpern weights (one case: one per iteration).
  double* wt = reinterpret_cast<double*>(cluster_smem + l.wt);
  for (int32_t i = threadIdx.x; i < len; i += kClusterThreads) wt[i] = pe.w_table[i];
  lpe.w_table = wt;
  lde.w_table = wt;
  // Every CTA of the cluster is running, and every local copy and slice is
  // filled, before any CTA stores into another's shared memory.
  cluster_barrier();
  for (int32_t it = 0; it < len; ++it) {
    const uint32_t f = it == len - 1 ? last_flags : flags;
    lpe.it = it;
    lpe.flags = f;
    lde.it = it;
    lde.flags = f;
    cluster_phase<C>(st, ktr, rank, ys, lpe, xbs);
    cluster_barrier();
    cluster_phase<C>(sk, kr, rank, xbs, lde, ys);
    cluster_barrier();
  }
  // The last barrier also ordered every thread's step-vector writes.
  const bool delta = (last_flags & kWriteDelta) != 0;
  primal_out(pe, ep, ktr.max_rows, st.rb, st.re, accumulate, delta);
  dual_out(de, ed, kr.max_rows, sk.rb, sk.re, accumulate, delta);
}

}  // namespace anu
