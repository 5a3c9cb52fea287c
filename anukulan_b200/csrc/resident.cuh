// The resident iteration kernel for case stacks.
//
// One cooperative launch runs a whole check period of PDHG iterations for K
// cases sharing a small matrix. Each CTA (one per SM) owns a fixed set of
// columns and a fixed set of rows - whole segment-schedule units of K' and of
// K - and keeps their iteration state in shared memory for the launch:
//
//   columns:  x (offset), c, lower, upper, Halpern anchor, averaged sum
//   rows:     y, q, K x, anchors of y and K x, dual floor, averaged sum
//
// Per iteration there are two phases, each ending in a grid barrier:
//
//   primal  gather y (global, written by the row owners last phase) through
//           the CTA's K' segments, finish the columns' step in shared memory,
//           publish x_bar to global;
//   dual    gather x_bar through the K segments, finish the rows' step in
//           shared memory, publish y.
//
// The gathers read data other SMs wrote during this launch, so they bypass
// L1 (ld.global.cg). The matrix and the schedule are read-only for the
// launch and are served from L1 after the first iteration. The barrier is a
// monotonic arrival counter with a bounded spin: a CTA that waits longer
// than kSpinLimit polls sets the shared error word and returns, and every
// other CTA returns at its next poll of that word, so a fault cannot hang the
// GPU. The arithmetic of the step is the same as PrimalEpi / DualEpi.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.cuh"

namespace anu {

constexpr int kResidentThreads = 1024;
constexpr uint32_t kSpinLimit = 1u << 24;  // x 64 ns backoff ~ one second

// Per-CTA ownership tables, flattened over the grid (offsets per CTA).
struct ResidentSide {
  const int32_t* __restrict__ seg_off;   // G+1: the CTA's segments
  const int32_t* __restrict__ segs;      // global segment ids
  const int32_t* __restrict__ row_off;   // G+1: the CTA's rows
  const int32_t* __restrict__ rows;      // global row ids
  const int32_t* __restrict__ row_lseg;  // per owned row: first local segment (+1 sentinel per CTA)
};

template <class T>
struct ResidentArgs {
  CsrView<T> kt;  // primal side gathers through K'
  CsrView<T> k;   // dual side gathers through K
  ResidentSide ps;
  ResidentSide ds;
  int32_t K;
  int32_t num_eq;
  int32_t len;        // iterations in this launch
  uint32_t flags_last;  // flags of the last iteration (delta writes)
  uint32_t flags;       // flags of every iteration (averaging)
  const StepParams* __restrict__ params;
  // global state (case-interleaved)
  T* x;
  T* x_bar;
  const T* __restrict__ c;
  const T* __restrict__ lo;
  const T* __restrict__ hi;
  T* anchor_x;
  T* dx;
  T* sum_x;
  T* y;
  const T* __restrict__ q;
  T* kx;
  T* anchor_y;
  T* anchor_kx;
  T* dy;
  T* sum_y;
  const T* __restrict__ ylo;
  // barrier
  unsigned int* counter;
  int* error;
  // shared memory layout (elements)
  int32_t max_cols;   // largest owned column count over the CTAs
  int32_t max_rows;
  int32_t max_segs;   // largest owned segment count over both sides
};

__device__ __forceinline__ bool grid_barrier(unsigned int* counter, unsigned int target,
                                             int* error) {
  __shared__ int fail;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(counter, 1u);
    int f = 0;
    uint32_t spins = 0;
    for (;;) {
      const unsigned int v = *reinterpret_cast<volatile unsigned int*>(counter);
      if (v >= target) break;
      if (*reinterpret_cast<volatile int*>(error) != 0) {
        f = 1;
        break;
      }
      if (++spins > kSpinLimit) {
        atomicExch(error, 1);
        f = 1;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
    fail = f;
  }
  __syncthreads();
  return fail == 0;
}

template <class T>
__device__ __forceinline__ T ldcg(const T* p) {
  return __ldcg(p);
}

// Segment partial sums of the CTA's segments of one side: group of L lanes
// per segment, lanes over cases; partials to part[local segment][case].
template <class T, int L, int CPL>
__device__ __forceinline__ void gather_side(const CsrView<T>& a, const ResidentSide& side,
                                            const T* src, int32_t K, T* part) {
  constexpr int kGroups = kResidentThreads / L;
  const int32_t s0 = side.seg_off[blockIdx.x];
  const int32_t s1 = side.seg_off[blockIdx.x + 1];
  const int group = threadIdx.x / L;
  const int lane = threadIdx.x % L;
  for (int32_t sb = s0; sb < s1; sb += kGroups) {
    const int32_t ls = sb + group;
    const bool active = ls < s1;
    const int32_t g = active ? side.segs[ls] : 0;
    const int32_t b = active ? a.seg_begin[g] : 0;
    const int32_t e = active ? a.seg_begin[g + 1] : 0;
    const int32_t len = e - b;
    T acc[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) acc[c] = 0;
    const int32_t warp_len = __reduce_max_sync(0xffffffffu, static_cast<unsigned>(len));
    for (int32_t base = 0; base < warp_len; base += L) {
      int32_t idx = 0;
      T val = 0;
      if (base + lane < len) {
        idx = __ldg(a.index + b + base + lane);
        val = __ldg(a.value + b + base + lane);
      }
      const int32_t cnt = min(L, warp_len - base);
#pragma unroll 8
      for (int t = 0; t < cnt; ++t) {
        const int32_t col = __shfl_sync(0xffffffffu, idx, t, L);
        const T v = __shfl_sync(0xffffffffu, val, t, L);
        if (base + t < len) {
          const T* xc = src + (size_t)col * K;
#pragma unroll
          for (int c = 0; c < CPL; ++c) {
            const int32_t cs = lane + c * L;
            if (cs < K) acc[c] = madd(acc[c], v, ldcg(xc + cs));
          }
        }
      }
    }
    if (active) {
#pragma unroll
      for (int c = 0; c < CPL; ++c) part[(ls - s0) * kMaxCaseLanes + lane + c * L] = acc[c];
    }
  }
}

template <class T, int L, int CPL>
__global__ void __launch_bounds__(kResidentThreads, 1)
    resident_chunk_kernel(ResidentArgs<T> A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int32_t K = A.K;
  const int32_t cols0 = A.ps.row_off[blockIdx.x];
  const int32_t ncols = A.ps.row_off[blockIdx.x + 1] - cols0;
  const int32_t rows0 = A.ds.row_off[blockIdx.x];
  const int32_t nrows = A.ds.row_off[blockIdx.x + 1] - rows0;
  const bool accumulate = (A.flags & kAccumulate) != 0;
  // layout
  double* w_case = reinterpret_cast<double*>(smem_raw);                 // K
  T* part = reinterpret_cast<T*>(w_case + kMaxCaseLanes);               // max_segs * 64
  T* sx = part + (size_t)A.max_segs * kMaxCaseLanes;                    // columns x K each
  const size_t cstride = (size_t)A.max_cols * K;
  T* sc = sx + cstride;
  T* slo = sc + cstride;
  T* shi = slo + cstride;
  T* sax = shi + cstride;
  T* ssx = sax + cstride;  // averaged sum (used only when accumulating)
  const size_t rstride = (size_t)A.max_rows * K;
  T* sq = ssx + cstride;
  T* skx = sq + rstride;
  T* say = skx + rstride;
  T* sak = say + rstride;
  T* sylo = sak + rstride;
  T* ssy = sylo + rstride;
  T* sy = ssy + rstride;

  // Load the owned state.
  for (int32_t t = threadIdx.x; t < ncols * K; t += blockDim.x) {
    const int32_t lr = t / K, k = t % K;
    const size_t e = (size_t)A.ps.rows[cols0 + lr] * K + k;
    sx[t] = A.x[e];
    sc[t] = A.c[e];
    slo[t] = A.lo[e];
    shi[t] = A.hi[e];
    sax[t] = A.anchor_x[e];
    if (accumulate) ssx[t] = A.sum_x[e];
  }
  for (int32_t t = threadIdx.x; t < nrows * K; t += blockDim.x) {
    const int32_t lr = t / K, k = t % K;
    const size_t e = (size_t)A.ds.rows[rows0 + lr] * K + k;
    sq[t] = A.q[e];
    skx[t] = A.kx[e];
    say[t] = A.anchor_y[e];
    sak[t] = A.anchor_kx[e];
    sylo[t] = A.ylo ? A.ylo[e] : static_cast<T>(0);
    if (accumulate) ssy[t] = A.sum_y[e];
    sy[t] = A.y[e];
  }
  unsigned int target = 0;
  for (int32_t it = 0; it < A.len; ++it) {
    const uint32_t flags = A.flags | (it == A.len - 1 ? A.flags_last : 0u);
    // Halpern weights of this iteration per case: (k+1)/(k+2), k counted
    // from the epoch's first blended step.
    for (int32_t k = threadIdx.x; k < K; k += blockDim.x) {
      const StepParams& P = A.params[k];
      const int32_t kk = P.reset_pending ? it - 1 : P.k_base + it;
      w_case[k] = static_cast<double>(kk + 1) / static_cast<double>(kk + 2);
    }
    // ---- primal phase
    gather_side<T, L, CPL>(A.kt, A.ps, A.y, K, part);
    __syncthreads();
    {
      const int32_t s0 = A.ps.seg_off[blockIdx.x];
      for (int32_t t = threadIdx.x; t < ncols * K; t += blockDim.x) {
        const int32_t lr = t / K, k = t % K;
        const StepParams& P = A.params[k];
        if (!P.active) continue;
        const int32_t gr = cols0 + lr;
        T kty = 0;
        for (int32_t ls = A.ps.row_lseg[gr + blockIdx.x]; ls < A.ps.row_lseg[gr + blockIdx.x + 1]; ++ls)
          kty = add(kty, part[(ls - s0) * kMaxCaseLanes + k]);
        const T xj = sx[t];
        T v = sub(xj, mul(static_cast<T>(P.tau), sub(sc[t], kty)));
        if (v < slo[t]) v = slo[t];
        if (v > shi[t]) v = shi[t];
        const T d = sub(v, xj);
        const size_t e = (size_t)A.ps.rows[gr] * K + k;
        if (flags & kWriteDelta) A.dx[e] = d;
        __stcg(A.x_bar + e, add(v, d));
        T next = v;
        if (P.gamma != 0.0) next = add(next, mul(static_cast<T>(P.gamma), d));
        const bool reset_now = P.reset_pending && it == 0;
        if (P.halpern && !reset_now) {
          const double w = w_case[k];
          next = add(mul(static_cast<T>(w), next), mul(static_cast<T>(1.0 - w), sax[t]));
        }
        sx[t] = next;
        if (P.halpern && reset_now) sax[t] = next;
        if (accumulate) ssx[t] = add(ssx[t], mul(static_cast<T>(P.eta), next));
      }
    }
    target += gridDim.x;
    if (!grid_barrier(A.counter, target, A.error)) return;
    // ---- dual phase
    gather_side<T, L, CPL>(A.k, A.ds, A.x_bar, K, part);
    __syncthreads();
    {
      const int32_t s0 = A.ds.seg_off[blockIdx.x];
      for (int32_t t = threadIdx.x; t < nrows * K; t += blockDim.x) {
        const int32_t lr = t / K, k = t % K;
        const StepParams& P = A.params[k];
        if (!P.active) continue;
        const int32_t gr = rows0 + lr;
        T bar = 0;
        for (int32_t ls = A.ds.row_lseg[gr + blockIdx.x]; ls < A.ds.row_lseg[gr + blockIdx.x + 1]; ++ls)
          bar = add(bar, part[(ls - s0) * kMaxCaseLanes + k]);
        const int32_t i = A.ds.rows[gr];
        const size_t e = (size_t)i * K + k;
        const T yi = sy[t];
        const T kxv = skx[t];
        T v = add(yi, mul(static_cast<T>(P.sigma), sub(sq[t], bar)));
        if (i >= A.num_eq && v < sylo[t]) v = sylo[t];
        const T d = sub(v, yi);
        const T kd = mul(static_cast<T>(0.5), sub(bar, kxv));
        if (flags & kWriteDelta) A.dy[e] = d;
        T next_y = v;
        T next_k = mul(static_cast<T>(0.5), add(bar, kxv));
        if (P.gamma != 0.0) {
          next_y = add(next_y, mul(static_cast<T>(P.gamma), d));
          next_k = add(next_k, mul(static_cast<T>(P.gamma), kd));
        }
        const bool reset_now = P.reset_pending && it == 0;
        if (P.halpern && !reset_now) {
          const double w = w_case[k];
          const T wt = static_cast<T>(w), wc = static_cast<T>(1.0 - w);
          next_y = add(mul(wt, next_y), mul(wc, say[t]));
          next_k = add(mul(wt, next_k), mul(wc, sak[t]));
        }
        sy[t] = next_y;
        __stcg(A.y + e, next_y);
        skx[t] = next_k;
        if (P.halpern && reset_now) {
          say[t] = next_y;
          sak[t] = next_k;
        }
        if (accumulate) ssy[t] = add(ssy[t], mul(static_cast<T>(P.eta), next_y));
      }
    }
    target += gridDim.x;
    if (!grid_barrier(A.counter, target, A.error)) return;
  }
  // Write the owned state back.
  for (int32_t t = threadIdx.x; t < ncols * K; t += blockDim.x) {
    const int32_t lr = t / K, k = t % K;
    const size_t e = (size_t)A.ps.rows[cols0 + lr] * K + k;
    A.x[e] = sx[t];
    A.anchor_x[e] = sax[t];
    if (accumulate) A.sum_x[e] = ssx[t];
  }
  for (int32_t t = threadIdx.x; t < nrows * K; t += blockDim.x) {
    const int32_t lr = t / K, k = t % K;
    const size_t e = (size_t)A.ds.rows[rows0 + lr] * K + k;
    A.kx[e] = skx[t];
    A.anchor_y[e] = say[t];
    A.anchor_kx[e] = sak[t];
    if (accumulate) A.sum_y[e] = ssy[t];
  }
}

}  // namespace anu
