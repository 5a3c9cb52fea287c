// The case-resident iteration kernel for case stacks.
//
// One launch runs a whole check period of PDHG iterations with one CTA per
// case. Cases never exchange data, so a CTA needs nothing from any other CTA:
// it loads its case's iteration state and data into shared memory once,
//
//   columns:  x (offset), Halpern anchor, x_bar, c, lower, upper
//   rows:     y, K x, anchors of y and K x, q, dual floor
//
// runs the iterations with __syncthreads between the primal half (K'y
// gathered from shared memory, column step) and the dual half (K x_bar
// gathered from shared memory, row step), and writes the state back. The only
// global traffic per iteration is the shared matrix, read-only and streamed
// from L2 by every CTA; a vector of V lanes walks each row (coalesced index
// and value loads) and reduces with shuffles. There is no inter-CTA wait of
// any kind. The step arithmetic is PrimalEpi / DualEpi's.
//
// Eligible: FP32 iterates, no averaged-restart sums, 6 (n + m) floats per
// case within the shared-memory budget.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.cuh"

namespace anu {

constexpr int kCaseThreads = 1024;

template <class T>
struct CaseChunkArgs {
  CsrView<T> kt;  // primal side: rows of K' are columns of the LP
  CsrView<T> k;   // dual side
  int32_t K;      // cases in the stack (interleave stride of the globals)
  int32_t m;
  int32_t n;
  int32_t num_eq;
  int32_t len;
  uint32_t flags_last;  // flags of the last iteration (delta writes)
  const StepParams* __restrict__ params;
  T* x;
  const T* __restrict__ c;
  const T* __restrict__ lo;
  const T* __restrict__ hi;
  T* anchor_x;
  T* dx;
  T* y;
  const T* __restrict__ q;
  T* kx;
  T* anchor_y;
  T* anchor_kx;
  T* dy;
  const T* __restrict__ ylo;  // null: zero
};

// Sum over one CSR row by V lanes; the result is valid in the group's lane 0.
template <class T, int V>
__device__ __forceinline__ T row_dot(const CsrView<T>& a, int32_t row, bool valid, int lane,
                                     const T* __restrict__ src) {
  T acc = 0;
  if (valid) {
    const int32_t b = __ldg(a.start + row), e = __ldg(a.start + row + 1);
    for (int32_t p = b + lane; p < e; p += V)
      acc = madd(acc, __ldg(a.value + p), src[__ldg(a.index + p)]);
  }
#pragma unroll
  for (int off = V / 2; off > 0; off >>= 1) acc = add(acc, __shfl_down_sync(0xffffffffu, acc, off, V));
  return acc;
}

template <class T, int VP, int VD>
__global__ void __launch_bounds__(kCaseThreads, 1) case_chunk_kernel(CaseChunkArgs<T> A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int32_t k = blockIdx.x;
  const StepParams P = A.params[k];
  if (!P.active) return;
  const int32_t n = A.n, m = A.m, K = A.K;
  T* sx = reinterpret_cast<T*>(smem_raw);
  T* sax = sx + n;
  T* sxb = sax + n;
  T* sc = sxb + n;
  T* slo = sc + n;
  T* shi = slo + n;
  T* sy = shi + n;
  T* skx = sy + m;
  T* say = skx + m;
  T* sak = say + m;
  T* sq = sak + m;
  T* sylo = sq + m;
  for (int32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const size_t e = (size_t)j * K + k;
    sx[j] = A.x[e];
    sax[j] = A.anchor_x[e];
    sc[j] = A.c[e];
    slo[j] = A.lo[e];
    shi[j] = A.hi[e];
  }
  for (int32_t i = threadIdx.x; i < m; i += blockDim.x) {
    const size_t e = (size_t)i * K + k;
    sy[i] = A.y[e];
    skx[i] = A.kx[e];
    say[i] = A.anchor_y[e];
    sak[i] = A.anchor_kx[e];
    sq[i] = A.q[e];
    sylo[i] = A.ylo ? A.ylo[e] : static_cast<T>(0);
  }
  __syncthreads();
  const T tau = static_cast<T>(P.tau), sigma = static_cast<T>(P.sigma);
  const T gamma = static_cast<T>(P.gamma);
  for (int32_t it = 0; it < A.len; ++it) {
    const bool last = it == A.len - 1;
    const bool write_delta = last && (A.flags_last & kWriteDelta);
    const bool reset_now = P.reset_pending && it == 0;
    const bool blend = P.halpern && !reset_now;
    const int32_t kk = P.reset_pending ? it - 1 : P.k_base + it;
    const double w = blend ? static_cast<double>(kk + 1) / static_cast<double>(kk + 2) : 1.0;
    const T wt = static_cast<T>(w), wc = static_cast<T>(1.0 - w);
    // ---- primal half: columns j = rows of K'
    {
      constexpr int kGroups = kCaseThreads / VP;
      const int group = threadIdx.x / VP, lane = threadIdx.x % VP;
      for (int32_t r0 = 0; r0 < n; r0 += kGroups) {
        const int32_t j = r0 + group;
        const bool valid = j < n;
        const T kty = row_dot<T, VP>(A.kt, j, valid, lane, sy);
        if (valid && lane == 0) {
          const T xj = sx[j];
          T v = sub(xj, mul(tau, sub(sc[j], kty)));
          if (v < slo[j]) v = slo[j];
          if (v > shi[j]) v = shi[j];
          const T d = sub(v, xj);
          if (write_delta) A.dx[(size_t)j * K + k] = d;
          sxb[j] = add(v, d);
          T next = v;
          if (P.gamma != 0.0) next = add(next, mul(gamma, d));
          if (blend) next = add(mul(wt, next), mul(wc, sax[j]));
          sx[j] = next;
          if (P.halpern && reset_now) sax[j] = next;
        }
      }
    }
    __syncthreads();
    // ---- dual half: rows i of K
    {
      constexpr int kGroups = kCaseThreads / VD;
      const int group = threadIdx.x / VD, lane = threadIdx.x % VD;
      for (int32_t r0 = 0; r0 < m; r0 += kGroups) {
        const int32_t i = r0 + group;
        const bool valid = i < m;
        const T bar = row_dot<T, VD>(A.k, i, valid, lane, sxb);
        if (valid && lane == 0) {
          const T yi = sy[i];
          const T kxv = skx[i];
          T v = add(yi, mul(sigma, sub(sq[i], bar)));
          if (i >= A.num_eq && v < sylo[i]) v = sylo[i];
          const T d = sub(v, yi);
          const T kd = mul(static_cast<T>(0.5), sub(bar, kxv));
          if (write_delta) A.dy[(size_t)i * K + k] = d;
          T next_y = v;
          T next_k = mul(static_cast<T>(0.5), add(bar, kxv));
          if (P.gamma != 0.0) {
            next_y = add(next_y, mul(gamma, d));
            next_k = add(next_k, mul(gamma, kd));
          }
          if (blend) {
            next_y = add(mul(wt, next_y), mul(wc, say[i]));
            next_k = add(mul(wt, next_k), mul(wc, sak[i]));
          }
          sy[i] = next_y;
          skx[i] = next_k;
          if (P.halpern && reset_now) {
            say[i] = next_y;
            sak[i] = next_k;
          }
        }
      }
    }
    __syncthreads();
  }
  for (int32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const size_t e = (size_t)j * K + k;
    A.x[e] = sx[j];
    A.anchor_x[e] = sax[j];
  }
  for (int32_t i = threadIdx.x; i < m; i += blockDim.x) {
    const size_t e = (size_t)i * K + k;
    A.y[e] = sy[i];
    A.kx[e] = skx[i];
    A.anchor_y[e] = say[i];
    A.anchor_kx[e] = sak[i];
  }
}

inline int vector_width(int32_t rows, int32_t nnz) {
  if (rows <= 0 || nnz <= 0) return 4;
  const double per_row = static_cast<double>(nnz) / rows;
  int v = 4;
  while (v < 32 && v < per_row) v *= 2;
  return v;
}

inline size_t case_chunk_smem(int32_t m, int32_t n, size_t elem) {
  return elem * 6 * (static_cast<size_t>(m) + n);
}

}  // namespace anu
