// sm_100a kernels of the PDHG engine.
//
// Two sparse-product shapes, both reading A through a CSR with int32 indices:
//
//  * rows_kernel - one LP. CSR-adaptive: each CTA takes one row block (a run
//    of consecutive rows holding at most kBlockNnz nonzeros, or one longer
//    row). The block's value*x products are staged into shared memory with
//    coalesced loads of the index and value arrays, summed per row (one
//    thread per short row, a warp per long row, a CTA-wide tree for a row
//    longer than the block), and the row sums feed
//    an epilogue over the block's rows - contiguous, so the epilogue's vector
//    traffic is coalesced too. The epilogue is where the PDHG step is fused:
//    the primal step, bound projection, reflection and Halpern blend after
//    K'y, the dual step, cone projection and K x bookkeeping after K x_bar.
//
//  * seg_kernel - a case stack of K LPs sharing A, vectors case-interleaved
//    (element (row, case) at row*K + case). Rows are cut into segments of a
//    few nonzeros; a group of lanes takes a segment, and lane l owns cases
//    l, l+L, ... Every nonzero of A is loaded once per segment and serves
//    all K cases; the x loads of the K cases are one contiguous run.
//
// Sums are deterministic: the order depends only on the row-block schedule,
// never on timing. FP64 arithmetic in the epilogues and sums is written with
// explicit round-to-nearest intrinsics so nvcc does not contract it into
// FMAs; that keeps the FP64 path on the reference's own arithmetic
// (src/anukulan/backend.cpp:60-111 runs without contraction on x86-64).
#pragma once

#include <type_traits>
#include <utility>
#include <cuda_runtime.h>
#include <stdint.h>

namespace anu {

constexpr int kThreads = 256;
// Single-LP product: threads per CTA, and the most nonzeros and rows a row
// block holds.
constexpr int kRowThreads = 128;
constexpr int kBlockNnz = 1024;
constexpr int kBlockRows = 128;
// Case-stack product: nonzeros per segment, segments per CTA, rows per CTA,
// and the most cases one launch carries.
// The segment shape is a build-time choice (-DANU_SEG_NNZ, -DANU_SEG_PER_CTA)
// so it can be swept; a CTA has one warp per segment at 32 lanes. On the
// 60-case refinery stack (two half-stacks of 30) 4 segments of at most 16
// nonzeros per 128-thread CTA measured fastest: 4.96 us per launch against
// 5.30 at 8 per CTA, 5.40 at 2, and 6.62 with 8-nonzero segments.
#ifndef ANU_SEG_NNZ
#define ANU_SEG_NNZ 16
#endif
#ifndef ANU_SEG_PER_CTA
#define ANU_SEG_PER_CTA 4
#endif
constexpr int kSegNnz = ANU_SEG_NNZ;
constexpr int kSegPerCta = ANU_SEG_PER_CTA;
constexpr int kSegThreads = 32 * kSegPerCta;
// A matrix may carry another segment shape (the unrolled adjoint's does);
// seg_kernel takes it from the schedule, up to this many segments per CTA.
constexpr int kSegPerCtaMax = 16;
static_assert(kSegPerCta <= kSegPerCtaMax, "segment shape");
constexpr int kSegRows = 64;
constexpr int kMaxCaseLanes = 64;

// ------------------------------------------------------------------ math

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return a * b; }
__device__ __forceinline__ float add(float a, float b) { return a + b; }
__device__ __forceinline__ float sub(float a, float b) { return a - b; }
// acc + a*b: contracted to an FMA in FP32, two rounded operations in FP64.
__device__ __forceinline__ double madd(double acc, double a, double b) { return add(acc, mul(a, b)); }
__device__ __forceinline__ float madd(float acc, float a, float b) { return fmaf(a, b, acc); }

template <class T> __device__ __forceinline__ T load(const T* p) { return __ldg(p); }

// Programmatic dependent launch. A kernel launched with programmatic stream
// serialisation may start while its predecessor drains; it must not touch
// the predecessor's output before pdl_wait(), and it lets its own successor
// start only after that wait, so anything two launches back is complete when
// a kernel starts. Outside such a launch both are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// -------------------------------------------------------------- matrices

struct RowBlockDev {
  int32_t row_begin;
  int32_t row_end;
  int32_t nz_begin;  // start[row_begin], stored so a CTA's first index load
  int32_t nz_end;    // does not wait on a load of start[]
};

template <class V>
struct CsrView {
  int32_t rows;
  int32_t cols;
  const int32_t* __restrict__ start;
  const int32_t* __restrict__ index;
  const V* __restrict__ value;
  const RowBlockDev* __restrict__ blocks;
  int32_t num_blocks;
  // Segment schedule of the case-stack product: every row cut into
  // segments of at most a few nonzeros (seg_begin, in nonzero order; the
  // segments of row r are row_seg[r] .. row_seg[r+1]-1), and consecutive rows
  // grouped so a CTA holds at most seg_per_cta segments (cta_row, cta_seg).
  // seg_kernel runs 32 * seg_per_cta threads per CTA.
  const int32_t* __restrict__ seg_begin;
  const int32_t* __restrict__ row_seg;
  const int32_t* __restrict__ cta_row;
  const int32_t* __restrict__ cta_seg;
  int32_t num_ctas;
  int32_t seg_per_cta;
  // kEllWidth when every row holds exactly that many nonzeros (start[r] =
  // kEllWidth * r), so ell_kernel can take the product; 0 otherwise.
  int32_t uniform_len;
  // CTA size of the single-LP product (one of kTileThreads); `blocks` is
  // the row-block schedule for it.
  int32_t tile_threads;
};

// ------------------------------------------------------- per-case state

// What one case's step needs, read by every thread of the iteration kernels.
// Written by the host before each iteration chunk.
struct StepParams {
  double tau;
  double sigma;
  double gamma;        // reflection, 0 when off
  double eta;          // step size, for the averaged scheme's running sums
  int32_t active;      // 0: retired, its lanes do nothing
  int32_t halpern;     // Halpern blending on for this case
  int32_t reset_pending;  // the chunk's first step starts a new epoch
  int32_t k_base;         // Halpern counter at the chunk's first step
};

enum : uint32_t {
  kWriteDelta = 1u,   // write dx / dy (and k_dx)
  kAccumulate = 2u,   // running sums of the averaged scheme
};

// ------------------------------------------------------------ epilogues

// out[row*K + case] = sum
template <class Out>
struct StoreEpi {
  int32_t K;
  Out* __restrict__ out;
  struct Pre {};
  __device__ __forceinline__ Pre prefetch(int32_t, int32_t) const { return Pre{}; }
  template <class Acc>
  __device__ __forceinline__ void finish(int32_t r, int32_t k, Acc s, const Pre&) const {
    out[(size_t)r * K + k] = static_cast<Out>(s);
  }
  template <class Acc>
  __device__ __forceinline__ void operator()(int32_t r, int32_t k, Acc s) const {
    out[(size_t)r * K + k] = static_cast<Out>(s);
  }
};

// The primal side of one reflected Halpern PDHG step on column j of case k,
// given kty = (K'y)_j (backend.hpp:89-93, backend.cpp:60-79):
//   v = clamp(x - tau (c - kty), lower, upper); dx = v - x; x_bar = v + dx;
//   next = v + gamma dx; next = w next + (1-w) anchor  (when blending)
template <class T>
struct PrimalEpi {
  int32_t K;
  int32_t it;
  uint32_t flags;
  const StepParams* __restrict__ p;
  const double* __restrict__ w_table;  // Halpern weight per (it, case)
  const T* x_in;
  T* x_out;
  const T* __restrict__ c;
  const T* __restrict__ lo;
  const T* __restrict__ hi;
  T* __restrict__ x_bar;
  T* anchor;
  T* __restrict__ dx;
  T* __restrict__ sum_x;

  // The column's vectors the step reads besides (K'y)_j, loaded before the
  // kernel waits on the product's input. The per-case parameters stay in L1
  // and are read again in finish().
  struct Pre {
    T x, c, lo, hi, anchor, sum;
    double w;  // this iteration's Halpern weight (when blending)
  };
  // A retired case's lanes neither gather nor step.
  __device__ __forceinline__ bool live(int32_t k) const { return p[k].active != 0; }
  __device__ __forceinline__ Pre prefetch(int32_t j, int32_t k) const {
    Pre r{};
    const StepParams& P = p[k];
    if (!P.active) return r;
    const size_t e = (size_t)j * K + k;
    r.x = x_in[e];
    r.c = c[e];
    r.lo = lo[e];
    r.hi = hi[e];
    const bool blend = P.halpern && !(P.reset_pending && it == 0);
    r.anchor = blend ? anchor[e] : static_cast<T>(0);
    r.w = blend ? w_table[(size_t)it * K + k] : 1.0;
    r.sum = (flags & kAccumulate) ? sum_x[e] : static_cast<T>(0);
    return r;
  }
  // Returns the new x_bar entry (0 for a retired case).
  __device__ __forceinline__ T finish(int32_t j, int32_t k, T kty, const Pre& r) const {
    const StepParams& P = p[k];
    if (!P.active) return static_cast<T>(0);
    const size_t e = (size_t)j * K + k;
    const T xj = r.x;
    T v = sub(xj, mul(static_cast<T>(P.tau), sub(r.c, kty)));
    if (v < r.lo) v = r.lo;
    if (v > r.hi) v = r.hi;
    const T d = sub(v, xj);
    if (flags & kWriteDelta) dx[e] = d;
    const T xb = add(v, d);
    x_bar[e] = xb;
    T next = v;
    if (P.gamma != 0.0) next = add(next, mul(static_cast<T>(P.gamma), d));
    const bool reset_now = P.reset_pending && it == 0;
    if (P.halpern && !reset_now) {
      const double w = r.w;
      next = add(mul(static_cast<T>(w), next), mul(static_cast<T>(1.0 - w), r.anchor));
    }
    x_out[e] = next;
    if (P.halpern && reset_now) anchor[e] = next;
    if (flags & kAccumulate) sum_x[e] = add(r.sum, mul(static_cast<T>(P.eta), next));
    return xb;
  }
  __device__ __forceinline__ void operator()(int32_t j, int32_t k, T kty) const {
    finish(j, k, kty, prefetch(j, k));
  }
};

// The dual side on row i of case k, given bar = (K x_bar)_i
// (backend.hpp:114-119, backend.cpp:81-111):
//   v = y + sigma (q - bar), projected to v >= ylo on inequality rows
//   dy = v - y; k_dx = (bar - kx)/2; next_y = v + gamma dy;
//   next_k = (bar + kx)/2 + gamma k_dx; both blended with their anchors.
// ylo is zero except in a refinement correction solve.
template <class T>
struct DualEpi {
  int32_t K;
  int32_t it;
  uint32_t flags;
  int32_t num_eq;
  const StepParams* __restrict__ p;
  const double* __restrict__ w_table;
  const T* y_in;
  T* y_out;
  const T* __restrict__ q;
  const T* kx_in;
  T* kx_out;
  T* anchor_y;
  T* anchor_kx;
  T* __restrict__ dy;
  T* __restrict__ k_dx;
  T* __restrict__ sum_y;
  const T* __restrict__ ylo;  // may be null (zero)

  // The row's vectors, loaded before the kernel waits on the product's input.
  struct Pre {
    T y, q, kx, anchor_y, anchor_kx, floor_v, sum;
    double w;  // this iteration's Halpern weight (when blending)
  };
  // A retired case's lanes neither gather nor step.
  __device__ __forceinline__ bool live(int32_t k) const { return p[k].active != 0; }
  __device__ __forceinline__ Pre prefetch(int32_t i, int32_t k) const {
    Pre r{};
    const StepParams& P = p[k];
    if (!P.active) return r;
    const size_t e = (size_t)i * K + k;
    r.y = y_in[e];
    r.q = q[e];
    r.kx = kx_in[e];
    r.floor_v = (i >= num_eq && ylo) ? ylo[e] : static_cast<T>(0);
    const bool blend = P.halpern && !(P.reset_pending && it == 0);
    r.anchor_y = blend ? anchor_y[e] : static_cast<T>(0);
    r.anchor_kx = blend ? anchor_kx[e] : static_cast<T>(0);
    r.w = blend ? w_table[(size_t)it * K + k] : 1.0;
    r.sum = (flags & kAccumulate) ? sum_y[e] : static_cast<T>(0);
    return r;
  }
  // Returns the new y entry (0 for a retired case).
  __device__ __forceinline__ T finish(int32_t i, int32_t k, T bar, const Pre& r) const {
    const StepParams& P = p[k];
    if (!P.active) return static_cast<T>(0);
    const size_t e = (size_t)i * K + k;
    const T yi = r.y;
    const T kx = r.kx;
    T v = add(yi, mul(static_cast<T>(P.sigma), sub(r.q, bar)));
    if (i >= num_eq && v < r.floor_v) v = r.floor_v;
    const T d = sub(v, yi);
    const T kd = mul(static_cast<T>(0.5), sub(bar, kx));
    if (flags & kWriteDelta) {
      dy[e] = d;
      if (k_dx) k_dx[e] = kd;
    }
    T next_y = v;
    T next_k = mul(static_cast<T>(0.5), add(bar, kx));
    if (P.gamma != 0.0) {
      next_y = add(next_y, mul(static_cast<T>(P.gamma), d));
      next_k = add(next_k, mul(static_cast<T>(P.gamma), kd));
    }
    const bool reset_now = P.reset_pending && it == 0;
    if (P.halpern && !reset_now) {
      const double w = r.w;
      const T wt = static_cast<T>(w);
      const T wc = static_cast<T>(1.0 - w);
      next_y = add(mul(wt, next_y), mul(wc, r.anchor_y));
      next_k = add(mul(wt, next_k), mul(wc, r.anchor_kx));
    }
    y_out[e] = next_y;
    kx_out[e] = next_k;
    if (P.halpern && reset_now) {
      anchor_y[e] = next_y;
      anchor_kx[e] = next_k;
    }
    if (flags & kAccumulate) sum_y[e] = add(r.sum, mul(static_cast<T>(P.eta), next_y));
    return next_y;
  }
  __device__ __forceinline__ void operator()(int32_t i, int32_t k, T bar) const {
    finish(i, k, bar, prefetch(i, k));
  }
};

// ------------------------------------------------------- block reductions

template <int kWidth, class Acc>
__device__ __forceinline__ Acc block_sum(Acc v, Acc* scratch) {
  // Deterministic tree over a CTA of kWidth threads.
  scratch[threadIdx.x] = v;
  __syncthreads();
  for (int s = kWidth / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) scratch[threadIdx.x] = add(scratch[threadIdx.x], scratch[threadIdx.x + s]);
    __syncthreads();
  }
  const Acc r = scratch[0];
  __syncthreads();
  return r;
}

// ----------------------------------------------------------- rows_kernel

// One LP, one row block per CTA. Each thread first loads its share of the
// block's indices and values into registers (kPerThread of each, all issued
// before any is used), together with the epilogue's vectors for its row;
// none of that depends on the previous launch, so under programmatic
// dependent launch it overlaps the predecessor's tail. After the wait it
// gathers x for all its nonzeros at once and stores the products in shared
// memory. Rows of at most kSerialRow nonzeros are then summed by their own
// thread, left to right from zero - the reference's order, so FP64 sums of
// short rows match it bit for bit. Longer rows are listed in row order and
// taken by whole warps (lane-strided partial sums, then a fixed shuffle
// tree). A row longer than the block has a CTA to itself.
//
// The products sit in shared memory with one pad word after every 32
// (prod_slot). A row's owner thread reads its products consecutively, so in
// a block of equal-length rows the 32 threads of a warp read at a stride of
// the row length: for 8-nonzero rows, unpadded, that is 4 distinct banks and
// an 8-way conflict on every step of the sum. Padded, the warp's reads fall
// in 32 distinct banks. Only the addresses change, not the order of a sum.
constexpr int kSerialRow = 32;
constexpr int kPerThread = kBlockNnz / kRowThreads;
// A row longer than kLongRow takes a CTA to itself and is summed over
// kLongWidth virtual lanes (lane v adds nonzeros v, v + kLongWidth, ... in
// order), then by a fixed tree over those lanes. Both are constants, not the
// CTA size, so every tile size (kTileThreads) sums every row the same way.
constexpr int kLongRow = kBlockNnz;
constexpr int kLongWidth = kRowThreads;
__device__ __forceinline__ int prod_slot(int k) { return k + (k >> 5); }
static_assert(kBlockRows <= kRowThreads, "one epilogue row per thread");
static_assert(kBlockNnz >= kRowThreads, "block_sum scratch");

// The CTA sizes the single-LP kernels are built for. A tile of T threads
// holds up to T * kPerThread nonzeros in at most T rows (rows_kernel), or T
// rows (ell_kernel). The tuner picks one per matrix at set-up.
constexpr int kTileThreads[] = {128, 256};

template <int kThreads>
struct RowTile {
  static_assert(kThreads >= kLongWidth, "the long-row sum needs kLongWidth threads");
  static constexpr int kNnz = kThreads * kPerThread;
  static constexpr int kRows = kThreads;
  static constexpr int kSlots = kNnz + kNnz / 32;
};

template <class V, class X, class Acc, class Epi, int kThreads = kRowThreads>
__global__ void __launch_bounds__(kThreads)
    rows_kernel(CsrView<V> a, const X* __restrict__ x, Epi epi) {
  using Tile = RowTile<kThreads>;
  constexpr int kWarps = kThreads / 32;
  __shared__ Acc prod[Tile::kSlots];
  __shared__ Acc rowsum[Tile::kRows];
  __shared__ int32_t long_rows[Tile::kRows];
  __shared__ int32_t long_b[Tile::kRows], long_e[Tile::kRows];  // their bounds in the block
  __shared__ int32_t warp_long[kWarps];
  const RowBlockDev blk = a.blocks[blockIdx.x];
  const int32_t r0 = blk.row_begin;
  const int32_t nrows = blk.row_end - r0;
  const int32_t nz0 = blk.nz_begin;
  const int32_t nnz = blk.nz_end - nz0;
  const int t = threadIdx.x;
  if (nrows == 1 && nnz > kLongRow) {
    // One long row: strided partial sums over kLongWidth virtual lanes, then
    // a fixed-order tree over them.
    typename Epi::Pre pre{};
    if (t == 0) pre = epi.prefetch(r0, 0);
    pdl_wait();
    pdl_launch();
    Acc s = 0;
    const int32_t end = nz0 + nnz;
    if (t < kLongWidth) {
      for (int32_t base = nz0; base < end; base += kLongWidth * kPerThread) {
        int32_t col[kPerThread];
        Acc val[kPerThread];
#pragma unroll
        for (int q = 0; q < kPerThread; ++q) {
          const int32_t k = base + q * kLongWidth + t;
          col[q] = k < end ? a.index[k] : -1;
          val[q] = k < end ? static_cast<Acc>(a.value[k]) : static_cast<Acc>(0);
        }
        Acc xv[kPerThread];
#pragma unroll
        for (int q = 0; q < kPerThread; ++q)
          xv[q] = col[q] >= 0 ? static_cast<Acc>(x[col[q]]) : static_cast<Acc>(0);
#pragma unroll
        for (int q = 0; q < kPerThread; ++q)
          if (col[q] >= 0) s = madd(s, val[q], xv[q]);
      }
      prod[t] = s;
    }
    __syncthreads();
    for (int w = kLongWidth / 2; w > 0; w >>= 1) {
      if (t < w) prod[t] = add(prod[t], prod[t + w]);
      __syncthreads();
    }
    if (t == 0) epi.finish(r0, 0, prod[0], pre);
    return;
  }
  // ---- independent of the previous launch
  int32_t col[kPerThread];
  V val[kPerThread];
#pragma unroll
  for (int q = 0; q < kPerThread; ++q) {
    const int32_t k = q * kThreads + t;
    col[q] = k < nnz ? a.index[nz0 + k] : -1;
    val[q] = k < nnz ? a.value[nz0 + k] : static_cast<V>(0);
  }
  const bool has_row = t < nrows;
  int32_t rb = 0, re = 0;
  typename Epi::Pre pre{};
  if (has_row) {
    rb = a.start[r0 + t] - nz0;
    re = a.start[r0 + t + 1] - nz0;
    pre = epi.prefetch(r0 + t, 0);
  }
  // ---- the gather reads the previous launch's output
  pdl_wait();
  pdl_launch();
  Acc xv[kPerThread];
#pragma unroll
  for (int q = 0; q < kPerThread; ++q)
    xv[q] = col[q] >= 0 ? static_cast<Acc>(x[col[q]]) : static_cast<Acc>(0);
#pragma unroll
  for (int q = 0; q < kPerThread; ++q)
    if (col[q] >= 0) prod[prod_slot(q * kThreads + t)] = mul(static_cast<Acc>(val[q]), xv[q]);
  __syncthreads();
  const bool is_long = has_row && re - rb > kSerialRow;
  if (has_row && !is_long) {
    Acc s = 0;
    for (int32_t k = rb; k < re; ++k) s = add(s, prod[prod_slot(k)]);
    rowsum[t] = s;
  }
  const int warp = t / 32;
  const int lane = t % 32;
  const unsigned ballot = __ballot_sync(0xffffffffu, is_long);
  if (lane == 0) warp_long[warp] = __popc(ballot);
  __syncthreads();
  int32_t before = 0, nlong = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    const int32_t c = warp_long[w];
    if (w < warp) before += c;
    nlong += c;
  }
  if (is_long) {
    const int32_t slot = before + __popc(ballot & ((1u << lane) - 1u));
    long_rows[slot] = t;
    long_b[slot] = rb;
    long_e[slot] = re;
  }
  __syncthreads();
  for (int32_t i = warp; i < nlong; i += kWarps) {
    const int32_t row = long_rows[i];
    const int32_t b = long_b[i];
    const int32_t e = long_e[i];
    Acc s = 0;
    for (int32_t k = b + lane; k < e; k += 32) s = add(s, prod[prod_slot(k)]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s = add(s, __shfl_down_sync(0xffffffffu, s, off));
    if (lane == 0) rowsum[row] = s;
  }
  __syncthreads();
  if (has_row) epi.finish(r0 + t, 0, rowsum[t], pre);
}

// ------------------------------------------------------------ ell_kernel

// One LP, a matrix whose rows all hold exactly kEllWidth nonzeros (the
// transpose of an LP with that many nonzeros per column, such as K~' of the
// power-law LP). Row r's nonzeros sit at kEllWidth * r, so one thread per row
// loads its indices and values with 128-bit loads straight into registers
// (before the PDL wait: they do not depend on the previous launch), issues
// its kEllWidth gathers together, and sums the products left to right from
// zero in registers with explicitly rounded multiplies and adds - the order
// and roundings of rows_kernel's short-row path and of the reference, so the
// result is the same bit for bit. No shared memory, no barrier.
constexpr int kEllWidth = 8;

__device__ __forceinline__ float strict_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float strict_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double strict_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double strict_add(double a, double b) { return __dadd_rn(a, b); }

template <class V>
__device__ __forceinline__ void load_ell_row(const int32_t* __restrict__ index,
                                             const V* __restrict__ value, int32_t r,
                                             int32_t (&col)[kEllWidth], V (&val)[kEllWidth]) {
  static_assert(kEllWidth % 4 == 0, "whole 16-byte vectors per row");
  const int4* ip = reinterpret_cast<const int4*>(index + static_cast<size_t>(r) * kEllWidth);
#pragma unroll
  for (int v = 0; v < kEllWidth / 4; ++v) {
    const int4 c = __ldg(ip + v);
    col[4 * v] = c.x;
    col[4 * v + 1] = c.y;
    col[4 * v + 2] = c.z;
    col[4 * v + 3] = c.w;
  }
  if constexpr (sizeof(V) == 4) {
    const float4* vp = reinterpret_cast<const float4*>(value + static_cast<size_t>(r) * kEllWidth);
#pragma unroll
    for (int v = 0; v < kEllWidth / 4; ++v) {
      const float4 w = __ldg(vp + v);
      val[4 * v] = w.x;
      val[4 * v + 1] = w.y;
      val[4 * v + 2] = w.z;
      val[4 * v + 3] = w.w;
    }
  } else {
    const double2* vp =
        reinterpret_cast<const double2*>(value + static_cast<size_t>(r) * kEllWidth);
#pragma unroll
    for (int v = 0; v < kEllWidth / 2; ++v) {
      const double2 w = __ldg(vp + v);
      val[2 * v] = w.x;
      val[2 * v + 1] = w.y;
    }
  }
}

template <class V, class X, class Acc, class Epi, int kThreads = kRowThreads>
__global__ void __launch_bounds__(kThreads)
    ell_kernel(CsrView<V> a, const X* __restrict__ x, Epi epi) {
  const int32_t r = static_cast<int32_t>(blockIdx.x) * kThreads + static_cast<int32_t>(threadIdx.x);
  const bool has_row = r < a.rows;
  int32_t col[kEllWidth];
  V val[kEllWidth];
  typename Epi::Pre pre{};
  if (has_row) {
    load_ell_row(a.index, a.value, r, col, val);
    pre = epi.prefetch(r, 0);
  }
  // ---- the gathers read the previous launch's output
  pdl_wait();
  pdl_launch();
  if (!has_row) return;
  Acc xv[kEllWidth];
#pragma unroll
  for (int q = 0; q < kEllWidth; ++q) xv[q] = static_cast<Acc>(x[col[q]]);
  Acc s = 0;
#pragma unroll
  for (int q = 0; q < kEllWidth; ++q)
    s = strict_add(s, strict_mul(static_cast<Acc>(val[q]), xv[q]));
  epi.finish(r, 0, s, pre);
}

// ------------------------------------------------------------ seg_kernel

// Whether the lanes of case k take part in a product: an epilogue that can
// retire cases says so through live(k); any other takes every case.
template <class E, class = void>
struct HasLive : std::false_type {};
template <class E>
struct HasLive<E, std::void_t<decltype(std::declval<const E&>().live(0))>> : std::true_type {};
template <class E>
__device__ __forceinline__ bool case_live(const E& e, int32_t k) {
  if constexpr (HasLive<E>::value) return e.live(k);
  else return true;
}

// The case-stack product in segments. A CTA owns a run of rows and their
// segments; each group of L lanes takes one segment at a time: the group
// loads the segment's indices and values once (one coalesced load), then
// walks them by shuffle, so the x loads of successive nonzeros are
// independent and overlap instead of waiting on an index load each. Lane l
// accumulates cases l, l+L, ... The segment partial sums meet in shared
// memory and are added per row in segment order (deterministic), and the
// epilogue runs over (row, case) pairs of the CTA - case-contiguous, so its
// vector traffic is coalesced.
//
// A CTA has 32 * a.seg_per_cta threads (at most kMaxThreads, the bound the
// instantiation is compiled for), so at least one lane group per segment at
// any L; the segment partials live in dynamic shared memory (seg_per_cta x
// kMaxCaseLanes values).
template <class V, class X, class Acc, class Epi, int L, int CPL, int kMaxThreads>
__global__ void __launch_bounds__(kMaxThreads)
    seg_kernel(CsrView<V> a, const X* __restrict__ x, int32_t K, Epi epi) {
  constexpr int kPrefetch = 2;  // epilogue items prefetched per thread
  extern __shared__ __align__(16) unsigned char seg_smem[];
  Acc* part = reinterpret_cast<Acc*>(seg_smem);
  const int32_t threads = static_cast<int32_t>(blockDim.x);
  const int32_t cta = blockIdx.x;
  const int32_t r0 = a.cta_row[cta];
  const int32_t r1 = a.cta_row[cta + 1];
  const int32_t s0 = a.cta_seg[cta];
  const int32_t s1 = a.cta_seg[cta + 1];
  const int group = threadIdx.x / L;
  const int lane = threadIdx.x % L;
  // ---- independent of the previous launch: the schedule, this group's
  // first indices and values, and the epilogue's own vectors.
  const int32_t sg = s0 + group;
  const bool active = sg < s1;
  const int32_t b = active ? a.seg_begin[sg] : 0;
  const int32_t e = active ? a.seg_begin[sg + 1] : 0;
  const int32_t len = e - b;
  int32_t idx0 = 0;
  Acc val0 = 0;
  if (lane < len) {
    idx0 = a.index[b + lane];
    val0 = static_cast<Acc>(a.value[b + lane]);
  }
  const int32_t items = (r1 - r0) * K;
  typename Epi::Pre pre[kPrefetch];
  // The segment range of each prefetched item's row, also schedule data.
  int32_t g_lo[kPrefetch], g_hi[kPrefetch];
#pragma unroll
  for (int q = 0; q < kPrefetch; ++q) {
    const int32_t t = threadIdx.x + q * threads;
    g_lo[q] = g_hi[q] = 0;
    if (t < items) {
      const int32_t row = r0 + t / K;
      pre[q] = epi.prefetch(row, t % K);
      g_lo[q] = a.row_seg[row];
      g_hi[q] = a.row_seg[row + 1];
    }
  }
  // Retired cases skip their gathers too, not only their epilogue: near the
  // end of a stack most lanes belong to retired cases. The per-case flags are
  // written before the chunk, so they are read before the wait.
  bool live[CPL];
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    const int32_t cs = lane + c * L;
    live[c] = cs < K && case_live(epi, cs);
  }
  // ---- the gather reads the previous launch's output.
  pdl_wait();
  pdl_launch();
  Acc acc[CPL];
#pragma unroll
  for (int c = 0; c < CPL; ++c) acc[c] = 0;
  const int32_t warp_len = __reduce_max_sync(0xffffffffu, static_cast<unsigned>(len));
  for (int32_t base = 0; base < warp_len; base += L) {
    int32_t idx = idx0;
    Acc val = val0;
    if (base > 0) {
      idx = 0;
      val = 0;
      if (base + lane < len) {
        idx = a.index[b + base + lane];
        val = static_cast<Acc>(a.value[b + base + lane]);
      }
    }
    const int32_t cnt = min(L, warp_len - base);
#pragma unroll 8
    for (int t = 0; t < cnt; ++t) {
      const int32_t col = __shfl_sync(0xffffffffu, idx, t, L);
      const Acc v = __shfl_sync(0xffffffffu, val, t, L);
      if (base + t < len) {
        const X* xc = x + (size_t)col * K;
#pragma unroll
        for (int c = 0; c < CPL; ++c)
          if (live[c]) acc[c] = madd(acc[c], v, static_cast<Acc>(xc[lane + c * L]));
      }
    }
  }
  if (active) {
#pragma unroll
    for (int c = 0; c < CPL; ++c) part[(sg - s0) * kMaxCaseLanes + lane + c * L] = acc[c];
  }
  __syncthreads();
  for (int32_t t = threadIdx.x, q = 0; t < items; t += threads, ++q) {
    const int32_t row = r0 + t / K;
    const int32_t k = t % K;
    int32_t lo = 0, hi = 0;
    if (q < kPrefetch) {
#pragma unroll
      for (int qq = 0; qq < kPrefetch; ++qq)
        if (qq == q) {
          lo = g_lo[qq];
          hi = g_hi[qq];
        }
    } else {
      lo = a.row_seg[row];
      hi = a.row_seg[row + 1];
    }
    Acc sum = 0;
    for (int32_t g = lo; g < hi; ++g) sum = add(sum, part[(g - s0) * kMaxCaseLanes + k]);
    if (q < kPrefetch) {
      typename Epi::Pre r;
#pragma unroll
      for (int qq = 0; qq < kPrefetch; ++qq)
        if (qq == q) r = pre[qq];
      epi.finish(row, k, sum, r);
    } else {
      epi.finish(row, k, sum, epi.prefetch(row, k));
    }
  }
}

// ------------------------------------------------------------ chunk_kernel

// A chunk of iterations of a case stack in ONE cooperative launch. The two
// products of an iteration (K'y with the primal step, K x_bar with the dual
// step) are separated by grid barriers instead of launch boundaries, which
// removes the per-launch latency that bounds seg_kernel on stacks whose
// matrix fits in one wave of CTAs. Each CTA owns the same slice of both
// segment schedules for the whole chunk: its lanes load their segment's
// index and value once into registers and keep them, so an iteration's
// critical path is barrier -> gather -> segment sums -> epilogue. The
// epilogue inputs of a phase are this thread's own elements (written by the
// same thread in the previous iteration), so they are prefetched before the
// barrier that precedes the phase. Vectors written by other CTAs during the
// chunk (y for the K'y gather, x_bar for the K x_bar gather) are read with
// plain loads ordered after the barrier's acquire, never through the
// read-only path, which could return a line cached before the barrier.
//
// Every CTA must be resident at once: the launch is cooperative and the
// host sizes the grid to fit one wave. Each barrier wait gives up after a
// bounded number of polls, records kSyncTimedOut and returns, and a CTA
// that sees another's failure returns too, so a grid that cannot meet ends
// with an error status instead of spinning.
struct GridSync {
  unsigned int* arrived;  // arrivals so far; zeroed before each launch
  int* status;            // 0, or kSyncTimedOut once a wait gave up
};
constexpr int kSyncTimedOut = 1;
constexpr unsigned kBarrierFastPolls = 4096;
constexpr unsigned kBarrierPollLimit = 1u << 24;  // ~1 s of 64 ns sleeps

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Waits until `target` arrivals (this CTA's included) have been counted.
// False when the wait gave up; the caller returns.
__device__ __forceinline__ bool grid_barrier(const GridSync& g, unsigned target, int* ok_flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    // Release: the CTA's writes (ordered before this thread by the
    // __syncthreads above) before its arrival.
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(g.arrived) : "memory");
    unsigned polls = 0;
    while (ld_acquire_u32(g.arrived) < target) {
      ++polls;
      if (polls > kBarrierFastPolls) {
        if ((polls & 255u) == 0 && *reinterpret_cast<volatile int*>(g.status) != 0) {
          ok = 0;
          break;
        }
        if (polls > kBarrierPollLimit) {
          atomicExch(g.status, kSyncTimedOut);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    // The acquire load that saw the last arrival orders the other CTAs'
    // writes before this CTA's reads (after the __syncthreads below).
    *ok_flag = ok;
  }
  __syncthreads();
  return *ok_flag != 0;
}

// A plain (weak, L1-cacheable) global load. The compiler may not turn it
// into a read-only-path load, whose cache is not kept coherent with writes
// made during the kernel; a weak load after the barrier's acquire sees every
// write from before the other CTAs' arrivals.
__device__ __forceinline__ float ld_weak(const float* p) {
  float v;
  asm volatile("ld.global.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ double ld_weak(const double* p) {
  double v;
  asm volatile("ld.global.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}

// One CTA's slice of a segment schedule, held for the whole chunk. Lane
// groups are whole warps (32 lanes); each lane keeps one of the segment's
// first 32 nonzeros. Segments are longer only in rows of more than
// kSegNnz * kSegPerCta nonzeros; their remaining nonzeros are loaded again
// in each phase.
template <class V>
struct SegSlice {
  int32_t r0 = 0, r1 = 0, s0 = 0, s1 = 0, seg = 0, b = 0, len = 0, idx = 0;
  V val = 0;
  bool active = false;
  __device__ __forceinline__ void load(const CsrView<V>& a, int32_t cta) {
    if (cta >= a.num_ctas) return;
    r0 = a.cta_row[cta];
    r1 = a.cta_row[cta + 1];
    s0 = a.cta_seg[cta];
    s1 = a.cta_seg[cta + 1];
    seg = s0 + static_cast<int32_t>(threadIdx.x / 32);
    active = seg < s1;
    if (!active) return;
    b = a.seg_begin[seg];
    len = a.seg_begin[seg + 1] - b;
    const int lane = threadIdx.x % 32;
    if (lane < len) {
      idx = a.index[b + lane];
      val = a.value[b + lane];
    }
  }
};

constexpr int kChunkPrefetch = 2;  // epilogue items prefetched per thread
// Resident CTAs per SM the chunk kernel is compiled for: 1,024 threads per
// SM, so 8 x 148 = 1,184 slices of 4 segments at the default shape, enough
// for schedules of up to ~75,000 nonzeros in either product.
constexpr int kChunkCtasPerSm = 1024 / kSegThreads;

template <class V, class Epi>
__device__ __forceinline__ void chunk_prefetch(const SegSlice<V>& s, int32_t K, const Epi& epi,
                                               typename Epi::Pre* pre) {
  const int32_t items = (s.r1 - s.r0) * K;
#pragma unroll
  for (int q = 0; q < kChunkPrefetch; ++q) {
    const int32_t t = threadIdx.x + q * kSegThreads;
    if (t < items) pre[q] = epi.prefetch(s.r0 + t / K, t % K);
  }
}

template <class V, int CPL, class Epi>
__device__ __forceinline__ void chunk_phase(const CsrView<V>& a, const SegSlice<V>& s,
                                            const V* x, int32_t K, const Epi& epi,
                                            const typename Epi::Pre* pre,
                                            V (*part)[kMaxCaseLanes]) {
  const int lane = threadIdx.x % 32;
  V acc[CPL];
#pragma unroll
  for (int c = 0; c < CPL; ++c) acc[c] = 0;
  // s.len is uniform over the warp. Unrolled so the x loads of successive
  // nonzeros are in flight together.
  for (int32_t base = 0; base < s.len; base += 32) {
    int32_t idx = s.idx;
    V val = s.val;
    if (base > 0) {
      idx = 0;
      val = 0;
      if (base + lane < s.len) {
        idx = a.index[s.b + base + lane];
        val = a.value[s.b + base + lane];
      }
    }
    const int32_t cnt = min(32, s.len - base);
#pragma unroll 8
    for (int32_t t = 0; t < cnt; ++t) {
      const int32_t col = __shfl_sync(0xffffffffu, idx, t);
      const V v = __shfl_sync(0xffffffffu, val, t);
      const V* xc = x + (size_t)col * K;
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        const int32_t cs = lane + c * 32;
        if (cs < K) acc[c] = madd(acc[c], v, ld_weak(xc + cs));
      }
    }
  }
  if (s.active) {
#pragma unroll
    for (int c = 0; c < CPL; ++c)
      if (lane + c * 32 < kMaxCaseLanes) part[s.seg - s.s0][lane + c * 32] = acc[c];
  }
  __syncthreads();
  const int32_t items = (s.r1 - s.r0) * K;
  for (int32_t t = threadIdx.x, q = 0; t < items; t += kSegThreads, ++q) {
    const int32_t row = s.r0 + t / K;
    const int32_t k = t % K;
    V sum = 0;
    for (int32_t g = a.row_seg[row]; g < a.row_seg[row + 1]; ++g) sum = add(sum, part[g - s.s0][k]);
    if (q < kChunkPrefetch) {
      typename Epi::Pre r;
#pragma unroll
      for (int qq = 0; qq < kChunkPrefetch; ++qq)
        if (qq == q) r = pre[qq];
      epi.finish(row, k, sum, r);
    } else {
      epi.finish(row, k, sum, epi.prefetch(row, k));
    }
  }
}

// `len` iterations over cases 0..K-1 (17 <= K <= 32*CPL) of a stack with
// vectors case-interleaved; y and x_bar are the gather sources of the two
// products (the dual iterate and the primal extrapolation). The last
// iteration runs with `last_flags`, the others with `flags`.
template <class T, int CPL>
__global__ void __launch_bounds__(kSegThreads, kChunkCtasPerSm)
    chunk_kernel(CsrView<T> kt, CsrView<T> k, const T* y, const T* x_bar, int32_t K, int32_t len,
                 uint32_t flags, uint32_t last_flags, PrimalEpi<T> pe, DualEpi<T> de,
                 GridSync sync) {
  static_assert(kSegNnz <= 32 && kSegThreads / 32 >= kSegPerCta, "one warp per segment");
  __shared__ T part[kSegPerCta][kMaxCaseLanes];
  __shared__ int ok_flag;
  SegSlice<T> sa, sb;
  sa.load(kt, blockIdx.x);
  sb.load(k, blockIdx.x);
  const unsigned G = gridDim.x;
  unsigned target = 0;
  for (int32_t it = 0; it < len; ++it) {
    const uint32_t f = it == len - 1 ? last_flags : flags;
    PrimalEpi<T> ep = pe;
    ep.it = it;
    ep.flags = f;
    typename PrimalEpi<T>::Pre pre_a[kChunkPrefetch];
    chunk_prefetch(sa, K, ep, pre_a);
    if (it > 0) {  // the previous dual step wrote y
      target += G;
      if (!grid_barrier(sync, target, &ok_flag)) return;
    }
    chunk_phase<T, CPL>(kt, sa, y, K, ep, pre_a, part);
    DualEpi<T> ed = de;
    ed.it = it;
    ed.flags = f;
    typename DualEpi<T>::Pre pre_b[kChunkPrefetch];
    chunk_prefetch(sb, K, ed, pre_b);
    target += G;  // the primal step wrote x_bar
    if (!grid_barrier(sync, target, &ok_flag)) return;
    chunk_phase<T, CPL>(k, sb, x_bar, K, ed, pre_b, part);
  }
}

// ------------------------------------------------------- term reductions

// Stage 1 of a per-case reduction over `len` rows (or columns): groups of L
// lanes walk rows, lane l owns cases l, l+L, ...; each thread keeps NT
// accumulators per owned case; the CTA combines its groups in a fixed tree
// and writes partial[block][case][term].
template <class Terms, int L, int CPL>
__global__ void __launch_bounds__(kThreads) terms_stage1(int32_t len, int32_t K, Terms t,
                                                          double* __restrict__ partial) {
  constexpr int NT = Terms::NT;
  constexpr int kGroups = kThreads / L;
  constexpr int kSlots = L * CPL;
  __shared__ double red[kGroups][kSlots][NT];
  const int group = threadIdx.x / L;
  const int lane = threadIdx.x % L;
  double acc[CPL][NT];
#pragma unroll
  for (int c = 0; c < CPL; ++c) Terms::init(acc[c]);
  for (int64_t r = blockIdx.x * (int64_t)kGroups + group; r < len;
       r += (int64_t)gridDim.x * kGroups) {
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      const int32_t cs = lane + c * L;
      if (cs < K) t.add(acc[c], r, cs);
    }
  }
#pragma unroll
  for (int c = 0; c < CPL; ++c)
#pragma unroll
    for (int q = 0; q < NT; ++q) red[group][lane + c * L][q] = acc[c][q];
  __syncthreads();
  for (int s = kGroups / 2; s > 0; s >>= 1) {
    for (int idx = threadIdx.x; idx < s * kSlots * NT; idx += kThreads) {
      const int g = idx / (kSlots * NT);
      const int rem = idx % (kSlots * NT);
      const int slot = rem / NT;
      const int q = rem % NT;
      red[g][slot][q] = Terms::combine(q, red[g][slot][q], red[g + s][slot][q]);
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < kSlots * NT; idx += kThreads) {
    const int slot = idx / NT;
    const int q = idx % NT;
    // slot = lane + c*L -> case index is the slot itself.
    if (slot < K) partial[((size_t)blockIdx.x * K + slot) * NT + q] = red[0][slot][q];
  }
}

// Stage 2: out[case*stride + offset + term] = the blocks' partials combined
// by one warp per (case, term): lane l folds blocks l, l+32, ... in order,
// then a fixed shuffle tree - the same order on every run.
template <class Terms>
__global__ void terms_stage2(int32_t blocks, int32_t K, const double* __restrict__ partial,
                             double* __restrict__ out, int32_t stride, int32_t offset) {
  constexpr int NT = Terms::NT;
  const int32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
  const int lane = threadIdx.x % 32;
  if (warp >= K * NT) return;
  const int32_t k = warp / NT;
  const int q = warp % NT;
  double acc = Terms::identity(q);
  for (int32_t b = lane; b < blocks; b += 32)
    acc = Terms::combine(q, acc, partial[((size_t)b * K + k) * NT + q]);
  for (int off = 16; off > 0; off >>= 1)
    acc = Terms::combine(q, acc, __shfl_down_sync(0xffffffffu, acc, off));
  if (lane == 0) out[(size_t)k * stride + offset + q] = acc;
}

// ------------------------------------------------------------ check terms

// Row side of a termination check, per case (backend.cpp:143-161 and the
// row half of pdhg.cpp:191-221), plus the squared norms the step-size rule,
// the restart test and the primal-weight update read. `y_pt` is the point
// judged (FP64 when it combines a refinement base with the iterate), `y_it`
// the iterate whose restart distances the primal weight reads.
// Terms: 0 primal_sq, 1 primal_inf (max), 2 q_dot_y, 3 dy_sq, 4 dyr_sq
// (|y - y_restart|^2), 5 dypr_sq (|y - y_prev_restart|^2), 6 inf_scale (max
// |dy|), 7 inf_badcone (max of indicator), 8 inf_rhs (sum q~ dy).
template <class TP, class TI, class KX>
struct RowCheckTerms {
  static constexpr int NT = 9;
  int32_t K;
  int32_t num_eq;
  const KX* __restrict__ kx;       // K~ x~ (scaled) of the judged point
  const TP* __restrict__ y_pt;
  const TI* __restrict__ y_it;
  const TI* __restrict__ dy;
  const TI* __restrict__ y_restart;
  const TI* __restrict__ y_prev;
  const double* __restrict__ q;        // original, per case
  const double* __restrict__ q_scaled; // for the Farkas test
  const double* __restrict__ row_scale;  // shared, may be null (unit)
  __device__ static void init(double* a) {
#pragma unroll
    for (int i = 0; i < NT; ++i) a[i] = 0.0;
  }
  __device__ static double identity(int) { return 0.0; }
  __device__ static double combine(int q, double a, double b) {
    return (q == 1 || q == 6 || q == 7) ? fmax(a, b) : anu::add(a, b);
  }
  __device__ void add(double* a, int32_t i, int32_t k) const {
    const size_t e = (size_t)i * K + k;
    const double scale = row_scale ? row_scale[i] : 1.0;
    const double kxv = static_cast<double>(kx[e]);
    const double row = scale != 0.0 ? kxv / scale : kxv;
    const double qi = q[e];
    const double slack = anu::sub(row, qi);
    const double viol = (i < num_eq) ? slack : fmin(slack, 0.0);
    a[0] = anu::add(a[0], mul(viol, viol));
    a[1] = fmax(a[1], fabs(viol));
    const double yi = static_cast<double>(y_pt[e]);
    a[2] = anu::add(a[2], mul(qi, mul(scale, yi)));
    const double d = dy ? static_cast<double>(dy[e]) : 0.0;
    a[3] = anu::add(a[3], mul(d, d));
    const double yit = y_it ? static_cast<double>(y_it[e]) : 0.0;
    if (y_restart) {
      const double r = anu::sub(yit, static_cast<double>(y_restart[e]));
      a[4] = anu::add(a[4], mul(r, r));
    }
    if (y_prev) {
      const double r = anu::sub(yit, static_cast<double>(y_prev[e]));
      a[5] = anu::add(a[5], mul(r, r));
    }
    a[6] = fmax(a[6], fabs(d));
    if (i >= num_eq && d < 0.0) a[7] = 1.0;
    if (q_scaled) a[8] = anu::add(a[8], mul(q_scaled[e], d));
  }
};

// Column side (backend.cpp:163-198 and the column half of the Farkas test).
// Terms: 0 dual_sq, 1 dual_inf (max), 2 bound_term, 3 c_dot_x, 4 dx_sq,
// 5 dxr_sq, 6 dxpr_sq, 7 inf_support, 8 inf_unbounded (max of indicator).
template <class TP, class TI>
struct ColCheckTerms {
  static constexpr int NT = 9;
  int32_t K;
  const double* __restrict__ kty;   // K~' y~ (scaled) of the judged point
  const TP* __restrict__ x_pt;
  const TI* __restrict__ x_it;
  const TI* __restrict__ dx;
  const TI* __restrict__ x_restart;
  const TI* __restrict__ x_prev;
  const double* __restrict__ c;      // original, per case
  const double* __restrict__ lower;  // original
  const double* __restrict__ upper;  // original
  const double* __restrict__ col_scale;  // may be null
  const double* __restrict__ kt_dy;      // K~' dy, may be null
  const double* __restrict__ lower_scaled;
  const double* __restrict__ upper_scaled;
  __device__ static void init(double* a) {
#pragma unroll
    for (int i = 0; i < NT; ++i) a[i] = 0.0;
  }
  __device__ static double identity(int) { return 0.0; }
  __device__ static double combine(int q, double a, double b) {
    return (q == 1 || q == 8) ? fmax(a, b) : anu::add(a, b);
  }
  __device__ void add(double* a, int32_t j, int32_t k) const {
    const size_t e = (size_t)j * K + k;
    const double scale = col_scale ? col_scale[j] : 1.0;
    const double p = kty[e];
    const double product = scale != 0.0 ? p / scale : p;
    const double cj = c[e];
    const double lambda = anu::sub(cj, product);
    const double lo = lower[e];
    const double hi = upper[e];
    const bool has_lo = lo > -INFINITY;
    const bool has_hi = hi < INFINITY;
    double leftover = 0.0;
    if (has_lo && has_hi) leftover = 0.0;
    else if (has_lo) leftover = fmin(lambda, 0.0);
    else if (has_hi) leftover = fmax(lambda, 0.0);
    else leftover = lambda;
    a[0] = anu::add(a[0], mul(leftover, leftover));
    a[1] = fmax(a[1], fabs(leftover));
    const double absorbed = anu::sub(lambda, leftover);
    if (absorbed > 0.0) a[2] = anu::add(a[2], mul(absorbed, lo));
    else if (absorbed < 0.0) a[2] = anu::add(a[2], mul(absorbed, hi));
    const double xj = static_cast<double>(x_pt[e]);
    a[3] = anu::add(a[3], mul(cj, mul(scale, xj)));
    const double d = dx ? static_cast<double>(dx[e]) : 0.0;
    a[4] = anu::add(a[4], mul(d, d));
    const double xit = x_it ? static_cast<double>(x_it[e]) : 0.0;
    if (x_restart) {
      const double r = anu::sub(xit, static_cast<double>(x_restart[e]));
      a[5] = anu::add(a[5], mul(r, r));
    }
    if (x_prev) {
      const double r = anu::sub(xit, static_cast<double>(x_prev[e]));
      a[6] = anu::add(a[6], mul(r, r));
    }
    if (kt_dy) {
      const double lam = kt_dy[e];
      if (lam > 0.0) {
        const double u = upper_scaled[e];
        if (u >= INFINITY) a[8] = 1.0;
        else a[7] = anu::add(a[7], mul(lam, u));
      } else if (lam < 0.0) {
        const double l = lower_scaled[e];
        if (l <= -INFINITY) a[8] = 1.0;
        else a[7] = anu::add(a[7], mul(lam, l));
      }
    }
  }
};

// Weighted KKT error terms on the scaled problem (pdhg.cpp:295-340):
// row side 0 primal_sq, 1 q_dot_y; column side 0 dual_sq, 1 bound_term,
// 2 c_dot_x.
template <class T>
struct RowKktTerms {
  static constexpr int NT = 2;
  int32_t K;
  int32_t num_eq;
  const double* __restrict__ kx;
  const T* __restrict__ y;
  const double* __restrict__ q;
  __device__ static void init(double* a) { a[0] = a[1] = 0.0; }
  __device__ static double identity(int) { return 0.0; }
  __device__ static double combine(int, double a, double b) { return anu::add(a, b); }
  __device__ void add(double* a, int32_t i, int32_t k) const {
    const size_t e = (size_t)i * K + k;
    const double s = anu::sub(kx[e], q[e]);
    const double v = (i < num_eq) ? s : fmin(s, 0.0);
    a[0] = anu::add(a[0], mul(v, v));
    a[1] = anu::add(a[1], mul(q[e], static_cast<double>(y[e])));
  }
};

template <class T>
struct ColKktTerms {
  static constexpr int NT = 3;
  int32_t K;
  const double* __restrict__ kty;
  const T* __restrict__ x;
  const double* __restrict__ c;
  const double* __restrict__ lower;
  const double* __restrict__ upper;
  __device__ static void init(double* a) { a[0] = a[1] = a[2] = 0.0; }
  __device__ static double identity(int) { return 0.0; }
  __device__ static double combine(int, double a, double b) { return anu::add(a, b); }
  __device__ void add(double* a, int32_t j, int32_t k) const {
    const size_t e = (size_t)j * K + k;
    const double lambda = anu::sub(c[e], kty[e]);
    const double lo = lower[e], hi = upper[e];
    const bool has_lo = lo > -INFINITY, has_hi = hi < INFINITY;
    double leftover = 0.0;
    if (has_lo && has_hi) leftover = 0.0;
    else if (has_lo) leftover = fmin(lambda, 0.0);
    else if (has_hi) leftover = fmax(lambda, 0.0);
    else leftover = lambda;
    a[0] = anu::add(a[0], mul(leftover, leftover));
    const double absorbed = anu::sub(lambda, leftover);
    if (absorbed > 0.0) a[1] = anu::add(a[1], mul(absorbed, lo));
    else if (absorbed < 0.0) a[1] = anu::add(a[1], mul(absorbed, hi));
    a[2] = anu::add(a[2], mul(c[e], static_cast<double>(x[e])));
  }
};

// ------------------------------------------------------------ elementwise

// dst[e] = src[e] for the elements of cases whose mask is set (mask null:
// all). len is rows or columns; the arrays hold len*K elements.
template <class D, class S>
__global__ void masked_copy_kernel(int64_t total, int32_t K, const int32_t* __restrict__ mask,
                                   const S* __restrict__ src, D* __restrict__ dst) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    if (mask == nullptr || mask[e % K]) dst[e] = static_cast<D>(src[e]);
  }
}

template <class D>
__global__ void masked_fill_kernel(int64_t total, int32_t K, const int32_t* __restrict__ mask,
                                   D value, D* __restrict__ dst) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    if (mask == nullptr || mask[e % K]) dst[e] = value;
  }
}

// out = sum / weight per case (the averaged iterate), weights per case.
template <class T>
__global__ void average_kernel(int64_t total, int32_t K, const double* __restrict__ weight,
                               const T* __restrict__ sum, T* __restrict__ out) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const double w = weight[e % K];
    out[e] = static_cast<T>(static_cast<double>(sum[e]) / w);
  }
}

// ------------------------------------------------------------ refinement
//
// FP32 iterates are offsets from an FP64 base point, x = x* + x^, y = y* + y^.
// PDHG's step, projection, reflection and Halpern blend all commute with a
// shift of origin, so running the iteration on the offsets of the LP
//   min (c - K'y*)' x^  s.t.  K x^ (=,>=) q - K x*,  l - x* <= x^ <= u - x*,
//   dual floor -y* on the inequality rows
// follows the same trajectory; re-forming that correction LP from the FP64
// residual at every check and folding the offset into the base keeps the FP32
// numbers as small as the movement since the last check, so their rounding
// no longer floors the accuracy.

// The judged point: base + offset, in FP64.
template <class T>
__global__ void combine_kernel(int64_t total, const double* __restrict__ base,
                               const T* __restrict__ it, double* __restrict__ out) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x)
    out[e] = add(base[e], static_cast<double>(it[e]));
}

// Column side of a re-centring, for the masked cases: the offset moves into
// the base (kept inside the bounds), every column vector of the iteration
// state is shifted by it, the offset restarts at zero and the bounds follow
// the base. sum_weight is the averaged scheme's running weight per case;
// shift_out receives the column shift for the K x bookkeeping. Masked-out
// cases leave shift_out untouched, so it must start at zero for them.
template <class T>
__global__ void recenter_columns_kernel(int64_t total, int32_t K, const int32_t* __restrict__ mask,
                                        const double* __restrict__ l0,
                                        const double* __restrict__ u0, double* __restrict__ xb,
                                        T* __restrict__ x, T* __restrict__ anchor,
                                        T* __restrict__ restart, T* __restrict__ prev,
                                        T* __restrict__ sum, const double* __restrict__ sum_weight,
                                        T* __restrict__ lo, T* __restrict__ hi,
                                        double* __restrict__ lo64, double* __restrict__ hi64,
                                        double* __restrict__ shift_out) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int32_t k = static_cast<int32_t>(e % K);
    if (!mask[k]) continue;
    const double off = static_cast<double>(x[e]);
    double base = add(xb[e], off);
    const double l = l0[e], u = u0[e];
    if (base < l) base = l;
    if (base > u) base = u;
    const double shift = sub(base, xb[e]);
    shift_out[e] = shift;
    xb[e] = base;
    x[e] = static_cast<T>(sub(off, shift));
    anchor[e] = static_cast<T>(sub(static_cast<double>(anchor[e]), shift));
    restart[e] = static_cast<T>(sub(static_cast<double>(restart[e]), shift));
    if (prev) prev[e] = static_cast<T>(sub(static_cast<double>(prev[e]), shift));
    if (sum) sum[e] = static_cast<T>(sub(static_cast<double>(sum[e]), mul(sum_weight[k], shift)));
    const double lo_new = sub(l, base);
    const double hi_new = sub(u, base);
    lo[e] = static_cast<T>(lo_new);
    hi[e] = static_cast<T>(hi_new);
    if (lo64) lo64[e] = lo_new;
    if (hi64) hi64[e] = hi_new;
  }
}

// Row side: the same for y (kept in the cone on inequality rows), the dual
// floor -y*, and K x, whose shift is K times the column shift (kshift).
template <class T>
__global__ void recenter_rows_kernel(int64_t total, int32_t K, int32_t num_eq,
                                     const int32_t* __restrict__ mask, double* __restrict__ yb,
                                     T* __restrict__ y, T* __restrict__ anchor_y,
                                     T* __restrict__ restart, T* __restrict__ prev,
                                     T* __restrict__ sum, const double* __restrict__ sum_weight,
                                     T* __restrict__ ylo, T* __restrict__ kx,
                                     T* __restrict__ anchor_kx, const double* __restrict__ kshift) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int32_t k = static_cast<int32_t>(e % K);
    if (!mask[k]) continue;
    const int64_t i = e / K;
    const double off = static_cast<double>(y[e]);
    double base = add(yb[e], off);
    if (i >= num_eq && base < 0.0) base = 0.0;
    const double shift = sub(base, yb[e]);
    yb[e] = base;
    y[e] = static_cast<T>(sub(off, shift));
    anchor_y[e] = static_cast<T>(sub(static_cast<double>(anchor_y[e]), shift));
    restart[e] = static_cast<T>(sub(static_cast<double>(restart[e]), shift));
    if (prev) prev[e] = static_cast<T>(sub(static_cast<double>(prev[e]), shift));
    if (sum) sum[e] = static_cast<T>(sub(static_cast<double>(sum[e]), mul(sum_weight[k], shift)));
    ylo[e] = static_cast<T>(i >= num_eq ? -base : 0.0);
    const double ks = kshift[e];
    kx[e] = static_cast<T>(sub(static_cast<double>(kx[e]), ks));
    anchor_kx[e] = static_cast<T>(sub(static_cast<double>(anchor_kx[e]), ks));
  }
}

// The correction LP's cost c~ - K'y* and right-hand side q~ - K x* from the
// base's FP64 products, for the masked cases.
template <class T>
__global__ void correction_data_kernel(int64_t total_n, int64_t total_m, int32_t K,
                                       const int32_t* __restrict__ mask,
                                       const double* __restrict__ c0,
                                       const double* __restrict__ ktyb, T* __restrict__ c,
                                       const double* __restrict__ q0,
                                       const double* __restrict__ kxb, T* __restrict__ q,
                                       double* __restrict__ q64) {
  const int64_t total = total_n + total_m;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = t < total_n ? t : t - total_n;
    const int32_t k = static_cast<int32_t>(e % K);
    if (!mask[k]) continue;
    if (t < total_n) {
      c[e] = static_cast<T>(sub(c0[e], ktyb[e]));
    } else {
      const double v = sub(q0[e], kxb[e]);
      q[e] = static_cast<T>(v);
      if (q64) q64[e] = v;
    }
  }
}

}  // namespace anu
