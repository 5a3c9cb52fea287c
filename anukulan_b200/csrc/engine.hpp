// Internal declarations of the engine (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/anu_pdhg.h"
#include "kernels.cuh"
#include "launch.cuh"
#include "prep.hpp"

namespace anu {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t status, const char* what);
#define ANU_CUDA(call) ::anu::cuda_check((call), #call)

void set_last_error(int code, const std::string& message);
void clear_last_error();

// Device and pinned host blocks kept for reuse by one problem handle. A
// solve allocates its working vectors, host staging buffers and polishing
// sub-stacks again and again; without the pool each of those is a
// cudaMalloc/cudaFree (or cudaMallocHost/cudaFreeHost) pair, and a free
// waits for the whole device. Blocks are sized in powers of two. The pool
// is consulted only inside a PoolScope, whose work all runs on the
// problem's one stream, so a block handed from one allocation to the next
// is ordered by that stream; the scope synchronises the stream when it
// ends, so no copy from a pinned block is still pending when the host
// writes into it again.
//
// A pool that is destroyed hands its idle blocks to a process-wide cache
// (per device for device blocks) instead of freeing them, and a pool that
// misses takes from that cache before it allocates: a create-solve-destroy
// cycle of handles of like size then allocates and frees nothing after the
// first. The destroying handle has synchronised its stream, and the pool
// synchronises its device before the hand-over, so no work of the old
// handle can still touch a block the next handle receives.
class MemoryPool {
 public:
  MemoryPool() = default;
  MemoryPool(const MemoryPool&) = delete;
  MemoryPool& operator=(const MemoryPool&) = delete;
  ~MemoryPool();
  // A block of at least `bytes`; *rounded receives its size class.
  void* get(bool pinned, size_t bytes, size_t* rounded);
  void put(bool pinned, void* p, size_t rounded);

 private:
  std::mutex lock_;
  std::multimap<size_t, void*> free_[2];
  size_t cached_[2] = {0, 0};
  int device_ = -1;  // device of the device blocks, set by the first one
};

// Frees every block in the process-wide cache; returns the bytes freed.
size_t release_cached_blocks();

// Held by a stack while a cooperative chunk kernel of it may run on
// `device`, so this process never has two of them in flight on one device.
std::mutex& cooperative_mutex(int device);

// The pool of the innermost PoolScope on this thread, or null.
MemoryPool* current_pool();

class PoolScope {
 public:
  PoolScope(MemoryPool* pool, cudaStream_t stream);
  ~PoolScope();
  PoolScope(const PoolScope&) = delete;
  PoolScope& operator=(const PoolScope&) = delete;

 private:
  MemoryPool* previous_;
  cudaStream_t stream_;
};

// Device memory owned by RAII; from the current pool when there is one.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  MemoryPool* pool = nullptr;
  size_t bytes = 0;  // size class of a pooled block
  DevBuf() = default;
  explicit DevBuf(size_t count) { alloc(count); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), pool(o.pool), bytes(o.bytes) {
    o.p = nullptr;
    o.n = 0;
    o.pool = nullptr;
    o.bytes = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      pool = o.pool;
      bytes = o.bytes;
      o.p = nullptr;
      o.n = 0;
      o.pool = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(size_t count) {
    release();
    n = count;
    if (count == 0) return;
    if (MemoryPool* mp = current_pool()) {
      p = static_cast<T*>(mp->get(false, sizeof(T) * count, &bytes));
      pool = mp;
      return;
    }
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * count);
    if (e != cudaSuccess) {
      p = nullptr;
      n = 0;
      throw Error(ANU_ERR_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
  }
  void release() {
    if (p) {
      if (pool) pool->put(false, p, bytes);
      else cudaFree(p);
    }
    p = nullptr;
    n = 0;
    pool = nullptr;
    bytes = 0;
  }
  T* get() const { return p; }
};

// One sparse matrix on the device: structure, FP64 values, optional FP32
// values, and the row-block schedule of the staged SpMV.
struct DevCsr {
  int32_t rows = 0, cols = 0, nnz = 0;
  DevBuf<int32_t> start, index;
  DevBuf<double> v64;
  DevBuf<float> v32;
  // The single-LP product's row-block schedule for each tile size of
  // kTileThreads, both built at upload. tile_threads selects one; blocks and
  // num_blocks are the selected schedule.
  DevBuf<RowBlockDev> tile_blocks[2];
  int32_t tile_num_blocks[2] = {0, 0};
  const RowBlockDev* blocks = nullptr;
  int32_t num_blocks = 0;
  DevBuf<int32_t> seg_begin, row_seg, cta_row, cta_seg;
  int32_t num_ctas = 0;
  int32_t seg_per_cta = kSegPerCta;
  int32_t uniform_len = 0;  // kEllWidth when every row has that many nonzeros
  int32_t tile_threads = kRowThreads;  // CTA size of the single-LP product
  // seg_nnz, seg_per_cta: the segment schedule's shape (at most
  // kSegPerCtaMax segments per CTA).
  void upload(const HostCsr& a, bool with_fp32, cudaStream_t s, int32_t seg_nnz = kSegNnz,
              int32_t seg_per_cta = kSegPerCta);
  // Row schedules of the cluster-resident single-LP chunk
  // (cluster_chunk_kernel) for clusters of 16 and of 8 CTAs, and the
  // longest row; built by prepare_cluster on first use.
  DevBuf<int32_t> cl_bounds[2], cl_warp_start[2], cl_warp_rows[2];
  int32_t cl_max_rows[2] = {0, 0}, cl_max_nnz[2] = {0, 0};  // per CTA
  int32_t max_row = 0;
  bool cl_ready = false;
  void prepare_cluster(const HostCsr& a, cudaStream_t s);
  // Selects the single-LP product tile of `threads` (one of kTileThreads).
  void set_tile(int32_t threads);
  // The cluster schedule for clusters of `ctas` (16 or 8) CTAs.
  ClusterRows cluster_rows(int ctas) const;
  template <class V>
  CsrView<V> view() const;
};

// A relabelling of the rows and columns of K that gives the gathers of the
// two products locality. Rows are ordered by decreasing length, within the
// equality block and within the inequality block, so the first num_equalities
// rows are still the equalities. Columns are ordered by the first relabelled
// row they touch, so the columns of one long row sit together. row_old[r] is
// the original row of relabelled row r and row_new its inverse; likewise for
// the columns. Every row of K and of K' keeps its nonzeros in their original
// order, so each product entry is summed in the same order as without it.
struct Relabel {
  std::vector<int32_t> row_old, row_new, col_old, col_new;
  bool empty() const { return row_old.empty() || col_old.empty(); }
};

// The relabelling of `lp`'s matrix (empty when it has no rows or columns).
Relabel locality_relabel(const anu_lp& lp);

// Everything that depends on the matrix alone: the scaled matrix and its
// transpose (host and device), the scaling, ||K~||, the stream.
struct Problem : Exec {
  MemoryPool pool;  // declared first: outlives every other member
  int32_t m = 0, n = 0, num_eq = 0;
  int precision = ANU_PRECISION_FP64;
  HostCsr k;   // scaled K~
  HostCsr kt;  // its transpose
  Scaling scaling;
  ScalingSweeps sweeps;
  bool unit_scaling = false;  // sub-solves run on already-scaled data
  DevCsr dk, dkt;
  DevBuf<double> row_scale, col_scale;
  double matrix_norm = 0.0;
  bool owns_stream = false;
  int device = 0;
  int32_t seg_nnz = kSegNnz, seg_per_cta = kSegPerCta;  // segment schedule shape
  // Original column of each column when the problem is relabelled (empty
  // otherwise); the power iteration's start vector follows it.
  std::vector<int32_t> col_old;
  // One of many problems that host threads solve at once (a packed batch):
  // its single-LP checks run on one stream, without a second branch, and
  // launch directly for the first kConcurrentDirect checks of a solve.
  bool concurrent = false;
  // CTAs per cluster cluster_chunk_kernel runs with on this problem (16, 8,
  // or 0 where it does not fit); -1 until first asked.
  int cluster_ctas = -1;
  ~Problem();
};

// One case: the unscaled data the convergence test judges, the scaled data
// the iteration runs on.
struct CaseData {
  std::vector<double> c, q, lower, upper;      // original
  std::vector<double> cs, qs, ls, us;          // scaled
  std::vector<double> ylo;                     // dual floor (refinement), empty = 0
  double objective_scale = 1.0;
  double objective_offset = 0.0;
};

struct CaseResult {
  anu_pdhg_result r{};
  std::vector<double> x;  // unscaled
  std::vector<double> y;
  std::vector<double> xs;  // scaled iterate the result came from
  std::vector<double> ys;
};

// Builds the problem from a validated LP: copies, scales, uploads, and
// estimates ||K~|| unless known_matrix_norm is given.
// seg_nnz, seg_per_cta: the shape of the case-stack segment schedule.
// relabel: when given and not empty, the scaled matrix, its transpose and the
// scaling are relabelled after scaling (which runs in the original order);
// every case vector handed to this problem must then be relabelled too.
std::unique_ptr<Problem> make_problem(const anu_lp& lp, const anu_pdhg_options& o,
                                      double* scaling_seconds, double* norm_seconds,
                                      int32_t seg_nnz = kSegNnz, int32_t seg_per_cta = kSegPerCta,
                                      const Relabel* relabel = nullptr);
// scale_matrix_sweeps on the device: the same norms, factors and roundings,
// so the scaled matrix and the factors are bit-identical to the host's.
// Scales *k in place and writes its transpose to *kt.
Scaling scale_matrix_sweeps_device(Exec& ex, HostCsr* k, HostCsr* kt, int ruiz_iterations,
                                   bool pock_chambolle, ScalingSweeps* sweeps);

// A second problem on its own stream and memory pool with the same scaled
// matrix (host and device copies), scaling and norm, made without scaling or
// power iteration again.
std::unique_ptr<Problem> clone_problem(const Problem& src);

// Case stacks of at least this many cases run as two half-stacks at once,
// unless they run persistent chunks.
constexpr int kSplitStack = 16;

// Checks a single LP of a packed batch launches directly before its check
// graphs are captured.
constexpr int kConcurrentDirect = 100;

// Whether run_cases takes a stack of K cases on `p` through chunk_kernel.
bool stack_runs_persistent(const Problem& p, int K, const anu_pdhg_options& o);

CaseData make_case(const Problem& p, const double* c, const double* q, const double* lower,
                   const double* upper, double objective_scale, double objective_offset);

// Runs K cases sharing `problem` to termination (solve_pdhg semantics per
// case). warm_x / warm_y: per case, scaled-space starts or empty.
void run_cases(Problem& problem, const std::vector<const CaseData*>& cases,
               const anu_pdhg_options& options,
               const std::vector<const std::vector<double>*>& warm_x,
               const std::vector<const std::vector<double>*>& warm_y,
               std::vector<CaseResult>* results, double start_time);

// A rolling case stack: the first `slots` cases start; whenever a case
// retires at a termination check its slot takes the next waiting case.
// results[i] is case i's result. Each case runs the iteration it would run
// in a stack of its own (its iteration count starts at its admission).
void run_cases_rolling(Problem& problem, const std::vector<const CaseData*>& cases, int slots,
                       const anu_pdhg_options& options,
                       const std::vector<const std::vector<double>*>& warm_x,
                       const std::vector<const std::vector<double>*>& warm_y,
                       std::vector<CaseResult>* results, double start_time);

// A streaming case stack of at most `slots` cases on `problem`. next_case
// gives the next case (its id through the argument) or null when it has none
// now; it is asked for the first cases, and again whenever a slot frees at a
// termination check and nothing is waiting. deliver takes each case's result
// as the case retires, on the calling thread, before the freed slot is
// refilled, so it may decide what next_case hands out. Cases start cold.
// release gets back each case whose slot has taken a new case; the stack no
// longer reads it.
void run_cases_streaming(Problem& problem, int slots, const anu_pdhg_options& options,
                         const std::function<const CaseData*(int32_t*)>& next_case,
                         const std::function<void(int32_t, CaseResult&)>& deliver,
                         const std::function<void(const CaseData*)>& release,
                         double start_time);

// Picks each matrix's single-LP product tile: options.tile_threads, or, when
// it is 0 and `trial` (the LP's case) is given for a large enough LP, the
// pair that runs short trial solves of it fastest. Results do not depend on
// the choice. Returns whether trial solves ran.
constexpr int64_t kTuneNnz = int64_t(1) << 20;
constexpr int kTuneChunks = 4;
constexpr double kTuneMargin = 0.01;
bool choose_tiles(Problem& p, const anu_pdhg_options& o, const CaseData* trial);

// ||K~|| by power iteration on the device, FP64 (pdhg.cpp:223-282).
double device_matrix_norm(Problem& p, int iterations, double tolerance);

// Cases one run of the case-stack kernels carries (lanes x cases per lane).
constexpr int kMaxCasesPerRun = 64;

// FP64 convergence measures of one point against an unscaled LP held by a
// unit-scaled problem (evaluate_residual, pdhg.cpp:112-174).
void evaluate_point(Problem& p, const CaseData& cd, const std::vector<double>& x,
                    const std::vector<double>& y, anu_pdhg_residual* out);

int copy_last_error(char* buf, int32_t size);

std::string validate_lp(const anu_lp& lp);
void validate_options(const anu_pdhg_options& o);

}  // namespace anu
