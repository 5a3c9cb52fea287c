// The PDHG engine: device problem setup, the lockstep case-stack solver and
// the single-LP / case-stack entry points of the C ABI.
//
// The control flow of run_cases restates solve_pdhg
// (src/anukulan/pdhg.cpp:377-1285) once per case: the same step-size and
// primal-weight initialisation, Halpern epochs with reflection, the
// fixed-point (or KKT) restart test with cuPDLP's three conditions, the PID
// primal weight, feasibility polishing with its geometric schedule and exit
// polish, the Farkas infeasibility test, the time limit and the stop flag.
// What changes is where the work runs: the iteration is two fused kernels
// (K'y + primal step, K x_bar + dual step) launched as CUDA-graph chunks of
// one check period, and every check is a handful of device reductions whose
// results (18 doubles per case) are the only thing that crosses the bus.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <numeric>
#include <thread>
#include <unordered_map>
#include <utility>

#include "engine.hpp"

namespace anu {

// ------------------------------------------------------------- errors

namespace {
thread_local std::string g_error;
thread_local int g_error_code = ANU_OK;
}  // namespace

void set_last_error(int code, const std::string& message) {
  g_error_code = code;
  g_error = message;
}
void clear_last_error() {
  g_error_code = ANU_OK;
  g_error.clear();
}
int copy_last_error(char* buf, int32_t size) {
  if (buf != nullptr && size > 0) std::snprintf(buf, static_cast<size_t>(size), "%s", g_error.c_str());
  return g_error_code;
}

void cuda_check(cudaError_t status, const char* what) {
  if (status != cudaSuccess) {
    const int code = (status == cudaErrorNoDevice || status == cudaErrorInsufficientDriver)
                         ? ANU_ERR_NO_DEVICE
                         : (status == cudaErrorMemoryAllocation ? ANU_ERR_MEMORY : ANU_ERR_CUDA);
    throw Error(code, std::string(what) + ": " + cudaGetErrorString(status));
  }
}

// ------------------------------------------------------------ matrices

void DevCsr::upload(const HostCsr& a, bool with_fp32, cudaStream_t s, int32_t seg_nnz,
                    int32_t seg_per) {
  if (seg_nnz < 1 || seg_per < 1 || seg_per > kSegPerCtaMax)
    throw Error(ANU_ERR_INTERNAL, "segment shape out of range");
  rows = a.rows;
  cols = a.cols;
  nnz = a.nnz();
  start.alloc(static_cast<size_t>(rows) + 1);
  index.alloc(std::max<size_t>(nnz, 1));
  v64.alloc(std::max<size_t>(nnz, 1));
  ANU_CUDA(cudaMemcpyAsync(start.p, a.start.data(), sizeof(int32_t) * (rows + 1),
                           cudaMemcpyHostToDevice, s));
  std::vector<float> f;
  if (nnz > 0) {
    ANU_CUDA(cudaMemcpyAsync(index.p, a.index.data(), sizeof(int32_t) * nnz,
                             cudaMemcpyHostToDevice, s));
    ANU_CUDA(cudaMemcpyAsync(v64.p, a.value.data(), sizeof(double) * nnz,
                             cudaMemcpyHostToDevice, s));
  }
  if (with_fp32) {
    v32.alloc(std::max<size_t>(nnz, 1));
    f.resize(nnz);
    for (int32_t k = 0; k < nnz; ++k) f[k] = static_cast<float>(a.value[k]);
    if (nnz > 0)
      ANU_CUDA(cudaMemcpyAsync(v32.p, f.data(), sizeof(float) * nnz, cudaMemcpyHostToDevice, s));
  }
  // Every row exactly kEllWidth long: ell_kernel takes the single-LP product.
  bool uniform = rows > 0 && nnz == kEllWidth * rows;
  for (int32_t r = 0; uniform && r <= rows; ++r) uniform = a.start[r] == kEllWidth * r;
  uniform_len = uniform ? kEllWidth : 0;
  for (int i = 0; i < 2; ++i) {
    const int32_t threads = kTileThreads[i];
    const std::vector<RowBlock> b = row_blocks(a, threads * kPerThread, threads, kLongRow);
    std::vector<RowBlockDev> bd(b.size());
    for (size_t j = 0; j < b.size(); ++j)
      bd[j] = {b[j].row_begin, b[j].row_end, a.start[b[j].row_begin], a.start[b[j].row_end]};
    tile_num_blocks[i] = static_cast<int32_t>(bd.size());
    tile_blocks[i].alloc(std::max<size_t>(bd.size(), 1));
    if (!bd.empty())
      ANU_CUDA(cudaMemcpyAsync(tile_blocks[i].p, bd.data(), sizeof(RowBlockDev) * bd.size(),
                               cudaMemcpyHostToDevice, s));
  }
  set_tile(kRowThreads);
  const SegmentSchedule sch = segment_schedule(a, seg_nnz, seg_per, kSegRows);
  seg_per_cta = seg_per;
  num_ctas = static_cast<int32_t>(sch.cta_row.size()) - 1;
  auto put = [&](DevBuf<int32_t>& d, const std::vector<int32_t>& h) {
    d.alloc(std::max<size_t>(h.size(), 1));
    if (!h.empty())
      ANU_CUDA(cudaMemcpyAsync(d.p, h.data(), sizeof(int32_t) * h.size(), cudaMemcpyHostToDevice, s));
  };
  put(seg_begin, sch.seg_begin);
  put(row_seg, sch.row_seg);
  put(cta_row, sch.cta_row);
  put(cta_seg, sch.cta_seg);
  ANU_CUDA(cudaStreamSynchronize(s));
}

void DevCsr::set_tile(int32_t threads) {
  const int i = threads == kTileThreads[1] ? 1 : 0;
  if (threads != kTileThreads[i]) throw Error(ANU_ERR_INVALID, "tile size must be 128 or 256 threads");
  blocks = tile_blocks[i].p;
  num_blocks = tile_num_blocks[i];
  tile_threads = threads;
}

void DevCsr::prepare_cluster(const HostCsr& a, cudaStream_t s) {
  if (cl_ready) return;
  auto put_rows = [&](DevBuf<int32_t>& d, const std::vector<int32_t>& h) {
    d.alloc(std::max<size_t>(h.size(), 1));
    if (!h.empty())
      ANU_CUDA(cudaMemcpyAsync(d.p, h.data(), sizeof(int32_t) * h.size(), cudaMemcpyHostToDevice, s));
  };
  for (int i = 0; i < 2; ++i) {
    const ClusterSchedule c = cluster_schedule(a, i == 0 ? 16 : 8, kSerialRow);
    put_rows(cl_bounds[i], c.bounds);
    put_rows(cl_warp_start[i], c.warp_start);
    put_rows(cl_warp_rows[i], c.warp_rows);
    cl_max_rows[i] = c.max_part_rows;
    cl_max_nnz[i] = c.max_part_nnz;
    max_row = c.max_row;
  }
  ANU_CUDA(cudaStreamSynchronize(s));
  cl_ready = true;
}

ClusterRows DevCsr::cluster_rows(int ctas) const {
  const int i = ctas == 16 ? 0 : 1;
  return {cl_bounds[i].p, cl_warp_start[i].p, cl_warp_rows[i].p, cl_max_rows[i], cl_max_nnz[i]};
}

template <>
CsrView<double> DevCsr::view<double>() const {
  return {rows, cols, start.p, index.p, v64.p, blocks, num_blocks,
          seg_begin.p, row_seg.p, cta_row.p, cta_seg.p, num_ctas, seg_per_cta, uniform_len,
          tile_threads};
}
template <>
CsrView<float> DevCsr::view<float>() const {
  return {rows, cols, start.p, index.p, v32.p, blocks, num_blocks,
          seg_begin.p, row_seg.p, cta_row.p, cta_seg.p, num_ctas, seg_per_cta, uniform_len,
          tile_threads};
}

Problem::~Problem() {
  // The pool, destroyed after this body, frees its blocks on this device.
  cudaSetDevice(device);
  if (stream) cudaStreamSynchronize(stream);
  if (owns_stream && stream) cudaStreamDestroy(stream);
}

namespace {
thread_local MemoryPool* t_pool = nullptr;
// Most bytes a pool keeps cached per kind; blocks beyond it are freed.
constexpr size_t kPoolCap[2] = {size_t(4) << 30, size_t(256) << 20};

size_t size_class(size_t bytes) {
  size_t c = 256;
  while (c < bytes) c <<= 1;
  return c;
}
}  // namespace

MemoryPool* current_pool() { return t_pool; }

PoolScope::PoolScope(MemoryPool* pool, cudaStream_t stream) : previous_(t_pool), stream_(stream) {
  t_pool = pool;
}

PoolScope::~PoolScope() {
  if (stream_) cudaStreamSynchronize(stream_);
  t_pool = previous_;
}

// Idle blocks of destroyed pools, by (device, size class); pinned host
// blocks under device -1. Created on first use and never destroyed: at
// process exit the CUDA runtime may already be gone, and the driver
// reclaims the memory.
class BlockCache {
 public:
  void* take(int device, size_t cls) {
    std::lock_guard<std::mutex> g(lock_);
    auto it = free_.find({device, cls});
    if (it == free_.end()) return nullptr;
    void* p = it->second;
    free_.erase(it);
    bytes_[device < 0] -= cls;
    return p;
  }
  bool keep(int device, void* p, size_t cls) {
    std::lock_guard<std::mutex> g(lock_);
    if (bytes_[device < 0] + cls > kGlobalCap[device < 0]) return false;
    free_.emplace(std::make_pair(device, cls), p);
    bytes_[device < 0] += cls;
    return true;
  }
  size_t release() {
    std::multimap<std::pair<int, size_t>, void*> blocks;
    {
      std::lock_guard<std::mutex> g(lock_);
      blocks.swap(free_);
      bytes_[0] = bytes_[1] = 0;
    }
    int current = 0;
    cudaGetDevice(&current);
    size_t freed = 0;
    for (auto& b : blocks) {
      if (b.first.first < 0) {
        cudaFreeHost(b.second);
      } else {
        cudaSetDevice(b.first.first);
        cudaFree(b.second);
      }
      freed += b.first.second;
    }
    cudaSetDevice(current);
    return freed;
  }

 private:
  // Most bytes kept: device blocks (all devices together), pinned blocks.
  static constexpr size_t kGlobalCap[2] = {size_t(16) << 30, size_t(1) << 30};
  std::mutex lock_;
  std::multimap<std::pair<int, size_t>, void*> free_;
  size_t bytes_[2] = {0, 0};
};

BlockCache& block_cache() {
  static BlockCache* cache = new BlockCache();
  return *cache;
}

size_t release_cached_blocks() { return block_cache().release(); }

std::mutex& cooperative_mutex(int device) {
  static std::mutex locks[64];
  return locks[static_cast<unsigned>(device) % 64u];
}

void* MemoryPool::get(bool pinned, size_t bytes, size_t* rounded) {
  const size_t c = size_class(bytes);
  *rounded = c;
  {
    std::lock_guard<std::mutex> g(lock_);
    auto it = free_[pinned].find(c);
    if (it != free_[pinned].end()) {
      void* p = it->second;
      free_[pinned].erase(it);
      cached_[pinned] -= c;
      return p;
    }
  }
  int device = -1;
  if (!pinned) {
    ANU_CUDA(cudaGetDevice(&device));
    std::lock_guard<std::mutex> g(lock_);
    if (device_ < 0) device_ = device;
    if (device_ != device)
      throw Error(ANU_ERR_INTERNAL, "memory pool used on two devices");
  }
  if (void* p = block_cache().take(device, c)) return p;
  void* p = nullptr;
  cudaError_t e = pinned ? cudaMallocHost(&p, c) : cudaMalloc(&p, c);
  if (e == cudaErrorMemoryAllocation) {
    // Cached blocks of other sizes may be what fills the device: free them
    // and try once more.
    cudaGetLastError();
    block_cache().release();
    e = pinned ? cudaMallocHost(&p, c) : cudaMalloc(&p, c);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(ANU_ERR_MEMORY, std::string(pinned ? "cudaMallocHost: " : "cudaMalloc: ") +
                                    cudaGetErrorString(e));
  }
  return p;
}

void MemoryPool::put(bool pinned, void* p, size_t rounded) {
  {
    std::lock_guard<std::mutex> g(lock_);
    if (cached_[pinned] + rounded <= kPoolCap[pinned]) {
      free_[pinned].emplace(rounded, p);
      cached_[pinned] += rounded;
      return;
    }
  }
  // Over this pool's cap: freed at once (this pool's stream may still use
  // the block, and cudaFree waits for the device; the shared cache does not).
  if (pinned) cudaFreeHost(p);
  else cudaFree(p);
}

MemoryPool::~MemoryPool() {
  if (free_[0].empty() && free_[1].empty()) return;
  // All work that could read these blocks ends before any other pool may
  // receive them.
  int current = 0;
  cudaGetDevice(&current);
  if (device_ >= 0) {
    cudaSetDevice(device_);
    cudaDeviceSynchronize();
  } else {
    cudaDeviceSynchronize();
  }
  BlockCache& cache = block_cache();
  for (auto& b : free_[0])
    if (!cache.keep(device_, b.second, b.first)) cudaFree(b.second);
  for (auto& b : free_[1])
    if (!cache.keep(-1, b.second, b.first)) cudaFreeHost(b.second);
  cudaSetDevice(current);
}

// ------------------------------------------------------------- launches

namespace {

template <class T>
__global__ void accumulate_kernel(int64_t n, double weight, const T* __restrict__ v,
                                  T* __restrict__ sum) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    sum[i] = add(sum[i], mul(static_cast<T>(weight), v[i]));
}

// Sum of squares over one vector per case (power iteration, step terms).
template <class T>
struct SquareTerms {
  static constexpr int NT = 1;
  int32_t K;
  const T* __restrict__ v;
  __device__ static void init(double* a) { a[0] = 0.0; }
  __device__ static double identity(int) { return 0.0; }
  __device__ static double combine(int, double a, double b) { return anu::add(a, b); }
  __device__ void add(double* a, int32_t i, int32_t k) const {
    const double x = static_cast<double>(v[(size_t)i * K + k]);
    a[0] = anu::add(a[0], mul(x, x));
  }
};

// dy . k_dx and |dy|^2 (rows), for the adaptive step size.
template <class T>
struct StepRowTerms {
  static constexpr int NT = 2;
  const T* __restrict__ dy;
  const T* __restrict__ kdx;
  __device__ static void init(double* a) { a[0] = a[1] = 0.0; }
  __device__ static double identity(int) { return 0.0; }
  __device__ static double combine(int, double a, double b) { return anu::add(a, b); }
  __device__ void add(double* a, int32_t i, int32_t) const {
    const double d = static_cast<double>(dy[i]);
    a[0] = anu::add(a[0], mul(d, static_cast<double>(kdx[i])));
    a[1] = anu::add(a[1], mul(d, d));
  }
};

__global__ void normalize_kernel(int32_t n, const double* __restrict__ in,
                                 const double* __restrict__ sumsq, double* __restrict__ out,
                                 double* __restrict__ estimates, int32_t slot) {
  const double next = sqrt(sumsq[0]);
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x)
    out[j] = next != 0.0 ? in[j] / next : 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) estimates[slot] = next;
}

}  // namespace

// ------------------------------------------------------ ||K|| estimate

double device_matrix_norm(Problem& p, int iterations, double tolerance) {
  const int32_t n = p.n, m = p.m;
  if (n == 0 || m == 0 || p.dk.nnz == 0) return 0.0;
  // Deterministic non-uniform start, normalised on the host exactly as the
  // reference does (pdhg.cpp:233-238).
  // A relabelled problem starts from the same vector, entry for entry, so
  // the sum runs over the original order.
  std::vector<double> v(n);
  double ss = 0.0;
  for (int32_t j = 0; j < n; ++j) {
    const double a = 1.0 + 0.1 * static_cast<double>(j % 7);
    ss += a * a;
  }
  for (int32_t j = 0; j < n; ++j) {
    const int32_t orig = p.col_old.empty() ? j : p.col_old[j];
    v[j] = 1.0 + 0.1 * static_cast<double>(orig % 7);
  }
  const double norm = std::sqrt(ss);
  if (norm == 0.0) return 0.0;
  for (double& a : v) a /= norm;
  // Chunks of iterations between host looks; the convergence test reads the
  // estimates in order, so running past convergence (or past `iterations`,
  // in the last chunk) changes nothing. Estimate slots are per position in
  // the chunk, so after the first chunk (run directly, which also sizes the
  // reduction scratch) every chunk is the same work: one CUDA graph,
  // captured once and replayed.
  const int chunk = 16;
  DevBuf<double> dv(n), dkv(m), dktkv(n), partial, sumsq(1), est(chunk);
  ANU_CUDA(cudaMemcpyAsync(dv.p, v.data(), sizeof(double) * n, cudaMemcpyHostToDevice, p.stream));
  std::vector<double> h_est(chunk);
  auto enqueue = [&](int count) {
    for (int it = 0; it < count; ++it) {
      product<double, double, double>(p, p.dk, dv.p, 1, StoreEpi<double>{1, dkv.p});
      product<double, double, double>(p, p.dkt, dkv.p, 1, StoreEpi<double>{1, dktkv.p});
      reduce_terms(p, n, 1, SquareTerms<double>{1, dktkv.p}, partial, sumsq.p, 1, 0);
      normalize_kernel<<<grid_for(n, 256, 296), 256, 0, p.stream>>>(n, dktkv.p, sumsq.p, dv.p,
                                                                     est.p, it);
      ANU_CUDA(cudaGetLastError());
      ++p.launches;
    }
  };
  struct GraphGuard {
    cudaGraphExec_t exec = nullptr;
    ~GraphGuard() {
      if (exec) cudaGraphExecDestroy(exec);
    }
  } graph;
  int64_t graph_launches = 0;
  double sigma = 0.0;
  for (int base = 0; base < iterations; base += chunk) {
    const int count = std::min(chunk, iterations - base);
    if (base == 0) {
      enqueue(count);
    } else {
      if (graph.exec == nullptr) {
        const int64_t before = p.launches;
        ANU_CUDA(cudaStreamBeginCapture(p.stream, cudaStreamCaptureModeThreadLocal));
        try {
          enqueue(chunk);
        } catch (...) {
          cudaGraph_t broken = nullptr;
          cudaStreamEndCapture(p.stream, &broken);
          if (broken) cudaGraphDestroy(broken);
          throw;
        }
        cudaGraph_t g = nullptr;
        ANU_CUDA(cudaStreamEndCapture(p.stream, &g));
        const cudaError_t e = cudaGraphInstantiate(&graph.exec, g, 0);
        cudaGraphDestroy(g);
        ANU_CUDA(e);
        graph_launches = p.launches - before;
        p.launches = before;
      }
      ANU_CUDA(cudaGraphLaunch(graph.exec, p.stream));
      p.launches += graph_launches;
    }
    ANU_CUDA(cudaMemcpyAsync(h_est.data(), est.p, sizeof(double) * count,
                             cudaMemcpyDeviceToHost, p.stream));
    ANU_CUDA(cudaStreamSynchronize(p.stream));
    for (int it = base; it < base + count; ++it) {
      const double next = h_est[it - base];
      if (next == 0.0) return 0.0;
      const double estimate = std::sqrt(next);
      if (it > 0 && std::fabs(estimate - sigma) <= tolerance * estimate) return estimate;
      sigma = estimate;
    }
  }
  return sigma;
}

// ---------------------------------------------------------- validation

std::string validate_lp(const anu_lp& lp) {
  const std::string e = validate_csr(lp.k.rows, lp.k.cols, lp.k.nnz, lp.k.start, lp.k.index);
  if (!e.empty()) return e;
  if (lp.k.nnz > 0 && lp.k.value == nullptr) return "null matrix values";
  if (lp.k.cols > 0 && (lp.c == nullptr || lp.lower == nullptr || lp.upper == nullptr))
    return "null column vectors";
  if (lp.k.rows > 0 && lp.q == nullptr) return "null right-hand side";
  if (lp.num_equalities < 0 || lp.num_equalities > lp.k.rows) return "num_equalities out of range";
  for (int32_t j = 0; j < lp.k.cols; ++j)
    if (lp.lower[j] > lp.upper[j]) return "empty bound interval at column " + std::to_string(j);
  for (int32_t i = 0; i < lp.k.rows; ++i)
    if (!std::isfinite(lp.q[i])) return "rhs is not finite";
  return "";
}

void validate_options(const anu_pdhg_options& o) {
  if (o.termination_check_frequency < 1) throw Error(ANU_ERR_INVALID, "termination_check_frequency < 1");
  if (o.max_iterations < 0) throw Error(ANU_ERR_INVALID, "max_iterations < 0");
  if (o.precision != ANU_PRECISION_FP64 && o.precision != ANU_PRECISION_FP32)
    throw Error(ANU_ERR_INVALID, "unknown precision");
  if (o.ruiz_iterations < 0) throw Error(ANU_ERR_INVALID, "ruiz_iterations < 0");
  if (o.termination < 0 || o.termination > 2) throw Error(ANU_ERR_INVALID, "unknown termination");
  if (o.tile_threads != 0 && o.tile_threads != kTileThreads[0] && o.tile_threads != kTileThreads[1])
    throw Error(ANU_ERR_INVALID, "tile_threads must be 0 (tuned), 128 or 256");
  if (o.cluster_chunks != 0 && o.cluster_chunks != 1)
    throw Error(ANU_ERR_INVALID, "cluster_chunks must be 0 or 1");
}

// ------------------------------------------------------ product tiles

// The single-LP product tile of each matrix of `p`: options.tile_threads
// when set. Otherwise, for a single LP of at least kTuneNnz nonzeros (`trial`
// is its case), short solves of that LP run for each pair of tiles (one for
// K~, one for K~') and the pair with the least device time per iteration
// stays if it beats the default pair by kTuneMargin; smaller LPs keep
// kRowThreads, where the trials would cost more than they save. Every tile sums every row in the same order (a row longer than
// kLongRow always takes a CTA of its own and a fixed-width sum), so the
// choice changes timing only, never a result; the trial results are
// discarded. Returns whether trial solves ran.
bool choose_tiles(Problem& p, const anu_pdhg_options& o, const CaseData* trial) {
  const int32_t fixed = o.tile_threads != 0 ? o.tile_threads : kRowThreads;
  p.dk.set_tile(fixed);
  p.dkt.set_tile(fixed);
  if (o.tile_threads != 0 || trial == nullptr || !o.use_graphs || o.persistent_chunks ||
      p.k.nnz() < kTuneNnz)
    return false;
  anu_pdhg_options t = o;
  // Chunks of at most 64 iterations, so a long check period does not make
  // the trials long.
  t.termination_check_frequency = std::min<int32_t>(o.termination_check_frequency, 64);
  t.max_iterations = kTuneChunks * t.termination_check_frequency;
  t.tolerance = 0.0;  // runs the whole budget
  t.profile = 1;
  t.verbose = 0;
  t.polish_feasibility = 0;
  t.polish_on_exit = 0;
  const int64_t launches = p.launches;
  const std::vector<const std::vector<double>*> none(1, nullptr);
  auto per_iteration = [&](int32_t dk_threads, int32_t dkt_threads) {
    p.dk.set_tile(dk_threads);
    p.dkt.set_tile(dkt_threads);
    std::vector<CaseResult> res;
    run_cases(p, {trial}, t, none, none, &res, now_seconds());
    const anu_pdhg_result& r = res[0].r;
    return r.device_iterations > 0 ? r.device_iteration_seconds / r.device_iterations : INFINITY;
  };
  per_iteration(kRowThreads, kRowThreads);  // untimed: first touch of the pool and caches
  // Each pair twice, the second round in reverse order, keeping its faster
  // time: one trial varies by a percent or two, drift cancels.
  constexpr int kPairs = 4;
  double sec[kPairs];
  for (int rep = 0; rep < 2; ++rep)
    for (int k = 0; k < kPairs; ++k) {
      const int i = rep == 0 ? k : kPairs - 1 - k;
      const double t_i = per_iteration(kTileThreads[i / 2], kTileThreads[i % 2]);
      sec[i] = rep == 0 ? t_i : std::min(sec[i], t_i);
    }
  // Pair 0 is the default; another pair must beat it by kTuneMargin.
  int best = 0;
  for (int i = 1; i < kPairs; ++i)
    if (sec[i] < sec[best] && sec[i] < (1.0 - kTuneMargin) * sec[0]) best = i;
  p.dk.set_tile(kTileThreads[best / 2]);
  p.dkt.set_tile(kTileThreads[best % 2]);
  p.launches = launches;  // the trial launches belong to no solve
  return true;
}

// ------------------------------------------------ locality relabelling

Relabel locality_relabel(const anu_lp& lp) {
  const int32_t m = lp.k.rows, n = lp.k.cols, ne = lp.num_equalities;
  Relabel r;
  if (m == 0 || n == 0) return r;
  const int32_t* start = lp.k.start;
  r.row_old.resize(m);
  std::iota(r.row_old.begin(), r.row_old.end(), 0);
  const auto longer = [start](int32_t a, int32_t b) {
    return start[a + 1] - start[a] > start[b + 1] - start[b];
  };
  std::stable_sort(r.row_old.begin(), r.row_old.begin() + ne, longer);
  std::stable_sort(r.row_old.begin() + ne, r.row_old.end(), longer);
  r.row_new.resize(m);
  for (int32_t i = 0; i < m; ++i) r.row_new[r.row_old[i]] = i;
  // A column's key is the first relabelled row it appears in (m if none).
  std::vector<int32_t> key(n, m);
  for (int32_t i = 0; i < m; ++i)
    for (int32_t e = start[i]; e < start[i + 1]; ++e) {
      int32_t& k = key[lp.k.index[e]];
      k = std::min(k, r.row_new[i]);
    }
  r.col_old.resize(n);
  std::iota(r.col_old.begin(), r.col_old.end(), 0);
  std::stable_sort(r.col_old.begin(), r.col_old.end(),
                   [&key](int32_t a, int32_t b) { return key[a] < key[b]; });
  r.col_new.resize(n);
  for (int32_t j = 0; j < n; ++j) r.col_new[r.col_old[j]] = j;
  return r;
}

namespace {

// Rows taken in the order row_old, each with its nonzeros in stored order,
// column indices mapped through col_new.
HostCsr relabel_csr(const HostCsr& a, const std::vector<int32_t>& row_old,
                    const std::vector<int32_t>& col_new) {
  HostCsr b;
  b.rows = a.rows;
  b.cols = a.cols;
  b.start.assign(static_cast<size_t>(a.rows) + 1, 0);
  b.index.resize(a.index.size());
  b.value.resize(a.value.size());
  int32_t e = 0;
  for (int32_t r = 0; r < a.rows; ++r) {
    const int32_t i = row_old[r];
    for (int32_t s = a.start[i]; s < a.start[i + 1]; ++s, ++e) {
      b.index[e] = col_new[a.index[s]];
      b.value[e] = a.value[s];
    }
    b.start[r + 1] = e;
  }
  return b;
}

std::vector<double> take(const std::vector<double>& v, const std::vector<int32_t>& old) {
  std::vector<double> out(old.size());
  for (size_t i = 0; i < old.size(); ++i) out[i] = v[old[i]];
  return out;
}

std::vector<double> take(const double* v, const std::vector<int32_t>& old) {
  std::vector<double> out(old.size());
  for (size_t i = 0; i < old.size(); ++i) out[i] = v[old[i]];
  return out;
}

void apply_relabel(Problem& p, const Relabel& r) {
  p.k = relabel_csr(p.k, r.row_old, r.col_new);
  p.kt = relabel_csr(p.kt, r.col_old, r.row_new);
  p.scaling.row_scale = take(p.scaling.row_scale, r.row_old);
  p.scaling.col_scale = take(p.scaling.col_scale, r.col_old);
  for (auto& d : p.sweeps.d1) d = take(d, r.row_old);
  for (auto& d : p.sweeps.d2) d = take(d, r.col_old);
  p.col_old = r.col_old;
}

}  // namespace

// -------------------------------------------------------------- setup

std::unique_ptr<Problem> make_problem(const anu_lp& lp, const anu_pdhg_options& o,
                                      double* scaling_seconds, double* norm_seconds,
                                      int32_t seg_nnz, int32_t seg_per_cta,
                                      const Relabel* relabel) {
  int count = 0;
  const cudaError_t ce = cudaGetDeviceCount(&count);
  if (ce != cudaSuccess || count == 0)
    throw Error(ANU_ERR_NO_DEVICE, "no CUDA device is available; this engine has no CPU fallback");
  if (o.device < 0 || o.device >= count) throw Error(ANU_ERR_INVALID, "device ordinal out of range");
  ANU_CUDA(cudaSetDevice(o.device));
  auto p = std::make_unique<Problem>();
  p->device = o.device;
  ANU_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  p->owns_stream = true;
  // The matrices and the norm estimate's vectors come from the problem's
  // pool too, so they return to the shared cache with it.
  PoolScope scope(&p->pool, p->stream);
  p->m = lp.k.rows;
  p->n = lp.k.cols;
  p->num_eq = lp.num_equalities;
  p->precision = o.precision;
  double t0 = now_seconds();
  p->k = copy_csr(lp.k.rows, lp.k.cols, lp.k.nnz, lp.k.start, lp.k.index, lp.k.value);
  const int sweeps = o.ruiz_iterations + (o.pock_chambolle != 0 ? 1 : 0);
  if (o.scaling_on_device != 0 && sweeps > 0 && p->k.nnz() > 0) {
    p->scaling = scale_matrix_sweeps_device(*p, &p->k, &p->kt, o.ruiz_iterations,
                                            o.pock_chambolle != 0, &p->sweeps);
  } else {
    p->scaling = scale_matrix_sweeps(&p->k, o.ruiz_iterations, o.pock_chambolle != 0, &p->sweeps);
    p->kt = transpose(p->k);
  }
  if (relabel != nullptr && !relabel->empty()) apply_relabel(*p, *relabel);
  if (scaling_seconds) *scaling_seconds = now_seconds() - t0;
  const bool fp32 = o.precision == ANU_PRECISION_FP32;
  p->seg_nnz = seg_nnz;
  p->seg_per_cta = seg_per_cta;
  p->dk.upload(p->k, fp32, p->stream, seg_nnz, seg_per_cta);
  p->dkt.upload(p->kt, fp32, p->stream, seg_nnz, seg_per_cta);
  if (fp32) prepare_iteration_kernels<float>(p->stream);
  else prepare_iteration_kernels<double>(p->stream);
  p->row_scale.alloc(std::max(p->m, 1));
  p->col_scale.alloc(std::max(p->n, 1));
  if (p->m > 0)
    ANU_CUDA(cudaMemcpyAsync(p->row_scale.p, p->scaling.row_scale.data(), sizeof(double) * p->m,
                             cudaMemcpyHostToDevice, p->stream));
  if (p->n > 0)
    ANU_CUDA(cudaMemcpyAsync(p->col_scale.p, p->scaling.col_scale.data(), sizeof(double) * p->n,
                             cudaMemcpyHostToDevice, p->stream));
  ANU_CUDA(cudaStreamSynchronize(p->stream));
  t0 = now_seconds();
  p->matrix_norm = o.known_matrix_norm > 0.0 ? o.known_matrix_norm
                                              : device_matrix_norm(*p, 200, 1e-8);
  if (norm_seconds) *norm_seconds = now_seconds() - t0;
  return p;
}

bool stack_runs_persistent(const Problem& p, int K, const anu_pdhg_options& o) {
  const bool slow = (o.adaptive_step_size && !o.constant_step_size) || o.halpern_restart;
  if (!o.persistent_chunks || !o.use_graphs || slow) return false;
  ANU_CUDA(cudaSetDevice(p.device));
  return p.precision == ANU_PRECISION_FP32 ? chunk_fits<float>(p.dkt, p.dk, K)
                                           : chunk_fits<double>(p.dkt, p.dk, K);
}

std::unique_ptr<Problem> clone_problem(const Problem& src) {
  ANU_CUDA(cudaSetDevice(src.device));
  auto p = std::make_unique<Problem>();
  p->device = src.device;
  ANU_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  p->owns_stream = true;
  PoolScope scope(&p->pool, p->stream);
  p->m = src.m;
  p->n = src.n;
  p->num_eq = src.num_eq;
  p->precision = src.precision;
  p->k = src.k;
  p->kt = src.kt;
  p->scaling = src.scaling;
  p->sweeps = src.sweeps;
  p->unit_scaling = src.unit_scaling;
  p->matrix_norm = src.matrix_norm;
  p->col_old = src.col_old;
  const bool fp32 = p->precision == ANU_PRECISION_FP32;
  p->seg_nnz = src.seg_nnz;
  p->seg_per_cta = src.seg_per_cta;
  p->dk.upload(p->k, fp32, p->stream, p->seg_nnz, p->seg_per_cta);
  p->dkt.upload(p->kt, fp32, p->stream, p->seg_nnz, p->seg_per_cta);
  p->dk.set_tile(src.dk.tile_threads);
  p->dkt.set_tile(src.dkt.tile_threads);
  p->row_scale.alloc(std::max(p->m, 1));
  p->col_scale.alloc(std::max(p->n, 1));
  if (p->m > 0)
    ANU_CUDA(cudaMemcpyAsync(p->row_scale.p, p->scaling.row_scale.data(), sizeof(double) * p->m,
                             cudaMemcpyHostToDevice, p->stream));
  if (p->n > 0)
    ANU_CUDA(cudaMemcpyAsync(p->col_scale.p, p->scaling.col_scale.data(), sizeof(double) * p->n,
                             cudaMemcpyHostToDevice, p->stream));
  ANU_CUDA(cudaStreamSynchronize(p->stream));
  return p;
}

CaseData make_case(const Problem& p, const double* c, const double* q, const double* lower,
                   const double* upper, double objective_scale, double objective_offset) {
  CaseData d;
  d.c.assign(c, c + p.n);
  d.q.assign(q, q + p.m);
  d.lower.assign(lower, lower + p.n);
  d.upper.assign(upper, upper + p.n);
  d.cs = d.c;
  d.qs = d.q;
  d.ls = d.lower;
  d.us = d.upper;
  if (!p.unit_scaling)
    scale_vectors(p.sweeps, p.m, p.n, d.cs.data(), d.qs.data(), d.ls.data(), d.us.data());
  d.objective_scale = objective_scale;
  d.objective_offset = objective_offset;
  return d;
}

// ------------------------------------------------------------- solver

namespace {

double host_norm2(const std::vector<double>& v) {
  double s = 0.0;
  for (double a : v) s += a * a;
  return std::sqrt(s);
}
double host_norminf(const std::vector<double>& v) {
  double m = 0.0;
  for (double a : v) m = std::fmax(m, std::fabs(a));
  return m;
}

struct ResidualScales {
  double q_two, c_two, q_inf, c_inf;
};

// residual_from_terms (pdhg.cpp:70-87) from the row and column check terms.
anu_pdhg_residual residual_from_terms(const double* row, const double* col,
                                      const ResidualScales& s) {
  anu_pdhg_residual r{};
  r.primal_residual = std::sqrt(row[0]);
  r.primal_residual_inf = row[1];
  r.dual_residual = std::sqrt(col[0]);
  r.dual_residual_inf = col[1];
  r.primal_objective = col[3];
  r.dual_objective = row[2] + col[2];
  r.absolute_gap = std::fabs(r.primal_objective - r.dual_objective);
  r.relative_primal = r.primal_residual / (1.0 + s.q_two);
  r.relative_dual = r.dual_residual / (1.0 + s.c_two);
  r.relative_primal_inf = r.primal_residual_inf / (1.0 + s.q_inf);
  r.relative_dual_inf = r.dual_residual_inf / (1.0 + s.c_inf);
  r.relative_gap =
      r.absolute_gap / (1.0 + std::fabs(r.primal_objective) + std::fabs(r.dual_objective));
  return r;
}

bool primal_ok(const anu_pdhg_residual& r, double tol, double abs_tol, bool inf) {
  bool ok = r.relative_primal <= tol;
  if (inf) ok = ok && r.relative_primal_inf <= tol;
  if (abs_tol > 0.0) ok = ok && r.primal_residual_inf <= abs_tol;
  return ok;
}
bool dual_ok(const anu_pdhg_residual& r, double tol, double abs_tol, bool inf) {
  bool ok = r.relative_dual <= tol;
  if (inf) ok = ok && r.relative_dual_inf <= tol;
  if (abs_tol > 0.0) ok = ok && r.dual_residual_inf <= abs_tol;
  return ok;
}
bool converged(const anu_pdhg_residual& r, double tol, double abs_tol, bool inf, double gap_tol) {
  return primal_ok(r, tol, abs_tol, inf) && dual_ok(r, tol, abs_tol, inf) &&
         r.relative_gap <= (gap_tol > 0.0 ? gap_tol : tol);
}

void set_message(anu_pdhg_result* r, const std::string& m) {
  std::snprintf(r->message, sizeof(r->message), "%s", m.c_str());
}

constexpr int kRowTerms = RowCheckTerms<double, double, double>::NT;  // 9
constexpr int kColTerms = ColCheckTerms<double, double>::NT;          // 9
constexpr int kCheckTerms = kRowTerms + kColTerms;            // 18
constexpr int kKktTerms = 5;  // primal_sq, q_dot_y, dual_sq, bound_term, c_dot_x

// Pinned host staging that lives as long as a run.
template <class T>
struct Pinned {
  T* p = nullptr;
  size_t n = 0;
  MemoryPool* pool = nullptr;
  size_t bytes = 0;
  explicit Pinned(size_t count) : n(count) {
    if (!count) return;
    if (MemoryPool* mp = current_pool()) {
      p = static_cast<T*>(mp->get(true, sizeof(T) * count, &bytes));
      pool = mp;
      return;
    }
    ANU_CUDA(cudaMallocHost(reinterpret_cast<void**>(&p), sizeof(T) * count));
  }
  ~Pinned() {
    if (!p) return;
    if (pool) pool->put(true, p, bytes);
    else cudaFreeHost(p);
  }
  Pinned(const Pinned&) = delete;
  Pinned& operator=(const Pinned&) = delete;
};

// Evaluates the FP64 check terms of scaled points (x~, y~) of K cases: fresh
// products, then the row and column terms; returns terms[case][18] on host.
void eval_points_terms(Problem& p, bool unit, int K, const std::vector<const CaseData*>& cases,
                       const std::vector<std::vector<double>>& xs,
                       const std::vector<std::vector<double>>& ys, std::vector<double>* terms) {
  const int32_t n = p.n, m = p.m;
  std::vector<double> hx(static_cast<size_t>(n) * K), hy(static_cast<size_t>(m) * K);
  std::vector<double> hc(hx.size()), hl(hx.size()), hu(hx.size()), hq(hy.size());
  for (int k = 0; k < K; ++k) {
    for (int32_t j = 0; j < n; ++j) {
      const size_t e = static_cast<size_t>(j) * K + k;
      hx[e] = xs[k][j];
      hc[e] = cases[k]->c[j];
      hl[e] = cases[k]->lower[j];
      hu[e] = cases[k]->upper[j];
    }
    for (int32_t i = 0; i < m; ++i) {
      const size_t e = static_cast<size_t>(i) * K + k;
      hy[e] = ys[k][i];
      hq[e] = cases[k]->q[i];
    }
  }
  DevBuf<double> dx(std::max<size_t>(hx.size(), 1)), dy(std::max<size_t>(hy.size(), 1)),
      dc(dx.n), dl(dx.n), du(dx.n), dq(dy.n), kx(dy.n), kty(dx.n), out(kCheckTerms * K), part;
  auto up = [&](DevBuf<double>& d, const std::vector<double>& h) {
    if (!h.empty())
      ANU_CUDA(cudaMemcpyAsync(d.p, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice,
                               p.stream));
  };
  up(dx, hx);
  up(dy, hy);
  up(dc, hc);
  up(dl, hl);
  up(du, hu);
  up(dq, hq);
  product<double, double, double>(p, p.dk, dx.p, K, StoreEpi<double>{K, kx.p});
  product<double, double, double>(p, p.dkt, dy.p, K, StoreEpi<double>{K, kty.p});
  RowCheckTerms<double, double, double> rt{K, p.num_eq, kx.p, dy.p, nullptr, nullptr, nullptr,
                                           nullptr, dq.p, nullptr, unit ? nullptr : p.row_scale.p};
  ColCheckTerms<double, double> ct{K, kty.p, dx.p, nullptr, nullptr, nullptr, nullptr, dc.p, dl.p,
                                   du.p, unit ? nullptr : p.col_scale.p, nullptr, nullptr, nullptr};
  reduce_terms(p, m, K, rt, part, out.p, kCheckTerms, 0);
  reduce_terms(p, n, K, ct, part, out.p, kCheckTerms, kRowTerms);
  terms->resize(static_cast<size_t>(kCheckTerms) * K);
  ANU_CUDA(cudaMemcpyAsync(terms->data(), out.p, sizeof(double) * terms->size(),
                           cudaMemcpyDeviceToHost, p.stream));
  ANU_CUDA(cudaStreamSynchronize(p.stream));
}

// Per-case host state: the locals of solve_pdhg's loop (pdhg.cpp:466-757).
struct CaseState {
  double eta = 0.0, omega = 1.0;
  bool anchor_needs_reset = true;
  int32_t halpern_k = 0;
  double movement = 0.0, epoch_start_movement = 0.0;
  bool have_previous_restart = false;
  double kkt_at_restart = 0.0;
  double last_candidate_kkt = INFINITY;
  double residual_at_restart = INFINITY;
  double last_residual = INFINITY;
  double weight_error_sum = 0.0, weight_error_previous = 0.0;
  int32_t iterations_since_restart = 0;
  int32_t next_polish_iteration = 0;
  double sum_weight = 0.0;
  bool active = true;
  int32_t status = ANU_PDHG_ITERATION_LIMIT;
  int32_t final_iteration = 0;
  bool use_average = false;
  bool have_polished = false;
  std::vector<double> polished_x, polished_y;
  anu_pdhg_residual polished_residual{};
  ResidualScales scales{};
};

int32_t polish_budget(const anu_pdhg_options& o, int32_t at_iteration) {
  int32_t budget = static_cast<int32_t>(o.polish_iteration_factor * static_cast<double>(at_iteration + 1));
  budget = std::max(budget, o.polish_minimum_iterations);
  budget = std::min(budget, o.polish_maximum_iterations);
  return budget;
}

double kkt_value(const double* t, double omega) {
  // t: primal_sq, q_dot_y, dual_sq, bound_term, c_dot_x (pdhg.cpp:336-339)
  const double gap = t[4] - (t[1] + t[3]);
  const double value = omega * omega * t[0] + t[2] / (omega * omega) + gap * gap;
  return std::sqrt(value);
}

template <class T>
struct Workspace {
  int K = 0;
  int32_t m = 0, n = 0;
  // iteration vectors (case-interleaved)
  DevBuf<T> x, x_bar, anchor_x, dx, c, lo, hi, x_next, sum_x, avg_x, x_restart, x_prev;
  DevBuf<T> y, kx, anchor_y, anchor_kx, dy, q, k_dx, y_next, k_next, sum_y, avg_y, y_restart,
      y_prev, ylo;
  // FP64 island
  DevBuf<double> kty64, ktdy64, kx64, c0, lo0, hi0, q0, los, his, qs;
  // refinement: the FP64 base point, the judged point (base + offset), the
  // scaled data the correction LPs are formed from, K times a column shift,
  // and the averaged scheme's running weight per case
  DevBuf<double> xb, yb, x_comb, y_comb, c0s, q0s, l0s, u0s, kshift, sum_weight;
  DevBuf<StepParams> params;
  DevBuf<double> w_table;
  DevBuf<int32_t> mask;
  DevBuf<double> partial, partial2, terms, kkt, weights;
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
  // The device work of a termination check and of a re-centring, captured
  // as graphs once their buffers have settled and replayed at later checks.
  struct Replay {
    cudaGraphExec_t exec = nullptr;
    const double* partial = nullptr;  // reduction scratch the graph was captured with
    size_t partial_n = 0;
    const double* partial2 = nullptr;
    size_t partial2_n = 0;
    int64_t launches = 0;  // kernels in the graph
    int seen = 0;
    int direct = 0;  // calls run directly (a packed batch's LP, see replay)
  };
  Replay check_replay, recenter_replay;
  ~Workspace() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    if (check_replay.exec) cudaGraphExecDestroy(check_replay.exec);
    if (recenter_replay.exec) cudaGraphExecDestroy(recenter_replay.exec);
  }
};

// Case k's vector src[k] into dst, element (i, k) at i*K + k. The host
// staging is written in order (each case's vector is read sequentially), and
// the copy from pageable memory returns once the staging has been taken, so
// the buffer may go at once (the copy stays ordered on the stream).
template <class T>
void upload_interleaved(cudaStream_t s, DevBuf<T>& dst, int32_t len, int K,
                        const std::vector<const std::vector<double>*>& src) {
  std::vector<T> h(static_cast<size_t>(len) * K);
  std::vector<const double*> col(K);
  for (int k = 0; k < K; ++k) col[k] = src[k]->data();
  T* out = h.data();
  for (int32_t i = 0; i < len; ++i)
    for (int k = 0; k < K; ++k) *out++ = static_cast<T>(col[k][i]);
  dst.alloc(std::max<size_t>(h.size(), 1));
  if (!h.empty())
    ANU_CUDA(cudaMemcpyAsync(dst.p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s));
}

template <class T>
void download_case(cudaStream_t s, const DevBuf<T>& src, int32_t len, int K, int k,
                   std::vector<double>* out, std::vector<T>* staging) {
  staging->resize(static_cast<size_t>(len) * K);
  if (!staging->empty())
    ANU_CUDA(cudaMemcpyAsync(staging->data(), src.p, sizeof(T) * staging->size(),
                             cudaMemcpyDeviceToHost, s));
  ANU_CUDA(cudaStreamSynchronize(s));
  out->resize(len);
  for (int32_t i = 0; i < len; ++i) (*out)[i] = static_cast<double>((*staging)[static_cast<size_t>(i) * K + k]);
}

template <class T>
void download_all(cudaStream_t s, const DevBuf<T>& src, int32_t len, int K,
                  std::vector<std::vector<double>>* out) {
  std::vector<T> staging(static_cast<size_t>(len) * K);
  if (!staging.empty())
    ANU_CUDA(cudaMemcpyAsync(staging.data(), src.p, sizeof(T) * staging.size(),
                             cudaMemcpyDeviceToHost, s));
  ANU_CUDA(cudaStreamSynchronize(s));
  out->assign(K, std::vector<double>(len));
  for (int k = 0; k < K; ++k)
    for (int32_t i = 0; i < len; ++i)
      (*out)[k][i] = static_cast<double>(staging[static_cast<size_t>(i) * K + k]);
}

// A rolling case stack: the cases waiting for a slot and where the results
// of finished cases go. A slot whose case retires at a termination check is
// refilled there with the next waiting case (admission in place).
struct AdmissionQueue {
  std::vector<const CaseData*> pending;  // in admission order
  std::vector<int32_t> pending_index;    // their positions in the caller's list
  // Their warm starts (scaled space, as solve_pdhg takes them), null: cold.
  std::vector<const std::vector<double>*> pending_warm_x, pending_warm_y;
  size_t next = 0;
  std::vector<int32_t> slot_index;       // the caller's position of each slot's case, -1: none
  std::vector<CaseResult>* out = nullptr;  // results by the caller's position
  // Streaming stacks only. deliver: takes each result as its case retires,
  // in place of *out. refill: asked for more cases when `pending` is used up;
  // appends to it and returns false when it has none now.
  std::function<void(int32_t, CaseResult&)> deliver;
  std::function<bool(AdmissionQueue&)> refill;
  // Streaming stacks only: hands back a case whose slot has just been
  // refilled. Until then a retired slot still points at its case's vectors.
  std::function<void(const CaseData*)> release;
};

// One case's column of a case-interleaved device array (element (row, k) at
// row*K + k), written from host data.
template <class T>
void upload_slot(cudaStream_t s, T* dst, int32_t len, int K, int k, const std::vector<double>& src,
                 std::vector<std::vector<T>>* staging) {
  if (len == 0) return;
  staging->emplace_back(src.begin(), src.begin() + len);
  ANU_CUDA(cudaMemcpy2DAsync(dst + k, sizeof(T) * K, staging->back().data(), sizeof(T), sizeof(T),
                             len, cudaMemcpyHostToDevice, s));
}

// Keeps the cases `keep` (in that order) of a case-interleaved array of
// `len` rows and K cases, as an array of keep.size() cases. Unallocated
// arrays stay unallocated.
template <class T>
void keep_cases(cudaStream_t s, DevBuf<T>& buf, int32_t len, int K, const std::vector<int>& keep) {
  if (buf.p == nullptr || len <= 0) return;
  const int K2 = static_cast<int>(keep.size());
  DevBuf<T> kept(static_cast<size_t>(len) * K2);
  for (int j = 0; j < K2; ++j)
    ANU_CUDA(cudaMemcpy2DAsync(kept.p + j, sizeof(T) * K2, buf.p + keep[j], sizeof(T) * K,
                               sizeof(T), len, cudaMemcpyDeviceToDevice, s));
  buf = std::move(kept);
}

template <class T>
void zero_slot(cudaStream_t s, T* dst, int32_t len, int K, int k) {
  if (len == 0 || dst == nullptr) return;
  ANU_CUDA(cudaMemset2DAsync(dst + k, sizeof(T) * K, 0, sizeof(T), len, s));
}

template <class T>
void run_cases_t(Problem& p, const std::vector<const CaseData*>& cases,
                 const anu_pdhg_options& o, const std::vector<const std::vector<double>*>& warm_x,
                 const std::vector<const std::vector<double>*>& warm_y,
                 std::vector<CaseResult>* results, double start_time, bool unit,
                 const std::vector<double>* init_eta = nullptr,
                 const std::vector<double>* init_omega = nullptr,
                 AdmissionQueue* queue = nullptr);

// Feasibility polishing of a set of cases (pdhg.cpp:666-751): a primal
// sub-stack (c = 0) warm started from the seeds' x, then a dual sub-stack
// (q = 0, finite bounds = 0) from the seeds' y, both on the same device
// matrix with unit scaling and the parent's ||K~||, step and weight.
template <class T>
void run_polish(Problem& p, bool unit, const std::vector<const CaseData*>& parent,
                const std::vector<int>& which, const std::vector<std::vector<double>>& seed_x,
                const std::vector<std::vector<double>>& seed_y, int32_t budget,
                const std::vector<CaseState>& states, const anu_pdhg_options& o,
                double start_time, std::vector<std::vector<double>>* out_xs,
                std::vector<std::vector<double>>* out_ys,
                std::vector<std::vector<double>>* out_x, std::vector<std::vector<double>>* out_y,
                std::vector<anu_pdhg_residual>* out_r, std::vector<int32_t>* spent) {
  const size_t W = which.size();
  std::vector<CaseData> primal(W), dual(W);
  for (size_t w = 0; w < W; ++w) {
    const CaseData& src = *parent[which[w]];
    CaseData& a = primal[w];
    a.c.assign(p.n, 0.0);
    a.q = src.qs;
    a.lower = src.ls;
    a.upper = src.us;
    a.objective_scale = src.objective_scale;
    a.objective_offset = 0.0;
    a.cs = a.c;
    a.qs = a.q;
    a.ls = a.lower;
    a.us = a.upper;
    CaseData& b = dual[w];
    b.c = src.cs;
    b.q.assign(p.m, 0.0);
    b.lower = src.ls;
    b.upper = src.us;
    for (int32_t j = 0; j < p.n; ++j) {
      if (b.lower[j] > -kInf) b.lower[j] = 0.0;
      if (b.upper[j] < kInf) b.upper[j] = 0.0;
    }
    b.objective_scale = src.objective_scale;
    b.objective_offset = 0.0;
    b.cs = b.c;
    b.qs = b.q;
    b.ls = b.lower;
    b.us = b.upper;
  }
  anu_pdhg_options sub = o;
  sub.polish_feasibility = 0;
  sub.polish_on_exit = 0;
  sub.detect_infeasibility = 0;
  sub.verbose = 0;
  sub.known_matrix_norm = p.matrix_norm;
  sub.ruiz_iterations = 0;
  sub.pock_chambolle = 0;
  sub.max_iterations = budget;
  sub.termination_check_frequency =
      std::max<int32_t>(10, std::min(o.termination_check_frequency, budget / 4));
  sub.time_limit_seconds = std::fmax(0.0, o.time_limit_seconds - (now_seconds() - start_time));
  // One sub-stack per side for every polishing case, each case started from
  // its parent's step size and primal weight (pdhg.cpp:703-704).
  std::vector<const CaseData*> pp(W), dd(W);
  std::vector<std::vector<double>> zx(W, std::vector<double>(p.n, 0.0)),
      zy(W, std::vector<double>(p.m, 0.0));
  std::vector<const std::vector<double>*> wx(W), wy(W), wx2(W), wy2(W);
  std::vector<double> etas(W), omegas(W);
  for (size_t w = 0; w < W; ++w) {
    pp[w] = &primal[w];
    dd[w] = &dual[w];
    wx[w] = &seed_x[w];
    wy[w] = &zy[w];
    wx2[w] = &zx[w];
    wy2[w] = &seed_y[w];
    etas[w] = states[which[w]].eta;
    omegas[w] = states[which[w]].omega;
  }
  std::vector<CaseResult> pres, dres;
  sub.termination = ANU_TERMINATION_PRIMAL_FEASIBILITY;
  run_cases_t<T>(p, pp, sub, wx, wy, &pres, now_seconds(), true, &etas, &omegas);
  sub.termination = ANU_TERMINATION_DUAL_FEASIBILITY;
  run_cases_t<T>(p, dd, sub, wx2, wy2, &dres, now_seconds(), true, &etas, &omegas);
  out_xs->assign(W, {});
  out_ys->assign(W, {});
  out_x->assign(W, {});
  out_y->assign(W, {});
  spent->assign(W, 0);
  std::vector<const CaseData*> evc(W);
  for (size_t w = 0; w < W; ++w) {
    (*spent)[w] = pres[w].r.iterations + dres[w].r.iterations;
    (*out_xs)[w] = pres[w].x;  // unit-scaled sub-solve: its x is the scaled iterate
    (*out_ys)[w] = dres[w].y;
    (*out_x)[w].resize(p.n);
    (*out_y)[w].resize(p.m);
    for (int32_t j = 0; j < p.n; ++j)
      (*out_x)[w][j] = unit ? pres[w].x[j] : p.scaling.col_scale[j] * pres[w].x[j];
    for (int32_t i = 0; i < p.m; ++i)
      (*out_y)[w][i] = unit ? dres[w].y[i] : p.scaling.row_scale[i] * dres[w].y[i];
    evc[w] = parent[which[w]];
  }
  std::vector<double> terms;
  eval_points_terms(p, unit, static_cast<int>(W), evc, *out_xs, *out_ys, &terms);
  out_r->resize(W);
  for (size_t w = 0; w < W; ++w)
    (*out_r)[w] = residual_from_terms(&terms[w * kCheckTerms], &terms[w * kCheckTerms + kRowTerms],
                                      states[which[w]].scales);
}

// The cluster size cluster_chunk_kernel takes a single LP on `p` with, 0
// where it does not take it: options.cluster_chunks off, a packed batch's
// LP, a row longer than kLongRow, or y and x_bar too large for one CTA's
// shared memory.
template <class T>
int cluster_shape(Problem& p, const anu_pdhg_options& o) {
  if (!o.cluster_chunks || p.concurrent || p.m == 0 || p.n == 0) return 0;
  p.dk.prepare_cluster(p.k, p.stream);
  p.dkt.prepare_cluster(p.kt, p.stream);
  if (p.dk.max_row > kLongRow || p.dkt.max_row > kLongRow) return 0;
  if (p.cluster_ctas < 0)
    p.cluster_ctas =
        cluster_ctas_for<T>(ClusterLayout::of<T>(p.m, p.n, p.dkt.cluster_rows(16),
                                                 p.dk.cluster_rows(16)).total,
                            ClusterLayout::of<T>(p.m, p.n, p.dkt.cluster_rows(8),
                                                 p.dk.cluster_rows(8)).total);
  return p.cluster_ctas;
}

template <class T>
void run_cases_t(Problem& p, const std::vector<const CaseData*>& initial_cases,
                 const anu_pdhg_options& o, const std::vector<const std::vector<double>*>& warm_x,
                 const std::vector<const std::vector<double>*>& warm_y,
                 std::vector<CaseResult>* results, double start_time, bool unit,
                 const std::vector<double>* init_eta, const std::vector<double>* init_omega,
                 AdmissionQueue* queue) {
  // The case in each slot; a rolling stack replaces retired ones.
  std::vector<const CaseData*> cases(initial_cases);
  // Slots of the stack; a stack whose last cases run on alone is compacted
  // to fewer slots (compact() below), so K can shrink during the run.
  int K = static_cast<int>(cases.size());
  const int32_t n = p.n, m = p.m;
  results->assign(K, CaseResult{});
  if (K == 0) return;
  if (K > kMaxCasesPerRun) throw Error(ANU_ERR_INVALID, "a case stack holds at most 64 cases per run");
  double phase_mark = now_seconds();
  auto phase_end = [&phase_mark]() {
    const double now = now_seconds();
    const double s = now - phase_mark;
    phase_mark = now;
    return s;
  };
  const int64_t launches0 = p.launches;
  std::vector<CaseState> S(K);
  for (int k = 0; k < K; ++k) {
    S[k].scales = {host_norm2(cases[k]->q), host_norm2(cases[k]->c), host_norminf(cases[k]->q),
                   host_norminf(cases[k]->c)};
    S[k].next_polish_iteration = o.polish_first_iteration;
  }
  // The stack iteration at which each slot's case started (0 unless admitted
  // into a rolling stack); a case's own iteration count is measured from it.
  std::vector<int32_t> origin(K, 0);
  const double tolerance = o.tolerance;
  const double gap_tolerance = o.gap_tolerance > 0.0 ? o.gap_tolerance : tolerance;
  const bool inf_norm = o.require_inf_norm_termination != 0;
  auto passes = [&](const anu_pdhg_residual& r) {
    switch (o.termination) {
      case ANU_TERMINATION_PRIMAL_FEASIBILITY:
        return primal_ok(r, tolerance, o.absolute_tolerance, inf_norm);
      case ANU_TERMINATION_DUAL_FEASIBILITY:
        return dual_ok(r, tolerance, o.absolute_tolerance, inf_norm);
      default:
        return converged(r, tolerance, o.absolute_tolerance, inf_norm, gap_tolerance);
    }
  };

  // No constraint matrix content (pdhg.cpp:428-457): componentwise answer.
  if (p.matrix_norm <= 0.0) {
    std::vector<std::vector<double>> xs(K), ys(K);
    for (int k = 0; k < K; ++k) {
      const CaseData& cd = *cases[k];
      xs[k].assign(n, 0.0);
      ys[k].assign(m, 0.0);
      for (int32_t j = 0; j < n; ++j) {
        const double lo = cd.lower[j], hi = cd.upper[j], cj = cd.c[j];
        double v = 0.0;
        if (cj > 0.0) v = lo;
        else if (cj < 0.0) v = hi;
        else v = std::isfinite(lo) ? lo : (std::isfinite(hi) ? hi : 0.0);
        xs[k][j] = std::isfinite(v) ? v : 0.0;
      }
    }
    std::vector<std::vector<double>> sx = xs;
    if (!unit)
      for (int k = 0; k < K; ++k)
        for (int32_t j = 0; j < n; ++j) sx[k][j] = xs[k][j] / p.scaling.col_scale[j];
    std::vector<double> terms;
    eval_points_terms(p, unit, K, cases, sx, ys, &terms);
    for (int k = 0; k < K; ++k) {
      CaseResult& R = (*results)[k];
      R.r.residual = residual_from_terms(&terms[k * kCheckTerms], &terms[k * kCheckTerms + kRowTerms],
                                         S[k].scales);
      R.x = xs[k];
      R.y = ys[k];
      R.xs = sx[k];
      R.ys = ys[k];
      double cx = 0.0;
      for (int32_t j = 0; j < n; ++j) cx += cases[k]->c[j] * xs[k][j];
      R.r.objective = cases[k]->objective_scale * cx + cases[k]->objective_offset;
      R.r.status = converged(R.r.residual, tolerance, o.absolute_tolerance, inf_norm, 0.0)
                       ? ANU_PDHG_OPTIMAL
                       : ANU_PDHG_NUMERICAL_ERROR;
      set_message(&R.r, "no constraint matrix content");
      R.r.matrix_norm_estimate = p.matrix_norm;
      R.r.solve_seconds = now_seconds() - start_time;
      R.r.kernel_launches = static_cast<int32_t>(p.launches - launches0);
    }
    return;
  }

  const bool halpern = o.halpern && o.restarts;
  const double reflection = halpern ? o.reflection : 0.0;
  const bool adaptive = o.adaptive_step_size && !o.constant_step_size;
  const bool slow = adaptive || o.halpern_restart;
  const bool averaging = o.restarts && !halpern;
  const bool need_kkt_any = (o.restarts && !halpern) || (o.restarts && !o.restart_on_fixed_point) ||
                            o.verbose;
  const bool fp64 = std::is_same<T, double>::value;
  const bool refine = !fp64 && o.refinement != 0;
  const bool polish_on = o.polish_feasibility != 0;
  if (slow && K != 1)
    throw Error(ANU_ERR_INVALID,
                "adaptive step sizes and the Halpern restart test need a single case");

  // Step size and primal weight (pdhg.cpp:460-479), per case.
  for (int k = 0; k < K; ++k) {
    double eta = 0.9 / p.matrix_norm;
    if (o.constant_step_size) eta = o.constant_step_scale / p.matrix_norm;
    double omega = 1.0;
    if (o.primal_weight_updates) {
      const double cn = host_norm2(cases[k]->cs);
      const double qn = host_norm2(cases[k]->qs);
      if (cn > 1e-12 && qn > 1e-12) omega = cn / qn;
    }
    if (o.initial_step_size > 0.0) eta = o.initial_step_size;
    if (o.initial_primal_weight > 0.0) omega = o.initial_primal_weight;
    // Polishing sub-stacks hand each case its parent's values.
    if (init_eta != nullptr && (*init_eta)[k] > 0.0) eta = (*init_eta)[k];
    if (init_omega != nullptr && (*init_omega)[k] > 0.0) omega = (*init_omega)[k];
    S[k].eta = eta;
    S[k].omega = omega;
  }

  // Starting points (pdhg.cpp:481-503).
  std::vector<std::vector<double>> x0(K), y0(K);
  for (int k = 0; k < K; ++k) {
    const CaseData& cd = *cases[k];
    const bool warm = k < static_cast<int>(warm_x.size()) && warm_x[k] != nullptr &&
                      warm_y[k] != nullptr && warm_x[k]->size() == static_cast<size_t>(n) &&
                      warm_y[k]->size() == static_cast<size_t>(m);
    x0[k].assign(n, 0.0);
    y0[k].assign(m, 0.0);
    if (warm) {
      x0[k] = *warm_x[k];
      y0[k] = *warm_y[k];
      for (int32_t i = p.num_eq; i < m; ++i)
        if (!(y0[k][i] > 0.0)) y0[k][i] = 0.0;
    }
    for (int32_t j = 0; j < n; ++j) {
      const double lo = cd.ls[j], hi = cd.us[j];
      double v = warm ? x0[k][j] : 0.0;
      if (!std::isfinite(v)) v = 0.0;
      if (v < lo) v = std::isfinite(lo) ? lo : 0.0;
      if (v > hi) v = std::isfinite(hi) ? hi : 0.0;
      x0[k][j] = v;
    }
  }

  // Device working set.
  Workspace<T> w;
  w.K = K;
  w.m = m;
  w.n = n;
  const cudaStream_t st = p.stream;
  std::vector<const std::vector<double>*> vx(K), vy(K), vc(K), vl(K), vu(K), vq(K), oc(K),
      ol(K), ou(K), oq(K), ylo(K);
  bool any_ylo = false;
  for (int k = 0; k < K; ++k) {
    vx[k] = &x0[k];
    vy[k] = &y0[k];
    vc[k] = &cases[k]->cs;
    vl[k] = &cases[k]->ls;
    vu[k] = &cases[k]->us;
    vq[k] = &cases[k]->qs;
    oc[k] = &cases[k]->c;
    ol[k] = &cases[k]->lower;
    ou[k] = &cases[k]->upper;
    oq[k] = &cases[k]->q;
    if (!cases[k]->ylo.empty()) any_ylo = true;
  }
  size_t NK = static_cast<size_t>(std::max(n, 1)) * K;
  size_t MK = static_cast<size_t>(std::max(m, 1)) * K;
  upload_interleaved(st, w.x, n, K, vx);
  upload_interleaved(st, w.y, m, K, vy);
  upload_interleaved(st, w.c, n, K, vc);
  upload_interleaved(st, w.lo, n, K, vl);
  upload_interleaved(st, w.hi, n, K, vu);
  upload_interleaved(st, w.q, m, K, vq);
  upload_interleaved(st, w.c0, n, K, oc);
  upload_interleaved(st, w.lo0, n, K, ol);
  upload_interleaved(st, w.hi0, n, K, ou);
  upload_interleaved(st, w.q0, m, K, oq);
  if (o.detect_infeasibility) {
    upload_interleaved(st, w.los, n, K, vl);
    upload_interleaved(st, w.his, n, K, vu);
    upload_interleaved(st, w.qs, m, K, vq);
    w.ktdy64.alloc(NK);
  }
  if (refine) any_ylo = true;
  if (any_ylo) {
    std::vector<std::vector<double>> zeros(K);
    for (int k = 0; k < K; ++k) {
      if (cases[k]->ylo.empty()) {
        zeros[k].assign(m, 0.0);
        ylo[k] = &zeros[k];
      } else {
        ylo[k] = &cases[k]->ylo;
      }
    }
    upload_interleaved(st, w.ylo, m, K, ylo);
  }
  w.x_bar.alloc(NK);
  w.anchor_x.alloc(NK);
  w.dx.alloc(NK);
  w.kx.alloc(MK);
  w.anchor_y.alloc(MK);
  w.anchor_kx.alloc(MK);
  w.dy.alloc(MK);
  ANU_CUDA(cudaMemsetAsync(w.dx.p, 0, sizeof(T) * NK, st));
  ANU_CUDA(cudaMemsetAsync(w.dy.p, 0, sizeof(T) * MK, st));
  ANU_CUDA(cudaMemsetAsync(w.anchor_x.p, 0, sizeof(T) * NK, st));
  ANU_CUDA(cudaMemsetAsync(w.anchor_y.p, 0, sizeof(T) * MK, st));
  ANU_CUDA(cudaMemsetAsync(w.anchor_kx.p, 0, sizeof(T) * MK, st));
  w.x_restart.alloc(NK);
  w.y_restart.alloc(MK);
  ANU_CUDA(cudaMemcpyAsync(w.x_restart.p, w.x.p, sizeof(T) * NK, cudaMemcpyDeviceToDevice, st));
  ANU_CUDA(cudaMemcpyAsync(w.y_restart.p, w.y.p, sizeof(T) * MK, cudaMemcpyDeviceToDevice, st));
  if (!o.pid_primal_weight) {
    w.x_prev.alloc(NK);
    w.y_prev.alloc(MK);
    ANU_CUDA(cudaMemcpyAsync(w.x_prev.p, w.x.p, sizeof(T) * NK, cudaMemcpyDeviceToDevice, st));
    ANU_CUDA(cudaMemcpyAsync(w.y_prev.p, w.y.p, sizeof(T) * MK, cudaMemcpyDeviceToDevice, st));
  }
  if (slow) {
    w.x_next.alloc(NK);
    w.y_next.alloc(MK);
    w.k_next.alloc(MK);
    w.k_dx.alloc(MK);
    ANU_CUDA(cudaMemsetAsync(w.k_dx.p, 0, sizeof(T) * MK, st));
  }
  if (averaging) {
    w.sum_x.alloc(NK);
    w.sum_y.alloc(MK);
    w.avg_x.alloc(NK);
    w.avg_y.alloc(MK);
    ANU_CUDA(cudaMemsetAsync(w.sum_x.p, 0, sizeof(T) * NK, st));
    ANU_CUDA(cudaMemsetAsync(w.sum_y.p, 0, sizeof(T) * MK, st));
  }
  w.kty64.alloc(NK);
  w.kx64.alloc(MK);
  if (refine) {
    w.xb.alloc(NK);
    w.yb.alloc(MK);
    ANU_CUDA(cudaMemsetAsync(w.xb.p, 0, sizeof(double) * NK, st));
    ANU_CUDA(cudaMemsetAsync(w.yb.p, 0, sizeof(double) * MK, st));
    w.x_comb.alloc(NK);
    w.y_comb.alloc(MK);
    w.kshift.alloc(MK);
    w.sum_weight.alloc(K);
    upload_interleaved(st, w.c0s, n, K, vc);
    upload_interleaved(st, w.q0s, m, K, vq);
    upload_interleaved(st, w.l0s, n, K, vl);
    upload_interleaved(st, w.u0s, n, K, vu);
  }
  w.params.alloc(K);
  w.mask.alloc(K);
  w.terms.alloc(static_cast<size_t>(kCheckTerms) * K * 2);
  w.kkt.alloc(static_cast<size_t>(kKktTerms) * K * 2);
  w.weights.alloc(K);
  const int F = o.termination_check_frequency;
  w.w_table.alloc(static_cast<size_t>(std::max(F, 1)) * K);
  Pinned<StepParams> h_params(K);
  Pinned<double> h_w(static_cast<size_t>(std::max(F, 1)) * K);
  Pinned<double> h_terms(static_cast<size_t>(kCheckTerms) * K * 2);
  Pinned<double> h_kkt(static_cast<size_t>(kKktTerms) * K * 2);
  // Case masks go up through a ring of pinned staging slots, so a new mask
  // never waits for the copy of the previous one.
  constexpr int kMaskSlots = 4;
  Pinned<int32_t> h_mask(static_cast<size_t>(K) * kMaskSlots);
  int mask_slot = 0;
  Pinned<double> h_weights(K);


  // k_x = K~ x0 in FP64, rounded to T (pdhg.cpp:593).
  product<double, T, double>(p, p.dk, w.x.p, K, StoreEpi<double>{K, w.kx64.p});
  masked_copy<T, double>(p, m, K, nullptr, w.kx64.p, w.kx.p);

  // Weighted KKT terms of (x, y) on the scaled problem, for every case.
  auto kkt_terms = [&](const T* xv, const T* yv, double* out_dev) {
    product<double, T, double>(p, p.dk, xv, K, StoreEpi<double>{K, w.kx64.p});
    product<double, T, double>(p, p.dkt, yv, K, StoreEpi<double>{K, w.kty64.p});
    // The KKT error is measured on the scaled problem: scaled q, c, bounds.
    DevBuf<double>* qsc = &w.qs;
    DevBuf<double> tmpq, tmpc, tmpl, tmph;
    if (!o.detect_infeasibility) {
      upload_interleaved(st, tmpq, m, K, vq);
      upload_interleaved(st, tmpl, n, K, vl);
      upload_interleaved(st, tmph, n, K, vu);
      qsc = &tmpq;
    }
    upload_interleaved(st, tmpc, n, K, vc);
    RowKktTerms<T> rt{K, p.num_eq, w.kx64.p, yv, qsc->p};
    ColKktTerms<T> ct{K, w.kty64.p, xv, tmpc.p, o.detect_infeasibility ? w.los.p : tmpl.p,
                      o.detect_infeasibility ? w.his.p : tmph.p};
    reduce_terms(p, m, K, rt, w.partial, out_dev, kKktTerms, 0);
    reduce_terms(p, n, K, ct, w.partial, out_dev, kKktTerms, 2);
    ANU_CUDA(cudaStreamSynchronize(st));
  };

  if (o.restarts && !o.restart_on_fixed_point) {
    // pdhg.cpp:604 - the KKT error at the starting point.
    kkt_terms(w.x.p, w.y.p, w.kkt.p);
    // On the engine stream: a plain cudaMemcpy would not wait for it.
    ANU_CUDA(cudaMemcpyAsync(h_kkt.p, w.kkt.p, sizeof(double) * kKktTerms * K,
                             cudaMemcpyDeviceToHost, st));
    ANU_CUDA(cudaStreamSynchronize(st));
    for (int k = 0; k < K; ++k) S[k].kkt_at_restart = kkt_value(&h_kkt.p[k * kKktTerms], S[k].omega);
  }

  // Per-chunk parameter upload.
  auto upload_params = [&](int len) {
    for (int k = 0; k < K; ++k) {
      StepParams& P = h_params.p[k];
      P.tau = S[k].eta / S[k].omega;
      P.sigma = S[k].eta * S[k].omega;
      P.gamma = reflection;
      P.eta = S[k].eta;
      P.active = S[k].active ? 1 : 0;
      P.halpern = halpern ? 1 : 0;
      P.reset_pending = (halpern && S[k].anchor_needs_reset) ? 1 : 0;
      P.k_base = S[k].halpern_k;
      for (int it = 0; it < len; ++it) {
        double wv = 1.0;
        if (halpern) {
          const int32_t kk = P.reset_pending ? it - 1 : S[k].halpern_k + it;
          if (!(P.reset_pending && it == 0))
            wv = static_cast<double>(kk + 1) / static_cast<double>(kk + 2);
        }
        h_w.p[static_cast<size_t>(it) * K + k] = wv;
      }
    }
    ANU_CUDA(cudaMemcpyAsync(w.params.p, h_params.p, sizeof(StepParams) * K, cudaMemcpyHostToDevice, st));
    ANU_CUDA(cudaMemcpyAsync(w.w_table.p, h_w.p, sizeof(double) * len * K, cudaMemcpyHostToDevice, st));
  };

  const T* ylo_ptr = any_ylo ? w.ylo.p : nullptr;

  // One fast-path iteration (in place).
  auto launch_iteration = [&](int it, uint32_t flags) {
    PrimalEpi<T> pe{K, it, flags, w.params.p, w.w_table.p, w.x.p, w.x.p, w.c.p, w.lo.p, w.hi.p,
                    w.x_bar.p, w.anchor_x.p, w.dx.p, w.sum_x.p};
    product<T, T, T>(p, p.dkt, w.y.p, K, pe, true);
    DualEpi<T> de{K, it, flags, p.num_eq, w.params.p, w.w_table.p, w.y.p, w.y.p, w.q.p, w.kx.p,
                  w.kx.p, w.anchor_y.p, w.anchor_kx.p, w.dy.p, nullptr, w.sum_y.p, ylo_ptr};
    product<T, T, T>(p, p.dk, w.x_bar.p, K, de, true);
  };

  // Persistent chunks: one cooperative launch per chunk (chunk_kernel). At
  // most one runs per device at a time from this process: the lock is taken
  // before a launch and let go once the stream has been synchronised after
  // it, so two stacks never hold part of the device each while waiting for
  // the rest.
  const bool persistent = o.persistent_chunks != 0 && !slow && o.use_graphs &&
                          chunk_fits<T>(p.dkt, p.dk, K);
  // A single LP small enough runs each chunk as one cluster-resident launch
  // (cluster_chunk_kernel); so does a stack's last case once compacted.
  int cluster_c = (K == 1 && !persistent && !slow) ? cluster_shape<T>(p, o) : 0;
  DevBuf<uint32_t> sync_arrived;
  DevBuf<int32_t> sync_status;
  Pinned<int32_t> h_sync_status(persistent ? 1 : 0);
  std::unique_lock<std::mutex> coop_lock(cooperative_mutex(p.device), std::defer_lock);
  if (persistent) {
    sync_arrived.alloc(1);
    sync_status.alloc(1);
    ANU_CUDA(cudaMemsetAsync(sync_status.p, 0, sizeof(int32_t), st));
    h_sync_status.p[0] = 0;
  }
  // After a synchronisation of the stream: the chunks before it are done.
  auto chunks_done = [&]() {
    if (!persistent) return;
    if (coop_lock.owns_lock()) coop_lock.unlock();
    if (h_sync_status.p[0] != 0)
      throw Error(ANU_ERR_INTERNAL,
                  "chunk_kernel: a grid barrier wait gave up (the grid was not co-resident)");
  };

  // A polishing sub-stack, started from its parent's step sizes.
  const bool sub_run = init_eta != nullptr;

  // A refined check's products and reductions in two concurrent branches:
  // the row side on the engine stream, the column side (and the Farkas
  // product) on a second stream, joined before the terms are read back.
  // Each check kernel is latency-bound, so the branches overlap.
  struct CheckFork {
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, xcomb = nullptr, ycomb = nullptr, join = nullptr;
    ~CheckFork() {
      if (side) cudaStreamSynchronize(side);
      for (cudaEvent_t e : {fork, xcomb, ycomb, join})
        if (e) cudaEventDestroy(e);
      if (side) cudaStreamDestroy(side);
    }
  } fk;
  const bool fork_checks = refine && !sub_run && !slow && (K > 1 || !p.concurrent);
  if (fork_checks) {
    ANU_CUDA(cudaStreamCreateWithFlags(&fk.side, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&fk.fork, &fk.xcomb, &fk.ycomb, &fk.join})
      ANU_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  }
  // With profiling, a chunk is timed from just before its launch (after any
  // graph capture, which is host work) to its end.
  cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
  double device_iter_s = 0.0;
  int64_t device_iters = 0;
  if (o.profile) {
    ANU_CUDA(cudaEventCreate(&ev_begin));
    ANU_CUDA(cudaEventCreate(&ev_end));
  }
  struct EventGuard {
    cudaEvent_t a, b;
    ~EventGuard() {
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
    }
  } event_guard{ev_begin, ev_end};
  auto run_chunk_body = [&](int len, bool check_at_end) {
    const uint32_t base_flags = averaging ? kAccumulate : 0u;
    if (persistent) {
      if (!coop_lock.owns_lock()) coop_lock.lock();
      if (o.profile) ANU_CUDA(cudaEventRecord(ev_begin, st));
      PrimalEpi<T> pe{K, 0, 0u, w.params.p, w.w_table.p, w.x.p, w.x.p, w.c.p, w.lo.p, w.hi.p,
                      w.x_bar.p, w.anchor_x.p, w.dx.p, w.sum_x.p};
      DualEpi<T> de{K, 0, 0u, p.num_eq, w.params.p, w.w_table.p, w.y.p, w.y.p, w.q.p, w.kx.p,
                    w.kx.p, w.anchor_y.p, w.anchor_kx.p, w.dy.p, nullptr, w.sum_y.p, ylo_ptr};
      ANU_CUDA(cudaMemsetAsync(sync_arrived.p, 0, sizeof(uint32_t), st));
      launch_chunk<T>(p, p.dkt, p.dk, w.y.p, w.x_bar.p, K, len, base_flags,
                      base_flags | (check_at_end ? kWriteDelta : 0u), pe, de,
                      GridSync{sync_arrived.p, reinterpret_cast<int*>(sync_status.p)});
      ANU_CUDA(cudaMemcpyAsync(h_sync_status.p, sync_status.p, sizeof(int32_t),
                               cudaMemcpyDeviceToHost, st));
      return;
    }
    if (cluster_c > 0 && K == 1 && len <= kClusterMaxLen) {
      PrimalEpi<T> pe{K, 0, base_flags, w.params.p, w.w_table.p, w.x.p, w.x.p, w.c.p, w.lo.p,
                      w.hi.p, w.x_bar.p, w.anchor_x.p, w.dx.p, w.sum_x.p};
      DualEpi<T> de{K, 0, base_flags, p.num_eq, w.params.p, w.w_table.p, w.y.p, w.y.p, w.q.p,
                    w.kx.p, w.kx.p, w.anchor_y.p, w.anchor_kx.p, w.dy.p, nullptr, w.sum_y.p,
                    ylo_ptr};
      if (o.profile) ANU_CUDA(cudaEventRecord(ev_begin, st));
      launch_cluster_chunk<T>(p, cluster_c, p.dkt.view<T>(), p.dkt.cluster_rows(cluster_c),
                              p.dk.view<T>(), p.dk.cluster_rows(cluster_c), pe, de, len,
                              base_flags, base_flags | (check_at_end ? kWriteDelta : 0u));
      return;
    }
    if (o.use_graphs) {
      const auto key = std::make_pair(len, check_at_end ? 1 : 0);
      auto found = w.graphs.find(key);
      if (found == w.graphs.end()) {
        cudaGraph_t graph = nullptr;
        const int64_t before = p.launches;
        ANU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        for (int it = 0; it < len; ++it)
          launch_iteration(it, base_flags | ((check_at_end && it == len - 1) ? kWriteDelta : 0u));
        ANU_CUDA(cudaStreamEndCapture(st, &graph));
        cudaGraphExec_t exec = nullptr;
        ANU_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        cudaGraphDestroy(graph);
        p.launches = before;  // counted when launched
        found = w.graphs.emplace(key, exec).first;
      }
      if (o.profile) ANU_CUDA(cudaEventRecord(ev_begin, st));
      ANU_CUDA(cudaGraphLaunch(found->second, st));
      p.launches += 2 * len;
    } else {
      if (o.profile) ANU_CUDA(cudaEventRecord(ev_begin, st));
      for (int it = 0; it < len; ++it)
        launch_iteration(it, base_flags | ((check_at_end && it == len - 1) ? kWriteDelta : 0u));
    }
  };
  // With profiling, the chunk's events are read once the stream has passed
  // them (at the next read-back), so timing adds no wait of its own.
  int pending_timed = 0;
  // Only chunks at the stack's full width count: after tail compaction the
  // last case's single-LP chunks would mix another kernel into the mean.
  const int full_width = K;
  int pending_width = 0;
  auto collect_chunk_time = [&]() {
    if (!o.profile || pending_timed == 0) return;
    ANU_CUDA(cudaEventSynchronize(ev_end));
    float ms = 0.0f;
    ANU_CUDA(cudaEventElapsedTime(&ms, ev_begin, ev_end));
    if (pending_width == full_width) {
      device_iter_s += 1e-3 * ms;
      device_iters += pending_timed;
    }
    pending_timed = 0;
  };
  auto run_chunk = [&](int len, bool check_at_end) {
    collect_chunk_time();
    run_chunk_body(len, check_at_end);
    if (o.profile) {
      ANU_CUDA(cudaEventRecord(ev_end, st));
      pending_timed = len;
      pending_width = K;
    }
  };

  // Check reductions for every case at once. `xv`, `yv` is the point judged
  // (the iterate or its average); kx_maint the maintained K x when it may be
  // reused. Writes terms[case][18] at `out_dev`.
  auto check_terms = [&](const T* xv, const T* yv, const T* kx_maint, bool fresh_kx,
                         double* out_dev) {
    const double* rs = unit ? nullptr : p.row_scale.p;
    const double* cs = unit ? nullptr : p.col_scale.p;
    const T* yprev = o.pid_primal_weight ? nullptr : w.y_prev.p;
    const T* xprev = o.pid_primal_weight ? nullptr : w.x_prev.p;
    const double* qsc = o.detect_infeasibility ? w.qs.p : nullptr;
    const double* ktdy = o.detect_infeasibility ? w.ktdy64.p : nullptr;
    const double* los = o.detect_infeasibility ? w.los.p : nullptr;
    const double* his = o.detect_infeasibility ? w.his.p : nullptr;
    if (refine && fork_checks) {
      // The judged point is base + offset, in FP64.
      const int64_t tn = static_cast<int64_t>(n) * K, tm = static_cast<int64_t>(m) * K;
      RowCheckTerms<double, T, double> rt{K, p.num_eq, w.kx64.p, w.y_comb.p, yv, w.dy.p,
                                          w.y_restart.p, yprev, w.q0.p, qsc, rs};
      ColCheckTerms<double, T> ct{K, w.kty64.p, w.x_comb.p, xv, w.dx.p, w.x_restart.p, xprev,
                                  w.c0.p, w.lo0.p, w.hi0.p, cs, ktdy, los, his};
      Exec side;
      side.stream = fk.side;
      ANU_CUDA(cudaEventRecord(fk.fork, st));
      ANU_CUDA(cudaStreamWaitEvent(fk.side, fk.fork, 0));
      // Column side: y~ = yb + y, K'y~ and K'dy; its terms also need x~.
      combine_kernel<T><<<grid_for(tm, 256, 1184), 256, 0, fk.side>>>(tm, w.yb.p, yv, w.y_comb.p);
      ANU_CUDA(cudaGetLastError());
      ANU_CUDA(cudaEventRecord(fk.ycomb, fk.side));
      product<double, double, double>(side, p.dkt, w.y_comb.p, K, StoreEpi<double>{K, w.kty64.p});
      if (o.detect_infeasibility)
        product<double, T, double>(side, p.dkt, w.dy.p, K, StoreEpi<double>{K, w.ktdy64.p});
      // Row side: x~ = xb + x and K x~; its terms also need y~.
      combine_kernel<T><<<grid_for(tn, 256, 1184), 256, 0, st>>>(tn, w.xb.p, xv, w.x_comb.p);
      ANU_CUDA(cudaGetLastError());
      ANU_CUDA(cudaEventRecord(fk.xcomb, st));
      product<double, double, double>(p, p.dk, w.x_comb.p, K, StoreEpi<double>{K, w.kx64.p});
      ANU_CUDA(cudaStreamWaitEvent(fk.side, fk.xcomb, 0));
      reduce_terms(side, n, K, ct, w.partial2, out_dev, kCheckTerms, kRowTerms);
      ANU_CUDA(cudaEventRecord(fk.join, fk.side));
      ANU_CUDA(cudaStreamWaitEvent(st, fk.ycomb, 0));
      reduce_terms(p, m, K, rt, w.partial, out_dev, kCheckTerms, 0);
      ANU_CUDA(cudaStreamWaitEvent(st, fk.join, 0));
      p.launches += side.launches + 2;
      return;
    }
    if (o.detect_infeasibility)
      product<double, T, double>(p, p.dkt, w.dy.p, K, StoreEpi<double>{K, w.ktdy64.p});
    if (refine) {
      // The judged point is base + offset, in FP64.
      const int64_t tn = static_cast<int64_t>(n) * K, tm = static_cast<int64_t>(m) * K;
      combine_kernel<T><<<grid_for(tn, 256, 1184), 256, 0, st>>>(tn, w.xb.p, xv, w.x_comb.p);
      combine_kernel<T><<<grid_for(tm, 256, 1184), 256, 0, st>>>(tm, w.yb.p, yv, w.y_comb.p);
      ANU_CUDA(cudaGetLastError());
      p.launches += 2;
      product<double, double, double>(p, p.dk, w.x_comb.p, K, StoreEpi<double>{K, w.kx64.p});
      product<double, double, double>(p, p.dkt, w.y_comb.p, K, StoreEpi<double>{K, w.kty64.p});
      RowCheckTerms<double, T, double> rt{K, p.num_eq, w.kx64.p, w.y_comb.p, yv, w.dy.p,
                                          w.y_restart.p, yprev, w.q0.p, qsc, rs};
      ColCheckTerms<double, T> ct{K, w.kty64.p, w.x_comb.p, xv, w.dx.p, w.x_restart.p, xprev,
                                  w.c0.p, w.lo0.p, w.hi0.p, cs, ktdy, los, his};
      reduce_terms(p, m, K, rt, w.partial, out_dev, kCheckTerms, 0);
      reduce_terms(p, n, K, ct, w.partial, out_dev, kCheckTerms, kRowTerms);
      return;
    }
    product<double, T, double>(p, p.dkt, yv, K, StoreEpi<double>{K, w.kty64.p});
    if (fresh_kx) {
      product<double, T, double>(p, p.dk, xv, K, StoreEpi<double>{K, w.kx64.p});
      RowCheckTerms<T, T, double> rt{K, p.num_eq, w.kx64.p, yv, yv, w.dy.p, w.y_restart.p, yprev,
                                     w.q0.p, qsc, rs};
      reduce_terms(p, m, K, rt, w.partial, out_dev, kCheckTerms, 0);
    } else {
      RowCheckTerms<T, T, T> rt{K, p.num_eq, kx_maint, yv, yv, w.dy.p, w.y_restart.p, yprev,
                                w.q0.p, qsc, rs};
      reduce_terms(p, m, K, rt, w.partial, out_dev, kCheckTerms, 0);
    }
    ColCheckTerms<T, T> ct{K, w.kty64.p, xv, xv, w.dx.p, w.x_restart.p, xprev, w.c0.p, w.lo0.p,
                           w.hi0.p, cs, ktdy, los, his};
    reduce_terms(p, n, K, ct, w.partial, out_dev, kCheckTerms, kRowTerms);
  };

  // Runs `body`, device work on the stream over the workspace's fixed
  // buffers, as a CUDA graph from its second call on: the same kernels with
  // the same arguments at every check, so one graph launch replaces a dozen
  // kernel launches. The first call runs directly and sizes the reduction
  // scratch; a graph whose scratch has since been reallocated is captured
  // again. Not where the iterate buffers swap (the host-driven path), and not
  // in polishing sub-stacks, whose few checks would not repay the capture. A
  // single LP of a packed batch, where many host threads would capture and
  // instantiate graphs at once, launches its first kConcurrentDirect checks
  // directly: about half of a batch's LPs end before that, and only the
  // longer ones capture.
  auto replay = [&](typename Workspace<T>::Replay& r, auto&& body) {
    if (!o.use_graphs || slow || sub_run ||
        (K == 1 && p.concurrent && r.direct++ < kConcurrentDirect)) {
      body();
      return;
    }
    if (r.exec && (r.partial != w.partial.p || r.partial_n != w.partial.n ||
                   r.partial2 != w.partial2.p || r.partial2_n != w.partial2.n)) {
      cudaGraphExecDestroy(r.exec);
      r.exec = nullptr;
    }
    if (r.exec == nullptr) {
      if (++r.seen < 2) {
        body();
        return;
      }
      const int64_t before = p.launches;
      cudaGraph_t graph = nullptr;
      ANU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      body();
      ANU_CUDA(cudaStreamEndCapture(st, &graph));
      const cudaError_t ie = cudaGraphInstantiate(&r.exec, graph, 0);
      cudaGraphDestroy(graph);
      ANU_CUDA(ie);
      r.launches = p.launches - before;
      p.launches = before;
      r.partial = w.partial.p;
      r.partial_n = w.partial.n;
      r.partial2 = w.partial2.p;
      r.partial2_n = w.partial2.n;
    }
    ANU_CUDA(cudaGraphLaunch(r.exec, st));
    p.launches += r.launches;
  };

  auto set_mask = [&](const std::vector<int32_t>& mk) {
    // Wrapping around the ring, the slot about to be refilled may still feed
    // a copy: drain the stream first.
    mask_slot = (mask_slot + 1) % kMaskSlots;
    if (mask_slot == 0) ANU_CUDA(cudaStreamSynchronize(st));
    int32_t* h = h_mask.p + static_cast<size_t>(mask_slot) * K;
    for (int k = 0; k < K; ++k) h[k] = mk[k];
    ANU_CUDA(cudaMemcpyAsync(w.mask.p, h, sizeof(int32_t) * K, cudaMemcpyHostToDevice, st));
  };

  // Adopting the averaged candidate moves it on the device (pdhg.cpp:981-987).
  auto adopt = [&](const std::vector<int32_t>& mk) {
    bool any = false;
    for (int k = 0; k < K; ++k) any = any || mk[k];
    if (!any) return;
    set_mask(mk);
    masked_copy<T, T>(p, n, K, w.mask.p, w.avg_x.p, w.x.p);
    masked_copy<T, T>(p, m, K, w.mask.p, w.avg_y.p, w.y.p);
  };

  std::vector<CaseResult>* R_ptr = results;
  // The caller's slot of each current slot: results stay in the caller's
  // order when the stack is compacted.
  std::vector<int> orig(K);
  std::iota(orig.begin(), orig.end(), 0);
  // Refinement at a check: fold every active case's FP32 offset into its FP64
  // base and re-form the correction LP from the FP64 residual there.
  auto recenter = [&]() {
    if (!refine) return;
    std::vector<int32_t> mk(K, 0);
    bool any = false;
    for (int k = 0; k < K; ++k)
      if (S[k].active) {
        mk[k] = 1;
        any = true;
      }
    if (!any) return;
    set_mask(mk);
    if (averaging) {
      for (int k = 0; k < K; ++k) h_weights.p[k] = S[k].sum_weight;
      ANU_CUDA(cudaMemcpyAsync(w.sum_weight.p, h_weights.p, sizeof(double) * K, cudaMemcpyHostToDevice, st));
    }
    const bool det = o.detect_infeasibility != 0;
    const int64_t tn = static_cast<int64_t>(n) * K, tm = static_cast<int64_t>(m) * K;
    replay(w.recenter_replay, [&]() {
      ANU_CUDA(cudaMemsetAsync(w.x_comb.p, 0, sizeof(double) * NK, st));
      recenter_columns_kernel<T><<<grid_for(tn, 256, 1184), 256, 0, st>>>(
          tn, K, w.mask.p, w.l0s.p, w.u0s.p, w.xb.p, w.x.p, w.anchor_x.p, w.x_restart.p,
          o.pid_primal_weight ? nullptr : w.x_prev.p, averaging ? w.sum_x.p : nullptr,
          w.sum_weight.p, w.lo.p, w.hi.p, det ? w.los.p : nullptr, det ? w.his.p : nullptr,
          w.x_comb.p);
      ANU_CUDA(cudaGetLastError());
      product<double, double, double>(p, p.dk, w.x_comb.p, K, StoreEpi<double>{K, w.kshift.p});
      recenter_rows_kernel<T><<<grid_for(tm, 256, 1184), 256, 0, st>>>(
          tm, K, p.num_eq, w.mask.p, w.yb.p, w.y.p, w.anchor_y.p, w.y_restart.p,
          o.pid_primal_weight ? nullptr : w.y_prev.p, averaging ? w.sum_y.p : nullptr,
          w.sum_weight.p, w.ylo.p, w.kx.p, w.anchor_kx.p, w.kshift.p);
      ANU_CUDA(cudaGetLastError());
      product<double, double, double>(p, p.dk, w.xb.p, K, StoreEpi<double>{K, w.kx64.p});
      product<double, double, double>(p, p.dkt, w.yb.p, K, StoreEpi<double>{K, w.kty64.p});
      correction_data_kernel<T><<<grid_for(tn + tm, 256, 1184), 256, 0, st>>>(
          tn, tm, K, w.mask.p, w.c0s.p, w.kty64.p, w.c.p, w.q0s.p, w.kx64.p, w.q.p,
          det ? w.qs.p : nullptr);
      ANU_CUDA(cudaGetLastError());
      p.launches += 3;
    });
    for (int k = 0; k < K; ++k)
      if (mk[k]) ++R_ptr->at(orig[k]).r.refinement_rounds;
  };

  int32_t iteration = 0;
  std::vector<CaseResult>& R = *results;
  for (int k = 0; k < K; ++k) {
    R[orig[k]].r.matrix_norm_estimate = p.matrix_norm;
  }
  double t_setup = phase_end();
  double t_iter = 0.0, t_checks = 0.0, t_polish = 0.0;

  auto any_active = [&]() {
    for (int k = 0; k < K; ++k)
      if (S[k].active) return true;
    return false;
  };

  // Results (pdhg.cpp:1205-1285) of the cases in slots `ks`: the final
  // iterate (or the polished point), its FP64 residual, exit polishing, the
  // objective. A rolling stack hands them to the queue and frees the slots.
  auto finalize = [&](const std::vector<int>& ks) {
    if (ks.empty()) return;
    std::vector<std::vector<double>> fx, fy;
    download_all(st, w.x, n, K, &fx);
    download_all(st, w.y, m, K, &fy);
    if (refine) {
      // The answer is base + offset.
      std::vector<std::vector<double>> bx, by;
      download_all(st, w.xb, n, K, &bx);
      download_all(st, w.yb, m, K, &by);
      for (int k : ks) {
        for (int32_t j = 0; j < n; ++j) fx[k][j] += bx[k][j];
        for (int32_t i = 0; i < m; ++i) fy[k][i] += by[k][i];
      }
    }
    std::vector<double> fterms;
    {
      std::vector<const CaseData*> ec;
      std::vector<std::vector<double>> ex, ey;
      for (int k : ks) {
        ec.push_back(cases[k]);
        ex.push_back(fx[k]);
        ey.push_back(fy[k]);
      }
      eval_points_terms(p, unit, static_cast<int>(ks.size()), ec, ex, ey, &fterms);
    }
    std::vector<int> pos(K, -1);
    for (size_t i = 0; i < ks.size(); ++i) pos[ks[i]] = static_cast<int>(i);
    std::vector<int> exit_polish;
    for (int k : ks) {
      CaseState& c = S[k];
      CaseResult& cr = R[orig[k]];
      if (c.have_polished) {
        cr.x = c.polished_x;
        cr.y = c.polished_y;
        cr.r.residual = c.polished_residual;
        continue;
      }
      cr.xs = fx[k];
      cr.ys = fy[k];
      cr.x.resize(n);
      cr.y.resize(m);
      for (int32_t j = 0; j < n; ++j) cr.x[j] = unit ? fx[k][j] : p.scaling.col_scale[j] * fx[k][j];
      for (int32_t i = 0; i < m; ++i) cr.y[i] = unit ? fy[k][i] : p.scaling.row_scale[i] * fy[k][i];
      cr.r.residual = residual_from_terms(&fterms[static_cast<size_t>(pos[k]) * kCheckTerms],
                                          &fterms[static_cast<size_t>(pos[k]) * kCheckTerms + kRowTerms],
                                          c.scales);
      const bool worth = polish_on && o.polish_on_exit &&
                         o.termination == ANU_TERMINATION_FULL && c.status != ANU_PDHG_OPTIMAL &&
                         c.status != ANU_PDHG_PRIMAL_INFEASIBLE &&
                         c.status != ANU_PDHG_NUMERICAL_ERROR &&
                         std::isfinite(cr.r.residual.primal_residual) &&
                         std::isfinite(cr.r.residual.dual_residual) &&
                         now_seconds() - start_time < o.time_limit_seconds;
      if (worth && polish_budget(o, c.final_iteration) > 0) exit_polish.push_back(k);
    }
    // Exit polishing, one sub-stack per budget (cases that stopped at the
    // same iteration count share one).
    std::map<int32_t, std::vector<int>> exit_groups;
    for (int k : exit_polish) exit_groups[polish_budget(o, S[k].final_iteration)].push_back(k);
    for (const auto& group : exit_groups) {
      const std::vector<int>& exits = group.second;
      std::vector<std::vector<double>> sx, sy;
      for (int k : exits) {
        sx.push_back(fx[k]);
        sy.push_back(fy[k]);
      }
      std::vector<std::vector<double>> pxs, pys, px, py;
      std::vector<anu_pdhg_residual> pr;
      std::vector<int32_t> spent;
      run_polish<T>(p, unit, cases, exits, sx, sy, group.first, S, o, start_time, &pxs, &pys, &px,
                    &py, &pr, &spent);
      t_polish += phase_end();
      for (size_t i = 0; i < exits.size(); ++i) {
        const int k = exits[i];
        CaseResult& cr = R[orig[k]];
        ++cr.r.polish_attempts;
        cr.r.polish_iterations += spent[i];
        const anu_pdhg_residual& cur = cr.r.residual;
        const anu_pdhg_residual& tr = pr[i];
        const double gap_ceiling = std::fmax(gap_tolerance, cur.relative_gap);
        const bool improved = tr.relative_primal <= cur.relative_primal &&
                              tr.relative_dual <= cur.relative_dual &&
                              (tr.relative_primal < cur.relative_primal ||
                               tr.relative_dual < cur.relative_dual);
        if (improved && tr.relative_gap <= gap_ceiling) {
          cr.x = px[i];
          cr.y = py[i];
          cr.xs = pxs[i];
          cr.ys = pys[i];
          cr.r.residual = tr;
          cr.r.polished = 1;
          if (converged(tr, tolerance, o.absolute_tolerance, inf_norm, gap_tolerance)) {
            S[k].status = ANU_PDHG_OPTIMAL;
            set_message(&cr.r, "converged after feasibility polishing");
          } else if (cr.r.message[0] == '\0') {
            set_message(&cr.r, "feasibility polished");
          } else {
            set_message(&cr.r, std::string(cr.r.message) + ", feasibility polished");
          }
        }
      }
    }
    t_checks += phase_end();
    for (int k : ks) {
      CaseResult& cr = R[orig[k]];
      double cx = 0.0;
      for (int32_t j = 0; j < n; ++j) cx += cases[k]->c[j] * cr.x[j];
      cr.r.objective = cases[k]->objective_scale * cx + cases[k]->objective_offset;
      cr.r.iterations = S[k].final_iteration;
      cr.r.status = S[k].status;
      cr.r.final_step_size = S[k].eta;
      cr.r.final_primal_weight = S[k].omega;
      cr.r.solve_seconds = now_seconds() - start_time;
      cr.r.phases.setup = t_setup;
      cr.r.phases.iterating = t_iter;
      cr.r.phases.checks = t_checks;
      cr.r.phases.polishing = t_polish;
      cr.r.kernel_launches = static_cast<int32_t>(p.launches - launches0);
      cr.r.device_iteration_seconds = device_iter_s;
      cr.r.device_iterations = device_iters;
      if (queue != nullptr) {
        if (queue->deliver) queue->deliver(queue->slot_index[k], cr);
        else (*queue->out)[queue->slot_index[k]] = std::move(cr);
        cr = CaseResult{};
        queue->slot_index[k] = -1;
      }
    }
  };

  // Admission of `d` (the caller's case `index`) into the free slot k of a
  // rolling stack, at a termination check: the slot's host state and every
  // case-interleaved device array start over as at the start of a solve.
  auto admit = [&](int k, int32_t index, const CaseData* d, const std::vector<double>* wx,
                   const std::vector<double>* wy) {
    const CaseData* outgoing = cases[k];
    cases[k] = d;
    queue->slot_index[k] = index;
    origin[k] = iteration;
    S[k] = CaseState{};
    S[k].scales = {host_norm2(d->q), host_norm2(d->c), host_norminf(d->q), host_norminf(d->c)};
    S[k].next_polish_iteration = o.polish_first_iteration;
    double eta = 0.9 / p.matrix_norm;
    if (o.constant_step_size) eta = o.constant_step_scale / p.matrix_norm;
    double omega = 1.0;
    if (o.primal_weight_updates) {
      const double cn = host_norm2(d->cs);
      const double qn = host_norm2(d->qs);
      if (cn > 1e-12 && qn > 1e-12) omega = cn / qn;
    }
    if (o.initial_step_size > 0.0) eta = o.initial_step_size;
    if (o.initial_primal_weight > 0.0) omega = o.initial_primal_weight;
    S[k].eta = eta;
    S[k].omega = omega;
    R[orig[k]] = CaseResult{};
    R[orig[k]].r.matrix_norm_estimate = p.matrix_norm;
    vc[k] = &d->cs;
    vl[k] = &d->ls;
    vu[k] = &d->us;
    vq[k] = &d->qs;
    oc[k] = &d->c;
    ol[k] = &d->lower;
    ou[k] = &d->upper;
    oq[k] = &d->q;
    // The starting point as at the start of a solve (pdhg.cpp:481-503).
    const bool warm = wx != nullptr && wy != nullptr && wx->size() == static_cast<size_t>(n) &&
                      wy->size() == static_cast<size_t>(m);
    std::vector<double> x0(n, 0.0), y0(m, 0.0);
    if (warm) {
      y0 = *wy;
      for (int32_t i = p.num_eq; i < m; ++i)
        if (!(y0[i] > 0.0)) y0[i] = 0.0;
    }
    for (int32_t j = 0; j < n; ++j) {
      double v = warm ? (*wx)[j] : 0.0;
      if (!std::isfinite(v)) v = 0.0;
      const double lo = d->ls[j], hi = d->us[j];
      if (v < lo) v = std::isfinite(lo) ? lo : 0.0;
      if (v > hi) v = std::isfinite(hi) ? hi : 0.0;
      x0[j] = v;
    }
    std::vector<std::vector<T>> staged;
    std::vector<std::vector<double>> staged64;
    upload_slot<T>(st, w.x.p, n, K, k, x0, &staged);
    upload_slot<T>(st, w.y.p, m, K, k, y0, &staged);
    upload_slot<T>(st, w.c.p, n, K, k, d->cs, &staged);
    upload_slot<T>(st, w.lo.p, n, K, k, d->ls, &staged);
    upload_slot<T>(st, w.hi.p, n, K, k, d->us, &staged);
    upload_slot<T>(st, w.q.p, m, K, k, d->qs, &staged);
    upload_slot<double>(st, w.c0.p, n, K, k, d->c, &staged64);
    upload_slot<double>(st, w.lo0.p, n, K, k, d->lower, &staged64);
    upload_slot<double>(st, w.hi0.p, n, K, k, d->upper, &staged64);
    upload_slot<double>(st, w.q0.p, m, K, k, d->q, &staged64);
    if (o.detect_infeasibility) {
      upload_slot<double>(st, w.los.p, n, K, k, d->ls, &staged64);
      upload_slot<double>(st, w.his.p, n, K, k, d->us, &staged64);
      upload_slot<double>(st, w.qs.p, m, K, k, d->qs, &staged64);
    }
    zero_slot<T>(st, w.ylo.p, m, K, k);
    zero_slot<T>(st, w.anchor_x.p, n, K, k);
    zero_slot<T>(st, w.anchor_y.p, m, K, k);
    zero_slot<T>(st, w.anchor_kx.p, m, K, k);
    zero_slot<T>(st, w.dx.p, n, K, k);
    zero_slot<T>(st, w.dy.p, m, K, k);
    upload_slot<T>(st, w.x_restart.p, n, K, k, x0, &staged);
    upload_slot<T>(st, w.y_restart.p, m, K, k, y0, &staged);
    if (!o.pid_primal_weight) {
      upload_slot<T>(st, w.x_prev.p, n, K, k, x0, &staged);
      upload_slot<T>(st, w.y_prev.p, m, K, k, y0, &staged);
    }
    zero_slot<T>(st, w.sum_x.p, n, K, k);
    zero_slot<T>(st, w.sum_y.p, m, K, k);
    if (refine) {
      zero_slot<double>(st, w.xb.p, n, K, k);
      zero_slot<double>(st, w.yb.p, m, K, k);
      upload_slot<double>(st, w.c0s.p, n, K, k, d->cs, &staged64);
      upload_slot<double>(st, w.q0s.p, m, K, k, d->qs, &staged64);
      upload_slot<double>(st, w.l0s.p, n, K, k, d->ls, &staged64);
      upload_slot<double>(st, w.u0s.p, n, K, k, d->us, &staged64);
    }
    // K x0 for this slot alone (pdhg.cpp:593).
    product<double, T, double>(p, p.dk, w.x.p, K, StoreEpi<double>{K, w.kx64.p});
    std::vector<int32_t> only(K, 0);
    only[k] = 1;
    set_mask(only);
    masked_copy<T, double>(p, m, K, w.mask.p, w.kx64.p, w.kx.p);
    if (o.restarts && !o.restart_on_fixed_point) {
      kkt_terms(w.x.p, w.y.p, w.kkt.p);
      ANU_CUDA(cudaMemcpyAsync(h_kkt.p, w.kkt.p, sizeof(double) * kKktTerms * K,
                               cudaMemcpyDeviceToHost, st));
      ANU_CUDA(cudaStreamSynchronize(st));
      S[k].kkt_at_restart = kkt_value(&h_kkt.p[static_cast<size_t>(k) * kKktTerms], S[k].omega);
    }
    // The staged host columns stay alive until the copies are done.
    ANU_CUDA(cudaStreamSynchronize(st));
    // Nothing in this run points at the outgoing case any more.
    if (queue->release && outgoing != nullptr && outgoing != d) queue->release(outgoing);
  };

  // The lockstep tail. A stack's cases retire at different iterations, and
  // its last case often runs on alone for half of the stack's time while the
  // launches still carry every slot. When a single case is left, the retired
  // cases are finalized and every per-case array is compacted to that case,
  // which then runs the single-LP kernels. Its state moves with it unchanged.
  // Only a single case gains: the stack kernel's lane groups narrow with the
  // case count, and a few cases walk each segment in more dependent rounds
  // than many do. FP32 stacks of at least kTailStack cases only: FP64 stacks
  // stay in their layout, whose results equal separate solves bit for bit.
  // Not for rolling stacks (their slots take new cases) or polishing
  // sub-stacks.
  constexpr int kTailStack = 8;
  const bool compact_tail = !fp64 && queue == nullptr && !persistent && !slow && !sub_run &&
                            K >= kTailStack;
  auto compact = [&]() {
    std::vector<int> keep, drop;
    for (int k = 0; k < K; ++k) (S[k].active ? keep : drop).push_back(k);
    finalize(drop);
    const int K2 = static_cast<int>(keep.size());
    for (DevBuf<T>* b : {&w.x, &w.x_bar, &w.anchor_x, &w.dx, &w.c, &w.lo, &w.hi, &w.x_next,
                         &w.sum_x, &w.avg_x, &w.x_restart, &w.x_prev})
      keep_cases(st, *b, n, K, keep);
    for (DevBuf<T>* b : {&w.y, &w.kx, &w.anchor_y, &w.anchor_kx, &w.dy, &w.q, &w.k_dx, &w.y_next,
                         &w.k_next, &w.sum_y, &w.avg_y, &w.y_restart, &w.y_prev, &w.ylo})
      keep_cases(st, *b, m, K, keep);
    for (DevBuf<double>* b : {&w.kty64, &w.ktdy64, &w.c0, &w.lo0, &w.hi0, &w.los, &w.his, &w.xb,
                              &w.x_comb, &w.c0s, &w.l0s, &w.u0s})
      keep_cases(st, *b, n, K, keep);
    for (DevBuf<double>* b : {&w.kx64, &w.q0, &w.qs, &w.yb, &w.y_comb, &w.q0s, &w.kshift})
      keep_cases(st, *b, m, K, keep);
    keep_cases(st, w.sum_weight, 1, K, keep);
    auto pick = [&](auto& v) {
      std::remove_reference_t<decltype(v)> kept;
      for (int k : keep) kept.push_back(std::move(v[k]));
      v = std::move(kept);
    };
    pick(S);
    pick(origin);
    pick(cases);
    pick(orig);
    for (auto* v : {&vx, &vy, &vc, &vl, &vu, &vq, &oc, &ol, &ou, &oq}) pick(*v);
    K = K2;
    w.K = K2;
    if (K == 1) cluster_c = cluster_shape<T>(p, o);
    NK = static_cast<size_t>(std::max(n, 1)) * K;
    MK = static_cast<size_t>(std::max(m, 1)) * K;
    ylo_ptr = any_ylo ? w.ylo.p : nullptr;
    // Graphs hold the old layout's pointers and widths.
    for (auto& g : w.graphs) cudaGraphExecDestroy(g.second);
    w.graphs.clear();
    for (auto* r : {&w.check_replay, &w.recenter_replay}) {
      if (r->exec) cudaGraphExecDestroy(r->exec);
      *r = typename Workspace<T>::Replay{};
    }
    ANU_CUDA(cudaStreamSynchronize(st));
  };

  while ((queue != nullptr || iteration < o.max_iterations) && any_active()) {
    int32_t last;
    bool is_check;
    int len;
    if (!slow) {
      const int32_t next_check = (iteration / F + 1) * F - 1;
      // A rolling stack checks every case's own limit at the checks.
      last = queue != nullptr ? next_check : std::min(next_check, o.max_iterations - 1);
      is_check = (last == next_check);
      len = last - iteration + 1;
      upload_params(len);
      run_chunk(len, is_check);
      for (int k = 0; k < K; ++k) {
        CaseState& c = S[k];
        if (!c.active) continue;
        c.iterations_since_restart += len;
        if (halpern) {
          if (c.anchor_needs_reset) {
            c.anchor_needs_reset = false;
            c.halpern_k = len - 1;
          } else {
            c.halpern_k += len;
          }
        }
        if (averaging)
          for (int i = 0; i < len; ++i) c.sum_weight += c.eta;
      }
    } else {
      // One iteration at a time, host-driven, as the reference does when the
      // step size adapts (pdhg.cpp:759-897). Single case.
      CaseState& c = S[0];
      last = iteration;
      len = 1;
      is_check = ((iteration + 1) % F == 0);
      const bool blend = halpern && !c.anchor_needs_reset;
      const double hw = blend ? static_cast<double>(c.halpern_k + 1) / static_cast<double>(c.halpern_k + 2) : 1.0;
      const bool need_movement = adaptive || o.halpern_restart || is_check;
      for (int attempt = 0;; ++attempt) {
        StepParams& P = h_params.p[0];
        P.tau = c.eta / c.omega;
        P.sigma = c.eta * c.omega;
        P.gamma = reflection;
        P.eta = c.eta;
        P.active = 1;
        P.halpern = blend ? 1 : 0;
        P.reset_pending = 0;
        P.k_base = 0;
        h_w.p[0] = hw;
        ANU_CUDA(cudaMemcpyAsync(w.params.p, h_params.p, sizeof(StepParams), cudaMemcpyHostToDevice, st));
        ANU_CUDA(cudaMemcpyAsync(w.w_table.p, h_w.p, sizeof(double), cudaMemcpyHostToDevice, st));
        PrimalEpi<T> pe{1, 0, kWriteDelta, w.params.p, w.w_table.p, w.x.p, w.x_next.p, w.c.p,
                        w.lo.p, w.hi.p, w.x_bar.p, w.anchor_x.p, w.dx.p, nullptr};
        product<T, T, T>(p, p.dkt, w.y.p, 1, pe);
        DualEpi<T> de{1, 0, kWriteDelta, p.num_eq, w.params.p, w.w_table.p, w.y.p, w.y_next.p,
                      w.q.p, w.kx.p, w.k_next.p, w.anchor_y.p, w.anchor_kx.p, w.dy.p, w.k_dx.p,
                      nullptr, ylo_ptr};
        product<T, T, T>(p, p.dk, w.x_bar.p, 1, de);
        double interaction = 0.0;
        if (!adaptive) {
          if (need_movement) {
            reduce_terms(p, n, 1, SquareTerms<T>{1, w.dx.p}, w.partial, w.kkt.p, 1, 0);
            reduce_terms(p, m, 1, SquareTerms<T>{1, w.dy.p}, w.partial, w.kkt.p + 1, 1, 0);
            ANU_CUDA(cudaMemcpyAsync(h_kkt.p, w.kkt.p, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
            ANU_CUDA(cudaStreamSynchronize(st));
            c.movement = c.omega * h_kkt.p[0] + h_kkt.p[1] / c.omega;
          }
          break;
        }
        reduce_terms(p, n, 1, SquareTerms<T>{1, w.dx.p}, w.partial, w.kkt.p, 1, 0);
        reduce_terms(p, m, 1, StepRowTerms<T>{w.dy.p, w.k_dx.p}, w.partial, w.kkt.p + 1, 2, 0);
        ANU_CUDA(cudaMemcpyAsync(h_kkt.p, w.kkt.p, sizeof(double) * 3, cudaMemcpyDeviceToHost, st));
        ANU_CUDA(cudaStreamSynchronize(st));
        interaction = std::fabs(h_kkt.p[1]);
        c.movement = c.omega * h_kkt.p[0] + h_kkt.p[2] / c.omega;
        double eta_bar = INFINITY;
        if (interaction > 0.0) eta_bar = c.movement / (2.0 * interaction);
        const double k1 = static_cast<double>(iteration + 1);
        double eta_next = c.eta;
        if (std::isfinite(eta_bar))
          eta_next = std::fmin((1.0 - std::pow(k1, -0.3)) * eta_bar, (1.0 + std::pow(k1, -0.6)) * c.eta);
        else
          eta_next = (1.0 + std::pow(k1, -0.6)) * c.eta;
        if (!(eta_next > 0.0) || !std::isfinite(eta_next)) eta_next = c.eta;
        const bool accept = (c.eta <= eta_bar);
        c.eta = eta_next;
        if (accept) break;
        if (attempt > 60) break;
      }
      std::swap(w.x, w.x_next);
      std::swap(w.y, w.y_next);
      std::swap(w.kx, w.k_next);
      ++c.iterations_since_restart;
      if (halpern) {
        if (c.anchor_needs_reset) {
          ANU_CUDA(cudaMemcpyAsync(w.anchor_x.p, w.x.p, sizeof(T) * n, cudaMemcpyDeviceToDevice, st));
          ANU_CUDA(cudaMemcpyAsync(w.anchor_y.p, w.y.p, sizeof(T) * m, cudaMemcpyDeviceToDevice, st));
          ANU_CUDA(cudaMemcpyAsync(w.anchor_kx.p, w.kx.p, sizeof(T) * m, cudaMemcpyDeviceToDevice, st));
          c.anchor_needs_reset = false;
          c.halpern_k = 0;
          c.epoch_start_movement = c.movement;
        } else {
          ++c.halpern_k;
        }
      }
      if (averaging) {
        accumulate_kernel<T><<<grid_for(n, 256, 296), 256, 0, st>>>(n, c.eta, w.x.p, w.sum_x.p);
        accumulate_kernel<T><<<grid_for(m, 256, 296), 256, 0, st>>>(m, c.eta, w.y.p, w.sum_y.p);
        ANU_CUDA(cudaGetLastError());
        p.launches += 2;
        c.sum_weight += c.eta;
      }
      if (halpern && o.halpern_restart && !c.anchor_needs_reset && c.epoch_start_movement > 0.0 &&
          c.halpern_k >= o.halpern_minimum_epoch) {
        if (c.movement <= c.epoch_start_movement / 7.389056098930650) {
          c.anchor_needs_reset = true;
          ++R[orig[0]].r.restarts;
        }
      }
    }
    iteration = last + 1;
    if (!is_check) continue;
    ANU_CUDA(cudaStreamSynchronize(st));
    chunks_done();
    t_iter += phase_end();

    // ------------------------------------------------------------- check
    const int32_t it_idx = last;
    std::vector<char> was_active(K);
    for (int k = 0; k < K; ++k) was_active[k] = S[k].active ? 1 : 0;
    bool any_avg = false;
    for (int k = 0; k < K; ++k) any_avg = any_avg || (S[k].active && averaging && S[k].sum_weight > 0.0);
    const bool fresh_kx = !fp64 || !o.reuse_products;
    replay(w.check_replay, [&]() { check_terms(w.x.p, w.y.p, w.kx.p, fresh_kx, w.terms.p); });
    const bool need_kkt = need_kkt_any;
    if (need_kkt) kkt_terms(w.x.p, w.y.p, w.kkt.p);
    if (any_avg) {
      for (int k = 0; k < K; ++k) h_weights.p[k] = S[k].sum_weight > 0.0 ? S[k].sum_weight : 1.0;
      ANU_CUDA(cudaMemcpyAsync(w.weights.p, h_weights.p, sizeof(double) * K, cudaMemcpyHostToDevice, st));
      average_kernel<T><<<grid_for(static_cast<int64_t>(n) * K, 256, 1184), 256, 0, st>>>(
          static_cast<int64_t>(n) * K, K, w.weights.p, w.sum_x.p, w.avg_x.p);
      average_kernel<T><<<grid_for(static_cast<int64_t>(m) * K, 256, 1184), 256, 0, st>>>(
          static_cast<int64_t>(m) * K, K, w.weights.p, w.sum_y.p, w.avg_y.p);
      ANU_CUDA(cudaGetLastError());
      p.launches += 2;
      kkt_terms(w.avg_x.p, w.avg_y.p, w.kkt.p + static_cast<size_t>(kKktTerms) * K);
      check_terms(w.avg_x.p, w.avg_y.p, nullptr, true, w.terms.p + static_cast<size_t>(kCheckTerms) * K);
    }
    ANU_CUDA(cudaMemcpyAsync(h_terms.p, w.terms.p, sizeof(double) * kCheckTerms * K * (any_avg ? 2 : 1),
                             cudaMemcpyDeviceToHost, st));
    if (need_kkt || any_avg)
      ANU_CUDA(cudaMemcpyAsync(h_kkt.p, w.kkt.p, sizeof(double) * kKktTerms * K * (any_avg ? 2 : 1),
                               cudaMemcpyDeviceToHost, st));
    ANU_CUDA(cudaStreamSynchronize(st));
    collect_chunk_time();

    std::vector<int32_t> adopt_mask(K, 0);
    std::vector<anu_pdhg_residual> rr(K);
    std::vector<double> candidate_kkt(K, 0.0);
    std::vector<int> polish_cases;
    for (int k = 0; k < K; ++k) {
      CaseState& c = S[k];
      if (!c.active) continue;
      const double* tc = &h_terms.p[static_cast<size_t>(k) * kCheckTerms];
      c.movement = c.omega * tc[kRowTerms + 4] + tc[3] / c.omega;
      if (o.detect_infeasibility) {
        const double scale = tc[6];
        const bool bad = tc[7] > 0.0 || tc[kRowTerms + 8] > 0.0 || !(scale > 0.0);
        if (!bad && (tc[8] - tc[kRowTerms + 7]) / scale > o.infeasibility_tolerance) {
          c.status = ANU_PDHG_PRIMAL_INFEASIBLE;
          set_message(&R[orig[k]].r, "Farkas certificate found in the dual iterate difference");
          c.final_iteration = it_idx + 1 - origin[k];
          c.active = false;
          continue;
        }
      }
      const bool need_average = averaging && c.sum_weight > 0.0;
      const double current_kkt = need_kkt ? kkt_value(&h_kkt.p[static_cast<size_t>(k) * kKktTerms], c.omega) : 0.0;
      c.use_average = false;
      candidate_kkt[k] = current_kkt;
      if (need_average) {
        const double average_kkt =
            kkt_value(&h_kkt.p[static_cast<size_t>(K + k) * kKktTerms], c.omega);
        if (average_kkt < current_kkt) {
          c.use_average = true;
          candidate_kkt[k] = average_kkt;
        }
      }
      const double* t = c.use_average ? &h_terms.p[static_cast<size_t>(K + k) * kCheckTerms] : tc;
      const anu_pdhg_residual r = residual_from_terms(t, t + kRowTerms, c.scales);
      rr[k] = r;
      if (!std::isfinite(r.primal_residual) || !std::isfinite(r.dual_residual)) {
        c.status = ANU_PDHG_NUMERICAL_ERROR;
        set_message(&R[orig[k]].r, "iterates stopped being finite");
        c.final_iteration = it_idx + 1 - origin[k];
        adopt_mask[k] = c.use_average;
        c.active = false;
        continue;
      }
      if (passes(r)) {
        c.status = ANU_PDHG_OPTIMAL;
        c.final_iteration = it_idx + 1 - origin[k];
        adopt_mask[k] = c.use_average;
        c.active = false;
        continue;
      }
      const int32_t done = it_idx + 1 - origin[k];
      if (polish_on && o.termination == ANU_TERMINATION_FULL &&
          done >= c.next_polish_iteration) {
        while (c.next_polish_iteration <= done) c.next_polish_iteration *= 2;
        const int32_t budget = polish_budget(o, done - 1);
        if (r.relative_gap <= gap_tolerance && budget > 0) polish_cases.push_back(k);
      }
    }
    adopt(adopt_mask);
    if (!polish_cases.empty()) {
      t_checks += phase_end();
      std::vector<std::vector<double>> cur_x, cur_y, avg_x, avg_y, bx, by;
      download_all(st, w.x, n, K, &cur_x);
      download_all(st, w.y, m, K, &cur_y);
      if (any_avg) {
        download_all(st, w.avg_x, n, K, &avg_x);
        download_all(st, w.avg_y, m, K, &avg_y);
      }
      if (refine) {
        // Seeds are points of the scaled LP: base + offset.
        download_all(st, w.xb, n, K, &bx);
        download_all(st, w.yb, m, K, &by);
        for (int k = 0; k < K; ++k) {
          for (int32_t j = 0; j < n; ++j) {
            cur_x[k][j] += bx[k][j];
            if (any_avg) avg_x[k][j] += bx[k][j];
          }
          for (int32_t i = 0; i < m; ++i) {
            cur_y[k][i] += by[k][i];
            if (any_avg) avg_y[k][i] += by[k][i];
          }
        }
      }
      // One primal and one dual sub-stack per budget (the cases of a stack
      // started together share one; a rolling stack's may differ).
      const size_t P = polish_cases.size();
      std::vector<std::vector<double>> pxs(P), pys(P), px(P), py(P);
      std::vector<anu_pdhg_residual> pr(P);
      std::vector<int32_t> spent(P);
      std::map<int32_t, std::vector<size_t>> groups;
      for (size_t i = 0; i < P; ++i)
        groups[polish_budget(o, it_idx - origin[polish_cases[i]])].push_back(i);
      for (const auto& group : groups) {
        std::vector<int> which;
        std::vector<std::vector<double>> sx, sy;
        for (size_t i : group.second) {
          const int k = polish_cases[i];
          which.push_back(k);
          sx.push_back(S[k].use_average ? avg_x[k] : cur_x[k]);
          sy.push_back(S[k].use_average ? avg_y[k] : cur_y[k]);
        }
        std::vector<std::vector<double>> gxs, gys, gx, gy;
        std::vector<anu_pdhg_residual> gr;
        std::vector<int32_t> gs;
        run_polish<T>(p, unit, cases, which, sx, sy, group.first, S, o, start_time, &gxs, &gys,
                      &gx, &gy, &gr, &gs);
        for (size_t g = 0; g < group.second.size(); ++g) {
          const size_t i = group.second[g];
          pxs[i] = std::move(gxs[g]);
          pys[i] = std::move(gys[g]);
          px[i] = std::move(gx[g]);
          py[i] = std::move(gy[g]);
          pr[i] = gr[g];
          spent[i] = gs[g];
        }
      }
      t_polish += phase_end();
      for (size_t i = 0; i < polish_cases.size(); ++i) {
        const int k = polish_cases[i];
        CaseState& c = S[k];
        ++R[orig[k]].r.polish_attempts;
        R[orig[k]].r.polish_iterations += spent[i];
        if (converged(pr[i], tolerance, o.absolute_tolerance, inf_norm, gap_tolerance)) {
          c.polished_x = px[i];
          c.polished_y = py[i];
          R[orig[k]].xs = pxs[i];
          R[orig[k]].ys = pys[i];
          c.polished_residual = pr[i];
          c.have_polished = true;
          R[orig[k]].r.polished = 1;
          c.status = ANU_PDHG_OPTIMAL;
          set_message(&R[orig[k]].r, "converged after feasibility polishing");
          c.final_iteration = it_idx + 1 - origin[k];
          c.active = false;
        }
      }
    }
    for (int k = 0; k < K; ++k) {
      if (!S[k].active || !o.verbose || o.log_frequency <= 0) continue;
      if ((it_idx + 1) % o.log_frequency == 0)
        std::printf("  iter %7d  primal %.3e  dual %.3e  gap %.3e  kkt %.3e  eta %.3e  w %.3e\n",
                    it_idx + 1, rr[k].relative_primal, rr[k].relative_dual, rr[k].relative_gap,
                    candidate_kkt[k], S[k].eta, S[k].omega);
    }
    const bool out_of_time = now_seconds() - start_time > o.time_limit_seconds ||
                             (o.stop != nullptr && __atomic_load_n(o.stop, __ATOMIC_ACQUIRE) != 0);
    std::fill(adopt_mask.begin(), adopt_mask.end(), 0);
    if (out_of_time) {
      for (int k = 0; k < K; ++k) {
        if (!S[k].active) continue;
        S[k].status = ANU_PDHG_TIME_LIMIT;
        S[k].final_iteration = it_idx + 1 - origin[k];
        adopt_mask[k] = S[k].use_average;
        S[k].active = false;
      }
      adopt(adopt_mask);
      t_checks += phase_end();
      break;
    }
    std::vector<int32_t> restart_mask(K, 0);
    bool any_restart = false;
    for (int k = 0; k < K && o.restarts; ++k) {
      CaseState& c = S[k];
      if (!c.active) continue;
      const double residual = std::sqrt(std::fmax(c.movement, 0.0));
      const bool by_residual = o.restart_on_fixed_point != 0;
      if (by_residual && !std::isfinite(c.residual_at_restart)) c.residual_at_restart = residual;
      const double measure = by_residual ? residual : candidate_kkt[k];
      const double at_restart = by_residual ? c.residual_at_restart : c.kkt_at_restart;
      const double previous = by_residual ? c.last_residual : c.last_candidate_kkt;
      const bool sufficient = measure <= 0.2 * at_restart;
      const bool necessary = measure <= 0.8 * at_restart && measure > previous;
      const bool too_long = static_cast<double>(c.iterations_since_restart) >=
                            0.36 * static_cast<double>(it_idx + 1 - origin[k]);
      c.last_candidate_kkt = candidate_kkt[k];
      c.last_residual = residual;
      if (!(sufficient || necessary || too_long)) continue;
      restart_mask[k] = 1;
      adopt_mask[k] = c.use_average;
      any_restart = true;
    }
    if (any_restart) {
      adopt(adopt_mask);
      // Fresh K x for the restarting cases (pdhg.cpp:1125).
      product<double, T, double>(p, p.dk, w.x.p, K, StoreEpi<double>{K, w.kx64.p});
      set_mask(restart_mask);
      masked_copy<T, double>(p, m, K, w.mask.p, w.kx64.p, w.kx.p);
      for (int k = 0; k < K; ++k) {
        if (!restart_mask[k]) continue;
        CaseState& c = S[k];
        const double* t = c.use_average ? &h_terms.p[static_cast<size_t>(K + k) * kCheckTerms]
                                        : &h_terms.p[static_cast<size_t>(k) * kCheckTerms];
        if (o.primal_weight_updates && c.have_previous_restart) {
          const double dxs = o.pid_primal_weight ? t[kRowTerms + 5] : t[kRowTerms + 6];
          const double dys = o.pid_primal_weight ? t[4] : t[5];
          const double delta_x = std::sqrt(dxs);
          const double delta_y = std::sqrt(dys);
          if (delta_x > 1e-12 && delta_y > 1e-12) {
            double candidate = 0.0;
            if (o.pid_primal_weight) {
              const double e = std::log(c.omega * delta_x / delta_y);
              c.weight_error_sum += e;
              const double correction = o.primal_weight_kp * e + o.primal_weight_ki * c.weight_error_sum +
                                        o.primal_weight_kd * (e - c.weight_error_previous);
              c.weight_error_previous = e;
              candidate = std::exp(std::log(c.omega) - correction);
            } else {
              candidate = std::exp(0.5 * std::log(delta_y / delta_x) + 0.5 * std::log(c.omega));
            }
            if (std::isfinite(candidate) && candidate > 1e-12 && candidate < 1e12) c.omega = candidate;
          }
        }
        c.have_previous_restart = true;
        c.sum_weight = 0.0;
        c.anchor_needs_reset = true;
        c.iterations_since_restart = 0;
        c.last_candidate_kkt = INFINITY;
        c.last_residual = INFINITY;
        c.residual_at_restart = std::sqrt(std::fmax(c.movement, 0.0));
        if (!o.restart_on_fixed_point) {
          const double* kt = c.use_average ? &h_kkt.p[static_cast<size_t>(K + k) * kKktTerms]
                                           : &h_kkt.p[static_cast<size_t>(k) * kKktTerms];
          c.kkt_at_restart = kkt_value(kt, c.omega);
        }
        ++R[orig[k]].r.restarts;
      }
      if (!o.pid_primal_weight) {
        masked_copy<T, T>(p, n, K, w.mask.p, w.x_restart.p, w.x_prev.p);
        masked_copy<T, T>(p, m, K, w.mask.p, w.y_restart.p, w.y_prev.p);
      }
      masked_copy<T, T>(p, n, K, w.mask.p, w.x.p, w.x_restart.p);
      masked_copy<T, T>(p, m, K, w.mask.p, w.y.p, w.y_restart.p);
      if (averaging) {
        masked_fill<T>(p, n, K, w.mask.p, static_cast<T>(0), w.sum_x.p);
        masked_fill<T>(p, m, K, w.mask.p, static_cast<T>(0), w.sum_y.p);
      }
    }
    recenter();
    if (queue != nullptr) {
      // Every case's own iteration limit; then the slots freed at this check
      // hand their results over and take the next waiting cases.
      for (int k = 0; k < K; ++k)
        if (S[k].active && it_idx + 1 - origin[k] >= o.max_iterations) {
          S[k].status = ANU_PDHG_ITERATION_LIMIT;
          S[k].final_iteration = it_idx + 1 - origin[k];
          S[k].active = false;
        }
      std::vector<int> retired;
      for (int k = 0; k < K; ++k)
        if (was_active[k] && !S[k].active && queue->slot_index[k] >= 0) retired.push_back(k);
      if (!retired.empty()) {
        t_checks += phase_end();
        finalize(retired);
        for (int k : retired) {
          if (queue->next >= queue->pending.size() && !(queue->refill && queue->refill(*queue)))
            break;
          const size_t q = queue->next;
          admit(k, queue->pending_index[q], queue->pending[q],
                q < queue->pending_warm_x.size() ? queue->pending_warm_x[q] : nullptr,
                q < queue->pending_warm_y.size() ? queue->pending_warm_y[q] : nullptr);
          ++queue->next;
        }
      }
    }
    t_checks += phase_end();
    if (compact_tail) {
      int active = 0;
      for (int k = 0; k < K; ++k) active += S[k].active ? 1 : 0;
      if (active == 1 && K > 1) {
        compact();
        t_checks += phase_end();
      }
    }
  }
  if (persistent) {
    ANU_CUDA(cudaStreamSynchronize(st));
    chunks_done();
  }
  for (int k = 0; k < K; ++k)
    if (S[k].active) {
      S[k].final_iteration = iteration - origin[k];
      S[k].status = ANU_PDHG_ITERATION_LIMIT;
    }

  collect_chunk_time();
  std::vector<int> remaining;
  for (int k = 0; k < K; ++k)
    if (queue == nullptr || queue->slot_index[k] >= 0) remaining.push_back(k);
  finalize(remaining);
}

}  // namespace

void evaluate_point(Problem& p, const CaseData& cd, const std::vector<double>& x,
                    const std::vector<double>& y, anu_pdhg_residual* out) {
  std::vector<std::vector<double>> xs(1, x), ys(1, y);
  std::vector<double> terms;
  eval_points_terms(p, true, 1, {&cd}, xs, ys, &terms);
  const ResidualScales s{host_norm2(cd.q), host_norm2(cd.c), host_norminf(cd.q),
                         host_norminf(cd.c)};
  *out = residual_from_terms(terms.data(), terms.data() + kRowTerms, s);
}

void run_cases(Problem& problem, const std::vector<const CaseData*>& cases,
               const anu_pdhg_options& options,
               const std::vector<const std::vector<double>*>& warm_x,
               const std::vector<const std::vector<double>*>& warm_y,
               std::vector<CaseResult>* results, double start_time) {
  ANU_CUDA(cudaSetDevice(problem.device));
  PoolScope scope(&problem.pool, problem.stream);
  if (problem.precision == ANU_PRECISION_FP32)
    run_cases_t<float>(problem, cases, options, warm_x, warm_y, results, start_time,
                       problem.unit_scaling);
  else
    run_cases_t<double>(problem, cases, options, warm_x, warm_y, results, start_time,
                        problem.unit_scaling);
}

void run_cases_rolling(Problem& problem, const std::vector<const CaseData*>& cases, int slots,
                       const anu_pdhg_options& options,
                       const std::vector<const std::vector<double>*>& warm_x,
                       const std::vector<const std::vector<double>*>& warm_y,
                       std::vector<CaseResult>* results, double start_time) {
  ANU_CUDA(cudaSetDevice(problem.device));
  PoolScope scope(&problem.pool, problem.stream);
  const int total = static_cast<int>(cases.size());
  const int K = std::max(1, std::min(slots, total));
  results->assign(total, CaseResult{});
  AdmissionQueue queue;
  queue.out = results;
  std::vector<const CaseData*> first(cases.begin(), cases.begin() + K);
  for (int k = 0; k < K; ++k) queue.slot_index.push_back(k);
  auto warm_of = [](const std::vector<const std::vector<double>*>& v, int i) {
    return i < static_cast<int>(v.size()) ? v[i] : nullptr;
  };
  std::vector<const std::vector<double>*> first_x(K), first_y(K);
  for (int k = 0; k < K; ++k) {
    first_x[k] = warm_of(warm_x, k);
    first_y[k] = warm_of(warm_y, k);
  }
  for (int i = K; i < total; ++i) {
    queue.pending.push_back(cases[i]);
    queue.pending_index.push_back(i);
    queue.pending_warm_x.push_back(warm_of(warm_x, i));
    queue.pending_warm_y.push_back(warm_of(warm_y, i));
  }
  std::vector<CaseResult> slot_results;
  if (problem.precision == ANU_PRECISION_FP32)
    run_cases_t<float>(problem, first, options, first_x, first_y, &slot_results, start_time,
                       problem.unit_scaling, nullptr, nullptr, &queue);
  else
    run_cases_t<double>(problem, first, options, first_x, first_y, &slot_results, start_time,
                        problem.unit_scaling, nullptr, nullptr, &queue);
  // Cases the time limit (or a stop request) kept from ever starting.
  for (size_t i = queue.next; i < queue.pending.size(); ++i) {
    CaseResult& r = (*results)[queue.pending_index[i]];
    r.r.status = ANU_PDHG_TIME_LIMIT;
    set_message(&r.r, "not started: the time limit ended the stack first");
    r.x.assign(problem.n, 0.0);
    r.y.assign(problem.m, 0.0);
    r.r.matrix_norm_estimate = problem.matrix_norm;
  }
}

void run_cases_streaming(Problem& problem, int slots, const anu_pdhg_options& options,
                         const std::function<const CaseData*(int32_t*)>& next_case,
                         const std::function<void(int32_t, CaseResult&)>& deliver,
                         const std::function<void(const CaseData*)>& release,
                         double start_time) {
  ANU_CUDA(cudaSetDevice(problem.device));
  PoolScope scope(&problem.pool, problem.stream);
  AdmissionQueue queue;
  std::vector<CaseResult> unused;
  queue.out = &unused;
  queue.deliver = deliver;
  queue.release = release;
  queue.refill = [&next_case](AdmissionQueue& q) {
    int32_t id = -1;
    const CaseData* d = next_case(&id);
    if (d == nullptr) return false;
    q.pending.push_back(d);
    q.pending_index.push_back(id);
    q.pending_warm_x.push_back(nullptr);
    q.pending_warm_y.push_back(nullptr);
    return true;
  };
  std::vector<const CaseData*> first;
  for (int k = 0; k < slots; ++k) {
    int32_t id = -1;
    const CaseData* d = next_case(&id);
    if (d == nullptr) break;
    first.push_back(d);
    queue.slot_index.push_back(id);
  }
  if (first.empty()) return;
  const std::vector<const std::vector<double>*> cold(first.size(), nullptr);
  std::vector<CaseResult> slot_results;
  if (problem.precision == ANU_PRECISION_FP32)
    run_cases_t<float>(problem, first, options, cold, cold, &slot_results, start_time,
                       problem.unit_scaling, nullptr, nullptr, &queue);
  else
    run_cases_t<double>(problem, first, options, cold, cold, &slot_results, start_time,
                        problem.unit_scaling, nullptr, nullptr, &queue);
  // Cases taken from the source that the time limit (or a stop request) kept
  // from ever starting.
  for (size_t i = queue.next; i < queue.pending.size(); ++i) {
    CaseResult r;
    r.r.status = ANU_PDHG_TIME_LIMIT;
    set_message(&r.r, "not started: the time limit ended the stack first");
    r.x.assign(problem.n, 0.0);
    r.y.assign(problem.m, 0.0);
    r.r.matrix_norm_estimate = problem.matrix_norm;
    deliver(queue.pending_index[i], r);
  }
}

}  // namespace anu

// =============================================================== C ABI

using anu::Error;

namespace {

template <class F>
int guarded(F&& body) {
  try {
    anu::clear_last_error();
    body();
    return ANU_OK;
  } catch (const Error& e) {
    anu::set_last_error(e.code, e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    anu::set_last_error(ANU_ERR_MEMORY, "host allocation failed");
    return ANU_ERR_MEMORY;
  } catch (const std::exception& e) {
    anu::set_last_error(ANU_ERR_INTERNAL, e.what());
    return ANU_ERR_INTERNAL;
  }
}

void fill_result(const anu::Problem& p, const anu::CaseResult& cr, double scaling_s, double norm_s,
                 anu_pdhg_result* out) {
  *out = cr.r;
  out->phases.scaling = scaling_s;
  out->phases.matrix_norm = norm_s;
  out->row_spread_before = p.scaling.row_spread_before;
  out->row_spread_after = p.scaling.row_spread_after;
  out->col_spread_before = p.scaling.col_spread_before;
  out->col_spread_after = p.scaling.col_spread_after;
  out->matrix_norm_estimate = p.matrix_norm;
  out->row_product_threads = p.dk.tile_threads;
  out->column_product_threads = p.dkt.tile_threads;
}

}  // namespace

struct anu_pdhg {
  std::unique_ptr<anu::Problem> problem;
  // Set when options.locality_order is on: the problem and its case data
  // are relabelled, and x, y and warm starts are mapped at the boundary.
  anu::Relabel relabel;
  anu::CaseData data;
  anu_pdhg_options options;
  double scaling_seconds = 0.0;
  double norm_seconds = 0.0;
  double trial_seconds = 0.0;  // the product tiles' trial solves
};

struct anu_pdhg_batch {
  std::unique_ptr<anu::Problem> problem;
  // The base LP's vectors: what a streamed case starts from.
  std::vector<double> base_c, base_q, base_lower, base_upper;
  double objective_scale = 1.0, objective_offset = 0.0;
  // A second problem on its own stream (same scaled matrix): larger stacks
  // run as two half-stacks at once, one per problem.
  std::unique_ptr<anu::Problem> twin;
  std::vector<anu::CaseData> cases;
  anu_pdhg_options options;
  double scaling_seconds = 0.0;
  double norm_seconds = 0.0;
};

extern "C" {

const char* anu_pdhg_version(void) { return "anu-pdhg-b200 0.1.0 sm_100a"; }

void anu_pdhg_default_options(anu_pdhg_options* o) {
  if (o == nullptr) return;
  std::memset(o, 0, sizeof(*o));
  o->tolerance = 1e-6;
  o->gap_tolerance = 0.0;
  o->max_iterations = 200000;
  o->time_limit_seconds = 300.0;
  o->termination_check_frequency = 40;
  o->absolute_tolerance = 0.0;
  o->require_inf_norm_termination = 1;
  o->adaptive_step_size = 1;
  o->primal_weight_updates = 1;
  o->restarts = 1;
  o->halpern = 1;
  o->halpern_restart = 0;
  o->halpern_minimum_epoch = 16;
  o->polish_feasibility = 1;
  o->polish_first_iteration = 100;
  o->polish_iteration_factor = 0.125;
  o->polish_minimum_iterations = 40;
  o->polish_maximum_iterations = 20000;
  o->polish_on_exit = 1;
  o->reflection = 1.0;
  o->constant_step_size = 1;
  o->constant_step_scale = 0.90;
  o->restart_on_fixed_point = 1;
  o->pid_primal_weight = 1;
  o->primal_weight_kp = 0.5;
  o->primal_weight_ki = 0.0;
  o->primal_weight_kd = 0.3;
  o->ruiz_iterations = 10;
  o->pock_chambolle = 1;
  o->reuse_products = 1;
  o->detect_infeasibility = 1;
  o->infeasibility_tolerance = 1e-8;
  o->termination = ANU_TERMINATION_FULL;
  o->known_matrix_norm = 0.0;
  o->initial_step_size = 0.0;
  o->initial_primal_weight = 0.0;
  o->verbose = 0;
  o->log_frequency = 5000;
  o->stop = nullptr;
  o->precision = ANU_PRECISION_FP64;
  o->refinement = 1;
  o->device = 0;
  o->use_graphs = 1;
  o->profile = 0;
  o->split_stacks = 1;
  o->persistent_chunks = 0;
  o->locality_order = 0;
  o->scaling_on_device = 1;
  o->tile_threads = 0;
  o->cluster_chunks = 0;
}

int anu_last_error(char* buf, int32_t size) { return anu::copy_last_error(buf, size); }

int64_t anu_release_cached_memory(void) {
  return static_cast<int64_t>(anu::release_cached_blocks());
}

int32_t anu_device_count(void) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return count;
}

int anu_pdhg_create(const anu_lp* lp, const anu_pdhg_options* options, anu_pdhg** handle) {
  return guarded([&] {
    if (lp == nullptr || options == nullptr || handle == nullptr)
      throw Error(ANU_ERR_INVALID, "null argument");
    *handle = nullptr;
    anu::validate_options(*options);
    const std::string e = anu::validate_lp(*lp);
    if (!e.empty()) throw Error(ANU_ERR_INVALID, "invalid LP: " + e);
    auto h = std::make_unique<anu_pdhg>();
    h->options = *options;
    if (options->locality_order != 0) h->relabel = anu::locality_relabel(*lp);
    h->problem = anu::make_problem(*lp, *options, &h->scaling_seconds, &h->norm_seconds,
                                   anu::kSegNnz, anu::kSegPerCta, &h->relabel);
    if (h->relabel.empty()) {
      h->data = anu::make_case(*h->problem, lp->c, lp->q, lp->lower, lp->upper,
                               lp->objective_scale, lp->objective_offset);
    } else {
      const anu::Relabel& r = h->relabel;
      const std::vector<double> c = anu::take(lp->c, r.col_old), q = anu::take(lp->q, r.row_old),
                                lo = anu::take(lp->lower, r.col_old),
                                up = anu::take(lp->upper, r.col_old);
      h->data = anu::make_case(*h->problem, c.data(), q.data(), lo.data(), up.data(),
                               lp->objective_scale, lp->objective_offset);
    }
    const double trial_start = anu::now_seconds();
    if (anu::choose_tiles(*h->problem, *options, &h->data))
      h->trial_seconds = anu::now_seconds() - trial_start;
    *handle = h.release();
  });
}

int anu_pdhg_run(anu_pdhg* h, const double* warm_x, const double* warm_y, double* x, double* y,
                 anu_pdhg_result* result) {
  return guarded([&] {
    if (h == nullptr || result == nullptr) throw Error(ANU_ERR_INVALID, "null argument");
    const double start = anu::now_seconds();
    std::vector<double> wx, wy;
    std::vector<const std::vector<double>*> vwx(1, nullptr), vwy(1, nullptr);
    const anu::Relabel& r = h->relabel;
    if (warm_x != nullptr && warm_y != nullptr) {
      if (r.empty()) {
        wx.assign(warm_x, warm_x + h->problem->n);
        wy.assign(warm_y, warm_y + h->problem->m);
      } else {
        wx = anu::take(warm_x, r.col_old);
        wy = anu::take(warm_y, r.row_old);
      }
      vwx[0] = &wx;
      vwy[0] = &wy;
    }
    std::vector<anu::CaseResult> res;
    anu::run_cases(*h->problem, {&h->data}, h->options, vwx, vwy, &res, start);
    fill_result(*h->problem, res[0], h->scaling_seconds, h->norm_seconds, result);
    result->tile_trial_seconds = h->trial_seconds;
    if (r.empty()) {
      if (x) std::copy(res[0].x.begin(), res[0].x.end(), x);
      if (y) std::copy(res[0].y.begin(), res[0].y.end(), y);
    } else {
      if (x)
        for (size_t j = 0; j < r.col_old.size(); ++j) x[r.col_old[j]] = res[0].x[j];
      if (y)
        for (size_t i = 0; i < r.row_old.size(); ++i) y[r.row_old[i]] = res[0].y[i];
    }
  });
}

int anu_pdhg_set_case(anu_pdhg* h, const double* c, const double* q, const double* lower,
                      const double* upper) {
  return guarded([&] {
    if (h == nullptr) throw Error(ANU_ERR_INVALID, "null argument");
    const anu::Problem& p = *h->problem;
    const anu::Relabel& r = h->relabel;
    // Each given vector in the problem's order; a NULL one keeps the case's.
    auto order = [&](const double* v, const std::vector<int32_t>& old, int32_t len,
                     const std::vector<double>& keep) {
      if (v == nullptr) return keep;
      if (r.empty()) return std::vector<double>(v, v + len);
      return anu::take(v, old);
    };
    const std::vector<double> cc = order(c, r.col_old, p.n, h->data.c);
    const std::vector<double> qq = order(q, r.row_old, p.m, h->data.q);
    const std::vector<double> lo = order(lower, r.col_old, p.n, h->data.lower);
    const std::vector<double> up = order(upper, r.col_old, p.n, h->data.upper);
    for (int32_t j = 0; j < p.n; ++j) {
      if (!std::isfinite(cc[j])) throw Error(ANU_ERR_INVALID, "objective is not finite");
      if (lo[j] > up[j] || std::isnan(lo[j]) || std::isnan(up[j]))
        throw Error(ANU_ERR_INVALID, "empty or NaN bound interval");
    }
    for (int32_t i = 0; i < p.m; ++i)
      if (!std::isfinite(qq[i])) throw Error(ANU_ERR_INVALID, "rhs is not finite");
    h->data = anu::make_case(p, cc.data(), qq.data(), lo.data(), up.data(),
                             h->data.objective_scale, h->data.objective_offset);
  });
}

void anu_pdhg_destroy(anu_pdhg* h) { delete h; }

int anu_pdhg_solve(const anu_lp* lp, const anu_pdhg_options* options, const double* warm_x,
                   const double* warm_y, double* x, double* y, anu_pdhg_result* result) {
  const double t0 = anu::now_seconds();
  anu_pdhg* h = nullptr;
  int rc = anu_pdhg_create(lp, options, &h);
  if (rc != ANU_OK) return rc;
  rc = anu_pdhg_run(h, warm_x, warm_y, x, y, result);
  if (rc == ANU_OK) result->solve_seconds = anu::now_seconds() - t0;
  anu_pdhg_destroy(h);
  return rc;
}

int anu_locality_relabel(const anu_lp* lp, int32_t* row_old, int32_t* col_old) {
  return guarded([&] {
    if (lp == nullptr || (lp->k.rows > 0 && row_old == nullptr) ||
        (lp->k.cols > 0 && col_old == nullptr))
      throw Error(ANU_ERR_INVALID, "null argument");
    const std::string e = anu::validate_csr(lp->k.rows, lp->k.cols, lp->k.nnz, lp->k.start,
                                            lp->k.index);
    if (!e.empty()) throw Error(ANU_ERR_INVALID, "invalid matrix: " + e);
    if (lp->num_equalities < 0 || lp->num_equalities > lp->k.rows)
      throw Error(ANU_ERR_INVALID, "num_equalities out of range");
    const anu::Relabel r = anu::locality_relabel(*lp);
    for (int32_t i = 0; i < lp->k.rows; ++i) row_old[i] = r.empty() ? i : r.row_old[i];
    for (int32_t j = 0; j < lp->k.cols; ++j) col_old[j] = r.empty() ? j : r.col_old[j];
  });
}

int anu_estimate_matrix_norm(const anu_lp* lp, int32_t iterations, double tolerance,
                             double* norm) {
  return guarded([&] {
    if (lp == nullptr || norm == nullptr) throw Error(ANU_ERR_INVALID, "null argument");
    const std::string e = anu::validate_lp(*lp);
    if (!e.empty()) throw Error(ANU_ERR_INVALID, "invalid LP: " + e);
    anu_pdhg_options o;
    anu_pdhg_default_options(&o);
    o.ruiz_iterations = 0;
    o.pock_chambolle = 0;
    o.known_matrix_norm = 1.0;  // skip the default estimate; measured below
    auto p = anu::make_problem(*lp, o, nullptr, nullptr);
    *norm = anu::device_matrix_norm(*p, iterations, tolerance);
  });
}

int anu_evaluate_residual(const anu_lp* lp, const double* x, const double* y,
                          anu_pdhg_residual* out) {
  return guarded([&] {
    if (lp == nullptr || x == nullptr || y == nullptr || out == nullptr)
      throw Error(ANU_ERR_INVALID, "null argument");
    const std::string e = anu::validate_lp(*lp);
    if (!e.empty()) throw Error(ANU_ERR_INVALID, "invalid LP: " + e);
    anu_pdhg_options o;
    anu_pdhg_default_options(&o);
    o.ruiz_iterations = 0;
    o.pock_chambolle = 0;
    o.known_matrix_norm = 1.0;
    auto p = anu::make_problem(*lp, o, nullptr, nullptr);
    p->unit_scaling = true;
    anu::CaseData cd = anu::make_case(*p, lp->c, lp->q, lp->lower, lp->upper,
                                      lp->objective_scale, lp->objective_offset);
    anu::evaluate_point(*p, cd, std::vector<double>(x, x + lp->k.cols),
                        std::vector<double>(y, y + lp->k.rows), out);
  });
}

int anu_pdhg_batch_create(const anu_lp* base, int32_t num_cases, const double* c,
                          const double* q, const double* lower, const double* upper,
                          const anu_pdhg_options* options, anu_pdhg_batch** handle) {
  return guarded([&] {
    if (base == nullptr || options == nullptr || handle == nullptr)
      throw Error(ANU_ERR_INVALID, "null argument");
    *handle = nullptr;
    if (num_cases < 1) throw Error(ANU_ERR_INVALID, "num_cases < 1");
    anu::validate_options(*options);
    const std::string e = anu::validate_lp(*base);
    if (!e.empty()) throw Error(ANU_ERR_INVALID, "invalid LP: " + e);
    const int32_t n = base->k.cols, m = base->k.rows;
    for (int32_t k = 0; k < num_cases; ++k) {
      const double* lo = lower ? lower + static_cast<size_t>(k) * n : base->lower;
      const double* hi = upper ? upper + static_cast<size_t>(k) * n : base->upper;
      for (int32_t j = 0; j < n; ++j)
        if (lo[j] > hi[j]) throw Error(ANU_ERR_INVALID, "empty bound interval in case " + std::to_string(k));
      const double* qq = q ? q + static_cast<size_t>(k) * m : base->q;
      for (int32_t i = 0; i < m; ++i)
        if (!std::isfinite(qq[i])) throw Error(ANU_ERR_INVALID, "rhs is not finite in case " + std::to_string(k));
    }
    auto h = std::make_unique<anu_pdhg_batch>();
    h->options = *options;
    h->problem = anu::make_problem(*base, *options, &h->scaling_seconds, &h->norm_seconds);
    anu::choose_tiles(*h->problem, *options, nullptr);
    // A stack that runs persistent chunks is one stack: its chunk kernel
    // fills the device on its own, and two of them may not overlap.
    if (options->split_stacks && num_cases >= anu::kSplitStack &&
        !anu::stack_runs_persistent(*h->problem, std::min(num_cases, anu::kMaxCasesPerRun),
                                    *options))
      h->twin = anu::clone_problem(*h->problem);
    h->base_c.assign(base->c, base->c + n);
    h->base_q.assign(base->q, base->q + m);
    h->base_lower.assign(base->lower, base->lower + n);
    h->base_upper.assign(base->upper, base->upper + n);
    h->objective_scale = base->objective_scale;
    h->objective_offset = base->objective_offset;
    h->cases.reserve(num_cases);
    for (int32_t k = 0; k < num_cases; ++k) {
      h->cases.push_back(anu::make_case(
          *h->problem, c ? c + static_cast<size_t>(k) * n : base->c,
          q ? q + static_cast<size_t>(k) * m : base->q,
          lower ? lower + static_cast<size_t>(k) * n : base->lower,
          upper ? upper + static_cast<size_t>(k) * n : base->upper, base->objective_scale,
          base->objective_offset));
    }
    *handle = h.release();
  });
}

int anu_pdhg_batch_solve(anu_pdhg_batch* h, double* x, double* y, anu_pdhg_result* results) {
  return anu_pdhg_batch_solve_warm(h, nullptr, nullptr, x, y, results);
}

int anu_pdhg_batch_stream(anu_pdhg_batch* h, int32_t slots, anu_pdhg_case_source source,
                          anu_pdhg_case_sink sink, void* user) {
  return guarded([&] {
    if (h == nullptr || source == nullptr || sink == nullptr)
      throw Error(ANU_ERR_INVALID, "null argument");
    if (slots < 1 || slots > anu::kMaxCasesPerRun)
      throw Error(ANU_ERR_INVALID, "slots must be 1 to " + std::to_string(anu::kMaxCasesPerRun));
    const double start = anu::now_seconds();
    const int32_t n = h->problem->n, m = h->problem->m;
    // A streamed case lives until its slot takes the next case (the stack
    // hands it back then) or the stream ends, so a long stream holds about
    // `slots` cases on the host, not every case it has seen.
    std::unordered_map<const anu::CaseData*, std::unique_ptr<anu::CaseData>> owned;
    std::vector<double> c, q, lo, up;
    auto next_case = [&](int32_t* id) -> const anu::CaseData* {
      c = h->base_c;
      q = h->base_q;
      lo = h->base_lower;
      up = h->base_upper;
      int32_t case_id = -1;
      if (source(user, &case_id, c.data(), q.data(), lo.data(), up.data()) == 0) return nullptr;
      for (int32_t j = 0; j < n; ++j)
        if (lo[j] > up[j])
          throw Error(ANU_ERR_INVALID, "empty bound interval in streamed case " +
                                           std::to_string(case_id));
      for (int32_t i = 0; i < m; ++i)
        if (!std::isfinite(q[i]))
          throw Error(ANU_ERR_INVALID, "rhs is not finite in streamed case " +
                                           std::to_string(case_id));
      auto cd = std::make_unique<anu::CaseData>(anu::make_case(
          *h->problem, c.data(), q.data(), lo.data(), up.data(), h->objective_scale,
          h->objective_offset));
      const anu::CaseData* ptr = cd.get();
      owned.emplace(ptr, std::move(cd));
      *id = case_id;
      return ptr;
    };
    auto release = [&](const anu::CaseData* d) { owned.erase(d); };
    auto deliver = [&](int32_t id, anu::CaseResult& cr) {
      anu_pdhg_result r;
      fill_result(*h->problem, cr, h->scaling_seconds, h->norm_seconds, &r);
      sink(user, id, cr.x.data(), cr.y.data(), &r);
    };
    anu::run_cases_streaming(*h->problem, slots, h->options, next_case, deliver, release, start);
  });
}

int anu_pdhg_batch_solve_warm(anu_pdhg_batch* h, const double* warm_x, const double* warm_y,
                              double* x, double* y, anu_pdhg_result* results) {
  return guarded([&] {
    if (h == nullptr || results == nullptr) throw Error(ANU_ERR_INVALID, "null argument");
    const int32_t n = h->problem->n, m = h->problem->m;
    const int total = static_cast<int>(h->cases.size());
    const double start = anu::now_seconds();
    // One stack of the given cases on one problem: lockstep up to one run's
    // capacity, rolling beyond it.
    // Warm starts, case-major, both or neither.
    const bool warm = warm_x != nullptr && warm_y != nullptr;
    std::vector<std::vector<double>> wx(warm ? total : 0), wy(warm ? total : 0);
    for (int k = 0; warm && k < total; ++k) {
      wx[k].assign(warm_x + static_cast<size_t>(k) * n, warm_x + static_cast<size_t>(k + 1) * n);
      wy[k].assign(warm_y + static_cast<size_t>(k) * m, warm_y + static_cast<size_t>(k + 1) * m);
    }
    auto solve_part = [&](anu::Problem& prob, const std::vector<int>& idx,
                          std::vector<anu::CaseResult>* out) {
      std::vector<const anu::CaseData*> cs;
      std::vector<const std::vector<double>*> vx, vy;
      for (int k : idx) {
        cs.push_back(&h->cases[k]);
        vx.push_back(warm ? &wx[k] : nullptr);
        vy.push_back(warm ? &wy[k] : nullptr);
      }
      if (static_cast<int>(cs.size()) <= anu::kMaxCasesPerRun)
        anu::run_cases(prob, cs, h->options, vx, vy, out, start);
      else
        anu::run_cases_rolling(prob, cs, anu::kMaxCasesPerRun, h->options, vx, vy, out, start);
    };
    std::vector<anu::CaseResult> res(total);
    if (h->twin == nullptr) {
      std::vector<int> all(total);
      for (int k = 0; k < total; ++k) all[k] = k;
      solve_part(*h->problem, all, &res);
    } else {
      // Two half-stacks (alternate cases) at once, each on its own problem,
      // stream and host thread: every iteration kernel is latency-bound, so
      // two streams of them overlap.
      std::vector<int> part[2];
      for (int k = 0; k < total; ++k) part[k % 2].push_back(k);
      std::vector<anu::CaseResult> out[2];
      int code = 0;
      std::string message;
      std::thread other([&]() {
        try {
          solve_part(*h->twin, part[1], &out[1]);
        } catch (const Error& e) {
          code = e.code;
          message = e.what();
        } catch (const std::exception& e) {
          code = ANU_ERR_INTERNAL;
          message = e.what();
        }
      });
      try {
        solve_part(*h->problem, part[0], &out[0]);
      } catch (...) {
        other.join();
        throw;
      }
      other.join();
      if (code != 0) throw Error(code, message);
      for (int s = 0; s < 2; ++s)
        for (size_t i = 0; i < part[s].size(); ++i) res[part[s][i]] = std::move(out[s][i]);
    }
    for (int k = 0; k < total; ++k) {
      fill_result(*h->problem, res[k], h->scaling_seconds, h->norm_seconds, &results[k]);
      if (x) std::copy(res[k].x.begin(), res[k].x.end(), x + static_cast<size_t>(k) * n);
      if (y) std::copy(res[k].y.begin(), res[k].y.end(), y + static_cast<size_t>(k) * m);
    }
  });
}

void anu_pdhg_batch_destroy(anu_pdhg_batch* h) { delete h; }

}  // extern "C"
