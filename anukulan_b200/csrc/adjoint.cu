// Unrolled PDHG and its hand-written adjoint.
//
// The unrolled scheme is a fixed program: `iterations` steps of reflected
// Halpern PDHG (the step of anu_pdhg_solve with reflection 1) with step
// sizes fixed at their starting values (tau = eta/omega, sigma = eta*omega,
// eta = 0.9/||K~||, omega = ||c~||/||q~|| per case, as solve_pdhg starts, or
// options.initial_step_size / initial_primal_weight), and the Halpern
// anchor restarted at the new iterate every `checkpoint_every` steps. On the
// scaled problem, step t maps (x, y, anchors) to
//
//   u = x - tau (c - K'y),   v = clamp(u, l, u_b),   x_bar = 2v - x
//   s = y + sigma (q - K x_bar),   w = s (equality rows), max(s, 0) (others)
//   x+ = a (2v - x) + (1-a) x_anchor,   y+ = a (2w - y) + (1-a) y_anchor
//
// with a = j/(j+1) at the j-th step after a restart, and at a restart step
// (j = 0) x+ = 2v - x, y+ = 2w - y and the anchors set to them. It is
// piecewise linear in (c, q), so its derivative is exact away from the
// kinks of the projections.
//
// Forward: the steps run as the engine's fused SpMV launches over the case
// stack (case-interleaved vectors, every nonzero read serving all cases),
// with the state saved every `checkpoint_every` steps; a segment's launches
// are one CUDA graph, replayed segment after segment.
//
// Backward (reverse mode): segment by segment from the last, the segment is
// recomputed from its checkpoint with the projection masks recorded
// (clamp'(u) and the cone's max'(s), one byte per entry and step), then its
// steps are reversed. With hats for adjoints, step t reverses as
//
//   dual:    n = a y^+ (restart: y^+ + y_anchor^),  s^ = mask_s (2n),
//            y^ = -n + s^ + tau K u^,  q~^ += sigma s^,  z = sigma s^
//   primal:  m = a x^+ (restart: x^+ + x_anchor^),  x_bar^ = -K'z,
//            u^ = mask_u (2m + 2 x_bar^),  x^ = -m - x_bar^ + u^,
//            c~^ -= tau u^
//
// (anchor adjoints gather (1-a) of the state adjoint and restart at zero).
// That is two fused SpMV launches per reversed step: K'z with the primal
// reverse in its epilogue, then K u^ with the end of this step's dual
// reverse and the start of the previous step's. Gradients accumulate in
// FP64 and are mapped back to the unscaled c and q at the end.
#include <cmath>
#include <cstring>

#include "engine.hpp"

namespace anu {

// Segment shape of the unrolled handle's matrices. The forward and reverse
// epilogues do more per (row, case) item than the solver's step, and larger
// CTAs of shorter segments measured faster for them: 79 ms per 60-case,
// 2,000-step forward and backward against 104 ms at the solver's 4 x 16.
constexpr int32_t kAdjointSegNnz = 8;
constexpr int32_t kAdjointSegPerCta = 16;

namespace {

struct StepSchedule {
  bool restart;
  double a;
};

StepSchedule schedule(int t, int period) {
  const int j = t % period;
  if (j == 0) return {true, 1.0};
  return {false, static_cast<double>(j) / static_cast<double>(j + 1)};
}

// ---- forward step epilogues (record masks when `mask` is set)

template <class T>
struct UnrollPrimal {
  int32_t K;
  const double* __restrict__ tau;
  int32_t restart;
  double a;
  T* x;
  const T* __restrict__ c;
  const T* __restrict__ lo;
  const T* __restrict__ hi;
  T* anchor;
  T* __restrict__ x_bar;
  uint8_t* __restrict__ mask;
  struct Pre {};
  __device__ __forceinline__ Pre prefetch(int32_t, int32_t) const { return Pre{}; }
  __device__ __forceinline__ void finish(int32_t j, int32_t k, T kty, const Pre&) const {
    const size_t e = static_cast<size_t>(j) * K + k;
    const T xj = x[e];
    const T u = sub(xj, mul(static_cast<T>(tau[k]), sub(c[e], kty)));
    const T l = lo[e], h = hi[e];
    T v = u;
    if (v < l) v = l;
    if (v > h) v = h;
    if (mask) mask[e] = (u > l && u < h) ? 1 : 0;
    const T nxt = add(v, sub(v, xj));
    x_bar[e] = nxt;
    if (restart) {
      anchor[e] = nxt;
      x[e] = nxt;
    } else {
      x[e] = add(mul(static_cast<T>(a), nxt), mul(static_cast<T>(1.0 - a), anchor[e]));
    }
  }
  __device__ __forceinline__ void operator()(int32_t j, int32_t k, T s) const {
    finish(j, k, s, Pre{});
  }
};

template <class T>
struct UnrollDual {
  int32_t K;
  int32_t num_eq;
  const double* __restrict__ sigma;
  int32_t restart;
  double a;
  T* y;
  const T* __restrict__ q;
  T* anchor;
  uint8_t* __restrict__ mask;
  struct Pre {};
  __device__ __forceinline__ Pre prefetch(int32_t, int32_t) const { return Pre{}; }
  __device__ __forceinline__ void finish(int32_t i, int32_t k, T bar, const Pre&) const {
    const size_t e = static_cast<size_t>(i) * K + k;
    const T yi = y[e];
    const T s = add(yi, mul(static_cast<T>(sigma[k]), sub(q[e], bar)));
    const bool cone = i >= num_eq;
    T w = s;
    if (cone && w < static_cast<T>(0)) w = static_cast<T>(0);
    if (mask) mask[e] = (!cone || s > static_cast<T>(0)) ? 1 : 0;
    const T nxt = add(w, sub(w, yi));
    if (restart) {
      anchor[e] = nxt;
      y[e] = nxt;
    } else {
      y[e] = add(mul(static_cast<T>(a), nxt), mul(static_cast<T>(1.0 - a), anchor[e]));
    }
  }
  __device__ __forceinline__ void operator()(int32_t i, int32_t k, T s) const {
    finish(i, k, s, Pre{});
  }
};

// ---- reverse

// The dual half of reversing one step on entry (i, k), given y^+ = yh[e]:
// leaves the partial y^ (before the tau K u^ term) in yh, sigma s^ in z.
template <class T>
__device__ __forceinline__ void dual_reverse(size_t e, double sigma, int32_t restart, double a,
                                             uint8_t mask, T yplus, T* yh, T* ayh, T* z,
                                             double* gq) {
  T n;
  if (restart) {
    n = add(yplus, ayh[e]);
    ayh[e] = static_cast<T>(0);
  } else {
    n = mul(static_cast<T>(a), yplus);
    ayh[e] = add(ayh[e], mul(static_cast<T>(1.0 - a), yplus));
  }
  const T s = mask ? add(n, n) : static_cast<T>(0);
  yh[e] = sub(s, n);
  const T zs = mul(static_cast<T>(sigma), s);
  z[e] = zs;
  gq[e] += static_cast<double>(zs);
}

template <class T>
__global__ void dual_reverse_kernel(int64_t total, int32_t K, const double* __restrict__ sigma,
                                    int32_t restart, double a, const uint8_t* __restrict__ mask,
                                    T* yh, T* ayh, T* z, double* gq) {
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t k = static_cast<int32_t>(e % K);
    dual_reverse<T>(static_cast<size_t>(e), sigma[k], restart, a, mask[e], yh[e], yh, ayh, z, gq);
  }
}

// Epilogue of K'z over columns: the primal half of reversing step t.
template <class T>
struct RevPrimal {
  int32_t K;
  const double* __restrict__ tau;
  int32_t restart;
  double a;
  T* xh;
  T* axh;
  const uint8_t* __restrict__ mask;
  T* __restrict__ uh;
  double* __restrict__ gc;
  struct Pre {};
  __device__ __forceinline__ Pre prefetch(int32_t, int32_t) const { return Pre{}; }
  __device__ __forceinline__ void finish(int32_t j, int32_t k, T ktz, const Pre&) const {
    const size_t e = static_cast<size_t>(j) * K + k;
    const T xplus = xh[e];
    T m;
    if (restart) {
      m = add(xplus, axh[e]);
      axh[e] = static_cast<T>(0);
    } else {
      m = mul(static_cast<T>(a), xplus);
      axh[e] = add(axh[e], mul(static_cast<T>(1.0 - a), xplus));
    }
    const T xbh = -ktz;
    const T vh = add(add(m, m), add(xbh, xbh));
    const T u = mask[e] ? vh : static_cast<T>(0);
    xh[e] = add(sub(-m, xbh), u);
    uh[e] = u;
    gc[e] -= tau[k] * static_cast<double>(u);
  }
  __device__ __forceinline__ void operator()(int32_t j, int32_t k, T s) const {
    finish(j, k, s, Pre{});
  }
};

// Epilogue of K u^ over rows: y^ of step t complete; then, unless this is
// the first step of the segment, the dual half of reversing step t-1.
template <class T>
struct RevDual {
  int32_t K;
  const double* __restrict__ tau;
  const double* __restrict__ sigma;
  T* yh;
  T* ayh;
  T* z;
  double* gq;
  const uint8_t* __restrict__ mask_prev;  // null: no previous step here
  int32_t restart_prev;
  double a_prev;
  struct Pre {};
  __device__ __forceinline__ Pre prefetch(int32_t, int32_t) const { return Pre{}; }
  __device__ __forceinline__ void finish(int32_t i, int32_t k, T kuh, const Pre&) const {
    const size_t e = static_cast<size_t>(i) * K + k;
    const T yt = add(yh[e], mul(static_cast<T>(tau[k]), kuh));
    if (mask_prev == nullptr) {
      yh[e] = yt;
      return;
    }
    dual_reverse<T>(e, sigma[k], restart_prev, a_prev, mask_prev[e], yt, yh, ayh, z, gq);
  }
  __device__ __forceinline__ void operator()(int32_t i, int32_t k, T s) const {
    finish(i, k, s, Pre{});
  }
};

template <class T>
__global__ void scale_into_kernel(int64_t total, int32_t K, const double* __restrict__ scale,
                                  const double* __restrict__ src, T* __restrict__ dst) {
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[e] = static_cast<T>(scale ? scale[e / K] * src[e] : src[e]);
}

int grid_elems(int64_t n) { return grid_for(n, 256, 148 * 8); }

}  // namespace

namespace {
template <class T>
struct UnrollState;
}  // namespace

// The unrolled program of one case stack, held on the device.
struct Unrolled {
  std::unique_ptr<Problem> problem;
  std::vector<CaseData> cases;
  int K = 0;
  int32_t iterations = 0, period = 0;
  int precision = ANU_PRECISION_FP64;
  std::vector<double> tau, sigma;
  double scaling_seconds = 0.0, norm_seconds = 0.0;
  // The last forward pass's state and checkpoints (declared after the
  // problem, so released into its memory pool before the pool goes).
  std::unique_ptr<UnrollState<float>> state32;
  std::unique_ptr<UnrollState<double>> state64;
  ~Unrolled();
};

namespace {

template <class T>
void upload_cases(cudaStream_t s, DevBuf<T>& dst, int32_t len, int K,
                  const std::vector<std::vector<double>>& src) {
  std::vector<T> h(static_cast<size_t>(std::max(len, 1)) * K, static_cast<T>(0));
  for (int k = 0; k < K; ++k)
    for (int32_t i = 0; i < len; ++i) h[static_cast<size_t>(i) * K + k] = static_cast<T>(src[k][i]);
  dst.alloc(h.size());
  ANU_CUDA(cudaMemcpyAsync(dst.p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s));
  ANU_CUDA(cudaStreamSynchronize(s));
}

// Case-major host copy of a case-interleaved device vector, times `scale`.
template <class T>
void download_cases(cudaStream_t s, const DevBuf<T>& src, int32_t len, int K,
                    const std::vector<double>* scale, double* out) {
  std::vector<T> h(static_cast<size_t>(len) * K);
  if (!h.empty())
    ANU_CUDA(cudaMemcpyAsync(h.data(), src.p, sizeof(T) * h.size(), cudaMemcpyDeviceToHost, s));
  ANU_CUDA(cudaStreamSynchronize(s));
  for (int k = 0; k < K; ++k)
    for (int32_t i = 0; i < len; ++i)
      out[static_cast<size_t>(k) * len + i] =
          static_cast<double>(h[static_cast<size_t>(i) * K + k]) * (scale ? (*scale)[i] : 1.0);
}

// The device state of the unrolled program for one call.
template <class T>
struct UnrollState {
  DevBuf<T> x, y, ax, ay, x_bar, c, lo, hi, q;
  DevBuf<double> tau, sigma;
  DevBuf<T> ckpt;  // checkpoints: per segment x, y, ax, ay
  size_t nk = 0, mk = 0;
};

}  // namespace

Unrolled::~Unrolled() {
  state32.reset();
  state64.reset();
}

namespace {

template <class T>
void setup_state(Unrolled& u, UnrollState<T>& s) {
  Problem& p = *u.problem;
  const int K = u.K;
  const int32_t n = p.n, m = p.m;
  const cudaStream_t st = p.stream;
  s.nk = static_cast<size_t>(std::max(n, 1)) * K;
  s.mk = static_cast<size_t>(std::max(m, 1)) * K;
  std::vector<std::vector<double>> vc(K), vl(K), vh(K), vq(K), x0(K), y0(K);
  for (int k = 0; k < K; ++k) {
    const CaseData& d = u.cases[k];
    vc[k] = d.cs;
    vl[k] = d.ls;
    vh[k] = d.us;
    vq[k] = d.qs;
    x0[k].assign(n, 0.0);
    y0[k].assign(m, 0.0);
    // The starting point of solve_pdhg without a warm start (pdhg.cpp:481-503).
    for (int32_t j = 0; j < n; ++j) {
      double v = 0.0;
      const double lo = d.ls[j], hi = d.us[j];
      if (v < lo) v = std::isfinite(lo) ? lo : 0.0;
      if (v > hi) v = std::isfinite(hi) ? hi : 0.0;
      x0[k][j] = v;
    }
  }
  upload_cases(st, s.c, n, K, vc);
  upload_cases(st, s.lo, n, K, vl);
  upload_cases(st, s.hi, n, K, vh);
  upload_cases(st, s.q, m, K, vq);
  upload_cases(st, s.x, n, K, x0);
  upload_cases(st, s.y, m, K, y0);
  s.ax.alloc(s.nk);
  s.ay.alloc(s.mk);
  s.x_bar.alloc(s.nk);
  ANU_CUDA(cudaMemsetAsync(s.ax.p, 0, sizeof(T) * s.nk, st));
  ANU_CUDA(cudaMemsetAsync(s.ay.p, 0, sizeof(T) * s.mk, st));
  s.tau.alloc(K);
  s.sigma.alloc(K);
  ANU_CUDA(cudaMemcpyAsync(s.tau.p, u.tau.data(), sizeof(double) * K, cudaMemcpyHostToDevice, st));
  ANU_CUDA(cudaMemcpyAsync(s.sigma.p, u.sigma.data(), sizeof(double) * K, cudaMemcpyHostToDevice, st));
}

template <class T>
void forward_step(Problem& p, int K, UnrollState<T>& s, int t, int period, uint8_t* mx,
                  uint8_t* my) {
  const StepSchedule sc = schedule(t, period);
  product<T, T, T>(p, p.dkt, s.y.p, K,
                   UnrollPrimal<T>{K, s.tau.p, sc.restart ? 1 : 0, sc.a, s.x.p, s.c.p, s.lo.p,
                                   s.hi.p, s.ax.p, s.x_bar.p, mx});
  product<T, T, T>(p, p.dk, s.x_bar.p, K,
                   UnrollDual<T>{K, p.num_eq, s.sigma.p, sc.restart ? 1 : 0, sc.a, s.y.p, s.q.p,
                                 s.ay.p, my});
}

// Copies the state (x, y, ax, ay) into or out of checkpoint slot `seg`.
template <class T>
void checkpoint(Problem& p, UnrollState<T>& s, int seg, bool save) {
  T* base = s.ckpt.p + static_cast<size_t>(seg) * 2 * (s.nk + s.mk);
  T* parts[4] = {base, base + s.nk, base + 2 * s.nk, base + 2 * s.nk + s.mk};
  T* live[4] = {s.x.p, s.ax.p, s.y.p, s.ay.p};
  const size_t len[4] = {s.nk, s.nk, s.mk, s.mk};
  for (int i = 0; i < 4; ++i)
    ANU_CUDA(cudaMemcpyAsync(save ? parts[i] : live[i], save ? live[i] : parts[i],
                             sizeof(T) * len[i], cudaMemcpyDeviceToDevice, p.stream));
}

// A segment's launches as one CUDA graph: captured on first use, replayed
// for every later full segment (the launches and their arguments repeat
// from segment to segment; only the checkpoint copies between differ).
struct SegmentGraph {
  cudaGraphExec_t exec = nullptr;
  int64_t launches = 0;
  SegmentGraph() = default;
  SegmentGraph(const SegmentGraph&) = delete;
  SegmentGraph& operator=(const SegmentGraph&) = delete;
  ~SegmentGraph() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

template <class F>
void replay(Problem& p, SegmentGraph& g, F&& body) {
  if (g.exec == nullptr) {
    const int64_t before = p.launches;
    ANU_CUDA(cudaStreamBeginCapture(p.stream, cudaStreamCaptureModeThreadLocal));
    try {
      body();
    } catch (...) {
      cudaGraph_t broken = nullptr;
      cudaStreamEndCapture(p.stream, &broken);
      if (broken) cudaGraphDestroy(broken);
      throw;
    }
    cudaGraph_t graph = nullptr;
    ANU_CUDA(cudaStreamEndCapture(p.stream, &graph));
    const cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    ANU_CUDA(e);
    g.launches = p.launches - before;
    p.launches = before;
  }
  ANU_CUDA(cudaGraphLaunch(g.exec, p.stream));
  p.launches += g.launches;
}

template <class T>
void forward_t(Unrolled& u, UnrollState<T>& s, double* x_out, double* y_out) {
  Problem& p = *u.problem;
  const int segments = (u.iterations + u.period - 1) / u.period;
  setup_state(u, s);
  s.ckpt.alloc(static_cast<size_t>(std::max(segments, 1)) * 2 * (s.nk + s.mk));
  SegmentGraph graph;
  for (int seg = 0; seg < segments; ++seg) {
    const int s0 = seg * u.period;
    const int len = std::min(u.iterations - s0, u.period);
    checkpoint(p, s, seg, true);
    auto body = [&]() {
      for (int j = 0; j < len; ++j) forward_step(p, u.K, s, j, u.period, nullptr, nullptr);
    };
    if (len == u.period) replay(p, graph, body);
    else body();
  }
  if (x_out) download_cases(p.stream, s.x, p.n, u.K, &p.scaling.col_scale, x_out);
  if (y_out) download_cases(p.stream, s.y, p.m, u.K, &p.scaling.row_scale, y_out);
  ANU_CUDA(cudaStreamSynchronize(p.stream));
}

template <class T>
void backward_t(Unrolled& u, UnrollState<T>& s, const double* dx, const double* dy,
                double* grad_c, double* grad_q) {
  Problem& p = *u.problem;
  const cudaStream_t st = p.stream;
  const int K = u.K;
  const int32_t n = p.n, m = p.m;
  const int R = u.period;
  const int segments = (u.iterations + R - 1) / R;
  // Adjoint state, seeded with dL/dx~_T = D2 dL/dx and dL/dy~_T = D1 dL/dy.
  DevBuf<T> xh(s.nk), yh(s.mk), axh(s.nk), ayh(s.mk), z(s.mk), uh(s.nk);
  DevBuf<double> gc(s.nk), gq(s.mk), seed_x(s.nk), seed_y(s.mk), d2(std::max(n, 1)),
      d1(std::max(m, 1));
  ANU_CUDA(cudaMemcpyAsync(d2.p, p.scaling.col_scale.data(), sizeof(double) * n,
                           cudaMemcpyHostToDevice, st));
  ANU_CUDA(cudaMemcpyAsync(d1.p, p.scaling.row_scale.data(), sizeof(double) * m,
                           cudaMemcpyHostToDevice, st));
  std::vector<double> hx(s.nk, 0.0), hy(s.mk, 0.0);
  for (int k = 0; k < K; ++k) {
    for (int32_t j = 0; j < n && dx; ++j) hx[static_cast<size_t>(j) * K + k] = dx[static_cast<size_t>(k) * n + j];
    for (int32_t i = 0; i < m && dy; ++i) hy[static_cast<size_t>(i) * K + k] = dy[static_cast<size_t>(k) * m + i];
  }
  ANU_CUDA(cudaMemcpyAsync(seed_x.p, hx.data(), sizeof(double) * s.nk, cudaMemcpyHostToDevice, st));
  ANU_CUDA(cudaMemcpyAsync(seed_y.p, hy.data(), sizeof(double) * s.mk, cudaMemcpyHostToDevice, st));
  scale_into_kernel<T><<<grid_elems(s.nk), 256, 0, st>>>(static_cast<int64_t>(s.nk), K, d2.p,
                                                          seed_x.p, xh.p);
  scale_into_kernel<T><<<grid_elems(s.mk), 256, 0, st>>>(static_cast<int64_t>(s.mk), K, d1.p,
                                                          seed_y.p, yh.p);
  ANU_CUDA(cudaGetLastError());
  ANU_CUDA(cudaMemsetAsync(axh.p, 0, sizeof(T) * s.nk, st));
  ANU_CUDA(cudaMemsetAsync(ayh.p, 0, sizeof(T) * s.mk, st));
  ANU_CUDA(cudaMemsetAsync(gc.p, 0, sizeof(double) * s.nk, st));
  ANU_CUDA(cudaMemsetAsync(gq.p, 0, sizeof(double) * s.mk, st));
  DevBuf<uint8_t> mx(static_cast<size_t>(R) * s.nk), my(static_cast<size_t>(R) * s.mk);
  SegmentGraph recompute_graph, reverse_graph;
  for (int seg = segments - 1; seg >= 0; --seg) {
    const int s0 = seg * R;
    const int s1 = std::min(u.iterations, s0 + R);
    const int len = s1 - s0;
    // Recompute the segment from its checkpoint, recording the masks.
    checkpoint(p, s, seg, false);
    auto recompute = [&]() {
      for (int j = 0; j < len; ++j)
        forward_step(p, K, s, j, R, mx.p + static_cast<size_t>(j) * s.nk,
                     my.p + static_cast<size_t>(j) * s.mk);
    };
    // Then reverse it: the dual half of its last step, then step by step.
    auto reverse = [&]() {
      const StepSchedule sc = schedule(len - 1, R);
      dual_reverse_kernel<T><<<grid_elems(s.mk), 256, 0, st>>>(
          static_cast<int64_t>(s.mk), K, s.sigma.p, sc.restart ? 1 : 0, sc.a,
          my.p + static_cast<size_t>(len - 1) * s.mk, yh.p, ayh.p, z.p, gq.p);
      ANU_CUDA(cudaGetLastError());
      ++p.launches;
      for (int j = len - 1; j >= 0; --j) {
        const StepSchedule sj = schedule(j, R);
        product<T, T, T>(p, p.dkt, z.p, K,
                         RevPrimal<T>{K, s.tau.p, sj.restart ? 1 : 0, sj.a, xh.p, axh.p,
                                      mx.p + static_cast<size_t>(j) * s.nk, uh.p, gc.p});
        const bool more = j > 0;
        const StepSchedule sp = more ? schedule(j - 1, R) : StepSchedule{false, 0.0};
        product<T, T, T>(p, p.dk, uh.p, K,
                         RevDual<T>{K, s.tau.p, s.sigma.p, yh.p, ayh.p, z.p, gq.p,
                                    more ? my.p + static_cast<size_t>(j - 1) * s.mk : nullptr,
                                    sp.restart ? 1 : 0, sp.a});
      }
    };
    if (len == R) {
      replay(p, recompute_graph, recompute);
      replay(p, reverse_graph, reverse);
    } else {
      recompute();
      reverse();
    }
  }
  // Back to the unscaled data: c~ = D2 c, q~ = D1 q.
  std::vector<double> hc(s.nk), hq(s.mk);
  ANU_CUDA(cudaMemcpyAsync(hc.data(), gc.p, sizeof(double) * s.nk, cudaMemcpyDeviceToHost, st));
  ANU_CUDA(cudaMemcpyAsync(hq.data(), gq.p, sizeof(double) * s.mk, cudaMemcpyDeviceToHost, st));
  ANU_CUDA(cudaStreamSynchronize(st));
  for (int k = 0; k < K; ++k) {
    if (grad_c)
      for (int32_t j = 0; j < n; ++j)
        grad_c[static_cast<size_t>(k) * n + j] =
            p.scaling.col_scale[j] * hc[static_cast<size_t>(j) * K + k];
    if (grad_q)
      for (int32_t i = 0; i < m; ++i)
        grad_q[static_cast<size_t>(k) * m + i] =
            p.scaling.row_scale[i] * hq[static_cast<size_t>(i) * K + k];
  }
}

template <class F>
int guarded_unrolled(F&& body) {
  try {
    clear_last_error();
    body();
    return ANU_OK;
  } catch (const Error& e) {
    set_last_error(e.code, e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error(ANU_ERR_MEMORY, "host allocation failed");
    return ANU_ERR_MEMORY;
  } catch (const std::exception& e) {
    set_last_error(ANU_ERR_INTERNAL, e.what());
    return ANU_ERR_INTERNAL;
  }
}

}  // namespace
}  // namespace anu

struct anu_pdhg_unrolled {
  anu::Unrolled u;
};

using anu::Error;

extern "C" {

int anu_pdhg_unrolled_create(const anu_lp* base, int32_t num_cases, const double* c,
                             const double* q, const double* lower, const double* upper,
                             const anu_pdhg_options* options, int32_t iterations,
                             int32_t checkpoint_every, anu_pdhg_unrolled** handle) {
  return anu::guarded_unrolled([&] {
    if (base == nullptr || options == nullptr || handle == nullptr)
      throw Error(ANU_ERR_INVALID, "null argument");
    *handle = nullptr;
    if (num_cases < 1 || num_cases > anu::kMaxCasesPerRun)
      throw Error(ANU_ERR_INVALID, "num_cases must be in 1..64");
    if (iterations < 1) throw Error(ANU_ERR_INVALID, "iterations < 1");
    if (checkpoint_every < 1) throw Error(ANU_ERR_INVALID, "checkpoint_every < 1");
    anu::validate_options(*options);
    const std::string e = anu::validate_lp(*base);
    if (!e.empty()) throw Error(ANU_ERR_INVALID, "invalid LP: " + e);
    auto h = std::make_unique<anu_pdhg_unrolled>();
    anu::Unrolled& u = h->u;
    u.K = num_cases;
    u.iterations = iterations;
    u.period = checkpoint_every;
    u.precision = options->precision;
    u.problem = anu::make_problem(*base, *options, &u.scaling_seconds, &u.norm_seconds,
                                  anu::kAdjointSegNnz, anu::kAdjointSegPerCta);
    const int32_t n = base->k.cols, m = base->k.rows;
    for (int32_t k = 0; k < num_cases; ++k)
      u.cases.push_back(anu::make_case(
          *u.problem, c ? c + static_cast<size_t>(k) * n : base->c,
          q ? q + static_cast<size_t>(k) * m : base->q,
          lower ? lower + static_cast<size_t>(k) * n : base->lower,
          upper ? upper + static_cast<size_t>(k) * n : base->upper, base->objective_scale,
          base->objective_offset));
    // Step sizes as solve_pdhg starts (pdhg.cpp:460-479), then held fixed.
    const double norm = u.problem->matrix_norm;
    double eta = norm > 0.0 ? options->constant_step_scale / norm : 1.0;
    if (options->initial_step_size > 0.0) eta = options->initial_step_size;
    for (const anu::CaseData& d : u.cases) {
      double cn = 0.0, qn = 0.0;
      for (double v : d.cs) cn += v * v;
      for (double v : d.qs) qn += v * v;
      cn = std::sqrt(cn);
      qn = std::sqrt(qn);
      double omega = 1.0;
      if (options->primal_weight_updates && cn > 1e-12 && qn > 1e-12) omega = cn / qn;
      if (options->initial_primal_weight > 0.0) omega = options->initial_primal_weight;
      u.tau.push_back(eta / omega);
      u.sigma.push_back(eta * omega);
    }
    *handle = h.release();
  });
}

int anu_pdhg_unrolled_step_sizes(const anu_pdhg_unrolled* h, double* tau, double* sigma) {
  return anu::guarded_unrolled([&] {
    if (h == nullptr) throw Error(ANU_ERR_INVALID, "null argument");
    if (tau) std::copy(h->u.tau.begin(), h->u.tau.end(), tau);
    if (sigma) std::copy(h->u.sigma.begin(), h->u.sigma.end(), sigma);
  });
}

int anu_pdhg_forward_unrolled(anu_pdhg_unrolled* h, double* x, double* y) {
  return anu::guarded_unrolled([&] {
    if (h == nullptr) throw Error(ANU_ERR_INVALID, "null argument");
    anu::Unrolled& u = h->u;
    anu::Problem& p = *u.problem;
    ANU_CUDA(cudaSetDevice(p.device));
    anu::PoolScope scope(&p.pool, p.stream);
    if (u.precision == ANU_PRECISION_FP32) {
      u.state32 = std::make_unique<anu::UnrollState<float>>();
      anu::forward_t<float>(u, *u.state32, x, y);
    } else {
      u.state64 = std::make_unique<anu::UnrollState<double>>();
      anu::forward_t<double>(u, *u.state64, x, y);
    }
  });
}

int anu_pdhg_backward(anu_pdhg_unrolled* h, const double* dloss_dx, const double* dloss_dy,
                      double* grad_c, double* grad_q) {
  return anu::guarded_unrolled([&] {
    if (h == nullptr) throw Error(ANU_ERR_INVALID, "null argument");
    anu::Unrolled& u = h->u;
    anu::Problem& p = *u.problem;
    ANU_CUDA(cudaSetDevice(p.device));
    anu::PoolScope scope(&p.pool, p.stream);
    // The checkpoints of the last forward pass; without one, a forward pass
    // lays them down first.
    if (u.precision == ANU_PRECISION_FP32) {
      if (!u.state32) {
        u.state32 = std::make_unique<anu::UnrollState<float>>();
        anu::forward_t<float>(u, *u.state32, nullptr, nullptr);
      }
      anu::backward_t<float>(u, *u.state32, dloss_dx, dloss_dy, grad_c, grad_q);
    } else {
      if (!u.state64) {
        u.state64 = std::make_unique<anu::UnrollState<double>>();
        anu::forward_t<double>(u, *u.state64, nullptr, nullptr);
      }
      anu::backward_t<double>(u, *u.state64, dloss_dx, dloss_dy, grad_c, grad_q);
    }
  });
}

void anu_pdhg_unrolled_destroy(anu_pdhg_unrolled* h) { delete h; }

}  // extern "C"
