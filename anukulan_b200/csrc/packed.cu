// Packed batches of unequal LPs: many independent LPs of different shapes
// solved together on one GPU.
//
// Each LP keeps its own problem (scaled matrix and transpose on the device,
// its own stream and memory pool) and runs the same fused single-LP path as
// anu_pdhg_run: two kernels per iteration, CUDA-graph-captured between
// termination checks. The batch is fed to W host workers from one queue,
// largest LP first. A worker that finishes an LP (retires it) takes the next
// one (admits it) at once, so up to W LPs' kernel streams overlap on the GPU
// at any time. Small LPs fill only a few SMs each, and running many of them
// side by side is what fills the device.
//
// W is chosen by a short autotuning pass at creation unless the caller
// fixes it. Each candidate W runs W LPs, drawn evenly from the size order,
// for a fixed number of iterations at once; the W with the most nonzero x
// iterations per second of wall time wins. The single-LP product tile (128
// or 256 threads per CTA) is then chosen the same way at that W, unless
// options.tile_threads fixes it; the tile changes no result.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <numeric>
#include <thread>

#include "engine.hpp"

struct anu_pdhg_packed {
  std::vector<std::unique_ptr<anu::Problem>> problems;
  std::vector<anu::CaseData> data;
  std::vector<double> scaling_seconds, norm_seconds;
  std::vector<int32_t> order;  // most nonzeros first
  anu_pdhg_options options;
  int32_t workers = 0;
};

namespace anu {
namespace {

// Runs `items` (indices into the batch) on `workers` host threads, each
// taking the next item from a shared queue. The first error stops the queue
// and is rethrown here.
template <class F>
void run_queue(const std::vector<int32_t>& items, int workers, F&& solve_one) {
  std::atomic<size_t> next{0};
  std::mutex lock;
  int code = 0;
  std::string message;
  auto work = [&]() {
    for (;;) {
      const size_t i = next.fetch_add(1);
      if (i >= items.size()) return;
      try {
        solve_one(items[i]);
      } catch (const Error& e) {
        std::lock_guard<std::mutex> g(lock);
        if (code == 0) {
          code = e.code;
          message = e.what();
        }
        next.store(items.size());
      } catch (const std::exception& e) {
        std::lock_guard<std::mutex> g(lock);
        if (code == 0) {
          code = ANU_ERR_INTERNAL;
          message = e.what();
        }
        next.store(items.size());
      }
    }
  };
  const int w = std::max(1, std::min<int>(workers, static_cast<int>(items.size())));
  std::vector<std::thread> threads;
  threads.reserve(w - 1);
  for (int t = 1; t < w; ++t) threads.emplace_back(work);
  work();
  for (auto& t : threads) t.join();
  if (code != 0) throw Error(code, message);
}

int host_threads() {
  const unsigned h = std::thread::hardware_concurrency();
  return h == 0 ? 4 : static_cast<int>(h);
}

// Nonzero x iterations per second of `w` workers solving an even sample of
// w LPs of the batch for a few check periods each (a second pass, timed,
// after one that fills the sample LPs' memory pools: it measures how w
// solves share the device, not how w first-time allocations contend).
double sample_rate(anu_pdhg_packed& h, int w) {
  const int n = static_cast<int>(h.problems.size());
  anu_pdhg_options o = h.options;
  o.max_iterations = 4 * o.termination_check_frequency;
  o.polish_feasibility = 0;
  o.polish_on_exit = 0;
  o.profile = 0;
  o.tolerance = 1e-300;  // run the whole budget
  o.gap_tolerance = 1e-300;
  std::vector<int32_t> sample;
  for (int i = 0; i < w; ++i) sample.push_back(h.order[static_cast<size_t>(i) * n / w]);
  double work = 0.0;
  for (int32_t idx : sample)
    work += static_cast<double>(h.problems[idx]->k.nnz()) * o.max_iterations;
  auto pass = [&]() {
    run_queue(sample, w, [&](int32_t idx) {
      std::vector<CaseResult> r;
      run_cases(*h.problems[idx], {&h.data[idx]}, o, {nullptr}, {nullptr}, &r, now_seconds());
    });
  };
  pass();
  const double t0 = now_seconds();
  pass();
  return work / std::max(now_seconds() - t0, 1e-9);
}

// Candidate worker counts, each run briefly on an even sample of the batch.
int32_t tune_workers(anu_pdhg_packed& h) {
  const int n = static_cast<int>(h.problems.size());
  const int cap = std::min(n, 2 * host_threads());
  int32_t best = 1;
  double best_rate = -1.0;
  for (const int w : {1, 2, 4, 8, 12, 16, 24, 32, 48}) {
    if (w > cap) break;
    const double rate = sample_rate(h, w);
    if (rate > best_rate) {
      best_rate = rate;
      best = w;
    }
  }
  return best;
}

void set_tiles(anu_pdhg_packed& h, int32_t threads) {
  for (auto& p : h.problems) {
    p->dk.set_tile(threads);
    p->dkt.set_tile(threads);
  }
}

// The product tile of every LP of the batch at `w` workers: each tile's
// sample rate twice, alternating, keeping the better; 256 threads must beat
// 128 by kTuneMargin.
int32_t tune_tile(anu_pdhg_packed& h, int w) {
  double rate[2] = {0.0, 0.0};
  for (int rep = 0; rep < 2; ++rep)
    for (int i = 0; i < 2; ++i) {
      set_tiles(h, kTileThreads[i]);
      rate[i] = std::max(rate[i], sample_rate(h, w));
    }
  const int32_t best = rate[1] * (1.0 - kTuneMargin) > rate[0] ? kTileThreads[1] : kTileThreads[0];
  set_tiles(h, best);
  return best;
}

void fill_packed_result(const Problem& p, const CaseResult& cr, double scaling_s, double norm_s,
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

template <class F>
int guarded_packed(F&& body) {
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

using anu::Error;

extern "C" {

int anu_pdhg_packed_create(int32_t num_lps, const anu_lp* lps, const anu_pdhg_options* options,
                           int32_t workers, anu_pdhg_packed** handle) {
  return anu::guarded_packed([&] {
    if (lps == nullptr || options == nullptr || handle == nullptr)
      throw Error(ANU_ERR_INVALID, "null argument");
    *handle = nullptr;
    if (num_lps < 1) throw Error(ANU_ERR_INVALID, "num_lps < 1");
    if (workers < 0) throw Error(ANU_ERR_INVALID, "workers < 0");
    anu::validate_options(*options);
    for (int32_t i = 0; i < num_lps; ++i) {
      const std::string e = anu::validate_lp(lps[i]);
      if (!e.empty()) throw Error(ANU_ERR_INVALID, "invalid LP " + std::to_string(i) + ": " + e);
    }
    auto h = std::make_unique<anu_pdhg_packed>();
    h->options = *options;
    h->problems.resize(num_lps);
    h->data.resize(num_lps);
    h->scaling_seconds.assign(num_lps, 0.0);
    h->norm_seconds.assign(num_lps, 0.0);
    std::vector<int32_t> all(num_lps);
    std::iota(all.begin(), all.end(), 0);
    // Host scaling and upload of every LP, several at a time.
    anu::run_queue(all, anu::host_threads(), [&](int32_t i) {
      h->problems[i] = anu::make_problem(lps[i], *options, &h->scaling_seconds[i],
                                         &h->norm_seconds[i]);
      h->data[i] = anu::make_case(*h->problems[i], lps[i].c, lps[i].q, lps[i].lower,
                                  lps[i].upper, lps[i].objective_scale, lps[i].objective_offset);
    });
    for (const auto& p : h->problems) {
      p->concurrent = true;
      anu::choose_tiles(*p, *options, nullptr);
    }
    h->order = all;
    std::stable_sort(h->order.begin(), h->order.end(), [&](int32_t a, int32_t b) {
      return h->problems[a]->k.nnz() > h->problems[b]->k.nnz();
    });
    h->workers = workers > 0 ? workers : anu::tune_workers(*h);
    if (options->tile_threads == 0) anu::tune_tile(*h, h->workers);
    *handle = h.release();
  });
}

int anu_pdhg_packed_solve(anu_pdhg_packed* h, double* const* x, double* const* y,
                          anu_pdhg_result* results) {
  return anu::guarded_packed([&] {
    if (h == nullptr || results == nullptr) throw Error(ANU_ERR_INVALID, "null argument");
    anu::run_queue(h->order, h->workers, [&](int32_t i) {
      std::vector<anu::CaseResult> r;
      const double start = anu::now_seconds();
      anu::run_cases(*h->problems[i], {&h->data[i]}, h->options, {nullptr}, {nullptr}, &r, start);
      anu::fill_packed_result(*h->problems[i], r[0], h->scaling_seconds[i], h->norm_seconds[i],
                              &results[i]);
      if (x != nullptr && x[i] != nullptr) std::copy(r[0].x.begin(), r[0].x.end(), x[i]);
      if (y != nullptr && y[i] != nullptr) std::copy(r[0].y.begin(), r[0].y.end(), y[i]);
    });
  });
}

int32_t anu_pdhg_packed_workers(const anu_pdhg_packed* h) { return h == nullptr ? 0 : h->workers; }

void anu_pdhg_packed_destroy(anu_pdhg_packed* h) { delete h; }

}  // extern "C"
