// extern "C" entry points (include/usap.h).  Errors never escape as C++
// exceptions: each call returns a status and records a message for the
// calling thread.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/usap.h"
#include "job.h"

struct usap_ctx {
  std::unique_ptr<usap::Job> job;
};

namespace {

thread_local std::string g_last_error;

template <class F>
usap_status guarded(F&& f) {
  try {
    f();
    g_last_error.clear();
    return USAP_OK;
  } catch (const usap::Error& e) {
    g_last_error = e.what();
    return e.code();
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return USAP_ERR_OOM;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return USAP_ERR_INTERNAL;
  }
}

// Solver states kept for usap_partition: creating one (streams, events,
// pinned control buffers) costs milliseconds, which a one-shot solve would
// otherwise pay on every call.  At most kIdleJobs idle states per device.
constexpr size_t kIdleJobs = 4;
// The idle states are never destroyed: at process exit the CUDA runtime may
// already be gone.
std::mutex g_idle_mu;
std::vector<std::unique_ptr<usap::Job>>* const g_idle = new std::vector<std::unique_ptr<usap::Job>>[64];

std::unique_ptr<usap::Job> acquire_job(int device) {
  if (device >= 0 && device < 64) {
    std::lock_guard<std::mutex> lk(g_idle_mu);
    if (!g_idle[device].empty()) {
      std::unique_ptr<usap::Job> j = std::move(g_idle[device].back());
      g_idle[device].pop_back();
      return j;
    }
  }
  return std::make_unique<usap::Job>(device);
}

void release_job(std::unique_ptr<usap::Job> j) {
  const int device = j->device();
  j->detach();
  if (device < 0 || device >= 64) return;
  std::lock_guard<std::mutex> lk(g_idle_mu);
  if (g_idle[device].size() < kIdleJobs) g_idle[device].push_back(std::move(j));
}

void check_ctx(usap_ctx* ctx) {
  if (!ctx || !ctx->job) throw usap::Error(USAP_ERR_INVALID, "null context");
}

}  // namespace

int usap::call_guarded(const std::function<void()>& f) { return guarded(f); }

extern "C" {

const char* usap_version(void) { return "usap-b200 0.1 (sm_100a)"; }

const char* usap_last_error(void) { return g_last_error.c_str(); }

void usap_params_default(usap_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->beta = 3;
  p->block_size = 1024;
  p->num_agg_proposals_per_block = 10;
  p->num_block_reduction_rate = 0.5f;
  p->max_num_nodal_itr = 100;
  p->num_batch_nodal_update = 4;
  p->delta_entropy_threshold1 = 5e-4;
  p->delta_entropy_threshold2 = 1e-4;
  p->delta_entropy_moving_avg_window = 3;
  p->verbose = 0;
  p->dfs_depth = 20;
  p->t_block_num = 20;
  p->seed = 0;
  p->init_mode = 0;
  p->dense_max = 0;   // automatic: 4096, or 16384 with the float nodal dS (effective_dense_max)
  p->device = 0;
  p->stats = 0;
  p->persistent = 1;
  p->precision = 3;   // the reference's own float nodal dS (graph_parallel.hpp:1066-1215)
}

usap_status usap_partition(const usap_graph* g, const usap_params* p, int32_t* out_assign,
                           usap_result* out) {
  return guarded([&] {
    if (!g || !out_assign || !out) throw usap::Error(USAP_ERR_INVALID, "null argument");
    usap_params def;
    usap_params_default(&def);
    const usap_params& prm = p ? *p : def;
    std::unique_ptr<usap::Job> job = acquire_job(prm.device);
    const auto lc0 = usap::launch_count();
    job->load(*g);
    job->partition(prm, out_assign, out);
    out->ms_h2d = job->last_h2d_ms();
    out->h2d_bytes += job->last_h2d_bytes();
    out->kernel_launches = usap::launch_count().kernels - lc0.kernels;
    out->cub_calls = usap::launch_count().cub - lc0.cub;
    release_job(std::move(job));
  });
}

usap_status usap_evaluate(const int32_t* truth, const int32_t* given, int64_t n, usap_scores* out) {
  return guarded([&] {
    if (!truth || !given || !out) throw usap::Error(USAP_ERR_INVALID, "null argument");
    usap::evaluate_host(truth, given, n, out);
  });
}

usap_status usap_ctx_create(int32_t device, usap_ctx** out) {
  return guarded([&] {
    if (!out) throw usap::Error(USAP_ERR_INVALID, "null argument");
    *out = nullptr;
    auto ctx = std::make_unique<usap_ctx>();
    ctx->job = std::make_unique<usap::Job>(device);
    *out = ctx.release();
  });
}

usap_status usap_ctx_destroy(usap_ctx* ctx) {
  return guarded([&] { delete ctx; });
}

usap_status usap_ctx_load(usap_ctx* ctx, const usap_graph* g) {
  return guarded([&] {
    check_ctx(ctx);
    if (!g) throw usap::Error(USAP_ERR_INVALID, "null graph");
    ctx->job->load(*g);
  });
}

usap_status usap_ctx_load_tsv(usap_ctx* ctx, const char* text, int64_t len, int32_t n) {
  return guarded([&] {
    check_ctx(ctx);
    if (!text && len > 0) throw usap::Error(USAP_ERR_INVALID, "null text");
    if (n < 0) throw usap::Error(USAP_ERR_INVALID, "n must be >= 0");
    // parse and adjacency lists on the device; the host keeps a copy of the
    // lists for its own passes (initial blocks, work units)
    usap::HostGraph h;
    usap::TsvEdges t = usap::parse_tsv_device(ctx->job->device(), text ? text : "", len, n, &h);
    if (t.src.empty()) throw usap::Error(USAP_ERR_INVALID, "graph needs at least one edge");
    ctx->job->load_host(std::move(h));
  });
}

usap_status usap_ctx_num_nodes(usap_ctx* ctx, int32_t* n, int64_t* e) {
  return guarded([&] {
    check_ctx(ctx);
    if (n) *n = ctx->job->host_graph().n;
    if (e) *e = ctx->job->host_graph().e;
  });
}

usap_status usap_ctx_partition(usap_ctx* ctx, const usap_params* p, int32_t* out_assign,
                               usap_result* out) {
  return guarded([&] {
    check_ctx(ctx);
    if (!out) throw usap::Error(USAP_ERR_INVALID, "null result");
    usap_params def;
    usap_params_default(&def);
    ctx->job->partition(p ? *p : def, out_assign, out);
  });
}

usap_status usap_ctx_partition_from(usap_ctx* ctx, const usap_params* p, const int32_t* init,
                                    int32_t* out_assign, usap_result* out) {
  return guarded([&] {
    check_ctx(ctx);
    if (!init || !out) throw usap::Error(USAP_ERR_INVALID, "null argument");
    usap_params def;
    usap_params_default(&def);
    ctx->job->partition(p ? *p : def, out_assign, out, init);
  });
}

usap_status usap_ctx_add_edges(usap_ctx* ctx, const usap_graph* g) {
  return guarded([&] {
    check_ctx(ctx);
    if (!g) throw usap::Error(USAP_ERR_INVALID, "null graph");
    ctx->job->add_edges(*g);
  });
}

usap_status usap_ctx_evaluate(usap_ctx* ctx, const int32_t* truth, usap_scores* out) {
  return guarded([&] {
    check_ctx(ctx);
    if (!truth || !out) throw usap::Error(USAP_ERR_INVALID, "null argument");
    ctx->job->evaluate_last(truth, out);
  });
}

usap_status usap_evaluate_device(const int32_t* truth, const int32_t* given, int64_t n, int32_t device,
                                 usap_scores* out) {
  return guarded([&] {
    if (!truth || !given || !out) throw usap::Error(USAP_ERR_INVALID, "null argument");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
      throw usap::Error(USAP_ERR_NO_DEVICE, "no CUDA device available");
    if (device < 0 || device >= count) throw usap::Error(USAP_ERR_INVALID, "device index out of range");
    usap::evaluate_device(truth, given, n, device, out);
  });
}

usap_status usap_ctx_set_trace(usap_ctx* ctx, usap_trace_fn fn, void* user) {
  return guarded([&] {
    check_ctx(ctx);
    ctx->job->set_trace(fn, user);
  });
}

usap_status usap_ctx_adjacency(usap_ctx* ctx, int32_t* out_ptr, int32_t* out_idx, int32_t* out_w,
                               int32_t* in_ptr, int32_t* in_idx, int32_t* in_w, int32_t* kout, int32_t* kin) {
  return guarded([&] {
    check_ctx(ctx);
    const usap::HostGraph& h = ctx->job->host_graph();
    auto copy = [](int32_t* dst, const std::vector<int32_t>& v) {
      if (dst && !v.empty()) std::memcpy(dst, v.data(), sizeof(int32_t) * v.size());
    };
    auto weights = [&](int32_t* dst, const std::vector<int32_t>& v) {
      if (!dst) return;
      if (h.unit) std::fill(dst, dst + h.e, 1);
      else copy(dst, v);
    };
    copy(out_ptr, h.out_ptr);
    copy(out_idx, h.out_idx);
    weights(out_w, h.out_w);
    copy(in_ptr, h.in_ptr);
    copy(in_idx, h.in_idx);
    weights(in_w, h.in_w);
    copy(kout, h.kout);
    copy(kin, h.kin);
  });
}

usap_status usap_ctx_test_barrier_timeout(usap_ctx* ctx, int32_t hold_cta, int64_t timeout_ns) {
  return guarded([&] {
    check_ctx(ctx);
    if (hold_cta < 0) throw usap::Error(USAP_ERR_INVALID, "hold_cta must be >= 0");
    if (timeout_ns <= 0 || timeout_ns > 10000000000ll)
      throw usap::Error(USAP_ERR_INVALID, "timeout_ns must be in (0, 10 s]");
    ctx->job->arm_barrier_test(hold_cta, static_cast<unsigned long long>(timeout_ns));
  });
}

usap_status usap_batch_partition(const usap_graph* graphs, int32_t ngraphs, const usap_params* p,
                                 usap_batch_job* jobs, int32_t njobs, int32_t workers,
                                 int32_t device, usap_batch_stats* stats) {
  return guarded([&] {
    if (!graphs || ngraphs <= 0 || !jobs || njobs < 0) throw usap::Error(USAP_ERR_INVALID, "bad batch");
    for (int32_t j = 0; j < njobs; j++)
      if (jobs[j].graph < 0 || jobs[j].graph >= ngraphs)
        throw usap::Error(USAP_ERR_INVALID, "job names a graph outside the batch");
    usap_params def;
    usap_params_default(&def);
    const usap_params base = p ? *p : def;
    auto t0 = std::chrono::steady_clock::now();
    int hw = static_cast<int>(std::thread::hardware_concurrency());
    if (hw <= 0) hw = 8;
    // dense nodal phases of the concurrent solves run together in gang
    // launches; solves mostly wait there, so more of them than host threads
    std::unique_ptr<usap::NodalGang> gang;
    USAP_CUDA(cudaSetDevice(device));
    if (usap::nodal_gang_grid(device) > 0) gang = std::make_unique<usap::NodalGang>(device);
    int W = workers > 0 ? workers : (gang ? usap::kGangMax : std::min(32, 2 * hw));
    W = std::max(1, std::min(W, std::max(njobs, ngraphs)));
    // load every graph once, in parallel
    std::vector<std::shared_ptr<usap::GraphResident>> res(ngraphs);
    std::vector<std::string> load_err(ngraphs);
    {
      std::atomic<int32_t> next{0};
      std::vector<std::thread> th;
      for (int w = 0; w < std::min(W, static_cast<int>(ngraphs)); w++)
        th.emplace_back([&] {
          for (int32_t i = next++; i < ngraphs; i = next++) {
            try {
              res[i] = usap::load_graph(device, graphs[i]);
            } catch (const std::exception& e) {
              load_err[i] = e.what();
            }
          }
        });
      for (auto& t : th) t.join();
    }
    for (int32_t i = 0; i < ngraphs; i++)
      if (!res[i]) throw usap::Error(USAP_ERR_INVALID, "graph " + std::to_string(i) + ": " + load_err[i]);
    auto t1 = std::chrono::steady_clock::now();
    // largest graphs first (shortest makespan for a greedy pool)
    std::vector<int32_t> order(njobs);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
      return res[jobs[a].graph]->hg.e > res[jobs[b].graph]->hg.e;
    });
    // the first W solves (the largest graphs) would otherwise grow the memory
    // pool while other solves' kernels run, which is slow: reserve it now
    {
      int64_t want = 0;
      const int64_t dmax = usap::effective_dense_max(base);
      for (int32_t k = 0; k < std::min<int32_t>(W, njobs); k++) {
        const usap::HostGraph& hg = res[jobs[order[k]].graph]->hg;
        // initial blocks: one per vertex, or about N/7 from the SCC pass
        const int64_t b0 = base.init_mode == 1 ? hg.n : std::max<int64_t>(1, hg.n / 4);
        want += usap::solve_footprint_bytes(hg.n, hg.e, std::min<int64_t>(dmax, b0), !hg.unit, base.precision == 3);
      }
      usap::pool_reserve(device, want);
    }
    std::atomic<int32_t> next{0};
    std::atomic<long long> launches{0};
    std::vector<std::thread> th;
    for (int w = 0; w < std::min(W, std::max<int32_t>(njobs, 1)); w++)
      th.emplace_back([&] {
        const auto lc0 = usap::launch_count();
        std::unique_ptr<usap::Job> job;
        try {
          job = std::make_unique<usap::Job>(device);
        } catch (const std::exception&) {
          job.reset();
        }
        for (int32_t k = next++; k < njobs; k = next++) {
          usap_batch_job& bj = jobs[order[k]];
          if (!job) {
            bj.status = USAP_ERR_CUDA;
            continue;
          }
          struct GangSeat {   // counts this solve as in progress for the gang
            usap::NodalGang* g;
            explicit GangSeat(usap::NodalGang* gg) : g(gg) { if (g) g->enter(); }
            ~GangSeat() { if (g) g->leave(); }
          } seat(gang.get());
          try {
            job->set_gang(gang.get());
            job->attach(res[bj.graph]);
            usap_params prm = base;
            prm.persistent = 0;   // concurrent jobs: per-batch launches interleave
            prm.seed = bj.seed;
            job->partition(prm, bj.out_assign, &bj.result);
            bj.status = USAP_OK;
          } catch (const usap::Error& e) {
            bj.status = e.code();
          } catch (const std::exception&) {
            bj.status = USAP_ERR_INTERNAL;
          }
        }
        job.reset();
        launches += usap::launch_count().kernels - lc0.kernels;
      });
    for (auto& t : th) t.join();
    res.clear();
    if (stats) {
      stats->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      stats->ms_load = std::chrono::duration<double, std::milli>(t1 - t0).count();
      stats->workers = W;
      stats->kernel_launches = launches.load();
      stats->gang_launches = gang ? gang->launches() : 0;
      stats->gang_phases = gang ? gang->phases() : 0;
      stats->ms_gang = gang ? gang->ms() : 0.0;
    }
    for (int32_t j = 0; j < njobs; j++)
      if (jobs[j].status != USAP_OK) throw usap::Error(jobs[j].status, "a batch job failed");
  });
}

usap_status usap_op_scc(usap_ctx* ctx, int32_t dfs_depth, int32_t* part, int32_t* B) {
  return guarded([&] {
    check_ctx(ctx);
    if (!part || !B) throw usap::Error(USAP_ERR_INVALID, "null argument");
    *B = ctx->job->op_scc(dfs_depth, part);
  });
}

static void check_part(usap_ctx* ctx, const int32_t* part, int32_t B) {
  if (!part) throw usap::Error(USAP_ERR_INVALID, "null partition");
  const auto& hg = ctx->job->host_graph();
  if (hg.n <= 0) throw usap::Error(USAP_ERR_STATE, "no graph loaded");
  if (B < 1) throw usap::Error(USAP_ERR_INVALID, "B must be >= 1");
  for (int32_t v = 0; v < hg.n; v++)
    if (part[v] < 0 || part[v] >= B) throw usap::Error(USAP_ERR_INVALID, "block id out of range");
}

usap_status usap_op_build(usap_ctx* ctx, const int32_t* part, int32_t B, int32_t dense_max,
                          int32_t* M, int32_t* dout, int32_t* din) {
  return guarded([&] {
    check_ctx(ctx);
    check_part(ctx, part, B);
    if (!dout || !din) throw usap::Error(USAP_ERR_INVALID, "null degree buffer");
    ctx->job->op_build(part, B, dense_max > 0 ? dense_max : 4096, M, dout, din);
  });
}

usap_status usap_op_entropy(usap_ctx* ctx, const int32_t* part, int32_t B, int32_t dense_max,
                            int64_t* S_q) {
  return guarded([&] {
    check_ctx(ctx);
    check_part(ctx, part, B);
    if (!S_q) throw usap::Error(USAP_ERR_INVALID, "null output");
    *S_q = ctx->job->op_entropy(part, B, dense_max > 0 ? dense_max : 4096);
  });
}

usap_status usap_op_merge_phase(usap_ctx* ctx, const int32_t* part, int32_t B, int32_t K,
                                int32_t stage, uint64_t seed, int32_t* best_s, int64_t* best_q,
                                int32_t* prop_s, int64_t* prop_q) {
  return guarded([&] {
    check_ctx(ctx);
    check_part(ctx, part, B);
    if (!best_s || !best_q) throw usap::Error(USAP_ERR_INVALID, "null output");
    ctx->job->op_merge_phase(part, B, K, stage, seed, best_s, best_q, prop_s, prop_q);
  });
}

usap_status usap_op_merge_apply(usap_ctx* ctx, int32_t* part, int32_t B, const int32_t* best_s,
                                const int64_t* best_q, int32_t b_to_merge, int32_t* B_new,
                                int32_t* merged) {
  return guarded([&] {
    check_ctx(ctx);
    check_part(ctx, part, B);
    if (!best_s || !best_q || !B_new || !merged) throw usap::Error(USAP_ERR_INVALID, "null argument");
    ctx->job->op_merge_apply(part, B, best_s, best_q, b_to_merge, B_new, merged);
  });
}

usap_status usap_op_nodal_batch(usap_ctx* ctx, int32_t* part, int32_t B, int32_t dense_max,
                                int32_t beg, int32_t end, int32_t itr, int32_t stage,
                                uint64_t seed, int32_t* prop_s, int64_t* prop_q,
                                int32_t* prop_ninf, int64_t* cum_q, int32_t* cum_ninf,
                                int64_t* moves) {
  return guarded([&] {
    check_ctx(ctx);
    check_part(ctx, part, B);
    ctx->job->op_nodal_batch(part, B, dense_max > 0 ? dense_max : 4096, beg, end, itr, stage, seed,
                             prop_s, prop_q, prop_ninf, cum_q, cum_ninf, moves);
  });
}

usap_status usap_op_merge_phase_prec(usap_ctx* ctx, const int32_t* part, int32_t B, int32_t K,
                                     int32_t stage, uint64_t seed, int32_t precision, int32_t* best_s,
                                     int64_t* best_q, int32_t* prop_s, int64_t* prop_q, double* prop_f,
                                     int64_t* flips) {
  return guarded([&] {
    check_ctx(ctx);
    check_part(ctx, part, B);
    if (!best_s || !best_q) throw usap::Error(USAP_ERR_INVALID, "null output");
    // the path a solve takes at this B: the dense tile up to 4096 blocks
    ctx->job->op_merge_phase(part, B, K, stage, seed, best_s, best_q, prop_s, prop_q, precision, prop_f, flips,
                             4096);
  });
}

usap_status usap_op_nodal_batch_prec(usap_ctx* ctx, int32_t* part, int32_t B, int32_t dense_max,
                                     int32_t beg, int32_t end, int32_t itr, int32_t stage,
                                     uint64_t seed, int32_t precision, int32_t* prop_s, int64_t* prop_q,
                                     double* prop_f, int32_t* prop_ninf, int64_t* cum_q, int32_t* cum_ninf,
                                     int64_t* moves, int64_t* flips) {
  return guarded([&] {
    check_ctx(ctx);
    check_part(ctx, part, B);
    ctx->job->op_nodal_batch(part, B, dense_max > 0 ? dense_max : 4096, beg, end, itr, stage, seed,
                             prop_s, prop_q, prop_ninf, cum_q, cum_ninf, moves, precision, prop_f, flips);
  });
}

}  // extern "C"
