// Served form: a partition service on one GPU.
//
// Requests arrive at any time (usap_server_submit copies the edge list and
// returns a ticket at once).  A fixed set of worker threads, each owning a
// solver state with its own CUDA streams, takes requests in arrival order
// as soon as a worker is free and the request's device-memory footprint
// fits in what the running requests leave of the budget; requests that
// arrive while others run are admitted the moment a slot and memory free
// up, and their kernels overlap those of the running requests on the
// device.  Each request's graph, partition slots and block structures stay
// resident for all its golden-section stages.  A request's result does not
// depend on what else runs: the solve is deterministic in its inputs and
// seed.  Completion is read with usap_server_poll / usap_server_wait.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/usap.h"
#include "job.h"

namespace usap {
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t ticket = 0;
  std::vector<int32_t> src, dst, w;
  usap_graph g{};
  usap_params params{};
  int32_t* out_assign = nullptr;
  int64_t bytes = 0;
  usap_result result{};
  int status = USAP_OK;
  std::string error;
  bool done = false;
  Clock::time_point submitted, started, finished;
};

}  // namespace

// Upper estimate of the device memory one solve of a graph with n vertices
// and e edges holds: the graph (edge list, both adjacency lists, edge
// chunks, log table), the partition slots and per-vertex state, the sorted
// views' sort buffers, the dense tile for B <= dense_max, and with the
// float nodal dS its per-batch term tables (two floats per cell, B <= 4096).
int64_t solve_footprint_bytes(int64_t n, int64_t e, int64_t dense_max, bool weighted, bool float_ds) {
  const int64_t d = std::min(n, std::max<int64_t>(dense_max, 1));
  const int64_t graph = (weighted ? 48 : 32) * e + 64 * n + 8 * (e + 1);
  const int64_t state = 72 * n + 160 * n + 112 * e;
  const int64_t tile = 8 * (d + 4) * (d + 4) + 4 * d * ((d + 127) / 128 + 1);
  const int64_t dt = std::min<int64_t>(d, 4096);
  const int64_t tables = float_ds ? 8 * (dt + 4) * (dt + 4) : 0;
  return graph + state + tile + tables + (8ll << 20);
}

class Server {
 public:
  Server(const usap_server_config& cfg) : device_(cfg.device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
      throw Error(USAP_ERR_NO_DEVICE, "no CUDA device available");
    if (device_ < 0 || device_ >= count) throw Error(USAP_ERR_INVALID, "device index out of range");
    USAP_CUDA(cudaSetDevice(device_));
    size_t free_b = 0, total_b = 0;
    USAP_CUDA(cudaMemGetInfo(&free_b, &total_b));
    budget_ = cfg.memory_budget > 0 ? cfg.memory_budget : static_cast<int64_t>(0.8 * static_cast<double>(free_b));
    int hw = static_cast<int>(std::thread::hardware_concurrency());
    if (hw <= 0) hw = 8;
    const int nw = cfg.workers > 0 ? cfg.workers : std::min(32, 2 * hw);
    // the solver states are created up front, so that a missing or
    // unusable device fails here and not in a worker
    std::vector<std::unique_ptr<Job>> states;
    for (int i = 0; i < nw; i++) states.push_back(std::make_unique<Job>(device_));
    for (int i = 0; i < nw; i++) {
      workers_.emplace_back([this, st = states[i].release()] {
        std::unique_ptr<Job> job(st);
        work(job.get());
      });
    }
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stopping_ = true;
    }
    cv_work_.notify_all();
    for (auto& t : workers_) t.join();
  }

  int64_t submit(const usap_graph& g, const usap_params& p, int32_t* out_assign) {
    if (!g.src || !g.dst || g.e <= 0) throw Error(USAP_ERR_INVALID, "graph needs at least one edge");
    if (!out_assign) throw Error(USAP_ERR_INVALID, "null output");
    auto r = std::make_shared<Request>();
    r->src.assign(g.src, g.src + g.e);
    r->dst.assign(g.dst, g.dst + g.e);
    if (g.weight) r->w.assign(g.weight, g.weight + g.e);
    r->g = g;
    r->g.src = r->src.data();
    r->g.dst = r->dst.data();
    r->g.weight = g.weight ? r->w.data() : nullptr;
    r->params = p;
    r->params.persistent = 0;   // the cooperative kernel would hold every SM
    r->out_assign = out_assign;
    int64_t n = g.n;
    if (n <= 0) {
      const int32_t base = g.one_based ? 1 : 0;
      int64_t m = -1;
      // the largest id over both endpoints, as Job::load sizes the graph
      for (int64_t i = 0; i < g.e; i++)
        m = std::max<int64_t>(m, static_cast<int64_t>(std::max(g.src[i], g.dst[i])) - base);
      n = m + 1;
    }
    r->bytes = solve_footprint_bytes(n, g.e, effective_dense_max(p), g.weight != nullptr, p.precision == 3);
    if (r->bytes > budget_)
      throw Error(USAP_ERR_LIMIT, "request needs about " + std::to_string(r->bytes >> 20) +
                                      " MiB of device memory, more than the server's budget of " +
                                      std::to_string(budget_ >> 20) + " MiB");
    r->submitted = Clock::now();
    {
      std::lock_guard<std::mutex> lk(mu_);
      r->ticket = next_ticket_++;
      requests_[r->ticket] = r;
      queue_.push_back(r);
    }
    cv_work_.notify_all();
    return r->ticket;
  }

  // true when finished; then copies out the result and forgets the request
  // (a failed request sets *finished and throws its error)
  bool take(int64_t ticket, bool block, usap_result* result, usap_server_timing* timing, int32_t* finished) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = requests_.find(ticket);
    if (it == requests_.end()) throw Error(USAP_ERR_INVALID, "unknown ticket " + std::to_string(ticket));
    std::shared_ptr<Request> r = it->second;
    if (block) cv_done_.wait(lk, [&] { return r->done; });
    if (!r->done) return false;
    // another thread waiting on the same ticket may have taken it meanwhile
    if (requests_.erase(ticket) == 0) throw Error(USAP_ERR_INVALID, "ticket " + std::to_string(ticket) + " was already taken");
    lk.unlock();
    if (timing) {
      auto ms = [](Clock::time_point a, Clock::time_point b) {
        return std::chrono::duration<double, std::milli>(b - a).count();
      };
      timing->ms_queued = ms(r->submitted, r->started);
      timing->ms_running = ms(r->started, r->finished);
      timing->ms_latency = ms(r->submitted, r->finished);
    }
    if (finished) *finished = 1;
    if (r->status != USAP_OK) throw Error(r->status, r->error);
    if (result) *result = r->result;
    return true;
  }

  void stats(usap_server_stats* s) {
    std::lock_guard<std::mutex> lk(mu_);
    s->queued = static_cast<int32_t>(queue_.size());
    s->running = running_;
    s->workers = static_cast<int32_t>(workers_.size());
    s->completed = completed_;
    s->failed = failed_;
    s->admitted_bytes = admitted_;
    s->peak_admitted_bytes = peak_admitted_;
    s->peak_running = peak_running_;
    s->memory_budget = budget_;
  }

 private:
  void work(Job* job) {
    for (;;) {
      std::shared_ptr<Request> r;
      {
        std::unique_lock<std::mutex> lk(mu_);
        // arrival order; the oldest waiting request goes first as soon as
        // its footprint fits in the budget left by the running ones
        cv_work_.wait(lk, [&] {
          return (stopping_ && queue_.empty()) || (!queue_.empty() && admitted_ + queue_.front()->bytes <= budget_);
        });
        if (queue_.empty()) return;
        r = queue_.front();
        queue_.pop_front();
        admitted_ += r->bytes;
        running_++;
        peak_admitted_ = std::max(peak_admitted_, admitted_);
        peak_running_ = std::max(peak_running_, running_);
        r->started = Clock::now();
      }
      try {
        job->load(r->g);
        job->partition(r->params, r->out_assign, &r->result);
        r->result.ms_h2d = job->last_h2d_ms();
        r->result.h2d_bytes += job->last_h2d_bytes();
        r->status = USAP_OK;
      } catch (const Error& e) {
        r->status = e.code();
        r->error = e.what();
      } catch (const std::exception& e) {
        r->status = USAP_ERR_INTERNAL;
        r->error = e.what();
      }
      try {
        job->detach();
      } catch (const std::exception&) {
      }
      r->src.clear();
      r->src.shrink_to_fit();
      r->dst.clear();
      r->dst.shrink_to_fit();
      r->w.clear();
      r->w.shrink_to_fit();
      {
        std::lock_guard<std::mutex> lk(mu_);
        r->finished = Clock::now();
        r->done = true;
        admitted_ -= r->bytes;
        running_--;
        if (r->status == USAP_OK) completed_++;
        else failed_++;
      }
      cv_done_.notify_all();
      cv_work_.notify_all();
    }
  }

  int device_;
  int64_t budget_ = 0;
  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  std::deque<std::shared_ptr<Request>> queue_;
  std::unordered_map<int64_t, std::shared_ptr<Request>> requests_;
  std::vector<std::thread> workers_;
  int64_t next_ticket_ = 1;
  int64_t admitted_ = 0, peak_admitted_ = 0;
  int32_t running_ = 0, peak_running_ = 0;
  int64_t completed_ = 0, failed_ = 0;
  bool stopping_ = false;
};

}  // namespace usap

struct usap_server {
  std::unique_ptr<usap::Server> impl;
};

extern "C" {

void usap_server_config_default(usap_server_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
}

usap_status usap_server_create(const usap_server_config* cfg, usap_server** out) {
  return usap::call_guarded([&] {
    if (!out) throw usap::Error(USAP_ERR_INVALID, "null output");
    *out = nullptr;
    usap_server_config def;
    usap_server_config_default(&def);
    auto s = std::make_unique<usap_server>();
    s->impl = std::make_unique<usap::Server>(cfg ? *cfg : def);
    *out = s.release();
  });
}

void usap_server_destroy(usap_server* s) { delete s; }

usap_status usap_server_submit(usap_server* s, const usap_graph* g, const usap_params* p, int32_t* out_assign,
                               int64_t* ticket) {
  return usap::call_guarded([&] {
    if (!s || !s->impl || !g || !ticket) throw usap::Error(USAP_ERR_INVALID, "null argument");
    usap_params def;
    usap_params_default(&def);
    *ticket = s->impl->submit(*g, p ? *p : def, out_assign);
  });
}

usap_status usap_server_poll(usap_server* s, int64_t ticket, int32_t* done, usap_result* result,
                             usap_server_timing* timing) {
  return usap::call_guarded([&] {
    if (!s || !s->impl || !done) throw usap::Error(USAP_ERR_INVALID, "null argument");
    *done = 0;
    s->impl->take(ticket, false, result, timing, done);
  });
}

usap_status usap_server_wait(usap_server* s, int64_t ticket, usap_result* result, usap_server_timing* timing) {
  return usap::call_guarded([&] {
    if (!s || !s->impl) throw usap::Error(USAP_ERR_INVALID, "null server");
    s->impl->take(ticket, true, result, timing, nullptr);
  });
}

usap_status usap_server_get_stats(usap_server* s, usap_server_stats* out) {
  return usap::call_guarded([&] {
    if (!s || !s->impl || !out) throw usap::Error(USAP_ERR_INVALID, "null argument");
    s->impl->stats(out);
  });
}

}  // extern "C"
