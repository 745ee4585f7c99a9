// Minimal stand-in for the Taskflow API subset that uSAP's
// include/graph_parallel.hpp uses.  Taskflow itself (an un-vendored git
// submodule of the reference, include/taskflow/, commit unrecorded) is absent
// here, so the reference's own sources are compiled against this shim.
//
// It is written from Taskflow's documented semantics, not from its code:
//   * tf::Executor(n)            n worker threads; this_worker_id() in [0, n)
//                                inside work run by the pool, -1 elsewhere;
//   * Executor::run(tf).wait()   runs a graph to completion;
//   * Taskflow::emplace(f)       a static task (void()) or a condition task
//                                (int()); a condition task's successors are
//                                weak: returning i jumps to successor i;
//   * Taskflow::for_each_index(beg, end, step, f)
//                                a parallel loop whose bounds may be
//                                std::ref()'d and are read when it runs;
//   * Task::precede(...), Task::name(...).
// A node becomes ready when all its strong (non-condition) predecessors have
// finished; its join counter is then reset so the graph may loop.  Ready
// static/loop tasks that are independent run in parallel on the pool.
// This is test and baseline infrastructure only.
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>

namespace tf {

class Executor;

namespace shim_detail {

inline thread_local int tl_worker_id = -1;

template <typename T> struct unwrap { static T get(T v) { return v; } };
template <typename T> struct unwrap<std::reference_wrapper<T>> {
  static T get(std::reference_wrapper<T> v) { return v.get(); }
};
template <typename T> auto unwrap_value(T v) { return unwrap<T>::get(v); }

struct Node {
  enum Kind { kStatic, kCondition, kLoop } kind = kStatic;
  std::string name;
  std::function<void()> work;
  std::function<int()> cond;
  std::function<void(Executor&)> loop;
  std::vector<Node*> succ;
  int strong = 0;   // predecessors that are not condition tasks
  int weak = 0;     // predecessors that are condition tasks
  int join = 0;
};

}  // namespace shim_detail

class Task {
 public:
  Task() = default;
  explicit Task(shim_detail::Node* n) : _node(n) {}
  Task& name(const std::string& s) { _node->name = s; return *this; }
  const std::string& name() const { return _node->name; }
  template <typename... Ts>
  Task& precede(Ts&&... tasks) {
    (_add(std::forward<Ts>(tasks)), ...);
    return *this;
  }
 private:
  void _add(const Task& t) {
    _node->succ.push_back(t._node);
    if (_node->kind == shim_detail::Node::kCondition) t._node->weak++;
    else t._node->strong++;
  }
  shim_detail::Node* _node = nullptr;
};

class Taskflow {
 public:
  Taskflow() = default;
  explicit Taskflow(const std::string& name) : _name(name) {}

  template <typename C>
  Task emplace(C&& c) {
    auto n = std::make_unique<shim_detail::Node>();
    using R = std::invoke_result_t<C&>;
    if constexpr (std::is_void_v<R>) {
      n->kind = shim_detail::Node::kStatic;
      n->work = std::function<void()>(std::forward<C>(c));
    } else {
      n->kind = shim_detail::Node::kCondition;
      n->cond = [f = std::forward<C>(c)]() mutable { return static_cast<int>(f()); };
    }
    _nodes.push_back(std::move(n));
    return Task(_nodes.back().get());
  }

  template <typename B, typename E, typename S, typename C>
  Task for_each_index(B beg, E end, S step, C c);

  const std::string& name() const { return _name; }
  std::vector<std::unique_ptr<shim_detail::Node>>& nodes() { return _nodes; }

 private:
  std::string _name;
  std::vector<std::unique_ptr<shim_detail::Node>> _nodes;
};

class Future {
 public:
  void wait() const {}
  void get() const {}
};

class Executor {
 public:
  explicit Executor(size_t n = std::thread::hardware_concurrency())
      : _n(n == 0 ? 1 : n) {
    for (size_t i = 0; i < _n; i++) {
      _threads.emplace_back([this, i] { _worker(static_cast<int>(i)); });
    }
  }
  ~Executor() {
    {
      std::lock_guard<std::mutex> lk(_mu);
      _stop = true;
      _epoch.fetch_add(1, std::memory_order_release);
    }
    _cv.notify_all();
    for (auto& t : _threads) t.join();
  }
  Executor(const Executor&) = delete;
  Executor& operator=(const Executor&) = delete;

  size_t num_workers() const { return _n; }
  int this_worker_id() const { return shim_detail::tl_worker_id; }

  // Runs fn(worker_id) once on every worker and returns when all are done.
  void fork_join(const std::function<void(int)>& fn) {
    if (shim_detail::tl_worker_id >= 0) {   // nested call from a worker: run inline
      fn(shim_detail::tl_worker_id);
      return;
    }
    std::lock_guard<std::mutex> serial(_dispatch_mu);
    _job = &fn;
    _done.store(0, std::memory_order_relaxed);
    {
      std::lock_guard<std::mutex> lk(_mu);
      _epoch.fetch_add(1, std::memory_order_release);
    }
    _cv.notify_all();
    // the caller spins briefly, then yields, until every worker reports back
    size_t spins = 0;
    while (_done.load(std::memory_order_acquire) != _n) {
      if (++spins > 2000) std::this_thread::yield();
    }
    _job = nullptr;
  }

  // Parallel loop over [b, e) with the given step, dynamic chunks.
  template <typename F>
  void parallel_for(long b, long e, long step, F&& f) {
    if (step == 0 || (step > 0 && b >= e) || (step < 0 && b <= e)) return;
    long count = step > 0 ? (e - b + step - 1) / step : (b - e + (-step) - 1) / (-step);
    long chunk = count / (static_cast<long>(_n) * 8);
    if (chunk < 1) chunk = 1;
    std::atomic<long> next{0};
    fork_join([&](int) {
      while (true) {
        long k0 = next.fetch_add(chunk, std::memory_order_relaxed);
        if (k0 >= count) break;
        long k1 = k0 + chunk < count ? k0 + chunk : count;
        for (long k = k0; k < k1; k++) f(b + k * step);
      }
    });
  }

  Future run(Taskflow& flow) {
    using shim_detail::Node;
    auto& nodes = flow.nodes();
    std::deque<Node*> ready;
    for (auto& n : nodes) {
      n->join = n->strong;
      if (n->strong == 0 && n->weak == 0) ready.push_back(n.get());
    }
    auto finish = [&](Node* n, int branch) {
      n->join = n->strong;
      if (n->kind == Node::kCondition) {
        if (branch >= 0 && branch < static_cast<int>(n->succ.size())) {
          ready.push_back(n->succ[branch]);
        }
      } else {
        for (Node* s : n->succ) {
          if (--s->join == 0) ready.push_back(s);
        }
      }
    };
    while (!ready.empty()) {
      // independent static tasks that are ready together run in parallel
      std::vector<Node*> statics;
      while (!ready.empty() && ready.front()->kind == Node::kStatic) {
        statics.push_back(ready.front());
        ready.pop_front();
      }
      if (statics.size() == 1) {
        statics[0]->work();
        finish(statics[0], -1);
        continue;
      }
      if (statics.size() > 1) {
        parallel_for(0, static_cast<long>(statics.size()), 1,
                     [&](long i) { statics[i]->work(); });
        for (Node* n : statics) finish(n, -1);
        continue;
      }
      Node* n = ready.front();
      ready.pop_front();
      if (n->kind == Node::kCondition) {
        int r = n->cond();
        finish(n, r);
      } else {
        n->loop(*this);
        finish(n, -1);
      }
    }
    return Future{};
  }

 private:
  void _worker(int id) {
    shim_detail::tl_worker_id = id;
    uint64_t seen = 0;
    while (true) {
      // spin briefly on the epoch before sleeping, so tight loops stay cheap
      size_t spins = 0;
      uint64_t cur = _epoch.load(std::memory_order_acquire);
      while (cur == seen && spins < 20000) {
        ++spins;
        cur = _epoch.load(std::memory_order_acquire);
      }
      if (cur == seen) {
        std::unique_lock<std::mutex> lk(_mu);
        _cv.wait(lk, [&] { return _epoch.load(std::memory_order_acquire) != seen; });
        cur = _epoch.load(std::memory_order_acquire);
      }
      seen = cur;
      if (_stop) return;
      const std::function<void(int)>* job = _job;
      if (job) (*job)(id);
      _done.fetch_add(1, std::memory_order_acq_rel);
    }
  }

  size_t _n;
  std::vector<std::thread> _threads;
  std::mutex _mu;
  std::mutex _dispatch_mu;
  std::condition_variable _cv;
  std::atomic<uint64_t> _epoch{0};
  std::atomic<size_t> _done{0};
  const std::function<void(int)>* volatile _job = nullptr;
  std::atomic<bool> _stop{false};
};

template <typename B, typename E, typename S, typename C>
Task Taskflow::for_each_index(B beg, E end, S step, C c) {
  auto n = std::make_unique<shim_detail::Node>();
  n->kind = shim_detail::Node::kLoop;
  n->loop = [beg, end, step, c](Executor& ex) mutable {
    long b = static_cast<long>(shim_detail::unwrap_value(beg));
    long e = static_cast<long>(shim_detail::unwrap_value(end));
    long s = static_cast<long>(shim_detail::unwrap_value(step));
    ex.parallel_for(b, e, s, [&](long i) { c(static_cast<int>(i)); });
  };
  _nodes.push_back(std::move(n));
  return Task(_nodes.back().get());
}

}  // namespace tf
