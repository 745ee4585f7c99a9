// Host side of load_graph_from_tsv (graph_parallel.hpp:251-317): the edge
// list in file order becomes out- and in-adjacency lists whose entries keep
// the file order inside each list (:285-290).
//
// Both lists are stable counting sorts of the edges, by source and by
// target.  Large graphs use host threads: every thread counts the keys of
// its slice of the edge list, per-thread offsets follow from the counts in
// slice order, and every thread then scatters its slice in order, so the
// result equals the sequential stable sort.  An edge list already ordered
// by source (the usual TSV layout) is its own out-list, and its in-lists
// are then also ordered by source id, which is the transpose the initial
// SCC walk needs (:518-523), so that copy is skipped.
#include <algorithm>
#include <thread>
#include <utility>
#include <vector>

#include "job.h"

namespace usap {

namespace {

int host_threads(int64_t work) {
  if (work < (1 << 17)) return 1;
  const unsigned hw = std::thread::hardware_concurrency();
  return std::max(1, std::min<int>(16, hw ? static_cast<int>(hw) : 1));
}

template <class F>
void parallel(int T, F&& f) {
  if (T <= 1) {
    f(0);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(T - 1);
  for (int t = 1; t < T; t++) th.emplace_back([&f, t] { f(t); });
  f(0);
  for (auto& x : th) x.join();
}

// stable counting sort of the e edges by key[i] in [0, n): ptr (n + 1),
// idx[k] = val[edge], wout[k] = w[edge] when w is given
void stable_bucket(int32_t n, int64_t e, const int32_t* key, const int32_t* val, const int32_t* w, int T,
                   std::vector<int32_t>& ptr, std::vector<int32_t>& idx, std::vector<int32_t>* wout) {
  const int64_t cap = std::max<int64_t>(1, (int64_t{1} << 25) / (static_cast<int64_t>(n) + 1));
  T = static_cast<int>(std::min<int64_t>(T, cap));
  std::vector<int32_t> cnt(static_cast<size_t>(T) * n, 0);
  auto slice = [&](int t) { return std::make_pair(e * t / T, e * (t + 1) / T); };
  auto vslice = [&](int t) {
    return std::make_pair(static_cast<int32_t>(static_cast<int64_t>(n) * t / T),
                          static_cast<int32_t>(static_cast<int64_t>(n) * (t + 1) / T));
  };
  parallel(T, [&](int t) {
    const auto r = slice(t);
    int32_t* c = cnt.data() + static_cast<size_t>(t) * n;
    for (int64_t i = r.first; i < r.second; i++) c[key[i]]++;
  });
  ptr.assign(static_cast<size_t>(n) + 1, 0);
  parallel(T, [&](int t) {
    const auto r = vslice(t);
    for (int32_t v = r.first; v < r.second; v++) {
      int32_t s = 0;
      for (int u = 0; u < T; u++) s += cnt[static_cast<size_t>(u) * n + v];
      ptr[v + 1] = s;
    }
  });
  for (int32_t v = 0; v < n; v++) ptr[v + 1] += ptr[v];
  parallel(T, [&](int t) {
    const auto r = vslice(t);
    for (int32_t v = r.first; v < r.second; v++) {
      int32_t run = ptr[v];
      for (int u = 0; u < T; u++) {
        int32_t& c = cnt[static_cast<size_t>(u) * n + v];
        const int32_t k = c;
        c = run;
        run += k;
      }
    }
  });
  idx.resize(e);
  if (wout) wout->resize(e);
  parallel(T, [&](int t) {
    const auto r = slice(t);
    int32_t* c = cnt.data() + static_cast<size_t>(t) * n;
    for (int64_t i = r.first; i < r.second; i++) {
      const int32_t p = c[key[i]]++;
      idx[p] = val[i];
      if (wout) (*wout)[p] = w[i];
    }
  });
}

}  // namespace

void build_csr(HostGraph& h) {
  const int32_t n = h.n;
  const int64_t e = h.e;
  const int T = host_threads(e);
  const int32_t* w = h.unit ? nullptr : h.w.data();
  bool by_source = true;
  for (int64_t i = 1; i < e && by_source; i++) by_source = h.src[i - 1] <= h.src[i];
  if (by_source) {
    h.out_ptr.assign(static_cast<size_t>(n) + 1, 0);
    for (int64_t i = 0; i < e; i++) h.out_ptr[h.src[i] + 1]++;
    for (int32_t v = 0; v < n; v++) h.out_ptr[v + 1] += h.out_ptr[v];
    h.out_idx = h.dst;
    if (!h.unit) h.out_w = h.w;
  } else {
    stable_bucket(n, e, h.src.data(), h.dst.data(), w, T, h.out_ptr, h.out_idx, h.unit ? nullptr : &h.out_w);
  }
  stable_bucket(n, e, h.dst.data(), h.src.data(), w, T, h.in_ptr, h.in_idx, h.unit ? nullptr : &h.in_w);
  h.kout.assign(n, 0);
  h.kin.assign(n, 0);
  parallel(std::min(T, std::max(1, n / 4096)), [&](int t) {
    const int Tn = std::min(T, std::max(1, n / 4096));
    const int32_t v0 = static_cast<int32_t>(static_cast<int64_t>(n) * t / Tn);
    const int32_t v1 = static_cast<int32_t>(static_cast<int64_t>(n) * (t + 1) / Tn);
    for (int32_t v = v0; v < v1; v++) {
      if (h.unit) {
        h.kout[v] = h.out_ptr[v + 1] - h.out_ptr[v];
        h.kin[v] = h.in_ptr[v + 1] - h.in_ptr[v];
      } else {
        int32_t so = 0, si = 0;
        for (int32_t p = h.out_ptr[v]; p < h.out_ptr[v + 1]; p++) so += h.out_w[p];
        for (int32_t p = h.in_ptr[v]; p < h.in_ptr[v + 1]; p++) si += h.in_w[p];
        h.kout[v] = so;
        h.kin[v] = si;
      }
    }
  });
  h.transpose_is_in = by_source;
}

}  // namespace usap
