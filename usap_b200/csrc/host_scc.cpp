// Initial blocks: the reference's SCC-style initial merge
// (_dfs_itr, graph_parallel.hpp:573-603, then _scc, :514-556).
//
// 1. Iterative DFS over the out-graph, vertices in id order, neighbours in
//    edge order; a vertex is pushed once per unvisited in-edge and finishes
//    when it is popped grey, giving a finish stack.
// 2. Vertices are popped from the finish stack; each unvisited one starts a
//    DFS over the transposed graph (in-lists ordered by source id, as the
//    reference builds them at :518-523) that stops after `dfs_depth`
//    vertices; the vertices it reached form one block.
// Inherently sequential and O(N + E); it runs on the host.
#include <vector>

#include "job.h"

namespace usap {

void scc_prepare(HostGraph& g) {
  if (g.transpose_is_in) return;
  const int32_t n = g.n;
  g.tptr.assign(n + 1, 0);
  g.tidx.resize(g.e);
  for (int64_t i = 0; i < g.e; i++) g.tptr[g.out_idx[i] + 1]++;
  for (int32_t v = 0; v < n; v++) g.tptr[v + 1] += g.tptr[v];
  std::vector<int32_t> fill(g.tptr.begin(), g.tptr.end() - 1);
  for (int32_t i = 0; i < n; i++)
    for (int32_t p = g.out_ptr[i]; p < g.out_ptr[i + 1]; p++) g.tidx[fill[g.out_idx[p]]++] = i;
}

int32_t scc_host(const HostGraph& g, int32_t dfs_depth, int32_t* part) {
  const int32_t n = g.n;
  std::vector<uint8_t> color(n, 0);
  std::vector<int32_t> finish;
  finish.reserve(n);
  std::vector<int32_t> st;
  st.reserve(1024);
  for (int32_t v0 = 0; v0 < n; v0++) {
    if (color[v0]) continue;
    st.push_back(v0);
    while (!st.empty()) {
      int32_t v = st.back();
      if (color[v]) {
        st.pop_back();
        if (color[v] == 1) {
          finish.push_back(v);
          color[v] = 2;
        }
      } else {
        color[v] = 1;
        for (int32_t p = g.out_ptr[v]; p < g.out_ptr[v + 1]; p++) {
          int32_t t = g.out_idx[p];
          if (!color[t]) st.push_back(t);
        }
      }
    }
  }
  const int32_t* tptr = g.transpose_is_in ? g.in_ptr.data() : g.tptr.data();
  const int32_t* tidx = g.transpose_is_in ? g.in_idx.data() : g.tidx.data();
  std::vector<uint8_t> visited(n, 0);
  for (int32_t v = 0; v < n; v++) part[v] = -1;
  int32_t b = 0;
  std::vector<int32_t> st2;
  st2.reserve(256);
  while (!finish.empty()) {
    int32_t v = finish.back();
    finish.pop_back();
    if (visited[v]) continue;
    int32_t i = 0;
    st2.clear();
    st2.push_back(v);
    while (!st2.empty() && i < dfs_depth) {
      int32_t ni = st2.back();
      st2.pop_back();
      if (!visited[ni]) {
        visited[ni] = 1;
        part[ni] = b;
        i++;
        for (int32_t p = tptr[ni]; p < tptr[ni + 1]; p++) {
          int32_t t = tidx[p];
          if (!visited[t]) st2.push_back(t);
        }
      }
    }
    b++;
  }
  return b;
}

}  // namespace usap
