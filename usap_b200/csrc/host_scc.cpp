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
  const int32_t* tptr = g.transpose_is_in ? g.in_ptr.data() : g.tptr.data();
  const int32_t* tidx = g.transpose_is_in ? g.in_idx.data() : g.tidx.data();
  return scc_arrays(g.n, g.e, g.out_ptr.data(), g.out_idx.data(), tptr, tidx, dfs_depth, part);
}

int32_t scc_arrays(int32_t n, int64_t e, const int32_t* optr, const int32_t* oidx, const int32_t* tptr,
                   const int32_t* tidx, int32_t dfs_depth, int32_t* part) {
  // both passes use preallocated stacks: a vertex turns grey once and pushes
  // each out-neighbour at most once then, so the first pass pushes at most
  // E + N entries; the second is bounded by E + 1 per root
  std::vector<uint8_t> color(n, 0);
  std::vector<int32_t> finish(n);
  std::vector<int32_t> stack(static_cast<size_t>(e) + n + 1);
  uint8_t* col = color.data();
  int32_t* st = stack.data();
  int32_t nf = 0;
  for (int32_t v0 = 0; v0 < n; v0++) {
    if (col[v0]) continue;
    int64_t top = 0;
    st[top++] = v0;
    while (top) {
      const int32_t v = st[top - 1];
      const uint8_t c = col[v];
      if (c) {
        --top;
        if (c == 1) {
          finish[nf++] = v;
          col[v] = 2;
        }
      } else {
        col[v] = 1;
        for (const int32_t *it = oidx + optr[v], *end = oidx + optr[v + 1]; it != end; ++it) {
          const int32_t t = *it;
          if (!col[t]) st[top++] = t;
        }
      }
    }
  }
  std::vector<uint8_t> visited(n, 0);
  uint8_t* vis = visited.data();
  for (int32_t v = 0; v < n; v++) part[v] = -1;
  int32_t b = 0;
  while (nf > 0) {
    const int32_t v = finish[--nf];
    if (vis[v]) continue;
    int32_t i = 0;
    int64_t top = 0;
    st[top++] = v;
    while (top && i < dfs_depth) {
      const int32_t ni = st[--top];
      if (!vis[ni]) {
        vis[ni] = 1;
        part[ni] = b;
        i++;
        for (const int32_t *it = tidx + tptr[ni], *end = tidx + tptr[ni + 1]; it != end; ++it) {
          const int32_t t = *it;
          if (!vis[t]) st[top++] = t;
        }
      }
    }
    b++;
  }
  return b;
}

}  // namespace usap
