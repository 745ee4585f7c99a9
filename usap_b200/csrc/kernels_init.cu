// Initial blocks on the device (init_mode 2): a stand-in for the reference's
// sequential SCC/DFS pass (_scc + _dfs_itr, graph_parallel.hpp:514-603),
// which groups each vertex with the vertices a depth-limited DFS on the
// transpose reaches from it, about eight per block on the graphs here.  No
// parallel algorithm reproduces that DFS order, so this pass builds blocks
// of the same kind -- connected through edges, N/8 of them -- as the
// cells of a multi-source breadth-first search:
//   * one vertex in eight is a seed, chosen by a hash of its id (so the
//     result depends on the graph only, like the SCC pass);
//   * level by level, a vertex not yet reached joins the block of a
//     neighbour (out- or in-edge) reached at an earlier level, the one whose
//     seed has the highest hash; every level reads only earlier levels, so
//     the result does not depend on thread order;
//   * vertices no seed reaches (components without a seed) keep blocks of
//     their own.
// Blocks are then numbered in ascending order of their seed's id.  The host
// SCC pass stays the default; this one runs with no host pass and no copy
// of the partition across the bus.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "job.h"

namespace usap {
namespace {

constexpr int kThreads = 256;
constexpr uint32_t kSeedBelow = 0x20000000u;   // hash < 2^32 / 8: one vertex in eight is a seed
constexpr int kMaxLevels = 64;
constexpr int32_t kUnreached = 0x7fffffff;

__device__ __forceinline__ uint32_t vhash(uint32_t v) {
  // the murmur3 32-bit finaliser of the vertex id
  uint32_t h = v * 0x9E3779B1u + 0x7F4A7C15u;
  h ^= h >> 16;
  h *= 0x85EBCA6Bu;
  h ^= h >> 13;
  h *= 0xC2B2AE35u;
  h ^= h >> 16;
  return h;
}

__global__ void k_init_seeds(int32_t n, int32_t* __restrict__ label, int32_t* __restrict__ level) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const bool seed = vhash(static_cast<uint32_t>(v)) < kSeedBelow;
  label[v] = seed ? v : -1;
  level[v] = seed ? 0 : kUnreached;
}

// level L: unreached vertices next to a vertex reached before L
__global__ void k_init_grow(int32_t n, const int32_t* __restrict__ out_ptr, const int32_t* __restrict__ out_idx,
                            const int32_t* __restrict__ in_ptr, const int32_t* __restrict__ in_idx,
                            int32_t* __restrict__ label, int32_t* __restrict__ level, int32_t L,
                            int32_t* __restrict__ reached) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n || level[v] != kUnreached) return;
  uint32_t best_h = 0;
  int32_t best = -1;
  auto look = [&](int32_t x) {
    // a vertex reached in this level writes L: it is skipped either way
    if (level[x] < L) {
      const int32_t s = label[x];
      const uint32_t h = vhash(static_cast<uint32_t>(s));
      if (best < 0 || h > best_h || (h == best_h && s > best)) {
        best_h = h;
        best = s;
      }
    }
  };
  for (int32_t p = out_ptr[v]; p < out_ptr[v + 1]; p++) look(out_idx[p]);
  for (int32_t p = in_ptr[v]; p < in_ptr[v + 1]; p++) look(in_idx[p]);
  if (best >= 0) {
    label[v] = best;
    level[v] = L;
    atomicAdd(reached, 1);
  }
}

__global__ void k_init_present(int32_t n, int32_t* __restrict__ label, int32_t* __restrict__ present) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  if (label[v] < 0) label[v] = v;   // unreached: a block of its own
  present[v] = label[v] == v ? 1 : 0;
}

__global__ void k_init_compact(int32_t n, const int32_t* __restrict__ label, const int32_t* __restrict__ newid,
                               int32_t* __restrict__ part) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) part[v] = newid[label[v]];
}

}  // namespace

int32_t device_initial_blocks(const GraphDev& g, int32_t* part, cudaStream_t st, int* rounds_out) {
  const int32_t n = g.n;
  if (n <= 0) return 0;
  std::vector<void*> bufs;
  auto alloc = [&](size_t bytes) {
    void* p = dev_alloc(bytes, st);
    bufs.push_back(p);
    return p;
  };
  struct Free {
    std::vector<void*>& b;
    cudaStream_t st;
    ~Free() {
      for (void* p : b) dev_free(p, st);
    }
  } fr{bufs, st};
  int32_t* label = static_cast<int32_t*>(alloc(sizeof(int32_t) * n));
  int32_t* level = static_cast<int32_t*>(alloc(sizeof(int32_t) * n));
  int32_t* counter = static_cast<int32_t*>(alloc(sizeof(int32_t) * 2));
  int32_t* present = static_cast<int32_t*>(alloc(sizeof(int32_t) * (static_cast<size_t>(n) + 1)));
  int32_t* newid = static_cast<int32_t*>(alloc(sizeof(int32_t) * (static_cast<size_t>(n) + 1)));
  const unsigned blocks = static_cast<unsigned>((n + kThreads - 1) / kThreads);
  k_init_seeds<<<blocks, kThreads, 0, st>>>(n, label, level);
  USAP_LAUNCHED();
  int rounds = 0;
  for (int L = 1; L <= kMaxLevels; L++) {
    USAP_CUDA(cudaMemsetAsync(counter, 0, sizeof(int32_t), st));
    k_init_grow<<<blocks, kThreads, 0, st>>>(n, g.out_ptr, g.out_idx, g.in_ptr, g.in_idx, label, level, L, counter);
    USAP_LAUNCHED();
    int32_t reached = 0;
    USAP_CUDA(cudaMemcpyAsync(&reached, counter, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    USAP_CUDA(cudaStreamSynchronize(st));
    rounds++;
    if (reached == 0) break;
  }
  k_init_present<<<blocks, kThreads, 0, st>>>(n, label, present);
  USAP_LAUNCHED();
  USAP_CUDA(cudaMemsetAsync(present + n, 0, sizeof(int32_t), st));
  scan_exclusive_i32(present, static_cast<int64_t>(n) + 1, newid, st, alloc);
  k_init_compact<<<blocks, kThreads, 0, st>>>(n, label, newid, part);
  USAP_LAUNCHED();
  int32_t B = 0;
  USAP_CUDA(cudaMemcpyAsync(&B, newid + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  USAP_CUDA(cudaStreamSynchronize(st));
  if (rounds_out) *rounds_out = rounds;
  return B;
}

}  // namespace usap
