// Adjacency lists on the device from an edge list already in device memory
// (load_graph_from_tsv, graph_parallel.hpp:285-290): for every vertex its
// out-list (targets, weights) and in-list (sources, weights), each in the
// order the edges appear in the file, plus the weighted degrees.
//
// A stable counting sort by key (source for the out-lists, target for the
// in-lists):
//   1. counts per key (integer atomics), an exclusive scan -> ptr;
//   2. every edge lands in its key's bucket at ptr[key] + an atomic cursor
//      (arrival order, not file order), carrying its edge index;
//   3. one warp per bucket ranks its entries by edge index (the rank of an
//      entry is the number of entries of the bucket with a smaller index;
//      indices are distinct) and writes them at ptr[key] + rank.
// Step 3 costs the sum over vertices of degree^2 / 32 comparisons per warp
// lane, a few tens of millions for the largest graphs here; the result is
// the sequential stable sort's, whatever order the atomics took.
#include <algorithm>
#include <cstdint>
#include <functional>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "job.h"

namespace usap {
namespace {

constexpr int kThreads = 256;
constexpr int kScanTile = 1024;

__global__ void k_csr_count(const int32_t* __restrict__ key, const int32_t* __restrict__ w, int64_t e,
                            int32_t* __restrict__ cnt, int32_t* __restrict__ wdeg) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < e; i += stride) {
    const int32_t k = __ldg(key + i);
    atomicAdd(cnt + k, 1);
    atomicAdd(wdeg + k, w ? __ldg(w + i) : 1);
  }
}

// exclusive scan of one tile of kScanTile values per block; the tile's
// total goes to sums[blockIdx.x]
__global__ void __launch_bounds__(kScanTile) k_scan_tile(const int32_t* __restrict__ in, int64_t n,
                                                          int32_t* __restrict__ out, int32_t* __restrict__ sums) {
  __shared__ int32_t warp_tot[kScanTile / 32];
  const int64_t i = static_cast<int64_t>(blockIdx.x) * kScanTile + threadIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int32_t x = i < n ? in[i] : 0;
  const int32_t incl = warp_incl_scan(x, lane);
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    const int32_t t = warp_tot[lane];
    const int32_t ti = warp_incl_scan(t, lane);
    warp_tot[lane] = ti - t;
  }
  __syncthreads();
  const int32_t ex = incl - x + warp_tot[wid];
  if (i < n) out[i] = ex;
  if (threadIdx.x == kScanTile - 1) sums[blockIdx.x] = ex + x;
}

// exclusive scan of the tile totals by one block, chunk after chunk
__global__ void __launch_bounds__(kScanTile) k_scan_sums(int32_t* __restrict__ sums, int64_t tiles) {
  __shared__ int32_t warp_tot[kScanTile / 32];
  __shared__ int32_t carry;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < tiles; base += kScanTile) {
    const int64_t i = base + threadIdx.x;
    const int32_t x = i < tiles ? sums[i] : 0;
    const int32_t incl = warp_incl_scan(x, lane);
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      const int32_t t = warp_tot[lane];
      const int32_t ti = warp_incl_scan(t, lane);
      warp_tot[lane] = ti - t;
    }
    __syncthreads();
    const int32_t c = carry;
    const int32_t ex = incl - x + warp_tot[wid] + c;
    if (i < tiles) sums[i] = ex;
    __syncthreads();
    if (threadIdx.x == kScanTile - 1) carry = ex + x;
    __syncthreads();
  }
}

__global__ void k_scan_add(int32_t* __restrict__ out, int64_t n, const int32_t* __restrict__ sums) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] += sums[i / kScanTile];
}

// step 2: an edge into its bucket (arrival order), with its index
__global__ void k_csr_scatter(const int32_t* __restrict__ key, const int32_t* __restrict__ val, int64_t e,
                              const int32_t* __restrict__ ptr, int32_t* __restrict__ cursor,
                              int32_t* __restrict__ tmp_eid) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < e; i += stride) {
    const int32_t k = __ldg(key + i);
    const int32_t p = __ldg(ptr + k) + atomicAdd(cursor + k, 1);
    tmp_eid[p] = static_cast<int32_t>(i);
  }
}

// step 3: one warp per bucket; entry j goes to ptr[v] + (number of the
// bucket's entries with a smaller edge index)
__global__ void k_csr_rank(const int32_t* __restrict__ ptr, int32_t n, const int32_t* __restrict__ tmp_eid,
                           const int32_t* __restrict__ val, const int32_t* __restrict__ w,
                           int32_t* __restrict__ idx, int32_t* __restrict__ wout) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x / 32);
  for (int64_t v = static_cast<int64_t>(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5); v < n; v += warps) {
    const int32_t lo = __ldg(ptr + v), hi = __ldg(ptr + v + 1);
    for (int32_t j = lo + lane; j < hi; j += 32) {
      const int32_t ej = tmp_eid[j];
      int32_t rank = 0;
      for (int32_t k = lo; k < hi; k++) rank += tmp_eid[k] < ej ? 1 : 0;
      idx[lo + rank] = __ldg(val + ej);
      if (wout) wout[lo + rank] = __ldg(w + ej);
    }
  }
}

int grid_for(int64_t work, int per_block) {
  const int64_t g = (work + per_block - 1) / per_block;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(g, 148 * 16)));
}

}  // namespace

// exclusive scan of m int32 values (out[m - 1] + in[m - 1] = the total)
void scan_exclusive_i32(const int32_t* cnt, int64_t m, int32_t* ptr, cudaStream_t st,
                        const std::function<void*(size_t)>& alloc) {
  const int64_t tiles = (m + kScanTile - 1) / kScanTile;
  int32_t* sums = static_cast<int32_t*>(alloc(sizeof(int32_t) * tiles));
  k_scan_tile<<<static_cast<unsigned>(tiles), kScanTile, 0, st>>>(cnt, m, ptr, sums);
  USAP_LAUNCHED();
  k_scan_sums<<<1, kScanTile, 0, st>>>(sums, tiles);
  USAP_LAUNCHED();
  k_scan_add<<<static_cast<unsigned>((m + kThreads - 1) / kThreads), kThreads, 0, st>>>(ptr, m, sums);
  USAP_LAUNCHED();
}

namespace {

// one side (keyed by `key`): ptr (n + 1), idx and optional weights (e), the
// weighted degree per key
void csr_side(const int32_t* key, const int32_t* val, const int32_t* w, int64_t e, int32_t n, cudaStream_t st,
              const std::function<void*(size_t)>& alloc, std::vector<int32_t>& h_ptr, std::vector<int32_t>& h_idx,
              std::vector<int32_t>* h_w, std::vector<int32_t>& h_deg) {
  const int64_t m = static_cast<int64_t>(n) + 1;
  int32_t* cnt = static_cast<int32_t*>(alloc(sizeof(int32_t) * m));
  int32_t* deg = static_cast<int32_t*>(alloc(sizeof(int32_t) * m));
  int32_t* ptr = static_cast<int32_t*>(alloc(sizeof(int32_t) * m));
  int32_t* cursor = static_cast<int32_t*>(alloc(sizeof(int32_t) * m));
  int32_t* tmp = static_cast<int32_t*>(alloc(sizeof(int32_t) * e));
  int32_t* idx = static_cast<int32_t*>(alloc(sizeof(int32_t) * e));
  int32_t* wo = w ? static_cast<int32_t*>(alloc(sizeof(int32_t) * e)) : nullptr;
  USAP_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * m, st));
  USAP_CUDA(cudaMemsetAsync(deg, 0, sizeof(int32_t) * m, st));
  USAP_CUDA(cudaMemsetAsync(cursor, 0, sizeof(int32_t) * m, st));
  k_csr_count<<<grid_for(e, kThreads), kThreads, 0, st>>>(key, w, e, cnt, deg);
  USAP_LAUNCHED();
  scan_exclusive_i32(cnt, m, ptr, st, alloc);
  k_csr_scatter<<<grid_for(e, kThreads), kThreads, 0, st>>>(key, val, e, ptr, cursor, tmp);
  USAP_LAUNCHED();
  k_csr_rank<<<grid_for(static_cast<int64_t>(n) * 32, kThreads), kThreads, 0, st>>>(ptr, n, tmp, val, w, idx, wo);
  USAP_LAUNCHED();
  h_ptr.resize(m);
  h_idx.resize(e);
  h_deg.resize(n);
  USAP_CUDA(cudaMemcpyAsync(h_ptr.data(), ptr, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, st));
  USAP_CUDA(cudaMemcpyAsync(h_idx.data(), idx, sizeof(int32_t) * e, cudaMemcpyDeviceToHost, st));
  USAP_CUDA(cudaMemcpyAsync(h_deg.data(), deg, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
  if (w) {
    h_w->resize(e);
    USAP_CUDA(cudaMemcpyAsync(h_w->data(), wo, sizeof(int32_t) * e, cudaMemcpyDeviceToHost, st));
  }
}

}  // namespace

void build_csr_device(const int32_t* d_src, const int32_t* d_dst, const int32_t* d_w, HostGraph& h,
                      cudaStream_t st, const std::function<void*(size_t)>& alloc) {
  const int32_t* w = h.unit ? nullptr : d_w;
  csr_side(d_src, d_dst, w, h.e, h.n, st, alloc, h.out_ptr, h.out_idx, h.unit ? nullptr : &h.out_w, h.kout);
  csr_side(d_dst, d_src, w, h.e, h.n, st, alloc, h.in_ptr, h.in_idx, h.unit ? nullptr : &h.in_w, h.kin);
  USAP_CUDA(cudaStreamSynchronize(st));
  bool by_source = true;
  for (int64_t i = 1; i < h.e && by_source; i++) by_source = h.src[i - 1] <= h.src[i];
  h.transpose_is_in = by_source;
  h.csr_built = true;
}

}  // namespace usap
