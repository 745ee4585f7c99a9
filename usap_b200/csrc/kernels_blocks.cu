// Interblock edge counts M, block degrees and the description length.
//
// Reference: _initialize_edge_counts (graph_parallel.hpp:703-759) rebuilds M
// from scratch after every batch with one sequential pass over the edges;
// _compute_overall_entropy (:1281-1319) scans all B*B cells.  Here the dense
// tile is built by edge-parallel warp-aggregated atomics (edges of one warp
// that land in the same cell are summed in-warp first, so the many
// within-block edges of late stages cost one atomic per distinct cell), and
// later updated by deltas; the sparse views come from a radix sort of the
// (source block, target block) keys.  Entropy terms are Q32-rounded FP64
// and reduced with integer atomics.
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include <cub/cub.cuh>
#include <cuda/std/functional>

#include "common.cuh"
#include "engine.h"

namespace cg = cooperative_groups;

namespace usap {

namespace {

constexpr int kThreads = 256;

inline int grid_for(int64_t work, int per_block, int cap = 148 * 16) {
  int64_t g = (work + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return static_cast<int>(g);
}

// M[bs, bd] += w and Mt[bd, bs] += w over all edges, aggregated per warp.
__global__ void __launch_bounds__(kThreads) k_dense_build(int64_t E, const int32_t* __restrict__ src,
                                                         const int32_t* __restrict__ dst,
                                                         const int32_t* __restrict__ w,
                                                         const int32_t* __restrict__ part, int ld,
                                                         int* __restrict__ M, int* __restrict__ Mt) {
  auto tile = cg::tiled_partition<32>(cg::this_thread_block());
  int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x;
  for (; base < E; base += stride) {
    int64_t e = base + threadIdx.x;
    bool valid = e < E;
    int bs = valid ? __ldg(part + __ldg(src + e)) : 0;
    int bd = valid ? __ldg(part + __ldg(dst + e)) : 0;
    int ww = valid ? (w ? __ldg(w + e) : 1) : 0;
    long long key = valid ? static_cast<long long>(bs) * ld + bd : -1;
    auto grp = cg::labeled_partition(tile, key);
    int sum = cg::reduce(grp, ww, cg::plus<int>());
    if (valid && grp.thread_rank() == 0) {
      atomicAdd(M + static_cast<int64_t>(bs) * ld + bd, sum);
      atomicAdd(Mt + static_cast<int64_t>(bd) * ld + bs, sum);
    }
  }
}

// dout[b] = sum of kout over b's vertices, din likewise (aggregated per warp).
__global__ void __launch_bounds__(kThreads) k_degrees(int n, const int32_t* __restrict__ part,
                                                     const int32_t* __restrict__ kout,
                                                     const int32_t* __restrict__ kin,
                                                     int32_t* __restrict__ dout,
                                                     int32_t* __restrict__ din) {
  auto tile = cg::tiled_partition<32>(cg::this_thread_block());
  int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
    int v = base + threadIdx.x;
    bool valid = v < n;
    int b = valid ? __ldg(part + v) : -1;
    int ko = valid ? __ldg(kout + v) : 0;
    int ki = valid ? __ldg(kin + v) : 0;
    auto grp = cg::labeled_partition(tile, b);
    int so = cg::reduce(grp, ko, cg::plus<int>());
    int si = cg::reduce(grp, ki, cg::plus<int>());
    if (valid && grp.thread_rank() == 0) {
      atomicAdd(dout + b, so);
      atomicAdd(din + b, si);
    }
  }
}

// data term sum_{ij} q32(M_ij log(M_ij/(dout_i din_j))) over the dense tile
__global__ void __launch_bounds__(kThreads) k_entropy_dense(const double* __restrict__ L,
                                                           const int* __restrict__ M, int ld, int B,
                                                           const int32_t* __restrict__ dout,
                                                           const int32_t* __restrict__ din,
                                                           unsigned long long* acc) {
  long long part = 0;
  int64_t cells = static_cast<int64_t>(B) * B;
  int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < cells;
       c += stride) {
    int i = static_cast<int>(c / B), j = static_cast<int>(c - static_cast<int64_t>(i) * B);
    int m = __ldg(M + static_cast<int64_t>(i) * ld + j);
    if (m) part += q32(g_term(L, m, __ldg(din + j), __ldg(dout + i)));
  }
  part = warp_sum_ll(part);
  if ((threadIdx.x & 31) == 0 && part) atomicAdd(acc, static_cast<unsigned long long>(part));
}

__global__ void __launch_bounds__(kThreads) k_entropy_sorted(const double* __restrict__ L,
                                                            const int* __restrict__ nnz_dev,
                                                            const int32_t* __restrict__ rowof,
                                                            const int* __restrict__ col,
                                                            const int* __restrict__ val,
                                                            const int32_t* __restrict__ dout,
                                                            const int32_t* __restrict__ din,
                                                            unsigned long long* acc) {
  int nnz = *nnz_dev;
  long long part = 0;
  int stride = gridDim.x * blockDim.x;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += stride) {
    int m = __ldg(val + j);
    if (m) part += q32(g_term(L, m, __ldg(din + __ldg(col + j)), __ldg(dout + __ldg(rowof + j))));
  }
  part = warp_sum_ll(part);
  if ((threadIdx.x & 31) == 0 && part) atomicAdd(acc, static_cast<unsigned long long>(part));
}

// keys of (source block, target block) pairs; kind 0 rows, 1 columns,
// 2 symmetric (both orientations, 2E keys)
__global__ void k_make_keys(int64_t E, const int32_t* __restrict__ src,
                            const int32_t* __restrict__ dst, const int32_t* __restrict__ w,
                            const int32_t* __restrict__ part, int B, int kind,
                            unsigned long long* __restrict__ keys, int* __restrict__ vals) {
  int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < E; e += stride) {
    unsigned long long bs = static_cast<unsigned long long>(__ldg(part + __ldg(src + e)));
    unsigned long long bd = static_cast<unsigned long long>(__ldg(part + __ldg(dst + e)));
    int ww = w ? __ldg(w + e) : 1;
    if (kind == 1) {
      keys[e] = bd * B + bs;
    } else {
      keys[e] = bs * B + bd;
    }
    vals[e] = ww;
    if (kind == 2) {
      keys[E + e] = bd * B + bs;
      vals[E + e] = ww;
    }
  }
}

// row offsets, column ids and values from sorted unique keys
__global__ void k_offsets(const unsigned long long* __restrict__ ukeys, const int* __restrict__ uvals,
                          const int* __restrict__ nruns, int B, int* __restrict__ ptr,
                          int* __restrict__ idx, int* __restrict__ val, int32_t* __restrict__ rowof,
                          int* __restrict__ nnz_out) {
  int nnz = *nruns;
  int stride = gridDim.x * blockDim.x;
  int t0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (t0 == 0) {
    if (nnz_out) *nnz_out = nnz;
    if (nnz == 0)
      for (int rr = 0; rr <= B; rr++) ptr[rr] = 0;
  }
  for (int j = t0; j < nnz; j += stride) {
    unsigned long long key = ukeys[j];
    int r = static_cast<int>(key / B), c = static_cast<int>(key - static_cast<unsigned long long>(r) * B);
    idx[j] = c;
    if (val) val[j] = uvals[j];
    if (rowof) rowof[j] = r;
    int prev = j == 0 ? -1 : static_cast<int>(ukeys[j - 1] / B);
    for (int rr = prev + 1; rr <= r; rr++) ptr[rr] = j;
    if (j == nnz - 1)
      for (int rr = r + 1; rr <= B; rr++) ptr[rr] = nnz;
  }
}

int key_bits(int B) {
  unsigned long long m = static_cast<unsigned long long>(B) * B;
  int bits = 1;
  while (bits < 64 && (1ull << bits) < m) bits++;
  return bits;
}

// the log table as float pairs: hi = log k rounded to float, lo = the
// remainder rounded to float (log 0 = -inf has lo = 0)
__global__ void k_log_pairs(int64_t n, const double* __restrict__ L, float2* __restrict__ T) {
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double x = L[k];
    const float hi = __double2float_rn(x);
    const float lo = isinf(x) ? 0.0f : __double2float_rn(__dsub_rn(x, static_cast<double>(hi)));
    T[k] = make_float2(hi, lo);
  }
}

}  // namespace

void launch_log_pairs(const double* L, float2* T, int64_t n, cudaStream_t st) {
  if (n <= 0) return;
  int64_t blocks = (n + kThreads - 1) / kThreads;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_log_pairs<<<static_cast<int>(blocks), kThreads, 0, st>>>(n, L, T);
  USAP_LAUNCHED();
}

void launch_dense_build(const GraphDev& g, const int32_t* part, int B, int ld, int* M, int* Mt,
                        cudaStream_t st) {
  size_t bytes = sizeof(int) * static_cast<size_t>(ld) * ld;
  USAP_CUDA(cudaMemsetAsync(M, 0, bytes, st));
  USAP_CUDA(cudaMemsetAsync(Mt, 0, bytes, st));
  k_dense_build<<<grid_for(g.e, kThreads), kThreads, 0, st>>>(g.e, g.src, g.dst, g.w, part, ld, M, Mt);
  USAP_LAUNCHED();
}

void launch_degrees(const GraphDev& g, const int32_t* part, int B, int32_t* dout, int32_t* din,
                    cudaStream_t st) {
  USAP_CUDA(cudaMemsetAsync(dout, 0, sizeof(int32_t) * B, st));
  USAP_CUDA(cudaMemsetAsync(din, 0, sizeof(int32_t) * B, st));
  k_degrees<<<grid_for(g.n, kThreads), kThreads, 0, st>>>(g.n, part, g.kout, g.kin, dout, din);
  USAP_LAUNCHED();
}

void launch_entropy_dense(const GraphDev& g, DenseView v, int B, const int32_t* dout,
                          const int32_t* din, unsigned long long* acc, cudaStream_t st) {
  int64_t cells = static_cast<int64_t>(B) * B;
  k_entropy_dense<<<grid_for(cells, kThreads), kThreads, 0, st>>>(g.logk, v.M, v.ld, B, dout, din, acc);
  USAP_LAUNCHED();
}

void launch_entropy_sorted(const GraphDev& g, SortedView v, const int* nnz_dev, int64_t max_nnz,
                           const int32_t* rowof, const int32_t* dout, const int32_t* din,
                           unsigned long long* acc, cudaStream_t st) {
  k_entropy_sorted<<<grid_for(max_nnz, kThreads), kThreads, 0, st>>>(g.logk, nnz_dev, rowof, v.col,
                                                                      v.val, dout, din, acc);
  USAP_LAUNCHED();
}

// --- SortedBuilder --------------------------------------------------------------
void SortedBuilder::reserve(int64_t e, int bmax, cudaStream_t st) {
  if (keys_ && e <= e_ && bmax <= bmax_) return;   // the buffers already fit
  e = std::max(e, e_);
  bmax = std::max(bmax, bmax_);
  release(st);
  e_ = e;
  bmax_ = bmax;
  const int64_t e2 = 2 * e;
  auto a64 = [&](int64_t n) { return static_cast<unsigned long long*>(dev_alloc(sizeof(unsigned long long) * n, st)); };
  auto a32 = [&](int64_t n) { return static_cast<int*>(dev_alloc(sizeof(int) * n, st)); };
  keys_ = a64(e2);
  keys_alt_ = a64(e2);
  ukeys_ = a64(e2);
  vals_ = a32(e2);
  vals_alt_ = a32(e2);
  uvals_ = a32(e2);
  nruns_ = a32(4);
  nnz_ = a32(4);
  rowptr_ = a32(bmax + 1);
  col_ = a32(e);
  val_ = a32(e);
  rowof_ = a32(e);
  colptr_ = a32(bmax + 1);
  crow_ = a32(e);
  cval_ = a32(e);
  symptr_ = a32(bmax + 1);
  symcol_ = a32(e2);
  symcum_ = a32(e2);
  size_t b1 = 0, b2 = 0, b3 = 0;
  int n2 = static_cast<int>(e2);
  USAP_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b1, keys_, keys_alt_, vals_, vals_alt_, n2));
  USAP_CUDA(cub::DeviceReduce::ReduceByKey(nullptr, b2, keys_alt_, ukeys_, vals_alt_, uvals_, nruns_,
                                           cuda::std::plus<int>{}, n2));
  USAP_CUDA(cub::DeviceScan::InclusiveSum(nullptr, b3, uvals_, symcum_, n2));
  tmp_bytes_ = b1 > b2 ? b1 : b2;
  if (b3 > tmp_bytes_) tmp_bytes_ = b3;
  tmp_ = dev_alloc(tmp_bytes_, st);
}

void SortedBuilder::release(cudaStream_t st) {
  void* ptrs[] = {keys_, keys_alt_, ukeys_, vals_, vals_alt_, uvals_, nruns_, nnz_, rowptr_, col_, val_,
                  rowof_, colptr_, crow_, cval_, symptr_, symcol_, symcum_, tmp_};
  for (void* p : ptrs) dev_free(p, st);
  keys_ = keys_alt_ = ukeys_ = nullptr;
  vals_ = vals_alt_ = uvals_ = nruns_ = nnz_ = nullptr;
  rowptr_ = col_ = val_ = rowof_ = colptr_ = crow_ = cval_ = symptr_ = symcol_ = symcum_ = nullptr;
  tmp_ = nullptr;
  tmp_bytes_ = 0;
}

void SortedBuilder::sort_reduce(int64_t count, int B, int kind, cudaStream_t st) {
  int n = static_cast<int>(count);
  int bits = key_bits(B);
  size_t bytes = tmp_bytes_;
  USAP_CUB(cub::DeviceRadixSort::SortPairs(tmp_, bytes, keys_, keys_alt_, vals_, vals_alt_, n, 0,
                                           bits, st));
  bytes = tmp_bytes_;
  USAP_CUB(cub::DeviceReduce::ReduceByKey(tmp_, bytes, keys_alt_, ukeys_, vals_alt_, uvals_,
                                          nruns_ + kind, cuda::std::plus<int>{}, n, st));
}

void SortedBuilder::build(const GraphDev& g, const int32_t* part, int B, bool with_csc, bool with_sym,
                          cudaStream_t st) {
  if (B > bmax_) throw Error(-6, "SortedBuilder: B above reserved size");
  int grid = grid_for(g.e, kThreads);
  int ogrid = grid_for(2 * g.e, kThreads);
  // row view
  k_make_keys<<<grid, kThreads, 0, st>>>(g.e, g.src, g.dst, g.w, part, B, 0, keys_, vals_);
  USAP_LAUNCHED();
  sort_reduce(g.e, B, 0, st);
  k_offsets<<<grid, kThreads, 0, st>>>(ukeys_, uvals_, nruns_ + 0, B, rowptr_, col_, val_, rowof_, nnz_ + 0);
  USAP_LAUNCHED();
  has_csc_ = with_csc;
  if (with_csc) {
    k_make_keys<<<grid, kThreads, 0, st>>>(g.e, g.src, g.dst, g.w, part, B, 1, keys_, vals_);
    USAP_LAUNCHED();
    sort_reduce(g.e, B, 1, st);
    k_offsets<<<grid, kThreads, 0, st>>>(ukeys_, uvals_, nruns_ + 1, B, colptr_, crow_, cval_,
                                         nullptr, nnz_ + 1);
    USAP_LAUNCHED();
  }
  if (with_sym) {
    k_make_keys<<<grid, kThreads, 0, st>>>(g.e, g.src, g.dst, g.w, part, B, 2, keys_, vals_);
    USAP_LAUNCHED();
    sort_reduce(2 * g.e, B, 2, st);
    k_offsets<<<ogrid, kThreads, 0, st>>>(ukeys_, uvals_, nruns_ + 2, B, symptr_, symcol_, nullptr,
                                          nullptr, nnz_ + 2);
    USAP_LAUNCHED();
    size_t bytes = tmp_bytes_;
    USAP_CUB(cub::DeviceScan::InclusiveSum(tmp_, bytes, uvals_, symcum_, static_cast<int>(2 * g.e), st));
  }
}

SortedView SortedBuilder::view() const {
  SortedView v;
  v.rowptr = rowptr_;
  v.col = col_;
  v.val = val_;
  v.colptr = has_csc_ ? colptr_ : nullptr;
  v.row = has_csc_ ? crow_ : nullptr;
  v.cval = has_csc_ ? cval_ : nullptr;
  v.symptr = symptr_;
  v.symcol = symcol_;
  v.symcum = symcum_;
  return v;
}

}  // namespace usap
