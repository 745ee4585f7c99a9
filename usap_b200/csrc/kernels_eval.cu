// Partition scores on the device (bf::evaluate, include/evaluate.hpp:18-266):
// the contingency table, its row and column sums, the exact pair counts and
// the fixed-point information sums of eval_common.h, from device arrays of
// truth and given labels.  Only the sums (and, for the matching accuracy,
// the table when both sides have at most 2048 blocks) come back to the host,
// which forms the scores exactly as the host version does.
#include <vector>

#include "eval_common.h"
#include "job.h"

namespace usap {

namespace {

constexpr int kThreads = 256;
constexpr int64_t kMaxCells = int64_t(1) << 26;   // dense table limit (256 MiB of counts)

struct LabelInfo {
  int max_truth, max_given, bad;
  unsigned long long known;   // vertices with truth >= 0
};

__global__ void k_eval_labels(int64_t n, const int32_t* __restrict__ truth, const int32_t* __restrict__ given,
                              LabelInfo* info) {
  int mt = -1, mg = -1, bad = 0;
  unsigned long long known = 0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int t = truth[i], g = given[i];
    if (g < 0 || t < -1) bad = 1;
    mt = max(mt, t);
    mg = max(mg, g);
    known += t >= 0;
  }
  for (int o = 16; o > 0; o >>= 1) {
    mt = max(mt, __shfl_xor_sync(0xffffffffu, mt, o));
    mg = max(mg, __shfl_xor_sync(0xffffffffu, mg, o));
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    known += __shfl_xor_sync(0xffffffffu, known, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&info->max_truth, mt);
    atomicMax(&info->max_given, mg);
    if (bad) atomicOr(&info->bad, 1);
    if (known) atomicAdd(&info->known, known);
  }
}

// counts into the table (row-major b1 x b2) and the row/column sums; tables
// small enough for shared memory are privatised per CTA
__global__ void k_eval_count(int64_t n, const int32_t* __restrict__ truth, const int32_t* __restrict__ given, int b2,
                             int cells, unsigned* __restrict__ table, unsigned* __restrict__ rows,
                             unsigned* __restrict__ cols, int priv) {
  extern __shared__ unsigned s_tab[];
  if (priv) {
    for (int i = threadIdx.x; i < cells; i += blockDim.x) s_tab[i] = 0;
    __syncthreads();
  }
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int t = truth[i];
    if (t < 0) continue;
    const int g = given[i];
    const int64_t k = static_cast<int64_t>(t) * b2 + g;
    if (priv) atomicAdd(s_tab + k, 1u);
    else atomicAdd(table + k, 1u);
    atomicAdd(rows + t, 1u);
    atomicAdd(cols + g, 1u);
  }
  if (priv) {
    __syncthreads();
    for (int i = threadIdx.x; i < cells; i += blockDim.x)
      if (s_tab[i]) atomicAdd(table + i, s_tab[i]);
  }
}

__device__ __forceinline__ long long block_sum(long long v, long long* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  long long t = 0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < blockDim.x / 32 ? sh[threadIdx.x] : 0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  return t;   // valid in thread 0
}

// the exact sums over cells (items [0, cells)), rows and columns
__global__ void k_eval_sums(int b1, int b2, const unsigned* __restrict__ table, const unsigned* __restrict__ rows,
                            const unsigned* __restrict__ cols, const double* __restrict__ L, long long N,
                            EvalSums* out) {
  __shared__ long long sh[kThreads / 32];
  const double dN = static_cast<double>(N), LN = __ldg(L + N);
  long long sq = 0, same = 0, hgt = 0, htg = 0, mi = 0, sr = 0, s1 = 0, sc = 0, s2 = 0, h1 = 0, h2 = 0, nb1 = 0,
            nb2 = 0;
  const long long cells = static_cast<long long>(b1) * b2;
  const long long total = cells + b1 + b2;
  for (long long x = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; x < total;
       x += static_cast<long long>(gridDim.x) * blockDim.x) {
    if (x < cells) {
      const long long c = table[x];
      if (!c) continue;
      const int i = static_cast<int>(x / b2), j = static_cast<int>(x - static_cast<long long>(i) * b2);
      const long long r = rows[i], s = cols[j];
      const double Lc = __ldg(L + c), Lr = __ldg(L + r), Ls = __ldg(L + s);
      sq += c * c;
      same += c * (c - 1) / 2;
      hgt += ev_term(c, dN, Lc, Lr);
      htg += ev_term(c, dN, Lc, Ls);
      mi += ev_mi_term(c, dN, Lc, LN, Lr, Ls);
    } else if (x < cells + b1) {
      const long long r = rows[x - cells];
      if (!r) continue;
      sr += r * r;
      s1 += r * (r - 1) / 2;
      nb1++;
      h1 += ev_term(r, dN, __ldg(L + r), LN);
    } else {
      const long long s = cols[x - cells - b1];
      if (!s) continue;
      sc += s * s;
      s2 += s * (s - 1) / 2;
      nb2++;
      h2 += ev_term(s, dN, __ldg(L + s), LN);
    }
  }
  long long vals[13] = {sq, same, hgt, htg, mi, sr, s1, sc, s2, h1, h2, nb1, nb2};
  long long* dst[13] = {reinterpret_cast<long long*>(&out->sq), reinterpret_cast<long long*>(&out->same),
                        reinterpret_cast<long long*>(&out->h_gt_q), reinterpret_cast<long long*>(&out->h_tg_q),
                        reinterpret_cast<long long*>(&out->mi_q), reinterpret_cast<long long*>(&out->sr),
                        reinterpret_cast<long long*>(&out->s1), reinterpret_cast<long long*>(&out->sc),
                        reinterpret_cast<long long*>(&out->s2), reinterpret_cast<long long*>(&out->h_truth_q),
                        reinterpret_cast<long long*>(&out->h_given_q), reinterpret_cast<long long*>(&out->nb_truth),
                        reinterpret_cast<long long*>(&out->nb_given)};
#pragma unroll 1
  for (int k = 0; k < 13; k++) {
    const long long t = block_sum(vals[k], sh);
    if (threadIdx.x == 0 && t) atomicAdd(reinterpret_cast<unsigned long long*>(dst[k]), static_cast<unsigned long long>(t));
  }
}

int grid_for(int64_t items) {
  int64_t b = (items + kThreads - 1) / kThreads;
  if (b > 148 * 8) b = 148 * 8;
  return static_cast<int>(b < 1 ? 1 : b);
}

}  // namespace

void evaluate_device(const int32_t* truth, const int32_t* given, int64_t n, int device, usap_scores* s) {
  if (n < 2) throw Error(USAP_ERR_INVALID, "need at least two labelled vertices");
  USAP_CUDA(cudaSetDevice(device));
  pool_configure(device);
  cudaStream_t st = nullptr;
  USAP_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct Cleanup {
    cudaStream_t st;
    std::vector<void*> bufs;
    ~Cleanup() {
      for (void* p : bufs) cudaFreeAsync(p, st);
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
  } cl{st, {}};
  auto alloc = [&](size_t bytes) {
    void* p = dev_alloc(bytes, st);
    cl.bufs.push_back(p);
    return p;
  };
  LabelInfo* info = static_cast<LabelInfo*>(alloc(sizeof(LabelInfo)));
  const LabelInfo init{-1, -1, 0, 0};
  USAP_CUDA(cudaMemcpyAsync(info, &init, sizeof(init), cudaMemcpyHostToDevice, st));
  k_eval_labels<<<grid_for(n), kThreads, 0, st>>>(n, truth, given, info);
  USAP_LAUNCHED();
  LabelInfo h{};
  USAP_CUDA(cudaMemcpyAsync(&h, info, sizeof(h), cudaMemcpyDeviceToHost, st));
  USAP_CUDA(cudaStreamSynchronize(st));
  if (h.bad) throw Error(USAP_ERR_INVALID, "given labels must be >= 0 and truth labels >= -1");
  const int b1 = h.max_truth + 1, b2 = h.max_given + 1;
  const int64_t N = static_cast<int64_t>(h.known);
  if (b1 <= 0 || b2 <= 0 || N < 2) throw Error(USAP_ERR_INVALID, "need at least two vertices with known truth");
  const int64_t cells = static_cast<int64_t>(b1) * b2;
  if (cells > kMaxCells) throw Error(USAP_ERR_LIMIT, "contingency table above 2^26 cells");
  unsigned* table = static_cast<unsigned*>(alloc(sizeof(unsigned) * (cells + b1 + b2)));
  unsigned* rows = table + cells;
  unsigned* cols = rows + b1;
  USAP_CUDA(cudaMemsetAsync(table, 0, sizeof(unsigned) * (cells + b1 + b2), st));
  const int priv = cells <= 8192 ? 1 : 0;
  k_eval_count<<<grid_for(n), kThreads, priv ? sizeof(unsigned) * cells : 0, st>>>(n, truth, given, b2,
                                                                                   static_cast<int>(priv ? cells : 0),
                                                                                   table, rows, cols, priv);
  USAP_LAUNCHED();
  const std::shared_ptr<const std::vector<double>> Lp = log_table(N);
  double* L = static_cast<double*>(alloc(sizeof(double) * (N + 1)));
  USAP_CUDA(cudaMemcpyAsync(L, Lp->data(), sizeof(double) * (N + 1), cudaMemcpyHostToDevice, st));
  EvalSums* sums = static_cast<EvalSums*>(alloc(sizeof(EvalSums)));
  USAP_CUDA(cudaMemsetAsync(sums, 0, sizeof(EvalSums), st));
  k_eval_sums<<<grid_for(cells + b1 + b2), kThreads, 0, st>>>(b1, b2, table, rows, cols, L, N, sums);
  USAP_LAUNCHED();
  EvalSums e{};
  USAP_CUDA(cudaMemcpyAsync(&e, sums, sizeof(e), cudaMemcpyDeviceToHost, st));
  const int m = b1 > b2 ? b1 : b2;
  std::vector<unsigned> t;
  if (m <= 2048) {
    t.resize(static_cast<size_t>(cells));
    USAP_CUDA(cudaMemcpyAsync(t.data(), table, sizeof(unsigned) * cells, cudaMemcpyDeviceToHost, st));
  }
  USAP_CUDA(cudaStreamSynchronize(st));
  e.N = N;
  scores_from_sums(e, s);
  if (m <= 2048) {
    std::vector<int64_t> t64(t.begin(), t.end());
    s->accuracy = matching_accuracy(t64.data(), b1, b2, N);
  } else {
    s->accuracy = std::nan("");
  }
}

}  // namespace usap
