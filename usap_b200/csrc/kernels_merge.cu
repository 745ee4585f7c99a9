// Block-merge phase.
//
// Reference: block_merge task (graph_parallel.hpp:349-368) runs K proposals
// per block through _propose_new_partition_block (:761-988), O(B) each;
// _carry_out_best_merges (:1225-1279) then sorts the blocks by dS and merges
// them one at a time with a block_map relabel, O(B_to_merge*(B+N)).
//
// Here one warp handles one (block r, proposal k) pair: the neighbour block
// and the target are drawn by integer inverse-CDF over the block-id-sorted
// symmetric rows M[u,:]+M[:,u] (binary search on cumulative counts), and dS
// needs only the 2x2 entries of {r,s}, the block degrees and the columns
// where rows (columns) r and s are both non-zero (rows and columns that only
// one of them touches contribute count * log-ratio terms known from the
// degrees).  The merges are applied by a parallel restatement of the
// sequential walk: in sorted order a block r merges into the current
// representative of best_s[r] unless that representative is r itself.  With
// f(r) = best_s[r] a functional graph, the skipped blocks are exactly the
// last (in sorted order) member of each cycle of f; everything else points
// to best_s until the B_to_merge-th success.  Cycles and representatives
// are found by pointer jumping.
#include <cub/cub.cuh>

#include "common.cuh"
#include "engine.h"

namespace usap {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ int sv_get(const int* __restrict__ ptr, const int* __restrict__ idx,
                                      const int* __restrict__ val, int x, int y) {
  int lo = __ldg(ptr + x), hi = __ldg(ptr + x + 1);
  int p = find_sorted(idx, lo, hi, y);
  return p >= 0 ? __ldg(val + p) : 0;
}

// first entry of symmetric row u whose cumulative count exceeds t
__device__ __forceinline__ int sym_pick(const SortedView& v, int u, long long t) {
  int lo = __ldg(v.symptr + u), hi = __ldg(v.symptr + u + 1);
  long long base = lo > 0 ? __ldg(v.symcum + lo - 1) : 0;
  int j = upper_bound_i(v.symcum, lo, hi, t + base);
  if (j >= hi) j = hi - 1;   // t is below the row total; defensive clamp
  return __ldg(v.symcol + j);
}

// FP32 pair sum over the warp; every lane gets the same value
__device__ __forceinline__ FF warp_ffsum(FF f) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    f = ff_add(f, FF{__shfl_xor_sync(0xffffffffu, f.hi, o), __shfl_xor_sync(0xffffffffu, f.lo, o)});
  return f;
}

// P (precision mode 1 or 2): dS is also evaluated in FP32 and the merge key
// (argmin, merge order) is the FP32 value in Q32; the exact value is kept
// beside it
template <int P>
__global__ void __launch_bounds__(kThreads) k_merge_propose(SortedView v, MergeArgs a) {
  constexpr bool F32 = P > 0;
  __shared__ F32Tally s_f32;
  if (F32) {
    if (threadIdx.x == 0) s_f32 = F32Tally{0, 0, 0, 0.0};
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const long long items = static_cast<long long>(a.B) * a.K;
  const long long nwarps = static_cast<long long>(gridDim.x) * kWarps;
  for (long long item = static_cast<long long>(blockIdx.x) * kWarps + (threadIdx.x >> 5); item < items;
       item += nwarps) {
    const int r = static_cast<int>(item / a.K), k = static_cast<int>(item - static_cast<long long>(r) * a.K);
    const int B = a.B;
    Draws x = philox(static_cast<uint32_t>(r), static_cast<uint32_t>(k), a.stage, kTagMerge, a.seed);
    const long long dr_out = __ldg(a.dout + r), dr_in = __ldg(a.din + r);
    const long long ka = dr_out + dr_in;
    int s;
    if (ka == 0) {
      s = static_cast<int>(draw_below(x.x2, B));
    } else {
      int u = sym_pick(v, r, draw_below(x.x0, ka));
      long long dau = static_cast<long long>(__ldg(a.dout + u)) + __ldg(a.din + u);
      if (accept_uniform(x.x1, dau, B)) {
        s = skip_r(static_cast<int>(draw_below(x.x2, B)), r, B);
      } else {
        int lo = __ldg(v.symptr + u), hi = __ldg(v.symptr + u + 1);
        int pr = find_sorted(v.symcol, lo, hi, r);
        long long base = lo > 0 ? __ldg(v.symcum + lo - 1) : 0;
        long long c_ur = 0, before = 0;
        if (pr >= 0) {
          long long prev = pr > 0 ? __ldg(v.symcum + pr - 1) : 0;
          c_ur = __ldg(v.symcum + pr) - prev;
          before = prev - base;
        }
        long long wsum = dau - c_ur;
        if (wsum == 0) {
          s = skip_r(static_cast<int>(draw_below(x.x2, B)), r, B);
        } else {
          long long t2 = draw_below(x.x2, wsum);
          if (pr >= 0 && t2 >= before) t2 += c_ur;
          s = sym_pick(v, u, t2);
        }
      }
    }
    // --- dS of merging r into s ---
    const long long ds_out = __ldg(a.dout + s), ds_in = __ldg(a.din + s);
    const long long ds_out_n = ds_out + dr_out, ds_in_n = ds_in + dr_in;
    int e4 = 0;
    if (lane < 4) {
      int x0 = (lane < 2) ? r : s, y0 = (lane & 1) ? s : r;
      e4 = sv_get(v.rowptr, v.col, v.val, x0, y0);
    }
    const long long Mrr = __shfl_sync(0xffffffffu, e4, 0), Mrs = __shfl_sync(0xffffffffu, e4, 1);
    const long long Msr = __shfl_sync(0xffffffffu, e4, 2), Mss = __shfl_sync(0xffffffffu, e4, 3);
    long long acc = 0;
    FF f{0.0f, 0.0f};
    // rows: entries present in both row r and row s (h is symmetric)
    {
      int rlo = __ldg(v.rowptr + r), rhi = __ldg(v.rowptr + r + 1);
      int slo = __ldg(v.rowptr + s), shi = __ldg(v.rowptr + s + 1);
      bool iter_r = (rhi - rlo) <= (shi - slo);
      int ilo = iter_r ? rlo : slo, ihi = iter_r ? rhi : shi;
      int olo = iter_r ? slo : rlo, ohi = iter_r ? shi : rhi;
      for (int p = ilo + lane; p < ihi; p += 32) {
        int i = __ldg(v.col + p);
        if (i == r || i == s) continue;
        int q = find_sorted(v.col, olo, ohi, i);
        if (q >= 0) {
          const int x = __ldg(v.val + p), y = __ldg(v.val + q);
          acc += q32(h_term(a.L, x, y));
          if constexpr (F32) f = ff_add(f, h_term_ff<P>(a.L2, x, y));
        }
      }
    }
    // columns likewise, through the CSC
    {
      int rlo = __ldg(v.colptr + r), rhi = __ldg(v.colptr + r + 1);
      int slo = __ldg(v.colptr + s), shi = __ldg(v.colptr + s + 1);
      bool iter_r = (rhi - rlo) <= (shi - slo);
      int ilo = iter_r ? rlo : slo, ihi = iter_r ? rhi : shi;
      int olo = iter_r ? slo : rlo, ohi = iter_r ? shi : rhi;
      for (int p = ilo + lane; p < ihi; p += 32) {
        int i = __ldg(v.row + p);
        if (i == r || i == s) continue;
        int q = find_sorted(v.row, olo, ohi, i);
        if (q >= 0) {
          const int x = __ldg(v.cval + p), y = __ldg(v.cval + q);
          acc += q32(h_term(a.L, x, y));
          if constexpr (F32) f = ff_add(f, h_term_ff<P>(a.L2, x, y));
        }
      }
    }
    acc = warp_sum_ll(acc);
    if constexpr (F32) f = warp_ffsum(f);
    if (lane == 0) {
      acc += q32(g_term(a.L, Mrr, dr_in, dr_out));
      acc += q32(g_term(a.L, Mrs, ds_in, dr_out));
      acc += q32(g_term(a.L, Msr, dr_in, ds_out));
      acc += q32(g_term(a.L, Mss, ds_in, ds_out));
      acc -= q32(g_term(a.L, Mrr + Mrs + Msr + Mss, ds_in_n, ds_out_n));
      if constexpr (F32) {
        f = ff_add(f, g_term_ff<P>(a.L2, Mrr, dr_in, dr_out));
        f = ff_add(f, g_term_ff<P>(a.L2, Mrs, ds_in, dr_out));
        f = ff_add(f, g_term_ff<P>(a.L2, Msr, dr_in, ds_out));
        f = ff_add(f, g_term_ff<P>(a.L2, Mss, ds_in, ds_out));
        f = ff_sub(f, g_term_ff<P>(a.L2, Mrr + Mrs + Msr + Mss, ds_in_n, ds_out_n));
      }
      long long Ar, As, Cr, Cs;
      if (s != r) {
        Ar = dr_out - Mrr - Mrs;
        As = ds_out - Msr - Mss;
        Cr = dr_in - Mrr - Msr;
        Cs = ds_in - Mrs - Mss;
      } else {
        Ar = As = dr_out - Mrr;
        Cr = Cs = dr_in - Mrr;
      }
      acc += q32(coef_term(a.L, Ar, ds_out_n, dr_out));
      acc += q32(coef_term(a.L, As, ds_out_n, ds_out));
      acc += q32(coef_term(a.L, Cr, ds_in_n, dr_in));
      acc += q32(coef_term(a.L, Cs, ds_in_n, ds_in));
      a.prop_s[item] = s;
      if constexpr (F32) {
        const float2* __restrict__ T = a.L2;
        f = ff_add(f, coef_ff<P>(Ar, ld_ff(T, ds_out_n), ld_ff(T, dr_out)));
        f = ff_add(f, coef_ff<P>(As, ld_ff(T, ds_out_n), ld_ff(T, ds_out)));
        f = ff_add(f, coef_ff<P>(Cr, ld_ff(T, ds_in_n), ld_ff(T, dr_in)));
        f = ff_add(f, coef_ff<P>(Cs, ld_ff(T, ds_in_n), ld_ff(T, ds_in)));
        const double fv = ff_value(f);
        a.prop_q[item] = q32(fv);
        a.prop_x[item] = acc;
        a.prop_f[item] = fv;
        const double err = f32_err(fv, acc);
        atomicAdd(&s_f32.evals, 1ull);
        atomicMax(&s_f32.err_max, static_cast<unsigned long long>(__double_as_longlong(err)));
        atomicAdd(&s_f32.err_sum, err);
      } else {
        a.prop_q[item] = acc;
      }
    }
  }
  if (F32) {
    __syncthreads();
    if (threadIdx.x == 0) f32_tally_flush(&s_f32, a.f32);
  }
}

// first strict minimum over the K proposals of each block (:363-366).
// prop_x (precision modes 1, 2): the exact values, whose first strict minimum
// is found too; a block whose two choices differ counts as a flip, and
// best_x gets the exact value of the chosen proposal.
__global__ void k_merge_argmin(int B, int K, const int32_t* __restrict__ prop_s,
                               const long long* __restrict__ prop_q, const long long* __restrict__ prop_x,
                               int32_t* __restrict__ best_s, long long* __restrict__ best_q,
                               long long* __restrict__ best_x, F32Tally* f32) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= B) return;
  long long bq = LLONG_MAX, xq = LLONG_MAX;
  int bs = -1, bk = -1, xk = -1;
  for (int k = 0; k < K; k++) {
    const long long i = static_cast<long long>(r) * K + k;
    long long q = prop_q[i];
    if (q < bq) {
      bq = q;
      bs = prop_s[i];
      bk = k;
    }
    if (prop_x) {
      const long long x = prop_x[i];
      if (x < xq) {
        xq = x;
        xk = k;
      }
    }
  }
  best_s[r] = bs;
  best_q[r] = bq;
  if (prop_x) {
    best_x[r] = bk >= 0 ? prop_x[static_cast<long long>(r) * K + bk] : LLONG_MAX;
    if (bk != xk && (bk < 0 || xk < 0 || prop_s[static_cast<long long>(r) * K + bk] !=
                                             prop_s[static_cast<long long>(r) * K + xk]))
      atomicAdd(&f32->flips, 1ull);
  }
}

// precision modes 1, 2: adjacent pairs of the merge order (sorted by the FP32
// key) that the exact values would put the other way round
__global__ void k_order_flips(int B, const int32_t* __restrict__ order, const long long* __restrict__ best_x,
                              unsigned long long* count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i + 1 >= B) return;
  const int a = order[i], b = order[i + 1];
  const long long xa = best_x[a], xb = best_x[b];
  if (xa > xb || (xa == xb && a > b)) atomicAdd(count, 1ull);
}

__global__ void k_sort_keys(int B, const long long* __restrict__ best_q,
                            unsigned long long* __restrict__ keys, int32_t* __restrict__ idx) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= B) return;
  keys[r] = static_cast<unsigned long long>(best_q[r]) ^ 0x8000000000000000ull;  // order-preserving
  idx[r] = r;
}

// One CTA: cycles of f = best_s, skips, the stopping point and the final
// representative root[b] of every block.  `work` holds 8*B ints.
__global__ void __launch_bounds__(1024) k_merge_union(int B, const int32_t* __restrict__ order,
                                                      const int32_t* __restrict__ best_s, int btm,
                                                      int32_t* __restrict__ work,
                                                      int32_t* __restrict__ root,
                                                      int32_t* __restrict__ merged) {
  int32_t* pos = work;
  int32_t* F = work + B;
  int32_t* F2 = work + 2 * B;
  int32_t* MX = work + 3 * B;
  int32_t* MX2 = work + 4 * B;
  int32_t* cyc = work + 5 * B;
  int32_t* succ = work + 6 * B;   // success flag by sorted position
  int32_t* P2 = work + 7 * B;
  const int t = threadIdx.x, nt = blockDim.x;
  int rounds = 1;
  while ((1 << rounds) < B) rounds++;
  rounds++;
  for (int p = t; p < B; p += nt) pos[order[p]] = p;
  __syncthreads();
  for (int i = t; i < B; i += nt) {
    F[i] = best_s[i];
    MX[i] = pos[i];
    cyc[i] = 0;
  }
  __syncthreads();
  for (int k = 0; k < rounds; k++) {
    for (int i = t; i < B; i += nt) {
      int f = F[i];
      F2[i] = F[f];
      int m = MX[f];
      MX2[i] = MX[i] > m ? MX[i] : m;
    }
    __syncthreads();
    for (int i = t; i < B; i += nt) {
      F[i] = F2[i];
      MX[i] = MX2[i];
    }
    __syncthreads();
  }
  for (int i = t; i < B; i += nt) cyc[F[i]] = 1;   // f^(2^rounds)(i) lies on a cycle
  __syncthreads();
  for (int i = t; i < B; i += nt) {
    bool skip = cyc[i] && MX[i] == pos[i];        // last member of its cycle
    succ[pos[i]] = skip ? 0 : 1;
  }
  __syncthreads();
  // stopping point: first sorted position where the successes reach btm
  __shared__ int s_chunk[1024];
  __shared__ int s_stop;
  if (t == 0) s_stop = B;   // none
  __syncthreads();
  int carry = 0;
  for (int base = 0; base < B; base += nt) {
    int p = base + t;
    int v = p < B ? succ[p] : 0;
    s_chunk[t] = v;
    __syncthreads();
    for (int o = 1; o < nt; o <<= 1) {   // Hillis-Steele inclusive scan
      int add = t >= o ? s_chunk[t - o] : 0;
      __syncthreads();
      s_chunk[t] += add;
      __syncthreads();
    }
    int incl = carry + s_chunk[t];
    if (p < B && v && incl == btm) s_stop = p;   // unique position
    int chunk_total = s_chunk[nt - 1];
    __syncthreads();
    carry += chunk_total;
  }
  __syncthreads();
  // btm <= 0: nothing merges; fewer successes than btm: every block is
  // processed (the reference's walk would run past the end of its order)
  const int stop = btm <= 0 ? -1 : (s_stop < B ? s_stop : B - 1);
  if (t == 0) *merged = btm <= 0 ? 0 : (s_stop < B ? btm : carry);
  // parent pointers, then pointer jumping to the roots
  for (int i = t; i < B; i += nt) {
    bool ok = pos[i] <= stop && succ[pos[i]];
    F[i] = ok ? best_s[i] : i;
  }
  __syncthreads();
  for (int k = 0; k < rounds; k++) {
    for (int i = t; i < B; i += nt) P2[i] = F[F[i]];
    __syncthreads();
    for (int i = t; i < B; i += nt) F[i] = P2[i];
    __syncthreads();
  }
  for (int i = t; i < B; i += nt) root[i] = F[i];
}

__global__ void k_present(int n, const int32_t* __restrict__ part, const int32_t* __restrict__ root,
                          int32_t* __restrict__ present) {
  int stride = gridDim.x * blockDim.x;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) present[root[part[v]]] = 1;
}

__global__ void k_relabel(int n, int32_t* __restrict__ part, const int32_t* __restrict__ root,
                          const int32_t* __restrict__ newlabel) {
  int stride = gridDim.x * blockDim.x;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) part[v] = newlabel[root[part[v]]];
}

}  // namespace

void launch_merge_propose(const GraphDev& g, SortedView v, const MergeArgs& a, cudaStream_t st) {
  long long items = static_cast<long long>(a.B) * a.K;
  long long blocks = (items + kWarps - 1) / kWarps;
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  if (a.prec == 1) k_merge_propose<1><<<static_cast<int>(blocks), kThreads, 0, st>>>(v, a);
  else if (a.prec == 2) k_merge_propose<2><<<static_cast<int>(blocks), kThreads, 0, st>>>(v, a);
  else k_merge_propose<0><<<static_cast<int>(blocks), kThreads, 0, st>>>(v, a);
  USAP_LAUNCHED();
}

void launch_merge_argmin(int B, int K, const int32_t* prop_s, const long long* prop_q, const long long* prop_x,
                         int32_t* best_s, long long* best_q, long long* best_x, F32Tally* f32, cudaStream_t st) {
  k_merge_argmin<<<(B + 255) / 256, 256, 0, st>>>(B, K, prop_s, prop_q, prop_x, best_s, best_q, best_x, f32);
  USAP_LAUNCHED();
}

void launch_order_flips(int B, const int32_t* order, const long long* best_x, unsigned long long* count,
                        cudaStream_t st) {
  if (B < 2) return;
  k_order_flips<<<(B + 255) / 256, 256, 0, st>>>(B, order, best_x, count);
  USAP_LAUNCHED();
}

void launch_merge_union(int B, const int32_t* order, const int32_t* best_s, int btm, int32_t* work,
                        int32_t* root, int32_t* merged, cudaStream_t st) {
  k_merge_union<<<1, 1024, 0, st>>>(B, order, best_s, btm, work, root, merged);
  USAP_LAUNCHED();
}

void launch_merge_relabel(int n, int B, int32_t* part, const int32_t* root, int32_t* present,
                          int32_t* newlabel, void* cub_tmp, size_t cub_bytes, cudaStream_t st) {
  USAP_CUDA(cudaMemsetAsync(present, 0, sizeof(int32_t) * B, st));
  int grid = (n + 255) / 256;
  if (grid > 148 * 8) grid = 148 * 8;
  k_present<<<grid, 256, 0, st>>>(n, part, root, present);
  USAP_LAUNCHED();
  size_t bytes = cub_bytes;
  USAP_CUB(cub::DeviceScan::ExclusiveSum(cub_tmp, bytes, present, newlabel, B, st));
  k_relabel<<<grid, 256, 0, st>>>(n, part, root, newlabel);
  USAP_LAUNCHED();
}

// exposed for the engine: keys for the stable (dS, block) sort
void launch_merge_sort_keys(int B, const long long* best_q, unsigned long long* keys, int32_t* idx,
                            cudaStream_t st) {
  k_sort_keys<<<(B + 255) / 256, 256, 0, st>>>(B, best_q, keys, idx);
  USAP_LAUNCHED();
}

}  // namespace usap
