// Batched nodal update.
//
// Reference: the nodal_move task (graph_parallel.hpp:406-431) runs
// _propose_new_partition_nodal (:990-1222) for every vertex of a contiguous
// batch against the batch-start state, O(deg + B) per vertex (four length-B
// scratch rows are cleared and scanned); the update task (:433-458) applies
// the buffered moves, rebuilds M from scratch and tests convergence.
//
// Here one warp proposes for one vertex.  Its neighbour blocks are
// aggregated in a per-warp open-addressed hash in shared memory (or, for
// vertices whose degree does not fit, in a per-vertex region of global
// memory), so dS costs O(deg) lookups: each distinct neighbour block b gives
// the changed entries M[r,b], M[s,b] (out-neighbours) or M[b,r], M[b,s]
// (in-neighbours); the entries a move leaves unchanged contribute
// count * (log new degree - log old degree), with the counts known exactly
// from the degrees.  The reference's rule that in-edges from blocks r and s
// do not adjust the 2x2 row entries (the adjustment is commented out at
// :1135-1142) and that column sums skip i in {r,s} is kept.  Accepted moves
// are written to move_to[]; a second kernel applies them to the dense tile
// by +/-w deltas (exact integers, so order does not matter), a third commits
// the partition.  The convergence bookkeeping of the update task runs in a
// one-thread kernel so batches and sweeps queue without host round trips.
#include <cmath>

#include "common.cuh"
#include "engine.h"

namespace usap {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kHCap = 256;   // shared-memory hash slots per warp

struct DenseOps {
  DenseView v;
  int B;
  __device__ __forceinline__ int get(int x, int y) const {
    return __ldg(v.M + static_cast<long long>(x) * v.ld + y);
  }
  // first block i (block-id order) whose cumulative M[u,i]+M[i,u] exceeds t
  __device__ __forceinline__ int sym_sample(int u, long long t, int lane, int* scanned) const {
    const int* rowM = v.M + static_cast<long long>(u) * v.ld;
    const int* rowT = v.Mt + static_cast<long long>(u) * v.ld;
    long long run = 0;
    for (int base = 0; base < B; base += 32) {
      int i = base + lane;
      int val = i < B ? __ldg(rowM + i) + __ldg(rowT + i) : 0;
      int incl = warp_incl_scan(val, lane);
      int total = __shfl_sync(0xffffffffu, incl, 31);
      if (run + total > t) {
        unsigned m = __ballot_sync(0xffffffffu, run + incl > t);
        *scanned += base + 32;
        return base + __ffs(m) - 1;
      }
      run += total;
    }
    *scanned += B;
    return B - 1;
  }
};

struct SortedOps {
  SortedView v;
  int B;
  __device__ __forceinline__ int get(int x, int y) const {
    int lo = __ldg(v.rowptr + x), hi = __ldg(v.rowptr + x + 1);
    int p = find_sorted(v.col, lo, hi, y);
    return p >= 0 ? __ldg(v.val + p) : 0;
  }
  __device__ __forceinline__ int sym_sample(int u, long long t, int lane, int* scanned) const {
    int lo = __ldg(v.symptr + u), hi = __ldg(v.symptr + u + 1);
    long long base = lo > 0 ? __ldg(v.symcum + lo - 1) : 0;
    int j = upper_bound_i(v.symcum, lo, hi, t + base);
    if (j >= hi) j = hi - 1;   // t is below the row total; defensive clamp
    *scanned += 32 - __clz(hi - lo + 1);
    return __ldg(v.symcol + j);
  }
};

__device__ __forceinline__ unsigned hash_slot(int b, int lg) {
  return (static_cast<unsigned>(b) * 0x9E3779B1u) >> (32 - lg);
}

__device__ __forceinline__ int table_lookup_wo(const int* key, const int* wo, int cap, int lg, int b) {
  unsigned h = hash_slot(b, lg);
  while (true) {
    int k = key[h];
    if (k == b) return wo[h];
    if (k == -1) return 0;
    h = (h + 1) & (cap - 1);
  }
}

template <class Ops>
__global__ void __launch_bounds__(kThreads) k_nodal_propose(NodalArgs a, Ops ops) {
  __shared__ int s_key[kWarps][kHCap];
  __shared__ int s_wo[kWarps][kHCap];
  __shared__ int s_wi[kWarps][kHCap];
  if (*reinterpret_cast<volatile int*>(&a.ctl->done)) return;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nwarps = gridDim.x * kWarps;
  const int B = a.B;
  unsigned long long my_bytes = 0;
  for (int v = a.beg + blockIdx.x * kWarps + wib; v < a.end; v += nwarps) {
    const int r = __ldg(a.part + v);
    const long long kout = __ldg(a.kout + v), kin = __ldg(a.kin + v);
    const long long k = kout + kin;
    const int o0 = __ldg(a.out_ptr + v), dego = __ldg(a.out_ptr + v + 1) - o0;
    const int i0 = __ldg(a.in_ptr + v), degi = __ldg(a.in_ptr + v + 1) - i0;
    const int deg = dego + degi;
    Draws x = philox(static_cast<uint32_t>(v), a.itr, a.stage, kTagNodal, a.seed);
    int s;
    int scanned = 0;
    if (k == 0) {
      s = static_cast<int>(draw_below(x.x2, B));
    } else {
      long long t = draw_below(x.x0, k);
      int j;
      if (a.unit) {
        j = static_cast<int>(t);
      } else {   // weighted: first neighbour whose cumulative weight exceeds t
        long long run = 0;
        j = deg - 1;
        for (int base = 0; base < deg; base += 32) {
          int jj = base + lane;
          long long ww = 0;
          if (jj < deg) ww = jj < dego ? __ldg(a.out_w + o0 + jj) : __ldg(a.in_w + i0 + jj - dego);
          long long incl = warp_incl_scan_ll(ww, lane);
          long long total = __shfl_sync(0xffffffffu, incl, 31);
          if (run + total > t) {
            unsigned m = __ballot_sync(0xffffffffu, run + incl > t);
            j = base + __ffs(m) - 1;
            break;
          }
          run += total;
        }
      }
      const int nbr = j < dego ? __ldg(a.out_idx + o0 + j) : __ldg(a.in_idx + i0 + j - dego);
      const int u = __ldg(a.part + nbr);
      const long long dau = static_cast<long long>(__ldg(a.dout + u)) + __ldg(a.din + u);
      if (accept_uniform(x.x1, dau, B)) {
        s = static_cast<int>(draw_below(x.x2, B));
      } else {
        s = ops.sym_sample(u, draw_below(x.x2, dau), lane, &scanned);
      }
    }
    if (s == r) {
      if (a.prop_s && lane == 0) {
        a.prop_s[v - a.beg] = -1;
        a.prop_q[v - a.beg] = 0;
        a.prop_ninf[v - a.beg] = 0;
      }
      if (a.stats && lane == 0) my_bytes += 8 + 8ull * deg + 8ull * scanned;
      continue;
    }
    // --- aggregate the neighbour blocks: wo[b] (out-edges), wi[b] (in-edges)
    int lg = 5;
    while ((1 << lg) < 2 * deg) lg++;
    const int cap = 1 << lg;
    int *key, *two, *twi;
    if (cap <= kHCap) {
      key = s_key[wib];
      two = s_wo[wib];
      twi = s_wi[wib];
    } else {
      long long off = __ldg(a.hi_off + v);
      key = a.hkey + off;
      two = a.hwo + off;
      twi = a.hwi + off;
    }
    for (int i = lane; i < cap; i += 32) {
      key[i] = -1;
      two[i] = 0;
      twi[i] = 0;
    }
    __syncwarp();
    for (int j = lane; j < deg; j += 32) {
      const bool is_out = j < dego;
      const int nb = is_out ? __ldg(a.out_idx + o0 + j) : __ldg(a.in_idx + i0 + j - dego);
      const int ww = a.unit ? 1 : (is_out ? __ldg(a.out_w + o0 + j) : __ldg(a.in_w + i0 + j - dego));
      const int b = __ldg(a.part + nb);
      unsigned h = hash_slot(b, lg);
      while (true) {
        int prev = atomicCAS(key + h, -1, b);
        if (prev == -1 || prev == b) break;
        h = (h + 1) & (cap - 1);
      }
      atomicAdd(is_out ? two + h : twi + h, ww);
    }
    __syncwarp();
    // --- dS terms over the distinct neighbour blocks other than r and s
    const long long dr_out = __ldg(a.dout + r), dr_in = __ldg(a.din + r);
    const long long ds_out = __ldg(a.dout + s), ds_in = __ldg(a.din + s);
    const long long dr_out_n = dr_out - kout, ds_out_n = ds_out + kout;
    const long long dr_in_n = dr_in - kin, ds_in_n = ds_in + kin;
    long long acc = 0;
    int sXR = 0, sXS = 0, sYR = 0, sYS = 0, nb_distinct = 0;
    for (int i = lane; i < cap; i += 32) {
      const int b = key[i];
      if (b < 0) continue;
      nb_distinct++;
      if (b == r || b == s) continue;
      const int wo = two[i], wi = twi[i];
      if (wo > 0) {
        const int R = ops.get(r, b), S = ops.get(s, b);
        const long long dinb = __ldg(a.din + b);
        acc += q32(g_term(a.L, R, dinb, dr_out));
        acc += q32(g_term(a.L, S, dinb, ds_out));
        acc -= q32(g_term(a.L, R - wo, dinb, dr_out_n));
        acc -= q32(g_term(a.L, S + wo, dinb, ds_out_n));
        sXR += R;
        sXS += S;
      }
      if (wi > 0) {
        const int Rc = ops.get(b, r), Sc = ops.get(b, s);
        const long long doutb = __ldg(a.dout + b);
        acc += q32(g_term(a.L, Rc, dr_in, doutb));
        acc += q32(g_term(a.L, Sc, ds_in, doutb));
        acc -= q32(g_term(a.L, Rc - wi, dr_in_n, doutb));
        acc -= q32(g_term(a.L, Sc + wi, ds_in_n, doutb));
        sYR += Rc;
        sYS += Sc;
      }
    }
    acc = warp_sum_ll(acc);
    sXR = warp_sum_i(sXR);
    sXS = warp_sum_i(sXS);
    sYR = warp_sum_i(sYR);
    sYS = warp_sum_i(sYS);
    nb_distinct = warp_sum_i(nb_distinct);
    // 2x2 entries, fetched by four lanes
    int e4 = 0;
    if (lane < 4) e4 = ops.get(lane < 2 ? r : s, (lane & 1) ? s : r);
    const long long Rr = __shfl_sync(0xffffffffu, e4, 0), Rs = __shfl_sync(0xffffffffu, e4, 1);
    const long long Sr = __shfl_sync(0xffffffffu, e4, 2), Ss = __shfl_sync(0xffffffffu, e4, 3);
    if (lane == 0) {
      const long long wor = table_lookup_wo(key, two, cap, lg, r);
      const long long wos = table_lookup_wo(key, two, cap, lg, s);
      acc += q32(g_term(a.L, Rr, dr_in, dr_out));
      acc += q32(g_term(a.L, Rs, ds_in, dr_out));
      acc += q32(g_term(a.L, Sr, dr_in, ds_out));
      acc += q32(g_term(a.L, Ss, ds_in, ds_out));
      int ninf = 0;
      const double nt[4] = {g_term(a.L, Rr - wor, dr_in_n, dr_out_n), g_term(a.L, Rs - wos, ds_in_n, dr_out_n),
                            g_term(a.L, Sr + wor, dr_in_n, ds_out_n), g_term(a.L, Ss + wos, ds_in_n, ds_out_n)};
#pragma unroll
      for (int t = 0; t < 4; t++) {
        if (isinf(nt[t])) ninf = 1;
        else acc -= q32(nt[t]);
      }
      acc += q32(coef_term(a.L, dr_out - Rr - Rs - sXR, dr_out_n, dr_out));
      acc += q32(coef_term(a.L, ds_out - Sr - Ss - sXS, ds_out_n, ds_out));
      acc += q32(coef_term(a.L, dr_in - Rr - Sr - sYR, dr_in_n, dr_in));
      acc += q32(coef_term(a.L, ds_in - Rs - Ss - sYS, ds_in_n, ds_in));
      const bool accept = ninf || acc < 0;
      if (a.prop_s) {
        a.prop_s[v - a.beg] = s;
        a.prop_q[v - a.beg] = acc;
        a.prop_ninf[v - a.beg] = ninf;
      }
      if (accept) {
        a.move_to[v] = s;
        if (ninf) atomicOr(&a.ctl->cum_ninf, 1);
        else atomicAdd(&a.ctl->cum_q, static_cast<unsigned long long>(acc));
        atomicAdd(&a.ctl->moves, 1ull);
      }
      if (!ninf && acc <= kNearQ && acc >= -kNearQ) atomicAdd(&a.ctl->near, 1ull);
      if (a.stats) my_bytes += 8 + 8ull * deg + 48ull * nb_distinct + 48 + 8ull * scanned;
    }
    __syncwarp();
  }
  if (a.stats && lane == 0 && my_bytes) atomicAdd(&a.ctl->bytes, my_bytes);
}

// Apply accepted moves of [beg, end) to the dense tile by deltas.  An edge
// between two moved vertices is handled once, from its source's out-list.
__global__ void __launch_bounds__(kThreads) k_nodal_apply_dense(
    const int32_t* __restrict__ out_ptr, const int32_t* __restrict__ out_idx,
    const int32_t* __restrict__ out_w, const int32_t* __restrict__ in_ptr,
    const int32_t* __restrict__ in_idx, const int32_t* __restrict__ in_w,
    const int32_t* __restrict__ part, const int32_t* __restrict__ move_to, int beg, int end, int ld,
    int* __restrict__ M, int* __restrict__ Mt, const NodalCtl* ctl) {
  const int lane = threadIdx.x & 31;
  const int nwarps = gridDim.x * kWarps;
  for (int v = beg + blockIdx.x * kWarps + (threadIdx.x >> 5); v < end; v += nwarps) {
    const int s = move_to[v];
    if (s < 0) continue;
    const int r = part[v];
    const int o0 = out_ptr[v], o1 = out_ptr[v + 1];
    for (int p = o0 + lane; p < o1; p += 32) {
      const int y = out_idx[p];
      const int w = out_w ? out_w[p] : 1;
      const int oy = part[y];
      const int my = move_to[y];
      const int ny = my >= 0 ? my : oy;
      atomicAdd(M + static_cast<long long>(r) * ld + oy, -w);
      atomicAdd(Mt + static_cast<long long>(oy) * ld + r, -w);
      atomicAdd(M + static_cast<long long>(s) * ld + ny, w);
      atomicAdd(Mt + static_cast<long long>(ny) * ld + s, w);
    }
    const int i0 = in_ptr[v], i1 = in_ptr[v + 1];
    for (int p = i0 + lane; p < i1; p += 32) {
      const int y = in_idx[p];
      if (move_to[y] >= 0) continue;
      const int w = in_w ? in_w[p] : 1;
      const int oy = part[y];
      atomicAdd(M + static_cast<long long>(oy) * ld + r, -w);
      atomicAdd(Mt + static_cast<long long>(r) * ld + oy, -w);
      atomicAdd(M + static_cast<long long>(oy) * ld + s, w);
      atomicAdd(Mt + static_cast<long long>(s) * ld + oy, w);
    }
  }
}

__global__ void k_nodal_commit(int32_t* __restrict__ part, int32_t* __restrict__ move_to,
                               const int32_t* __restrict__ kout, const int32_t* __restrict__ kin,
                               int beg, int end, int update_degrees, int32_t* __restrict__ dout,
                               int32_t* __restrict__ din) {
  int stride = gridDim.x * blockDim.x;
  for (int v = beg + blockIdx.x * blockDim.x + threadIdx.x; v < end; v += stride) {
    const int s = move_to[v];
    if (s < 0) continue;
    const int r = part[v];
    if (update_degrees) {
      atomicSub(dout + r, kout[v]);
      atomicAdd(dout + s, kout[v]);
      atomicSub(din + r, kin[v]);
      atomicAdd(din + s, kin[v]);
    }
    part[v] = s;
    move_to[v] = -1;
  }
}

// prepare_batch (:381-395): S from the entropy kernel, the moving average
// of the previous sweeps' dS, and a fresh cumulative sum for this sweep
__global__ void k_ctl_sweep_start(NodalCtl* ctl, long long model_q, int itr, int W,
                                  const long long* ide_q, const int* ide_n) {
  if (ctl->done) return;
  ctl->S_q = model_q - static_cast<long long>(ctl->entropy_acc);
  ctl->S_ninf = 0;
  double mean = 0.0;
  if (itr >= W - 1) {
    long long sum = 0;
    int ninf = 0;
    for (int i = itr - W + 1; i < itr; i++) {
      sum += ide_q[i];
      ninf |= ide_n[i];
    }
    mean = ninf ? -INFINITY : (static_cast<double>(sum) / kQ32) / static_cast<double>(W - 1);
  }
  ctl->mean = mean;
  ctl->cum_q = 0;
  ctl->cum_ninf = 0;
  ctl->sweeps++;
}

// update (:433-458): the sweep's cumulative dS is recorded for this sweep
// and added to S after every batch (as the reference does), then the
// convergence test -mean < thr * S ends the nodal phase
__global__ void k_ctl_batch_end(NodalCtl* ctl, int itr, int W, double thr, long long* ide_q,
                                int* ide_n, long long batch_vertices, long long batch_edges) {
  if (ctl->done) return;
  const long long cum = static_cast<long long>(ctl->cum_q);
  ide_q[itr] = cum;
  ide_n[itr] = ctl->cum_ninf;
  ctl->S_q += cum;
  ctl->S_ninf |= ctl->cum_ninf;
  ctl->batches++;
  ctl->proposals += batch_vertices;
  ctl->edge_visits += batch_edges;
  if (itr >= W - 1) {
    double S_d = ctl->S_ninf ? -INFINITY : static_cast<double>(ctl->S_q) / kQ32;
    if (-ctl->mean < thr * S_d) ctl->done = 1;
  }
}

template <class Ops>
void launch_propose(const NodalArgs& a, Ops ops, cudaStream_t st) {
  int count = a.end - a.beg;
  if (count <= 0) return;
  int blocks = (count + kWarps - 1) / kWarps;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_nodal_propose<Ops><<<blocks, kThreads, 0, st>>>(a, ops);
  USAP_CUDA(cudaGetLastError());
}

}  // namespace

void launch_nodal_propose_dense(const NodalArgs& a, DenseView v, cudaStream_t st) {
  launch_propose(a, DenseOps{v, a.B}, st);
}

void launch_nodal_propose_sorted(const NodalArgs& a, SortedView v, cudaStream_t st) {
  launch_propose(a, SortedOps{v, a.B}, st);
}

void launch_nodal_apply_dense(const GraphDev& g, const int32_t* part, int32_t* move_to, int beg,
                              int end, int ld, int* M, int* Mt, int32_t* dout, int32_t* din,
                              const NodalCtl* ctl, cudaStream_t st) {
  int count = end - beg;
  if (count <= 0) return;
  int blocks = (count + kWarps - 1) / kWarps;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_nodal_apply_dense<<<blocks, kThreads, 0, st>>>(g.out_ptr, g.out_idx, g.out_w, g.in_ptr, g.in_idx,
                                                  g.in_w, part, move_to, beg, end, ld, M, Mt, ctl);
  USAP_CUDA(cudaGetLastError());
}

void launch_nodal_commit(const GraphDev& g, int32_t* part, int32_t* move_to, int beg, int end,
                         int update_degrees, int32_t* dout, int32_t* din, const NodalCtl* ctl,
                         cudaStream_t st) {
  int count = end - beg;
  if (count <= 0) return;
  int blocks = (count + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_nodal_commit<<<blocks, 256, 0, st>>>(part, move_to, g.kout, g.kin, beg, end, update_degrees, dout,
                                         din);
  USAP_CUDA(cudaGetLastError());
}

void launch_ctl_sweep_start(NodalCtl* ctl, long long model_q, int itr, int W, const long long* ide_q,
                            const int* ide_n, cudaStream_t st) {
  k_ctl_sweep_start<<<1, 1, 0, st>>>(ctl, model_q, itr, W, ide_q, ide_n);
  USAP_CUDA(cudaGetLastError());
}

void launch_ctl_batch_end(NodalCtl* ctl, int itr, int W, double thr, long long* ide_q, int* ide_n,
                          long long batch_vertices, long long batch_edges, cudaStream_t st) {
  k_ctl_batch_end<<<1, 1, 0, st>>>(ctl, itr, W, thr, ide_q, ide_n, batch_vertices, batch_edges);
  USAP_CUDA(cudaGetLastError());
}

}  // namespace usap
