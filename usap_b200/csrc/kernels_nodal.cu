// Batched nodal update.
//
// Reference: the nodal_move task (graph_parallel.hpp:406-431) runs
// _propose_new_partition_nodal (:990-1222) for every vertex of a contiguous
// batch against the batch-start state, O(deg + B) per vertex (four length-B
// scratch rows are cleared and scanned); the update task (:433-458) applies
// the buffered moves, rebuilds M from scratch and tests convergence.
//
// Here one warp proposes for one vertex (one CTA for vertices of degree
// above kHubDegree, so a hub does not set the batch's tail).  The target is
// drawn in block-id order: on the dense tile through per-row chunk sums of
// M[u,:]+M[:,u] (chunks of 128 blocks, kept current by the same delta
// updates as M), on the sparse views by binary search of cumulative counts.
// The vertex's neighbour blocks are aggregated in an open-addressed hash in
// shared memory (global memory for the largest hubs), so dS costs O(deg)
// lookups: each distinct neighbour block b gives the changed entries
// M[r,b], M[s,b] (out-neighbours) or M[b,r], M[b,s] (in-neighbours); the
// entries a move leaves unchanged contribute count * (log new degree - log
// old degree), with the counts known exactly from the degrees.  The
// reference's rule that in-edges from blocks r and s do not adjust the 2x2
// row entries (the adjustment is commented out at :1135-1142) and that
// column sums skip i in {r,s} is kept.  Accepted moves are written to
// move_to[]; a second kernel applies them to the dense tile by +/-w deltas
// (exact integers, so order does not matter), a third commits the
// partition.  The convergence bookkeeping of the update task runs in a
// one-thread kernel so batches and sweeps queue without host round trips.
#include <cmath>
#include <mutex>

#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include "common.cuh"
#include "engine.h"

namespace cg = cooperative_groups;

namespace usap {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kHCap = 256;          // shared-memory hash slots per warp
constexpr int kChunk = 128;         // blocks per chunk sum of a dense row
constexpr int kHubThreads = 512;    // threads of a hub CTA
constexpr int kHubWarps = kHubThreads / 32;

struct DenseOps {
  DenseView v;
  int B;
  __device__ __forceinline__ int get(int x, int y) const {
    return __ldg(v.M + static_cast<long long>(x) * v.ld + y);
  }
  // first block i (block-id order) whose cumulative M[u,i]+M[i,u] exceeds t:
  // a warp scan over the row's chunk sums, then over the 128 entries of the
  // chosen chunk (4 per lane, 16-byte loads; rows are padded to ld, a
  // multiple of 4, with zeros)
  __device__ __forceinline__ int sym_sample(int u, long long t, int lane, int* scanned) const {
    const int nch = (B + kChunk - 1) / kChunk;
    const int* cs = v.CS + static_cast<long long>(u) * v.cld;
    long long run = 0;
    int c = nch - 1;
    for (int base = 0; base < nch; base += 32) {
      const int cc = base + lane;
      const int val = cc < nch ? __ldg(cs + cc) : 0;
      const int incl = warp_incl_scan(val, lane);
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      if (run + total > t) {
        const unsigned m = __ballot_sync(0xffffffffu, run + incl > t);
        const int l = __ffs(m) - 1;
        c = base + l;
        run += __shfl_sync(0xffffffffu, incl - val, l);
        break;
      }
      run += total;
    }
    const int i0 = c * kChunk + lane * 4;
    int p0 = 0, p1 = 0, p2 = 0, p3 = 0;
    if (i0 < B) {
      const int4 a = __ldg(reinterpret_cast<const int4*>(v.M + static_cast<long long>(u) * v.ld + i0));
      const int4 b = __ldg(reinterpret_cast<const int4*>(v.Mt + static_cast<long long>(u) * v.ld + i0));
      p0 = a.x + b.x;
      p1 = p0 + a.y + b.y;
      p2 = p1 + a.z + b.z;
      p3 = p2 + a.w + b.w;
    }
    const int incl = warp_incl_scan(p3, lane);
    const long long before = run + incl - p3;
    const unsigned m = __ballot_sync(0xffffffffu, run + incl > t);
    const int l = m ? __ffs(m) - 1 : 31;
    int k = 3;
    if (before + p0 > t) k = 0;
    else if (before + p1 > t) k = 1;
    else if (before + p2 > t) k = 2;
    *scanned += nch + kChunk;
    int i = c * kChunk + l * 4 + __shfl_sync(0xffffffffu, k, l);
    return i < B ? i : B - 1;
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

__device__ __forceinline__ void table_insert(int* key, int* two, int* twi, int cap, int lg, int b,
                                             int ww, bool is_out) {
  unsigned h = hash_slot(b, lg);
  while (true) {
    int prev = atomicCAS(key + h, -1, b);
    if (prev == -1 || prev == b) break;
    h = (h + 1) & (cap - 1);
  }
  atomicAdd(is_out ? two + h : twi + h, ww);
}

struct VertexInfo {
  int r;
  long long kout, kin;
  int o0, dego, i0, degi;
};

__device__ __forceinline__ VertexInfo vertex_info(const NodalArgs& a, int v) {
  VertexInfo vi;
  vi.r = __ldg(a.part + v);
  vi.kout = __ldg(a.kout + v);
  vi.kin = __ldg(a.kin + v);
  vi.o0 = __ldg(a.out_ptr + v);
  vi.dego = __ldg(a.out_ptr + v + 1) - vi.o0;
  vi.i0 = __ldg(a.in_ptr + v);
  vi.degi = __ldg(a.in_ptr + v + 1) - vi.i0;
  return vi;
}

// target block of the proposal for v (warp-collective: all 32 lanes)
template <class Ops>
__device__ __forceinline__ int propose_target(const NodalArgs& a, const Ops& ops, int v,
                                              const VertexInfo& vi, int lane, int* scanned) {
  const int B = a.B;
  const Draws x = philox(static_cast<uint32_t>(v), static_cast<uint32_t>(a.ctl->itr), a.stage, kTagNodal,
                         a.seed);
  const long long k = vi.kout + vi.kin;
  if (k == 0) return static_cast<int>(draw_below(x.x2, B));
  const long long t = draw_below(x.x0, k);
  const int deg = vi.dego + vi.degi;
  int j;
  if (a.unit) {
    j = static_cast<int>(t);
  } else {   // weighted: first neighbour whose cumulative weight exceeds t
    long long run = 0;
    j = deg - 1;
    for (int base = 0; base < deg; base += 32) {
      const int jj = base + lane;
      long long ww = 0;
      if (jj < deg) ww = jj < vi.dego ? __ldg(a.out_w + vi.o0 + jj) : __ldg(a.in_w + vi.i0 + jj - vi.dego);
      const long long incl = warp_incl_scan_ll(ww, lane);
      const long long total = __shfl_sync(0xffffffffu, incl, 31);
      if (run + total > t) {
        const unsigned m = __ballot_sync(0xffffffffu, run + incl > t);
        j = base + __ffs(m) - 1;
        break;
      }
      run += total;
    }
  }
  const int nbr = j < vi.dego ? __ldg(a.out_idx + vi.o0 + j) : __ldg(a.in_idx + vi.i0 + j - vi.dego);
  const int u = __ldg(a.part + nbr);
  const long long dau = static_cast<long long>(__ldg(a.dout + u)) + __ldg(a.din + u);
  if (accept_uniform(x.x1, dau, B)) return static_cast<int>(draw_below(x.x2, B));
  return ops.sym_sample(u, draw_below(x.x2, dau), lane, scanned);
}

struct TermSums {
  long long acc;
  int sXR, sXS, sYR, sYS, nb;
};

// dS terms of one aggregated neighbour block b (b not in {r, s})
template <class Ops>
__device__ __forceinline__ void slot_terms(const NodalArgs& a, const Ops& ops, int r, int s, int b,
                                           int wo, int wi, long long dr_out, long long ds_out,
                                           long long dr_in, long long ds_in, long long dr_out_n,
                                           long long ds_out_n, long long dr_in_n, long long ds_in_n,
                                           TermSums& ts) {
  if (wo > 0) {
    const int R = ops.get(r, b), S = ops.get(s, b);
    const long long dinb = __ldg(a.din + b);
    ts.acc += q32(g_term(a.L, R, dinb, dr_out));
    ts.acc += q32(g_term(a.L, S, dinb, ds_out));
    ts.acc -= q32(g_term(a.L, R - wo, dinb, dr_out_n));
    ts.acc -= q32(g_term(a.L, S + wo, dinb, ds_out_n));
    ts.sXR += R;
    ts.sXS += S;
  }
  if (wi > 0) {
    const int Rc = ops.get(b, r), Sc = ops.get(b, s);
    const long long doutb = __ldg(a.dout + b);
    ts.acc += q32(g_term(a.L, Rc, dr_in, doutb));
    ts.acc += q32(g_term(a.L, Sc, ds_in, doutb));
    ts.acc -= q32(g_term(a.L, Rc - wi, dr_in_n, doutb));
    ts.acc -= q32(g_term(a.L, Sc + wi, ds_in_n, doutb));
    ts.sYR += Rc;
    ts.sYS += Sc;
  }
}

// 2x2 and unchanged-entry terms, the accept rule (dS < 0, -inf included)
// and the outputs; one thread
template <class Ops>
__device__ __forceinline__ void finalize(const NodalArgs& a, const Ops& ops, int v, int r, int s,
                                         const VertexInfo& vi, TermSums ts, long long wor,
                                         long long wos, long long Rr, long long Rs, long long Sr,
                                         long long Ss, int scanned, unsigned long long* my_bytes) {
  const long long dr_out = __ldg(a.dout + r), dr_in = __ldg(a.din + r);
  const long long ds_out = __ldg(a.dout + s), ds_in = __ldg(a.din + s);
  const long long dr_out_n = dr_out - vi.kout, ds_out_n = ds_out + vi.kout;
  const long long dr_in_n = dr_in - vi.kin, ds_in_n = ds_in + vi.kin;
  long long acc = ts.acc;
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
  acc += q32(coef_term(a.L, dr_out - Rr - Rs - ts.sXR, dr_out_n, dr_out));
  acc += q32(coef_term(a.L, ds_out - Sr - Ss - ts.sXS, ds_out_n, ds_out));
  acc += q32(coef_term(a.L, dr_in - Rr - Sr - ts.sYR, dr_in_n, dr_in));
  acc += q32(coef_term(a.L, ds_in - Rs - Ss - ts.sYS, ds_in_n, ds_in));
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
  if (a.stats) *my_bytes += 8 + 8ull * (vi.dego + vi.degi) + 48ull * ts.nb + 48 + 8ull * scanned;
}

__device__ __forceinline__ void record_stay(const NodalArgs& a, int v) {
  if (a.prop_s) {
    a.prop_s[v - a.beg] = -1;
    a.prop_q[v - a.beg] = 0;
    a.prop_ninf[v - a.beg] = 0;
  }
}

// one warp per vertex of degree <= kHubDegree; 5 CTAs per SM so that a
// batch of the bench workload (N/10 = 5000 vertices) runs in one wave
template <class Ops>
__global__ void __launch_bounds__(kThreads, 5) k_nodal_propose(NodalArgs a, Ops ops) {
  __shared__ int s_key[kWarps][kHCap];
  __shared__ int s_wo[kWarps][kHCap];
  __shared__ int s_wi[kWarps][kHCap];
  __shared__ int s_list[kWarps][kHubDegree];   // occupied slots other than r, s
  if (*reinterpret_cast<volatile int*>(&a.ctl->done)) return;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const unsigned lanes_below = (1u << lane) - 1u;
  const int nwarps = gridDim.x * kWarps;
  unsigned long long my_bytes = 0;
  for (int v = a.beg + blockIdx.x * kWarps + wib; v < a.end; v += nwarps) {
    const VertexInfo vi = vertex_info(a, v);
    const int deg = vi.dego + vi.degi;
    if (deg > kHubDegree) continue;   // handled by k_nodal_propose_hub
    const int r = vi.r;
    // aggregate the neighbour blocks first: these loads do not depend on
    // the target and overlap the sampling chain below
    int lg = 5;
    while ((1 << lg) < 2 * deg) lg++;
    const int cap = 1 << lg;   // <= kHCap since deg <= kHubDegree
    int* key = s_key[wib];
    int* two = s_wo[wib];
    int* twi = s_wi[wib];
    for (int i = lane; i < cap; i += 32) {
      key[i] = -1;
      two[i] = 0;
      twi[i] = 0;
    }
    __syncwarp();
    for (int j = lane; j < deg; j += 32) {
      const bool is_out = j < vi.dego;
      const int nb = is_out ? __ldg(a.out_idx + vi.o0 + j) : __ldg(a.in_idx + vi.i0 + j - vi.dego);
      const int ww = a.unit ? 1 : (is_out ? __ldg(a.out_w + vi.o0 + j) : __ldg(a.in_w + vi.i0 + j - vi.dego));
      table_insert(key, two, twi, cap, lg, __ldg(a.part + nb), ww, is_out);
    }
    int scanned = 0;
    const int s = propose_target(a, ops, v, vi, lane, &scanned);
    __syncwarp();
    if (s == r) {
      if (lane == 0) {
        record_stay(a, v);
        if (a.stats) my_bytes += 8 + 8ull * deg + 8ull * scanned;
      }
      __syncwarp();
      continue;
    }
    const long long dr_out = __ldg(a.dout + r), dr_in = __ldg(a.din + r);
    const long long ds_out = __ldg(a.dout + s), ds_in = __ldg(a.din + s);
    // compact the occupied slots so that each lane takes about one block
    int nlist = 0, noccupied = 0;
    for (int base = 0; base < cap; base += 32) {
      const int i = base + lane;
      const int b = i < cap ? key[i] : -1;
      const unsigned occ = __ballot_sync(0xffffffffu, b >= 0);
      const bool use = b >= 0 && b != r && b != s;
      const unsigned mu = __ballot_sync(0xffffffffu, use);
      if (use) s_list[wib][nlist + __popc(mu & lanes_below)] = i;
      nlist += __popc(mu);
      noccupied += __popc(occ);
    }
    __syncwarp();
    TermSums ts{0, 0, 0, 0, 0, 0};
    for (int t = lane; t < nlist; t += 32) {
      const int i = s_list[wib][t];
      slot_terms(a, ops, r, s, key[i], two[i], twi[i], dr_out, ds_out, dr_in, ds_in, dr_out - vi.kout,
                 ds_out + vi.kout, dr_in - vi.kin, ds_in + vi.kin, ts);
    }
    ts.acc = warp_sum_ll(ts.acc);
    ts.sXR = warp_sum_i(ts.sXR);
    ts.sXS = warp_sum_i(ts.sXS);
    ts.sYR = warp_sum_i(ts.sYR);
    ts.sYS = warp_sum_i(ts.sYS);
    ts.nb = noccupied;
    int e4 = 0;
    if (lane < 4) e4 = ops.get(lane < 2 ? r : s, (lane & 1) ? s : r);
    const long long Rr = __shfl_sync(0xffffffffu, e4, 0), Rs = __shfl_sync(0xffffffffu, e4, 1);
    const long long Sr = __shfl_sync(0xffffffffu, e4, 2), Ss = __shfl_sync(0xffffffffu, e4, 3);
    if (lane == 0) {
      const long long wor = table_lookup_wo(key, two, cap, lg, r);
      const long long wos = table_lookup_wo(key, two, cap, lg, s);
      finalize(a, ops, v, r, s, vi, ts, wor, wos, Rr, Rs, Sr, Ss, scanned, &my_bytes);
    }
    __syncwarp();
  }
  if (a.stats && lane == 0 && my_bytes) atomicAdd(&a.ctl->bytes, my_bytes);
}

// one CTA per vertex of degree > kHubDegree; the hash holds at most
// min(deg, B) distinct blocks and lives in dynamic shared memory
// (`smem_cap` slots) or, beyond that, in the vertex's global region
template <class Ops>
__global__ void __launch_bounds__(kHubThreads) k_nodal_propose_hub(NodalArgs a, Ops ops, const int32_t* hubs,
                                                                  int hub_lo, int hub_hi, int smem_cap) {
  extern __shared__ int dyn[];
  __shared__ long long s_acc[kHubWarps];
  __shared__ int s_sum[5][kHubWarps];
  __shared__ int s_target, s_scanned;
  if (*reinterpret_cast<volatile int*>(&a.ctl->done)) return;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  unsigned long long my_bytes = 0;
  for (int h = hub_lo + blockIdx.x; h < hub_hi; h += gridDim.x) {
    const int v = __ldg(hubs + h);
    const VertexInfo vi = vertex_info(a, v);
    const int deg = vi.dego + vi.degi;
    const int r = vi.r;
    if (wib == 0) {
      int scanned = 0;
      const int s = propose_target(a, ops, v, vi, lane, &scanned);
      if (lane == 0) {
        s_target = s;
        s_scanned = scanned;
      }
    }
    __syncthreads();
    const int s = s_target;
    if (s == r) {
      if (threadIdx.x == 0) {
        record_stay(a, v);
        if (a.stats) my_bytes += 8 + 8ull * deg + 8ull * s_scanned;
      }
      __syncthreads();
      continue;
    }
    const int distinct_max = deg < a.B ? deg : a.B;
    int lg = 5;
    while ((1 << lg) < 2 * distinct_max) lg++;
    const int cap = 1 << lg;
    int *key, *two, *twi;
    if (cap <= smem_cap) {
      key = dyn;
      two = dyn + smem_cap;
      twi = dyn + 2 * smem_cap;
    } else {
      const long long off = __ldg(a.hi_off + v);
      key = a.hkey + off;
      two = a.hwo + off;
      twi = a.hwi + off;
    }
    for (int i = threadIdx.x; i < cap; i += kHubThreads) {
      key[i] = -1;
      two[i] = 0;
      twi[i] = 0;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < deg; j += kHubThreads) {
      const bool is_out = j < vi.dego;
      const int nb = is_out ? __ldg(a.out_idx + vi.o0 + j) : __ldg(a.in_idx + vi.i0 + j - vi.dego);
      const int ww = a.unit ? 1 : (is_out ? __ldg(a.out_w + vi.o0 + j) : __ldg(a.in_w + vi.i0 + j - vi.dego));
      table_insert(key, two, twi, cap, lg, __ldg(a.part + nb), ww, is_out);
    }
    __syncthreads();
    const long long dr_out = __ldg(a.dout + r), dr_in = __ldg(a.din + r);
    const long long ds_out = __ldg(a.dout + s), ds_in = __ldg(a.din + s);
    TermSums ts{0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < cap; i += kHubThreads) {
      const int b = key[i];
      if (b < 0) continue;
      ts.nb++;
      if (b == r || b == s) continue;
      slot_terms(a, ops, r, s, b, two[i], twi[i], dr_out, ds_out, dr_in, ds_in, dr_out - vi.kout,
                 ds_out + vi.kout, dr_in - vi.kin, ds_in + vi.kin, ts);
    }
    ts.acc = warp_sum_ll(ts.acc);
    ts.sXR = warp_sum_i(ts.sXR);
    ts.sXS = warp_sum_i(ts.sXS);
    ts.sYR = warp_sum_i(ts.sYR);
    ts.sYS = warp_sum_i(ts.sYS);
    ts.nb = warp_sum_i(ts.nb);
    if (lane == 0) {
      s_acc[wib] = ts.acc;
      s_sum[0][wib] = ts.sXR;
      s_sum[1][wib] = ts.sXS;
      s_sum[2][wib] = ts.sYR;
      s_sum[3][wib] = ts.sYS;
      s_sum[4][wib] = ts.nb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      TermSums tot{0, 0, 0, 0, 0, 0};
      for (int w = 0; w < kHubWarps; w++) {
        tot.acc += s_acc[w];
        tot.sXR += s_sum[0][w];
        tot.sXS += s_sum[1][w];
        tot.sYR += s_sum[2][w];
        tot.sYS += s_sum[3][w];
        tot.nb += s_sum[4][w];
      }
      const long long Rr = ops.get(r, r), Rs = ops.get(r, s), Sr = ops.get(s, r), Ss = ops.get(s, s);
      const long long wor = table_lookup_wo(key, two, cap, lg, r);
      const long long wos = table_lookup_wo(key, two, cap, lg, s);
      finalize(a, ops, v, r, s, vi, tot, wor, wos, Rr, Rs, Sr, Ss, s_scanned, &my_bytes);
    }
    __syncthreads();
  }
  if (a.stats && threadIdx.x == 0 && my_bytes) atomicAdd(&a.ctl->bytes, my_bytes);
}

// chunk sums CS[u][c] = sum over the chunk's blocks i of M[u,i] + M[i,u]
__global__ void __launch_bounds__(kThreads) k_chunk_sums(int B, int ld, const int* __restrict__ M,
                                                        const int* __restrict__ Mt, int cld,
                                                        int* __restrict__ CS) {
  const int lane = threadIdx.x & 31;
  const int nch = (B + kChunk - 1) / kChunk;
  const long long items = static_cast<long long>(B) * nch;
  const long long nwarps = static_cast<long long>(gridDim.x) * kWarps;
  for (long long it = static_cast<long long>(blockIdx.x) * kWarps + (threadIdx.x >> 5); it < items;
       it += nwarps) {
    const int u = static_cast<int>(it / nch), c = static_cast<int>(it - static_cast<long long>(u) * nch);
    const int i0 = c * kChunk + lane * 4;
    int sum = 0;
    if (i0 < B) {
      const int4 a = *reinterpret_cast<const int4*>(M + static_cast<long long>(u) * ld + i0);
      const int4 b = *reinterpret_cast<const int4*>(Mt + static_cast<long long>(u) * ld + i0);
      sum = a.x + a.y + a.z + a.w + b.x + b.y + b.z + b.w;
    }
    sum = warp_sum_i(sum);
    if (lane == 0) CS[static_cast<long long>(u) * cld + c] = sum;
  }
}

// Sum of `val` over the lanes of `active` that hold the same key; *lead is
// set on one lane per key.
__device__ __forceinline__ int group_sum(unsigned active, long long key, int val, int lane, bool* lead) {
  const unsigned peers = __match_any_sync(active, key);
  *lead = (__ffs(peers) - 1) == lane;
  return __reduce_add_sync(peers, val);
}

// M[x,y] += w, keeping Mt and the chunk sums of rows x and y in step.
// Lanes that update the same cell (or the same chunk sum) are summed first,
// so a moved vertex with many edges into one block issues one atomic per
// distinct target per warp.
__device__ __forceinline__ void dense_add(unsigned active, int lane, int* M, int* Mt, int* CS, int ld,
                                          int cld, int x, int y, int w) {
  bool lead;
  int sum = group_sum(active, static_cast<long long>(x) * ld + y, w, lane, &lead);
  if (lead) {
    atomicAdd(M + static_cast<long long>(x) * ld + y, sum);
    atomicAdd(Mt + static_cast<long long>(y) * ld + x, sum);
  }
  sum = group_sum(active, static_cast<long long>(x) * cld + y / kChunk, w, lane, &lead);
  if (lead) atomicAdd(CS + static_cast<long long>(x) * cld + y / kChunk, sum);
  sum = group_sum(active, static_cast<long long>(y) * cld + x / kChunk, w, lane, &lead);
  if (lead) atomicAdd(CS + static_cast<long long>(y) * cld + x / kChunk, sum);
}

// Apply the accepted moves of a batch to the dense tile by deltas, one
// thread per edge of the batch: positions [0, n_out) walk the batch's
// out-edges (CSR positions o0 + i, owner out_src), [n_out, n_out + n_in)
// its in-edges (positions i0 + i, owner in_dst).  An edge between two moved
// vertices is applied once, from its source's out-list.
__global__ void __launch_bounds__(kThreads) k_nodal_apply_dense(
    const int32_t* __restrict__ out_src, const int32_t* __restrict__ out_idx,
    const int32_t* __restrict__ out_w, const int32_t* __restrict__ in_dst,
    const int32_t* __restrict__ in_idx, const int32_t* __restrict__ in_w,
    const int32_t* __restrict__ part, const int32_t* __restrict__ move_to, int o0, int n_out, int i0,
    int n_in, int ld, int* __restrict__ M, int* __restrict__ Mt, int cld, int* __restrict__ CS) {
  const int lane = threadIdx.x & 31;
  const long long total = static_cast<long long>(n_out) + n_in;
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31);
       base < total; base += stride) {
    const long long t = base + lane;
    const bool is_out = t < n_out;
    bool valid = t < total;
    int v = 0, y = 0, w = 1, s = -1;
    if (valid) {
      const int pos = is_out ? o0 + static_cast<int>(t) : i0 + static_cast<int>(t - n_out);
      v = is_out ? __ldg(out_src + pos) : __ldg(in_dst + pos);
      s = move_to[v];
      y = is_out ? __ldg(out_idx + pos) : __ldg(in_idx + pos);
      if (is_out ? out_w != nullptr : in_w != nullptr) w = is_out ? __ldg(out_w + pos) : __ldg(in_w + pos);
    }
    const int my = valid ? move_to[y] : -1;
    valid = valid && s >= 0 && (is_out || my < 0);
    const unsigned act_out = __ballot_sync(0xffffffffu, valid && is_out);
    const unsigned act_in = __ballot_sync(0xffffffffu, valid && !is_out);
    if (valid) {
      const int r = part[v];
      const int oy = part[y];
      if (is_out) {
        const int ny = my >= 0 ? my : oy;
        dense_add(act_out, lane, M, Mt, CS, ld, cld, r, oy, -w);
        dense_add(act_out, lane, M, Mt, CS, ld, cld, s, ny, w);
      } else {
        dense_add(act_in, lane, M, Mt, CS, ld, cld, oy, r, -w);
        dense_add(act_in, lane, M, Mt, CS, ld, cld, oy, s, w);
      }
    }
  }
}

__global__ void k_nodal_commit(int32_t* __restrict__ part, int32_t* __restrict__ move_to,
                               const int32_t* __restrict__ kout, const int32_t* __restrict__ kin,
                               int beg, int end, int update_degrees, int32_t* __restrict__ dout,
                               int32_t* __restrict__ din, NodalCtl* ctl, CtlArgs c);

// update (:433-458), second half: the sweep's cumulative dS is recorded for
// this sweep and added to S after every batch (as the reference does), then
// the convergence test -mean < thr * S ends the nodal phase
__device__ __forceinline__ void ctl_batch_end(NodalCtl* ctl, const CtlArgs& c) {
  if (ctl->done) return;
  const long long cum = static_cast<long long>(ctl->cum_q);
  const int itr = ctl->itr;
  c.ide_q[itr] = cum;
  c.ide_n[itr] = ctl->cum_ninf;
  ctl->S_q += cum;
  ctl->S_ninf |= ctl->cum_ninf;
  ctl->batches++;
  ctl->proposals += c.batch_vertices;
  ctl->edge_visits += c.batch_edges;
  if (itr >= c.W - 1) {
    double S_d = ctl->S_ninf ? -INFINITY : static_cast<double>(ctl->S_q) / kQ32;
    if (-ctl->mean < c.thr * S_d) ctl->done = 1;
  }
}

// commits the batch's moves (degrees, partition) and runs the batch-end
// bookkeeping in one launch; the bookkeeping reads only the control block
__global__ void k_nodal_commit(int32_t* __restrict__ part, int32_t* __restrict__ move_to,
                               const int32_t* __restrict__ kout, const int32_t* __restrict__ kin,
                               int beg, int end, int update_degrees, int32_t* __restrict__ dout,
                               int32_t* __restrict__ din, NodalCtl* ctl, CtlArgs c) {
  if (c.active && blockIdx.x == 0 && threadIdx.x == 0) ctl_batch_end(ctl, c);
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
__global__ void k_ctl_sweep_start(NodalCtl* ctl, long long model_q, int W, const long long* ide_q,
                                  const int* ide_n) {
  if (ctl->done) return;
  const int itr = static_cast<int>(ctl->sweeps);
  ctl->itr = itr;
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

// the hub CTAs run on a second stream, concurrently with the warp kernel
template <class Ops>
void launch_propose(const NodalArgs& a, Ops ops, const HubList& hubs, const StreamPair& sp) {
  const int count = a.end - a.beg;
  if (count <= 0) return;
  const bool has_hubs = hubs.hi > hubs.lo;
  if (has_hubs) {
    USAP_CUDA(cudaEventRecord(sp.fork, sp.main));
    USAP_CUDA(cudaStreamWaitEvent(sp.side, sp.fork, 0));
    const size_t smem = sizeof(int) * 3 * static_cast<size_t>(hubs.smem_cap);
    k_nodal_propose_hub<Ops><<<hubs.hi - hubs.lo, kHubThreads, smem, sp.side>>>(a, ops, hubs.ids, hubs.lo,
                                                                                hubs.hi, hubs.smem_cap);
    USAP_LAUNCHED();
  }
  int blocks = (count + kWarps - 1) / kWarps;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_nodal_propose<Ops><<<blocks, kThreads, 0, sp.main>>>(a, ops);
  USAP_LAUNCHED();
  if (has_hubs) {
    USAP_CUDA(cudaEventRecord(sp.join, sp.side));
    USAP_CUDA(cudaStreamWaitEvent(sp.main, sp.join, 0));
  }
}

}  // namespace

// the hub kernel's dynamic shared memory limit, set once per device
void nodal_configure(int device) {
  static std::once_flag once[64];
  if (device < 0 || device >= 64) return;
  std::call_once(once[device], [] {
    const int smem = static_cast<int>(sizeof(int) * 3 * kHubSmemSlots);
    USAP_CUDA(cudaFuncSetAttribute(k_nodal_propose_hub<DenseOps>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    USAP_CUDA(cudaFuncSetAttribute(k_nodal_propose_hub<SortedOps>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  });
}

void launch_nodal_propose_dense(const NodalArgs& a, DenseView v, const HubList& hubs,
                                const StreamPair& sp) {
  launch_propose(a, DenseOps{v, a.B}, hubs, sp);
}

void launch_nodal_propose_sorted(const NodalArgs& a, SortedView v, const HubList& hubs,
                                 const StreamPair& sp) {
  launch_propose(a, SortedOps{v, a.B}, hubs, sp);
}

void launch_chunk_sums(int B, DenseView v, int* CS, cudaStream_t st) {
  const int nch = (B + kChunk - 1) / kChunk;
  long long items = static_cast<long long>(B) * nch;
  long long blocks = (items + kWarps - 1) / kWarps;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  k_chunk_sums<<<static_cast<int>(blocks), kThreads, 0, st>>>(B, v.ld, v.M, v.Mt, v.cld, CS);
  USAP_LAUNCHED();
}

void launch_nodal_apply_dense(const GraphDev& g, const int32_t* part, int32_t* move_to, int o0,
                              int n_out, int i0, int n_in, int ld, int* M, int* Mt, int cld, int* CS,
                              cudaStream_t st) {
  const long long total = static_cast<long long>(n_out) + n_in;
  if (total <= 0) return;
  long long blocks = (total + kThreads - 1) / kThreads;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_nodal_apply_dense<<<static_cast<int>(blocks), kThreads, 0, st>>>(
      g.out_src, g.out_idx, g.out_w, g.in_dst, g.in_idx, g.in_w, part, move_to, o0, n_out, i0, n_in, ld, M,
      Mt, cld, CS);
  USAP_LAUNCHED();
}

void launch_nodal_commit(const GraphDev& g, int32_t* part, int32_t* move_to, int beg, int end,
                         int update_degrees, int32_t* dout, int32_t* din, NodalCtl* ctl,
                         const CtlArgs& c, cudaStream_t st) {
  int count = end - beg;
  int blocks = (count + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  if (blocks < 1) blocks = 1;
  k_nodal_commit<<<blocks, 256, 0, st>>>(part, move_to, g.kout, g.kin, beg, end, update_degrees, dout,
                                         din, ctl, c);
  USAP_LAUNCHED();
}

void launch_ctl_sweep_start(NodalCtl* ctl, long long model_q, int W, const long long* ide_q,
                            const int* ide_n, cudaStream_t st) {
  k_ctl_sweep_start<<<1, 1, 0, st>>>(ctl, model_q, W, ide_q, ide_n);
  USAP_LAUNCHED();
}


}  // namespace usap
