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
// move_to[]; they are applied to the dense tile by +/-w deltas (exact
// integers, so order does not matter) and committed together with the
// partition.  The convergence bookkeeping of the update task runs on the
// device, so batches and sweeps queue without host round trips.
//
// Two schedules run the same device code.  Per batch launches: a proposal
// kernel (hubs in a second kernel on a side stream) and an apply kernel.
// Persistent: one cooperative launch runs a stage's whole nodal phase,
// one 768-thread CTA per SM, with grid barriers between entropy, sweep
// start, proposals and apply; it removes the launch gaps that otherwise
// cost about half of each batch.  There each CTA applies the moves it
// accepted itself (listed in shared memory while proposing), and for small
// B the proposals read a per-batch copy of the tile in shared memory.
// State written inside that kernel (the partition, M, degrees, chunk sums,
// moves) is otherwise read through L2 (ld.cg); the non-coherent path is
// used only for data that no phase writes.  The gang kernel runs the same
// phase for many jobs at once.
#include <cmath>
#include <mutex>
#include <type_traits>

#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include "common.cuh"
#include "engine.h"

namespace cg = cooperative_groups;

namespace usap {

namespace {

// Load policies for the state a nodal batch reads: the partition, the
// block degrees and M.  LdNC (ld.global.nc) when the state is read-only
// for the whole launch; LdCG (L2, coherent) in the persistent kernel,
// whose later phases read what earlier phases wrote.
struct LdNC {
  template <class T>
  __device__ __forceinline__ static T ld(const T* p) { return __ldg(p); }
};
struct LdCG {
  template <class T>
  __device__ __forceinline__ static T ld(const T* p) { return __ldcg(p); }
};

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kHCap = 256;          // shared-memory hash slots per warp
constexpr int kChunk = 128;         // blocks per chunk sum of a dense row
constexpr int kHubThreads = 512;    // threads of a hub CTA
constexpr int kHubWarps = kHubThreads / 32;

// A group of G lanes of one warp (G = 16: a half-warp; G = 32: the warp)
// working on one vertex.  Shuffles use width G; ballots are returned as G
// bits of the caller's group.
template <int G>
struct Grp {
  int gl;          // lane within the group
  int base;        // first warp lane of the group
  unsigned mask;   // the group's lanes
  __device__ __forceinline__ explicit Grp(int lane)
      : gl(lane & (G - 1)), base(lane & ~(G - 1)),
        mask(G == 32 ? 0xffffffffu : (((1u << (G & 31)) - 1u) << (lane & ~(G - 1)))) {}
  __device__ __forceinline__ unsigned ballot(bool p) const { return __ballot_sync(mask, p) >> base; }
  __device__ __forceinline__ bool any(bool p) const { return __any_sync(mask, p) != 0; }
  __device__ __forceinline__ void sync() const { __syncwarp(mask); }
  template <class T>
  __device__ __forceinline__ T shfl(T v, int src) const { return __shfl_sync(mask, v, src, G); }
  template <class T>
  __device__ __forceinline__ T sum(T v) const {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
    return v;
  }
  // compensated FP32 sum over the group; every lane gets the same value
  __device__ __forceinline__ FF ffsum(FF f) const {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1)
      f = ff_add(f, FF{__shfl_xor_sync(mask, f.hi, o, G), __shfl_xor_sync(mask, f.lo, o, G)});
    return f;
  }
  template <class T>
  __device__ __forceinline__ T incl_scan(T v) const {
#pragma unroll
    for (int o = 1; o < G; o <<= 1) {
      const T n = __shfl_up_sync(mask, v, o, G);
      if (gl >= o) v += n;
    }
    return v;
  }
};

// P (precision mode 1 or 2): dS is also evaluated in FP32 and decisions
// are taken on that value; the exact FP64 value is kept beside it.
// Ld loads the partition, LdT the tile state (M, Mt, chunk sums, block
// degrees): the persistent kernel may read the latter from a per-batch
// copy in shared memory.
template <class LD, int P = 0, class LDT = LD>
struct DenseOpsT {
  using Ld = LD;
  using LdT = LDT;
  static constexpr int kP = P;
  DenseView v;
  int B;
  __device__ __forceinline__ int get(int x, int y) const {
    return LDT::ld(v.M + static_cast<long long>(x) * v.ld + y);
  }
  // M[y, x], read from row x of the transposed tile (coalesced over y)
  __device__ __forceinline__ int get_t(int x, int y) const {
    return LDT::ld(v.Mt + static_cast<long long>(x) * v.ld + y);
  }
  // first block i (block-id order) whose cumulative M[u,i]+M[i,u] exceeds t:
  // a group scan over the row's chunk sums, then over the 128 entries of the
  // chosen chunk (128 / G per lane, 16-byte loads; rows are padded to ld, a
  // multiple of 4, with zeros)
  template <int G>
  __device__ __forceinline__ int sym_sample(int u, long long t, const Grp<G>& g, int* scanned) const {
    constexpr int PER = kChunk / G;
    const int nch = (B + kChunk - 1) / kChunk;
    const int* cs = v.CS + static_cast<long long>(u) * v.cld;
    long long run = 0;
    int c = nch - 1;
    for (int base = 0; base < nch; base += G) {
      const int cc = base + g.gl;
      const int val = cc < nch ? LDT::ld(cs + cc) : 0;
      const int incl = g.incl_scan(val);
      const int total = g.shfl(incl, G - 1);
      if (run + total > t) {
        const unsigned m = g.ballot(run + incl > t);
        const int l = __ffs(m) - 1;
        c = base + l;
        run += g.shfl(incl - val, l);
        break;
      }
      run += total;
    }
    const int i0 = c * kChunk + g.gl * PER;
    int pr[PER];
#pragma unroll
    for (int k = 0; k < PER; k++) pr[k] = 0;
    const int* mrow = v.M + static_cast<long long>(u) * v.ld;
    const int* trow = v.Mt + static_cast<long long>(u) * v.ld;
#pragma unroll
    for (int q = 0; q < PER / 4; q++) {
      const int i = i0 + 4 * q;
      const int prev = q ? pr[4 * q - 1] : 0;
      if (i < B) {
        const int4 a = LDT::ld(reinterpret_cast<const int4*>(mrow + i));
        const int4 b = LDT::ld(reinterpret_cast<const int4*>(trow + i));
        pr[4 * q] = prev + a.x + b.x;
        pr[4 * q + 1] = pr[4 * q] + a.y + b.y;
        pr[4 * q + 2] = pr[4 * q + 1] + a.z + b.z;
        pr[4 * q + 3] = pr[4 * q + 2] + a.w + b.w;
      } else {
        pr[4 * q] = pr[4 * q + 1] = pr[4 * q + 2] = pr[4 * q + 3] = prev;
      }
    }
    const int last = pr[PER - 1];
    const int incl = g.incl_scan(last);
    const long long before = run + incl - last;
    const unsigned m = g.ballot(run + incl > t);
    const int l = m ? __ffs(m) - 1 : G - 1;
    int k = PER - 1;
#pragma unroll
    for (int kk = PER - 2; kk >= 0; kk--)
      if (before + pr[kk] > t) k = kk;
    *scanned += nch + kChunk;
    const int i = c * kChunk + l * PER + g.shfl(k, l);
    return i < B ? i : B - 1;
  }
};

template <int P = 0>
struct SortedOpsT {
  using Ld = LdNC;
  using LdT = LdNC;
  static constexpr int kP = P;
  SortedView v;
  int B;
  __device__ __forceinline__ int get(int x, int y) const {
    int lo = __ldg(v.rowptr + x), hi = __ldg(v.rowptr + x + 1);
    int p = find_sorted(v.col, lo, hi, y);
    return p >= 0 ? __ldg(v.val + p) : 0;
  }
  __device__ __forceinline__ int get_t(int x, int y) const { return get(y, x); }
  template <int G>
  __device__ __forceinline__ int sym_sample(int u, long long t, const Grp<G>&, int* scanned) const {
    int lo = __ldg(v.symptr + u), hi = __ldg(v.symptr + u + 1);
    long long base = lo > 0 ? __ldg(v.symcum + lo - 1) : 0;
    int j = upper_bound_i(v.symcum, lo, hi, t + base);
    if (j >= hi) j = hi - 1;   // t is below the row total; defensive clamp
    *scanned += 32 - __clz(hi - lo + 1);
    return __ldg(v.symcol + j);
  }
};

using DenseOps = DenseOpsT<LdNC>;
using SortedOps = SortedOpsT<0>;

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

template <class Ops>
__device__ __forceinline__ VertexInfo vertex_info(const NodalArgs& a, int v) {
  VertexInfo vi;
  vi.r = Ops::Ld::ld(a.part + v);
  vi.kout = __ldg(a.kout + v);
  vi.kin = __ldg(a.kin + v);
  vi.o0 = __ldg(a.out_ptr + v);
  vi.dego = __ldg(a.out_ptr + v + 1) - vi.o0;
  vi.i0 = __ldg(a.in_ptr + v);
  vi.degi = __ldg(a.in_ptr + v + 1) - vi.i0;
  return vi;
}

// target block once the chosen neighbour's block u is known
// (warp-collective): with probability B / (d_u + B) a uniform block, else
// a block drawn from row + column u of M
template <class Ops, int G>
__device__ __forceinline__ int target_from(const NodalArgs& a, const Ops& ops, const Draws& x, int u,
                                           const Grp<G>& g, int* scanned) {
  const long long dau = static_cast<long long>(Ops::LdT::ld(a.dout + u)) + Ops::LdT::ld(a.din + u);
  if (accept_uniform(x.x1, dau, a.B)) return static_cast<int>(draw_below(x.x2, a.B));
  return ops.template sym_sample<G>(u, draw_below(x.x2, dau), g, scanned);
}

// target block of the proposal for v (warp-collective), reading the
// vertex's adjacency from memory; used for hubs
template <class Ops>
__device__ __forceinline__ int propose_target(const NodalArgs& a, const Ops& ops, const Draws& x,
                                              const VertexInfo& vi, int lane, int* scanned) {
  const Grp<32> g(lane);
  const long long k = vi.kout + vi.kin;
  if (k == 0) return static_cast<int>(draw_below(x.x2, a.B));
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
  return target_from(a, ops, x, Ops::Ld::ld(a.part + nbr), g, scanned);
}

struct TermSums {
  long long acc;
  int sXR, sXS, sYR, sYS;
  FF f;   // FP32 value of the same terms (precision modes 1, 2)
};

// log of the degrees of r and s before and after the move
struct DegLogs {
  double r_out, s_out, r_out_n, s_out_n, r_in, s_in, r_in_n, s_in_n;
  FF fr_out, fs_out, fr_out_n, fs_out_n, fr_in, fs_in, fr_in_n, fs_in_n;   // precision modes 1, 2
};

template <int P>
__device__ __forceinline__ DegLogs deg_logs(const NodalArgs& a, long long dr_out, long long dr_in, long long ds_out,
                                            long long ds_in, long long kout, long long kin) {
  const double* __restrict__ L = a.L;
  DegLogs d{__ldg(L + dr_out), __ldg(L + ds_out), __ldg(L + dr_out - kout), __ldg(L + ds_out + kout),
            __ldg(L + dr_in),  __ldg(L + ds_in),  __ldg(L + dr_in - kin),   __ldg(L + ds_in + kin)};
  if constexpr (kPairTerms<P>) {
    const float2* __restrict__ T = a.L2;
    d.fr_out = ld_ff(T, dr_out);
    d.fs_out = ld_ff(T, ds_out);
    d.fr_out_n = ld_ff(T, dr_out - kout);
    d.fs_out_n = ld_ff(T, ds_out + kout);
    d.fr_in = ld_ff(T, dr_in);
    d.fs_in = ld_ff(T, ds_in);
    d.fr_in_n = ld_ff(T, dr_in - kin);
    d.fs_in_n = ld_ff(T, ds_in + kin);
  }
  return d;
}

// g(x, d1, d2) = x * ((L[x] - L[d1]) - L[d2]) from loaded log values,
// rounded exactly as g_term rounds it
__device__ __forceinline__ double g_val(long long x, double Lx, double L1, double L2) {
  if (x == 0) return 0.0;
  return __dmul_rn(static_cast<double>(x), __dsub_rn(__dsub_rn(Lx, L1), L2));
}

// dS terms of one aggregated neighbour block b (b not in {r, s}): v sends
// wo to b and receives wi from b
// the four terms of one changed pair of entries: + g(X) + g(Y) - g(X - w) - g(Y + w)
// (row entries M[r|s, b]: g(x, d_in[b], d_out[r|s]); column entries
// M[b, r|s]: g(x, d_in[r|s], d_out[b])); b's degree index is D
template <int P>
__device__ __forceinline__ void pair_terms(const NodalArgs& a, int X, int Y, int w, int D, const DegLogs& dl,
                                           bool col, TermSums& ts) {
  const double* __restrict__ L = a.L;
  const double LD = __ldg(L + D);
  const double a0 = col ? dl.r_in : dl.r_out, b0 = col ? dl.s_in : dl.s_out;
  const double a1 = col ? dl.r_in_n : dl.r_out_n, b1 = col ? dl.s_in_n : dl.s_out_n;
  const double LX = __ldg(L + X), LY = __ldg(L + Y), LXn = __ldg(L + X - w), LYn = __ldg(L + Y + w);
  ts.acc += q32(g_val(X, LX, col ? a0 : LD, col ? LD : a0));
  ts.acc += q32(g_val(Y, LY, col ? b0 : LD, col ? LD : b0));
  ts.acc -= q32(g_val(X - w, LXn, col ? a1 : LD, col ? LD : a1));
  ts.acc -= q32(g_val(Y + w, LYn, col ? b1 : LD, col ? LD : b1));
  if constexpr (kPairTerms<P>) {
    const float2* __restrict__ T = a.L2;
    const FF fD = ld_ff(T, D);
    const FF fa0 = col ? dl.fr_in : dl.fr_out, fb0 = col ? dl.fs_in : dl.fs_out;
    const FF fa1 = col ? dl.fr_in_n : dl.fr_out_n, fb1 = col ? dl.fs_in_n : dl.fs_out_n;
    ts.f = ff_add(ts.f, g_ff<P>(X, ld_ff(T, X), col ? fa0 : fD, col ? fD : fa0));
    ts.f = ff_add(ts.f, g_ff<P>(Y, ld_ff(T, Y), col ? fb0 : fD, col ? fD : fb0));
    ts.f = ff_sub(ts.f, g_ff<P>(X - w, ld_ff(T, X - w), col ? fa1 : fD, col ? fD : fa1));
    ts.f = ff_sub(ts.f, g_ff<P>(Y + w, ld_ff(T, Y + w), col ? fb1 : fD, col ? fD : fb1));
  }
}

template <class Ops>
__device__ __forceinline__ void slot_terms(const NodalArgs& a, const Ops& ops, int r, int s, int b, int wo,
                                           int wi, const DegLogs& dl, TermSums& ts) {
  if (wo > 0) {
    const int R = ops.get(r, b), S = ops.get(s, b);
    pair_terms<Ops::kP>(a, R, S, wo, Ops::LdT::ld(a.din + b), dl, false, ts);
    ts.sXR += R;
    ts.sXS += S;
  }
  if (wi > 0) {
    const int R = ops.get(b, r), S = ops.get(b, s);
    pair_terms<Ops::kP>(a, R, S, wi, Ops::LdT::ld(a.dout + b), dl, true, ts);
    ts.sYR += R;
    ts.sYS += S;
  }
}

// slot_terms from values already loaded: R = M[r,b], S = M[s,b], Di =
// d_in[b] (if wo > 0) and Rc = M[b,r], Sc = M[b,s], Do = d_out[b] (if wi > 0)
template <int P>
__device__ __forceinline__ void slot_terms_vals(const NodalArgs& a, int R, int S, int Rc, int Sc, int Di, int Do,
                                                int wo, int wi, const DegLogs& dl, TermSums& ts) {
  if (wo > 0) {
    pair_terms<P>(a, R, S, wo, Di, dl, false, ts);
    ts.sXR += R;
    ts.sXS += S;
  }
  if (wi > 0) {
    pair_terms<P>(a, Rc, Sc, wi, Do, dl, true, ts);
    ts.sYR += Rc;
    ts.sYS += Sc;
  }
}

// The 2x2 terms and the entries the move leaves unchanged, one term per
// lane (lanes 0-11), added to the warp-summed neighbour terms `ts`.  The
// four new 2x2 terms are subtracted; a -inf among them sets *ninf and is
// left out of the sum (the reference's dS is then -inf).  Every lane
// returns the same result.  P > 0: `fpart` is this lane's part of the
// FP32 sum of the neighbour terms; the group's FP32 dS goes to *f.
template <int G, int P = 0>
__device__ __forceinline__ long long finalize_grp(const NodalArgs& a, const Grp<G>& g, const TermSums& ts,
                                                   long long Rr, long long Rs, long long Sr, long long Ss,
                                                   long long wor, long long wos, long long dr_out,
                                                   long long dr_in, long long ds_out, long long ds_in,
                                                   long long kout, long long kin, int* ninf, FF fpart, double* f) {
  const double* __restrict__ L = a.L;
  const long long dr_out_n = dr_out - kout, ds_out_n = ds_out + kout;
  const long long dr_in_n = dr_in - kin, ds_in_n = ds_in + kin;
  // g lanes: mult * ((L[i0] - L[i1]) - L[i2]); coefficient lanes: mult * (L[i0] - L[i1])
  long long mult = 0, i0 = 0, i1 = 0, i2 = 0;
  bool coef = false, neg = false;
  switch (g.gl) {
    case 0: mult = Rr; i0 = Rr; i1 = dr_in; i2 = dr_out; break;
    case 1: mult = Rs; i0 = Rs; i1 = ds_in; i2 = dr_out; break;
    case 2: mult = Sr; i0 = Sr; i1 = dr_in; i2 = ds_out; break;
    case 3: mult = Ss; i0 = Ss; i1 = ds_in; i2 = ds_out; break;
    case 4: mult = Rr - wor; i0 = mult; i1 = dr_in_n; i2 = dr_out_n; neg = true; break;
    case 5: mult = Rs - wos; i0 = mult; i1 = ds_in_n; i2 = dr_out_n; neg = true; break;
    case 6: mult = Sr + wor; i0 = mult; i1 = dr_in_n; i2 = ds_out_n; neg = true; break;
    case 7: mult = Ss + wos; i0 = mult; i1 = ds_in_n; i2 = ds_out_n; neg = true; break;
    case 8: mult = dr_out - Rr - Rs - ts.sXR; i0 = dr_out_n; i1 = dr_out; coef = true; break;
    case 9: mult = ds_out - Sr - Ss - ts.sXS; i0 = ds_out_n; i1 = ds_out; coef = true; break;
    case 10: mult = dr_in - Rr - Sr - ts.sYR; i0 = dr_in_n; i1 = dr_in; coef = true; break;
    case 11: mult = ds_in - Rs - Ss - ts.sYS; i0 = ds_in_n; i1 = ds_in; coef = true; break;
    default: break;
  }
  const double La = __ldg(L + i0), Lb = __ldg(L + i1), Lc = __ldg(L + i2);
  double t = 0.0;
  if (mult != 0) {
    const double d = __dsub_rn(La, Lb);
    t = __dmul_rn(static_cast<double>(mult), coef ? d : __dsub_rn(d, Lc));
  }
  const bool inf = neg && isinf(t);
  long long q = inf ? 0 : q32(t);
  if (neg) q = -q;
  *ninf = g.any(inf) ? 1 : 0;
  if constexpr (kPairTerms<P>) {
    FF t32{0.0f, 0.0f};
    if (mult != 0 && !inf) {
      const FF A = ld_ff(a.L2, i0), Bv = ld_ff(a.L2, i1);
      t32 = coef ? coef_ff<P>(mult, A, Bv) : g_ff<P>(mult, A, Bv, ld_ff(a.L2, i2));
    }
    fpart = ff_add(fpart, neg ? ff_neg(t32) : t32);
    *f = ff_value(g.ffsum(fpart));
  }
  return ts.acc + g.sum(q);
}

// Precision mode 3: the reference's single-precision dS of v (block r)
// moving to s, _propose_new_partition_nodal (graph_parallel.hpp:1066-1215),
// in its float arithmetic and term order, by a group of G lanes:
//  1. the old terms of rows r, s and (i not in {r, s}) columns r, s, block
//     by block (:1096-1114);
//  2. the four new 2x2 terms, the row entries adjusted by v's out-edges only
//     (:1180-1195; the in-edge adjustment is commented out at :1135-1142);
//  3. the new terms of rows and columns for i not in {r, s} (:1196-1215),
//     the entries adjusted by v's out-weight (rows) and in-weight (columns)
//     towards block i, looked up in the group's neighbour-block table.
// A round covers G blocks: lane l loads the entries of block base + l of
// the four rows (the next round's loads are issued before this round's
// terms are evaluated).  The lanes evaluate the terms of their block, and
// the terms are then added to one float accumulator in
// the reference's order -- lane after lane, and within a lane in the
// reference's term order (float addition does not reassociate), through the
// group's shared-memory buffer `buf` (ref32_accumulate).  Rounds whose four
// rows are empty in every lane are skipped.  Every lane returns the same
// value.  Rr, Rs,
// Sr, Ss: M[r,r], M[r,s], M[s,r], M[s,s]; wor, wos: v's out-weight to
// blocks r and s.
// One round of the chain: lane l's four terms (0 where the reference skips
// a zero count) are staged in buf[4 l .. 4 l + 3] (buf: 4 G floats of the
// group's shared memory, 16-byte aligned), and every lane then adds (or
// subtracts) all 4 G of them to its copy of the accumulator in that order.
// Adding a zero term leaves the float sum unchanged: the accumulator starts
// at +0 and round-to-nearest never makes it -0, so x + 0 = x holds for every
// value it takes (infinities and NaN included).  The loop has the same trip
// count in every group, so the two half-warp groups of a warp run it in
// step, one shared-memory broadcast load per four terms.
template <int G>
__device__ __forceinline__ float ref32_accumulate(const Grp<G>& g, float dS, float t0, float t1, float t2,
                                                  float t3, bool sub, float* buf) {
  reinterpret_cast<float4*>(buf)[g.gl] = make_float4(t0, t1, t2, t3);
  g.sync();
#pragma unroll 8
  for (int j = 0; j < G; j++) {
    const float4 q = reinterpret_cast<const float4*>(buf)[j];
    if (sub) dS = __fsub_rn(__fsub_rn(__fsub_rn(__fsub_rn(dS, q.x), q.y), q.z), q.w);
    else dS = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(dS, q.x), q.y), q.z), q.w);
  }
  g.sync();   // the next round overwrites buf
  return dS;
}

// (not inlined: it runs after the group's other work is done, and a call
// gives it the registers the proposal code held)
template <class Ops, int G>
__device__ __noinline__ float ref32_nodal(const Ops ops, const int32_t* __restrict__ din_p,
                                          const int32_t* __restrict__ dout_p, const float* Trow,
                                          const float* Tcol, int tld, int r, int s, int dr_out, int dr_in,
                                          int ds_out, int ds_in, int kout, int kin, int Rr, int Rs, int Sr, int Ss,
                                          int wor, int wos, const int* key, const int* two, const int* twi, int cap,
                                          int lg, float* buf) {
  using LDT = typename Ops::LdT;
  const Grp<G> g(static_cast<int>(threadIdx.x & 31));
  const int B = ops.B;
  float dS = 0.0f;
  // Every round first issues the loads of the next round (pure reads of the
  // batch-start state), so that their L2 latency overlaps this round's
  // terms and chain.
  if (Trow) {
    // the old-state terms from the batch's tables (written in this launch: L2 loads)
    const float* tr = Trow + static_cast<long long>(r) * tld;
    const float* ts = Trow + static_cast<long long>(s) * tld;
    const float* cr = Tcol + static_cast<long long>(r) * tld;
    const float* cs = Tcol + static_cast<long long>(s) * tld;
    float n0, n1, n2, n3;
    auto tload = [&](int i) {
      const bool in = i < B, col = in && i != r && i != s;
      n0 = in ? __ldcg(tr + i) : 0.0f;
      n1 = in ? __ldcg(ts + i) : 0.0f;
      n2 = col ? __ldcg(cr + i) : 0.0f;
      n3 = col ? __ldcg(cs + i) : 0.0f;
    };
    tload(g.gl);
    for (int base = 0; base < B; base += G) {
      const float t0 = n0, t1 = n1, t2 = n2, t3 = n3;
      tload(base + G + g.gl);
      dS = ref32_accumulate<G>(g, dS, t0, t1, t2, t3, false, buf);
    }
  }
  // a round's entries of rows r, s (R, S), columns r, s (Rc, Sc) and the
  // degrees of its block (d_in: di, d_out: dn)
  int nR, nS, nRc, nSc, ndi, ndn;
  if (!Trow) {
    auto oload = [&](int i) {
      nR = nS = nRc = nSc = ndi = ndn = 0;
      if (i < B) {
        nR = ops.get(r, i);
        nS = ops.get(s, i);
        if (i != r && i != s) {   // columns skip i in {r, s}
          nRc = ops.get_t(r, i);
          nSc = ops.get_t(s, i);
        }
        ndi = LDT::ld(din_p + i);
        ndn = LDT::ld(dout_p + i);
      }
    };
    oload(g.gl);
    for (int base = 0; base < B; base += G) {
      const int R = nR, S = nS, Rc = nRc, Sc = nSc, di = ndi, dn = ndn;
      oload(base + G + g.gl);
      if (!g.any((R | S | Rc | Sc) != 0)) continue;
      const float t0 = ref_term_nz(R, static_cast<long long>(di) * dr_out);
      const float t1 = ref_term_nz(S, static_cast<long long>(di) * ds_out);
      const float t2 = ref_term_nz(Rc, static_cast<long long>(dn) * dr_in);
      const float t3 = ref_term_nz(Sc, static_cast<long long>(dn) * ds_in);
      dS = ref32_accumulate<G>(g, dS, t0, t1, t2, t3, false, buf);
    }
  }
  const int dor_n = dr_out - kout, dos_n = ds_out + kout;
  const int dir_n = dr_in - kin, dis_n = ds_in + kin;
  const int rr_r = Rr - wor, rr_s = Rs - wos, sr_r = Sr + wor, sr_s = Ss + wos;
  if (rr_r) dS = __fsub_rn(dS, ref_term(rr_r, static_cast<long long>(dir_n) * dor_n));
  if (rr_s) dS = __fsub_rn(dS, ref_term(rr_s, static_cast<long long>(dis_n) * dor_n));
  if (sr_r) dS = __fsub_rn(dS, ref_term(sr_r, static_cast<long long>(dir_n) * dos_n));
  if (sr_s) dS = __fsub_rn(dS, ref_term(sr_s, static_cast<long long>(dis_n) * dos_n));
  auto nload = [&](int i) {
    nR = nS = nRc = nSc = ndi = ndn = 0;
    if (i < B && i != r && i != s) {
      nR = ops.get(r, i);
      nS = ops.get(s, i);
      nRc = ops.get_t(r, i);
      nSc = ops.get_t(s, i);
      ndi = LDT::ld(din_p + i);
      ndn = LDT::ld(dout_p + i);
    }
  };
  nload(g.gl);
  for (int base = 0; base < B; base += G) {
    int R = nR, S = nS, Rc = nRc, Sc = nSc;
    const int di = ndi, dn = ndn;
    nload(base + G + g.gl);
    const int i = base + g.gl;
    // v's edges towards block i are part of M[r,i] (out) and M[i,r] (in)
    if (R > 0) {
      const int w = table_lookup_wo(key, two, cap, lg, i);
      R -= w;
      S += w;
    }
    if (Rc > 0) {
      const int w = table_lookup_wo(key, twi, cap, lg, i);
      Rc -= w;
      Sc += w;
    }
    if (!g.any((R | S | Rc | Sc) != 0)) continue;
    // (all four evaluated, the empty ones discarded: no branches, so the
    // four evaluations overlap)
    const float u0 = ref_term_nz(R, static_cast<long long>(di) * dor_n);
    const float u1 = ref_term_nz(S, static_cast<long long>(di) * dos_n);
    const float u2 = ref_term_nz(Rc, static_cast<long long>(dn) * dir_n);
    const float u3 = ref_term_nz(Sc, static_cast<long long>(dn) * dis_n);
    dS = ref32_accumulate<G>(g, dS, u0, u1, u2, u3, true, buf);
  }
  return dS;
}

// per-vertex outputs of a decided proposal; returns whether it is accepted
// (on the FP32 pair's value f in precision modes 1, 2, else on the exact
// FP64 value acc)
template <int P>
__device__ __forceinline__ bool emit(const NodalArgs& a, int v, int r, int s, long long acc, double f, int ninf) {
  const bool accept = ninf || (P > 0 ? f < 0.0 : acc < 0);
  a.move_to[v] = accept ? s : -1;
  a.from[v] = r;
  if (a.prop_s) {
    a.prop_s[v - a.beg] = s;
    a.prop_q[v - a.beg] = acc;
    a.prop_ninf[v - a.beg] = ninf;
    if (P > 0 && a.prop_f) a.prop_f[v - a.beg] = f;
  }
  return accept;
}

__device__ __forceinline__ void record_stay(const NodalArgs& a, int v, int r) {
  a.move_to[v] = -1;
  a.from[v] = r;
  if (a.prop_s) {
    a.prop_s[v - a.beg] = -1;
    a.prop_q[v - a.beg] = 0;
    a.prop_ninf[v - a.beg] = 0;
    if (a.prop_f) a.prop_f[v - a.beg] = 0.0;
  }
}

// accepted dS, moves and near-threshold proposals of one CTA, added to the
// control block once at the end of the kernel
// (the accepted dS summed for the convergence test is the exact FP64 value
// in precision modes 1 and 2, the reference's float value in mode 3)
struct CtaTally {
  unsigned long long cum, moves, near;
  int ninf;
  F32Tally f32;
  // persistent kernels: the edge chunks {v, own_tag | chunk} of the CTA's
  // accepted moves, so that its apply pass visits only those (null
  // elsewhere); *nown, shared by the CTA's tallies, counts past own_cap when
  // the list overflows; own_tag is the job index << 16 in the gang kernel
  int2* own;
  int* nown;
  int own_cap, own_tag;
};

// the accepted dS that the convergence test sums: the exact value, or in
// precision mode 3 the reference's float value (its update task sums the
// float dS it accepted, graph_parallel.hpp:428-434), in Q32
// |dS| <= 1e-9 for the value that decides: the exact one (Q32), or in
// precision 3 the float one
template <int P>
__device__ __forceinline__ bool near_threshold(long long acc, double f, int ninf) {
  if constexpr (P == 3) return !isinf(f) && fabs(f) <= 1e-9;
  return !ninf && acc <= kNearQ && acc >= -kNearQ;
}

template <int P>
__device__ __forceinline__ long long summed_dq(long long acc, double f) {
  if constexpr (P == 3) return q32(f);
  return acc;
}

template <int P>
__device__ __forceinline__ void tally(CtaTally* t, bool accept, long long acc, double f, int ninf, bool shadow) {
  if (accept) {
    if (ninf) atomicOr(&t->ninf, 1);
    else atomicAdd(&t->cum, static_cast<unsigned long long>(summed_dq<P>(acc, f)));
    atomicAdd(&t->moves, 1ull);
  }
  if (near_threshold<P>(acc, f, ninf)) atomicAdd(&t->near, 1ull);
  if constexpr (P > 0) {
    if (shadow && !ninf) f32_tally(&t->f32, f, acc);
  }
}

// the same straight into the control block (one proposal per CTA)
template <int P>
__device__ __forceinline__ void tally_ctl(NodalCtl* c, bool accept, long long acc, double f, int ninf,
                                          bool shadow) {
  if (accept) {
    if (ninf) atomicOr(&c->cum_ninf, 1);
    else atomicAdd(&c->cum_q, static_cast<unsigned long long>(summed_dq<P>(acc, f)));
    atomicAdd(&c->moves, 1ull);
  }
  if (near_threshold<P>(acc, f, ninf)) atomicAdd(&c->near, 1ull);
  if constexpr (P > 0) {
    if (shadow && !ninf) f32_tally(&c->f32, f, acc);
  }
}

__device__ __forceinline__ void tally_flush(const CtaTally* t, NodalCtl* ctl) {
  if (t->ninf) atomicOr(&ctl->cum_ninf, 1);
  if (t->cum) atomicAdd(&ctl->cum_q, t->cum);
  if (t->moves) atomicAdd(&ctl->moves, t->moves);
  if (t->near) atomicAdd(&ctl->near, t->near);
  f32_tally_flush(&t->f32, &ctl->f32);
}

// Proposal for one vertex of degree <= 4 * G by a group of G lanes (a
// warp, G = 32, or a half-warp, G = 16).  Each lane loads up to four
// neighbours at once (ids, then their blocks) and keeps them in registers:
// the hash of neighbour blocks and the target draw (whose chosen neighbour
// is among them) come from the same loads.  key/two/twi: the group's table
// of 8 * G slots; list: 4 * G ints.
template <class Ops, int G>
__device__ __forceinline__ void group_vertex(const NodalArgs& a, const Ops& ops, int v, uint32_t itr, int* key,
                                             int* two, int* twi, int* list, CtaTally* tl, const Grp<G>& g,
                                             unsigned long long* my_bytes) {
  using LD = typename Ops::Ld;
  using LDT = typename Ops::LdT;
  constexpr int KN = 4;   // neighbours per lane
  const unsigned lanes_below = (1u << g.gl) - 1u;
  const VertexInfo vi = vertex_info<Ops>(a, v);
  const int deg = vi.dego + vi.degi;
  if (deg > KN * G) return;   // proposed by a larger group or a whole CTA
  const int r = vi.r;
  const Draws x = philox(static_cast<uint32_t>(v), itr, a.stage, kTagNodal, a.seed);
  const long long dr_out = LDT::ld(a.dout + r), dr_in = LDT::ld(a.din + r);
  int lg = 5;
  while ((1 << lg) < 2 * deg) lg++;
  const int cap = 1 << lg;   // <= 8 * G
  for (int i = g.gl; i < cap; i += G) {
    key[i] = -1;
    two[i] = 0;
    twi[i] = 0;
  }
  g.sync();
  int nb[KN], wv[KN], pb[KN];
#pragma unroll
  for (int k = 0; k < KN; k++) {
    const int j = g.gl + G * k;
    nb[k] = 0;
    wv[k] = 0;
    if (j < deg) {
      const bool is_out = j < vi.dego;
      nb[k] = is_out ? __ldg(a.out_idx + vi.o0 + j) : __ldg(a.in_idx + vi.i0 + j - vi.dego);
      wv[k] = a.unit ? 1 : (is_out ? __ldg(a.out_w + vi.o0 + j) : __ldg(a.in_w + vi.i0 + j - vi.dego));
    }
  }
#pragma unroll
  for (int k = 0; k < KN; k++) pb[k] = g.gl + G * k < deg ? LD::ld(a.part + nb[k]) : 0;
#pragma unroll
  for (int k = 0; k < KN; k++) {
    const int j = g.gl + G * k;
    if (j < deg) table_insert(key, two, twi, cap, lg, pb[k], wv[k], j < vi.dego);
  }
  // the target: neighbour position j by weight, its block from registers
  int scanned = 0;
  int s;
  const long long ktot = vi.kout + vi.kin;
  if (ktot == 0) {
    s = static_cast<int>(draw_below(x.x2, a.B));
  } else {
    const long long t = draw_below(x.x0, ktot);
    int j;
    if (a.unit) {
      j = static_cast<int>(t);
    } else {
      long long run = 0;
      j = deg - 1;
#pragma unroll
      for (int k = 0; k < KN; k++) {
        if (G * k >= deg) break;
        const long long ww = g.gl + G * k < deg ? wv[k] : 0;
        const long long incl = g.incl_scan(ww);
        const long long total = g.shfl(incl, G - 1);
        if (run + total > t) {
          const unsigned m = g.ballot(run + incl > t);
          j = G * k + __ffs(m) - 1;
          break;
        }
        run += total;
      }
    }
    const int kq = j / G;
    const int pj = kq == 0 ? pb[0] : kq == 1 ? pb[1] : kq == 2 ? pb[2] : pb[3];
    s = target_from(a, ops, x, g.shfl(pj, j & (G - 1)), g, &scanned);
  }
  g.sync();
  if (s == r) {
    if (g.gl == 0) {
      record_stay(a, v, r);
      if (a.stats) *my_bytes += 8 + 8ull * deg + 8ull * scanned;
    }
    g.sync();
    return;
  }
  const long long ds_out = LDT::ld(a.dout + s), ds_in = LDT::ld(a.din + s);
  int e4 = 0;
  if (g.gl < 4) e4 = ops.get(g.gl < 2 ? r : s, (g.gl & 1) ? s : r);
  // the exact FP64 dS (decides in precision 0; in the others the shadow
  // value the FP32 decision is compared with, skipped in precision 3
  // unless asked for)
  const bool shadow = Ops::kP != 3 || a.shadow;
  int ninf = 0, noccupied = 0;
  double f = 0.0;
  long long acc = 0;
  if (shadow) {
    const DegLogs dl = deg_logs<Ops::kP>(a, dr_out, dr_in, ds_out, ds_in, vi.kout, vi.kin);
    // compact the occupied slots so that each lane takes about one block
    int nlist = 0;
    for (int base = 0; base < cap; base += G) {
      const int i = base + g.gl;
      const int b = i < cap ? key[i] : -1;
      const unsigned occ = g.ballot(b >= 0);
      const bool use = b >= 0 && b != r && b != s;
      const unsigned mu = g.ballot(use);
      if (use) list[nlist + __popc(mu & lanes_below)] = i;
      nlist += __popc(mu);
      noccupied += __popc(occ);
    }
    g.sync();
    // each lane has at most four slots (nlist <= 4 * G): their M entries
    // and degrees are loaded in two rounds of two, then the log terms
    TermSums ts{0, 0, 0, 0, 0};
#pragma unroll
    for (int k0 = 0; k0 < 4; k0 += 2) {
      int R[2], S[2], Rc[2], Sc[2], Di[2], Do[2], wo[2], wi[2];
#pragma unroll
      for (int k = 0; k < 2; k++) {
        const int t = g.gl + G * (k0 + k);
        R[k] = S[k] = Rc[k] = Sc[k] = Di[k] = Do[k] = wo[k] = wi[k] = 0;
        if (t < nlist) {
          const int i = list[t];
          const int b = key[i];
          wo[k] = two[i];
          wi[k] = twi[i];
          if (wo[k] > 0) {
            R[k] = ops.get(r, b);
            S[k] = ops.get(s, b);
            Di[k] = LDT::ld(a.din + b);
          }
          if (wi[k] > 0) {
            Rc[k] = ops.get(b, r);
            Sc[k] = ops.get(b, s);
            Do[k] = LDT::ld(a.dout + b);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < 2; k++)
        slot_terms_vals<Ops::kP>(a, R[k], S[k], Rc[k], Sc[k], Di[k], Do[k], wo[k], wi[k], dl, ts);
    }
    ts.acc = g.sum(ts.acc);
    ts.sXR = g.sum(ts.sXR);
    ts.sXS = g.sum(ts.sXS);
    ts.sYR = g.sum(ts.sYR);
    ts.sYS = g.sum(ts.sYS);
    const long long Rr = g.shfl(e4, 0), Rs = g.shfl(e4, 1);
    const long long Sr = g.shfl(e4, 2), Ss = g.shfl(e4, 3);
    const long long wor = table_lookup_wo(key, two, cap, lg, r);
    const long long wos = table_lookup_wo(key, two, cap, lg, s);
    acc = finalize_grp<G, Ops::kP>(a, g, ts, Rr, Rs, Sr, Ss, wor, wos, dr_out, dr_in, ds_out, ds_in, vi.kout,
                                   vi.kin, &ninf, ts.f, &f);
  }
  if constexpr (Ops::kP == 3) {
    const int Rr = g.shfl(e4, 0), Rs = g.shfl(e4, 1);
    const int Sr = g.shfl(e4, 2), Ss = g.shfl(e4, 3);
    const int wor = table_lookup_wo(key, two, cap, lg, r);
    const int wos = table_lookup_wo(key, two, cap, lg, s);
    f = ref32_nodal<Ops, G>(ops, a.din, a.dout, a.Trow, a.Tcol, a.tld, r, s, static_cast<int>(dr_out),
                            static_cast<int>(dr_in),
                            static_cast<int>(ds_out), static_cast<int>(ds_in), static_cast<int>(vi.kout),
                            static_cast<int>(vi.kin), static_cast<int>(Rr), static_cast<int>(Rs),
                            static_cast<int>(Sr), static_cast<int>(Ss), static_cast<int>(wor),
                            static_cast<int>(wos), key, two, twi, cap, lg, reinterpret_cast<float*>(list));
    // without the shadow the -inf of a new-state term x log(x / 0) comes
    // from the float sum itself (the term is +inf there, and every new-state
    // term is subtracted)
    if (!shadow) ninf = isinf(f) && f < 0.0 ? 1 : 0;
  }
  if (g.gl == 0) {
    const bool moved = emit<Ops::kP>(a, v, r, s, acc, f, ninf);
    tally<Ops::kP>(tl, moved, acc, f, ninf, shadow);
    if (moved && tl->own) {
      const int nch = deg > 32 ? (deg + 31) >> 5 : 1;   // the vertex's chunks (one even without edges)
      const int i0 = atomicAdd(tl->nown, nch);
      for (int c = 0; c < nch; c++)
        if (i0 + c < tl->own_cap) tl->own[i0 + c] = make_int2(v, tl->own_tag | c);
    }
    // precision 3 also reads, for the old-state and again for the new-state
    // terms, rows r and s and columns r and s of M and both degree arrays:
    // 2 x 24 bytes per block, as the reference's O(B) loops do
    if (a.stats)
      *my_bytes += 8 + 8ull * deg + 48ull * noccupied + 48 + 8ull * scanned + (Ops::kP == 3 ? 48ull * a.B : 0ull);
  }
  g.sync();
}

// One warp per vertex of degree <= kHubDegree; 5 CTAs per SM so that a
// batch of the bench workload (N/10 = 5000 vertices) runs in one wave.
template <class Ops>
__global__ void __launch_bounds__(kThreads, 5) k_nodal_propose(NodalArgs a, Ops ops) {
  __shared__ int s_key[kWarps][kHCap];
  __shared__ int s_wo[kWarps][kHCap];
  __shared__ int s_wi[kWarps][kHCap];
  __shared__ __align__(16) int s_list[kWarps][kHubDegree];   // occupied slots other than r, s; then the float dS's terms
  __shared__ CtaTally s_tally;
  if (a.ctl->done) return;   // written by earlier launches only
  const uint32_t itr = static_cast<uint32_t>(a.ctl->itr);
  if (threadIdx.x == 0) s_tally = CtaTally{0, 0, 0, 0};
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nwarps = gridDim.x * kWarps;
  unsigned long long my_bytes = 0;
  for (int v = a.beg + blockIdx.x * kWarps + wib; v < a.end; v += nwarps)
    group_vertex(a, ops, v, itr, s_key[wib], s_wo[wib], s_wi[wib], s_list[wib], &s_tally, Grp<32>(lane),
                 &my_bytes);
  __syncthreads();
  if (threadIdx.x == 0) tally_flush(&s_tally, a.ctl);
  if (a.stats && lane == 0 && my_bytes) atomicAdd(&a.ctl->bytes, my_bytes);
}

template <int NW>
struct HubShared {
  long long acc[NW];
  int sum[5][NW];
  float fhi[NW], flo[NW];   // FP32 partial sums (precision modes 1, 2)
  int target, scanned;
  __align__(16) float chain[128];   // precision 3: the float dS's staged terms (warp 0)
};

// Proposal for one vertex of degree > kHubDegree by a whole CTA of NT
// threads.  The last warp draws the target while the others fill the hash
// of neighbour blocks (at most min(deg, B) entries: in `stab`, a shared
// region of `scap` slots per array, or beyond that in the vertex's global
// region); each thread loads four neighbours at once, and up to four
// occupied slots at once for the terms.
template <class Ops, int NT>
__device__ __forceinline__ void hub_vertex(const NodalArgs& a, const Ops& ops, int v, uint32_t itr, int* stab,
                                           int scap, HubShared<NT / 32>* sh, unsigned long long* my_bytes) {
  using LD = typename Ops::Ld;
  using LDT = typename Ops::LdT;
  constexpr int NW = NT / 32;
  constexpr int kIns = NT - 32;   // threads that fill the table
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const VertexInfo vi = vertex_info<Ops>(a, v);
  const int deg = vi.dego + vi.degi;
  const int r = vi.r;
  const int distinct_max = deg < a.B ? deg : a.B;
  int lg = 5;
  while ((1 << lg) < 2 * distinct_max) lg++;
  const int cap = 1 << lg;
  int *key, *two, *twi;
  if (cap <= scap) {
    key = stab;
    two = stab + scap;
    twi = stab + 2 * scap;
  } else {
    const long long off = __ldg(a.hi_off + v);
    key = a.hkey + off;
    two = a.hwo + off;
    twi = a.hwi + off;
  }
  for (int i = threadIdx.x; i < cap; i += NT) {
    key[i] = -1;
    two[i] = 0;
    twi[i] = 0;
  }
  __syncthreads();
  if (wib == NW - 1) {
    const Draws x = philox(static_cast<uint32_t>(v), itr, a.stage, kTagNodal, a.seed);
    int scanned = 0;
    const int st = propose_target(a, ops, x, vi, lane, &scanned);
    if (lane == 0) {
      sh->target = st;
      sh->scanned = scanned;
    }
  } else {
    for (int j0 = threadIdx.x; j0 < deg; j0 += 4 * kIns) {
      int nb[4], wv[4], pb[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int j = j0 + k * kIns;
        nb[k] = 0;
        wv[k] = 0;
        if (j < deg) {
          const bool is_out = j < vi.dego;
          nb[k] = is_out ? __ldg(a.out_idx + vi.o0 + j) : __ldg(a.in_idx + vi.i0 + j - vi.dego);
          wv[k] = a.unit ? 1 : (is_out ? __ldg(a.out_w + vi.o0 + j) : __ldg(a.in_w + vi.i0 + j - vi.dego));
        }
      }
#pragma unroll
      for (int k = 0; k < 4; k++) pb[k] = j0 + k * kIns < deg ? LD::ld(a.part + nb[k]) : 0;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int j = j0 + k * kIns;
        if (j < deg) table_insert(key, two, twi, cap, lg, pb[k], wv[k], j < vi.dego);
      }
    }
  }
  __syncthreads();
  const int s = sh->target;
  if (s == r) {
    if (threadIdx.x == 0) {
      record_stay(a, v, r);
      if (a.stats) *my_bytes += 8 + 8ull * deg + 8ull * sh->scanned;
    }
    __syncthreads();
    return;
  }
  const long long dr_out = LDT::ld(a.dout + r), dr_in = LDT::ld(a.din + r);
  const long long ds_out = LDT::ld(a.dout + s), ds_in = LDT::ld(a.din + s);
  const DegLogs dl = deg_logs<Ops::kP>(a, dr_out, dr_in, ds_out, ds_in, vi.kout, vi.kin);
  TermSums ts{0, 0, 0, 0, 0};
  int nocc = 0;
  for (int i = threadIdx.x; i < cap;) {
    int sl[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      sl[k] = -1;
      while (i < cap) {
        const int b = key[i];
        i += NT;
        if (b < 0) continue;
        nocc++;
        if (b != r && b != s) {
          sl[k] = i - NT;
          break;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (sl[k] >= 0) slot_terms(a, ops, r, s, key[sl[k]], two[sl[k]], twi[sl[k]], dl, ts);
  }
  ts.acc = warp_sum_ll(ts.acc);
  ts.sXR = warp_sum_i(ts.sXR);
  ts.sXS = warp_sum_i(ts.sXS);
  ts.sYR = warp_sum_i(ts.sYR);
  ts.sYS = warp_sum_i(ts.sYS);
  nocc = warp_sum_i(nocc);
  if constexpr (kPairTerms<Ops::kP>) ts.f = Grp<32>(lane).ffsum(ts.f);
  if (lane == 0) {
    sh->acc[wib] = ts.acc;
    sh->fhi[wib] = ts.f.hi;
    sh->flo[wib] = ts.f.lo;
    sh->sum[0][wib] = ts.sXR;
    sh->sum[1][wib] = ts.sXS;
    sh->sum[2][wib] = ts.sYR;
    sh->sum[3][wib] = ts.sYS;
    sh->sum[4][wib] = nocc;
  }
  __syncthreads();
  if (wib == 0) {
    TermSums tot{0, 0, 0, 0, 0};
    int occ = 0;
    FF fpart{0.0f, 0.0f};
    if (lane < NW) {
      fpart = FF{sh->fhi[lane], sh->flo[lane]};
      tot.acc = sh->acc[lane];
      tot.sXR = sh->sum[0][lane];
      tot.sXS = sh->sum[1][lane];
      tot.sYR = sh->sum[2][lane];
      tot.sYS = sh->sum[3][lane];
      occ = sh->sum[4][lane];
    }
    tot.acc = warp_sum_ll(tot.acc);
    tot.sXR = warp_sum_i(tot.sXR);
    tot.sXS = warp_sum_i(tot.sXS);
    tot.sYR = warp_sum_i(tot.sYR);
    tot.sYS = warp_sum_i(tot.sYS);
    occ = warp_sum_i(occ);
    int e4 = 0;
    if (lane < 4) e4 = ops.get(lane < 2 ? r : s, (lane & 1) ? s : r);
    const long long Rr = __shfl_sync(0xffffffffu, e4, 0), Rs = __shfl_sync(0xffffffffu, e4, 1);
    const long long Sr = __shfl_sync(0xffffffffu, e4, 2), Ss = __shfl_sync(0xffffffffu, e4, 3);
    const long long wor = table_lookup_wo(key, two, cap, lg, r);
    const long long wos = table_lookup_wo(key, two, cap, lg, s);
    int ninf;
    double f = 0.0;
    const long long acc = finalize_grp<32, Ops::kP>(a, Grp<32>(lane), tot, Rr, Rs, Sr, Ss, wor, wos, dr_out,
                                                    dr_in, ds_out, ds_in, vi.kout, vi.kin, &ninf, fpart, &f);
    if constexpr (Ops::kP == 3)
      f = ref32_nodal<Ops, 32>(ops, a.din, a.dout, a.Trow, a.Tcol, a.tld, r, s, static_cast<int>(dr_out),
                               static_cast<int>(dr_in),
                               static_cast<int>(ds_out), static_cast<int>(ds_in), static_cast<int>(vi.kout),
                               static_cast<int>(vi.kin), static_cast<int>(Rr), static_cast<int>(Rs),
                               static_cast<int>(Sr), static_cast<int>(Ss), static_cast<int>(wor),
                               static_cast<int>(wos), key, two, twi, cap, lg, sh->chain);
    // (a hub's exact value is a CTA-parallel sum over its slots and is
    // always evaluated; without the shadow it is not reported, as for the
    // other vertices)
    const bool shadow = Ops::kP != 3 || a.shadow;
    if (!shadow) ninf = isinf(f) && f < 0.0 ? 1 : 0;
    if (lane == 0) {
      tally_ctl<Ops::kP>(a.ctl, emit<Ops::kP>(a, v, r, s, acc, f, ninf), acc, f, ninf, shadow);
      if (a.stats)
        *my_bytes += 8 + 8ull * deg + 48ull * occ + 48 + 8ull * sh->scanned + (Ops::kP == 3 ? 48ull * a.B : 0ull);
    }
  }
  __syncthreads();
}

// one CTA per vertex of degree > kHubDegree, hash in dynamic shared memory
// (`smem_cap` slots per array) or the vertex's global region
template <class Ops>
__global__ void __launch_bounds__(kHubThreads) k_nodal_propose_hub(NodalArgs a, Ops ops, const int32_t* hubs,
                                                                  int hub_lo, int hub_hi, int smem_cap) {
  extern __shared__ __align__(16) int dyn[];
  __shared__ HubShared<kHubWarps> sh;
  if (a.ctl->done) return;
  const uint32_t itr = static_cast<uint32_t>(a.ctl->itr);
  unsigned long long my_bytes = 0;
  for (int h = hub_lo + blockIdx.x; h < hub_hi; h += gridDim.x)
    hub_vertex<Ops, kHubThreads>(a, ops, __ldg(hubs + h), itr, dyn, smem_cap, &sh, &my_bytes);
  if (a.stats && threadIdx.x == 0 && my_bytes) atomicAdd(&a.ctl->bytes, my_bytes);
}

// --- block-merge proposals on the dense tile ------------------------------------
// The block_merge task (graph_parallel.hpp:349-368, _propose_new_partition_block
// :761-988) for B <= dense_max, reading the tile the nodal phase keeps (M, its
// transpose, the chunk sums) instead of sorted sparse views.  Draws, candidate
// order and the Q32 terms are those of the sparse kernel (kernels_merge.cu):
// the symmetric row M[u,:]+M[:,u] is walked in block-id order through the
// chunk sums, and the rows and columns of r and s are scanned whole, every
// column where both are non-zero giving one h term.

// sum of M[u,i] + M[i,u] over i < r (warp-collective, every lane returns it)
__device__ __forceinline__ long long sym_prefix(const DenseView& v, int u, int r, int lane) {
  const int c = r / kChunk;
  long long acc = 0;
  const int* cs = v.CS + static_cast<long long>(u) * v.cld;
  for (int q = lane; q < c; q += 32) acc += __ldg(cs + q);
  const int* mrow = v.M + static_cast<long long>(u) * v.ld;
  const int* trow = v.Mt + static_cast<long long>(u) * v.ld;
  for (int i = c * kChunk + lane; i < r; i += 32) acc += __ldg(mrow + i) + __ldg(trow + i);
  return warp_sum_ll(acc);
}

template <int P>
__global__ void __launch_bounds__(kThreads) k_merge_propose_dense(DenseView v, MergeArgs a) {
  constexpr bool F32 = P > 0;
  __shared__ F32Tally s_f32;
  if (F32) {
    if (threadIdx.x == 0) s_f32 = F32Tally{0, 0, 0, 0.0};
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const DenseOps ops{v, a.B};
  const Grp<32> g(lane);
  const long long items = static_cast<long long>(a.B) * a.K;
  const long long nwarps = static_cast<long long>(gridDim.x) * kWarps;
  for (long long item = static_cast<long long>(blockIdx.x) * kWarps + (threadIdx.x >> 5); item < items;
       item += nwarps) {
    const int r = static_cast<int>(item / a.K), k = static_cast<int>(item - static_cast<long long>(r) * a.K);
    const int B = a.B;
    const Draws x = philox(static_cast<uint32_t>(r), static_cast<uint32_t>(k), a.stage, kTagMerge, a.seed);
    const long long dr_out = __ldg(a.dout + r), dr_in = __ldg(a.din + r);
    const long long ka = dr_out + dr_in;
    int s;
    int scanned = 0;
    if (ka == 0) {
      s = static_cast<int>(draw_below(x.x2, B));
    } else {
      const int u = ops.sym_sample(r, static_cast<long long>(draw_below(x.x0, ka)), g, &scanned);
      const long long dau = static_cast<long long>(__ldg(a.dout + u)) + __ldg(a.din + u);
      if (accept_uniform(x.x1, dau, B)) {
        s = skip_r(static_cast<int>(draw_below(x.x2, B)), r, B);
      } else {
        // the multinomial over row u with r left out
        const long long c_ur = static_cast<long long>(ops.get(u, r)) + ops.get(r, u);
        const long long before = sym_prefix(v, u, r, lane);
        const long long wsum = dau - c_ur;
        if (wsum == 0) {
          s = skip_r(static_cast<int>(draw_below(x.x2, B)), r, B);
        } else {
          long long t2 = draw_below(x.x2, wsum);
          if (c_ur > 0 && t2 >= before) t2 += c_ur;
          s = ops.sym_sample(u, t2, g, &scanned);
        }
      }
    }
    // --- dS of merging r into s ---
    const long long ds_out = __ldg(a.dout + s), ds_in = __ldg(a.din + s);
    const long long ds_out_n = ds_out + dr_out, ds_in_n = ds_in + dr_in;
    int e4 = 0;
    if (lane < 4) e4 = ops.get(lane < 2 ? r : s, (lane & 1) ? s : r);
    const long long Mrr = __shfl_sync(0xffffffffu, e4, 0), Mrs = __shfl_sync(0xffffffffu, e4, 1);
    const long long Msr = __shfl_sync(0xffffffffu, e4, 2), Mss = __shfl_sync(0xffffffffu, e4, 3);
    long long acc = 0;
    FF f{0.0f, 0.0f};
    // rows r and s (M) and columns r and s (rows of Mt): columns i not in
    // {r, s} where both entries are non-zero
    const int* mr = v.M + static_cast<long long>(r) * v.ld;
    const int* ms = v.M + static_cast<long long>(s) * v.ld;
    const int* tr = v.Mt + static_cast<long long>(r) * v.ld;
    const int* ts = v.Mt + static_cast<long long>(s) * v.ld;
    for (int i = lane; i < B; i += 32) {
      if (i == r || i == s) continue;
      const int xr = __ldg(mr + i), xs = __ldg(ms + i);
      if (xr > 0 && xs > 0) {
        acc += q32(h_term(a.L, xr, xs));
        if constexpr (F32) f = ff_add(f, h_term_ff<P>(a.L2, xr, xs));
      }
      const int yr = __ldg(tr + i), ys = __ldg(ts + i);
      if (yr > 0 && ys > 0) {
        acc += q32(h_term(a.L, yr, ys));
        if constexpr (F32) f = ff_add(f, h_term_ff<P>(a.L2, yr, ys));
      }
    }
    acc = warp_sum_ll(acc);
    if constexpr (F32) f = g.ffsum(f);
    if (lane == 0) {
      acc += q32(g_term(a.L, Mrr, dr_in, dr_out));
      acc += q32(g_term(a.L, Mrs, ds_in, dr_out));
      acc += q32(g_term(a.L, Msr, dr_in, ds_out));
      acc += q32(g_term(a.L, Mss, ds_in, ds_out));
      acc -= q32(g_term(a.L, Mrr + Mrs + Msr + Mss, ds_in_n, ds_out_n));
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
        f = ff_add(f, g_term_ff<P>(T, Mrr, dr_in, dr_out));
        f = ff_add(f, g_term_ff<P>(T, Mrs, ds_in, dr_out));
        f = ff_add(f, g_term_ff<P>(T, Msr, dr_in, ds_out));
        f = ff_add(f, g_term_ff<P>(T, Mss, ds_in, ds_out));
        f = ff_sub(f, g_term_ff<P>(T, Mrr + Mrs + Msr + Mss, ds_in_n, ds_out_n));
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

// update (:433-458), second half: the sweep's cumulative dS is recorded for
// this sweep and added to S after every batch (as the reference does), then
// the convergence test -mean < thr * S ends the nodal phase.  One thread.
// The control block is read at once through L2 (ld.cg: the persistent
// kernel calls this after other CTAs wrote it), then written back.
__device__ __forceinline__ bool ctl_batch_end(NodalCtl* ctl, const CtlArgs& c) {
  const int done = __ldcg(&ctl->done);
  const long long cum = static_cast<long long>(__ldcg(&ctl->cum_q));
  const int itr = __ldcg(&ctl->itr);
  const int cum_ninf = __ldcg(&ctl->cum_ninf);
  const long long S_q = __ldcg(&ctl->S_q) + cum;
  const int S_ninf = __ldcg(&ctl->S_ninf) | cum_ninf;
  const unsigned long long batches = __ldcg(&ctl->batches);
  const unsigned long long proposals = __ldcg(&ctl->proposals);
  const unsigned long long edge_visits = __ldcg(&ctl->edge_visits);
  const double mean = __ldcg(&ctl->mean);
  if (done) return true;
  c.ide_q[itr] = cum;
  c.ide_n[itr] = cum_ninf;
  ctl->S_q = S_q;
  ctl->S_ninf = S_ninf;
  ctl->batches = batches + 1;
  ctl->proposals = proposals + static_cast<unsigned long long>(c.batch_vertices);
  ctl->edge_visits = edge_visits + static_cast<unsigned long long>(c.batch_edges);
  if (itr >= c.W - 1) {
    const double S_d = S_ninf ? -INFINITY : c.model_d + static_cast<double>(S_q) / kQ32;
    if (-mean < c.thr * S_d) {
      ctl->done = 1;
      return true;
    }
  }
  return false;
}

// prepare_batch (:381-395): the data term of S from the entropy
// accumulator (the model term is added where S is compared), the moving
// average of the previous sweeps' dS, and a fresh cumulative sum for this
// sweep.  One thread; reads as in ctl_batch_end.
__device__ __forceinline__ void ctl_sweep_start(NodalCtl* ctl, int W,
                                                const long long* ide_q, const int* ide_n) {
  const int done = __ldcg(&ctl->done);
  const unsigned long long sweeps = __ldcg(&ctl->sweeps);
  const unsigned long long eacc = __ldcg(&ctl->entropy_acc);
  if (done) return;
  const int itr = static_cast<int>(sweeps);
  double mean = 0.0;
  if (itr >= W - 1) {
    long long sum = 0;
    int ninf = 0;
    for (int i = itr - W + 1; i < itr; i++) {
      sum += __ldcg(ide_q + i);
      ninf |= __ldcg(ide_n + i);
    }
    mean = ninf ? -INFINITY : (static_cast<double>(sum) / kQ32) / static_cast<double>(W - 1);
  }
  ctl->itr = itr;
  ctl->S_q = -static_cast<long long>(eacc);
  ctl->S_ninf = 0;
  ctl->mean = mean;
  ctl->cum_q = 0;
  ctl->cum_ninf = 0;
  ctl->sweeps = sweeps + 1;
}

struct LdPlain {
  template <class T>
  __device__ __forceinline__ static T ld(const T* p) { return *p; }
};

// Accumulation of one CTA's tile deltas during an apply pass, in one of
// three modes.  All sums are exact integers, so the order of the updates
// does not matter.
//  kDeltaHashed: open-addressed tables in shared memory; `mkey/mval` hold
//    M[a][b] += d under the key a * ld + b; at the flush each entry updates
//    M and Mt and feeds the chunk sums of rows a and b, which are
//    accumulated in `ckey/cval` (key row * cld + chunk) and flushed last.  A
//    table that is full passes the update straight to global memory.
//  kDeltaDense (B * B <= the table region): a dense B x B array of deltas in
//    `mkey` (row stride dB = B) and the chunk-sum deltas in `ckey` (row *
//    cld + chunk); no probing, and a flush that scans B * B cells.  For
//    small B, where every CTA's updates fall on a few hundred cells and
//    global atomics would queue on them.
//  kDeltaGlobal: every update straight to M, Mt and the chunk sums; for
//    large B the updates spread over many cells and the per-CTA tables cost
//    more (clear, probes, flush) than they save.
constexpr int kDeltaHashed = 0, kDeltaGlobal = 1, kDeltaDense = 2;
struct DeltaTables {
  int *mkey, *mval, *ckey, *cval;
  int mlg, clg;   // capacities 1 << mlg, 1 << clg
  int tag = 0;    // job number << 24 when the tables serve several jobs
  int mode = kDeltaHashed;
  int dB = 0;     // kDeltaDense: B
};

// Adds d under key k; false when no slot was found within kProbeMax probes
// (the caller then adds straight to global memory), so a nearly full table
// costs a bounded number of probes per insert.
constexpr int kProbeMax = 32;

__device__ __forceinline__ bool table_add(int* key, int* val, int lg, int k, int d) {
  const int cap = 1 << lg;
  unsigned h = hash_slot(k, lg);
  const int probes = cap < kProbeMax ? cap : kProbeMax;
  for (int probe = 0; probe < probes; probe++) {
    const int prev = atomicCAS(key + h, -1, k);
    if (prev == -1 || prev == k) {
      atomicAdd(val + h, d);
      return true;
    }
    h = (h + 1) & (cap - 1);
  }
  return false;
}

__device__ __forceinline__ void cs_add(const DeltaTables& t, int* CS, int key, int d) {
  if (!table_add(t.ckey, t.cval, t.clg, t.tag | key, d)) atomicAdd(CS + key, d);
}

__device__ __forceinline__ void tile_add(const DeltaTables& t, int* M, int* Mt, int* CS, int ld, int cld, int x,
                                         int y, int d) {
  if (t.mode == kDeltaDense) {
    atomicAdd(t.mkey + x * t.dB + y, d);
    atomicAdd(t.ckey + x * cld + y / kChunk, d);
    atomicAdd(t.ckey + y * cld + x / kChunk, d);
    return;
  }
  if (t.mode == kDeltaGlobal) {
    atomicAdd(M + static_cast<long long>(x) * ld + y, d);
    atomicAdd(Mt + static_cast<long long>(y) * ld + x, d);
    atomicAdd(CS + x * cld + y / kChunk, d);
    atomicAdd(CS + y * cld + x / kChunk, d);
    return;
  }
  if (table_add(t.mkey, t.mval, t.mlg, t.tag | (x * ld + y), d)) return;
  atomicAdd(M + static_cast<long long>(x) * ld + y, d);
  atomicAdd(Mt + static_cast<long long>(y) * ld + x, d);
  cs_add(t, CS, x * cld + y / kChunk, d);
  cs_add(t, CS, y * cld + x / kChunk, d);
}

__device__ __forceinline__ void tables_clear(const DeltaTables& t) {
  for (int i = threadIdx.x; i < (1 << t.mlg); i += blockDim.x) {
    t.mkey[i] = -1;
    t.mval[i] = 0;
  }
  for (int i = threadIdx.x; i < (1 << t.clg); i += blockDim.x) {
    t.ckey[i] = -1;
    t.cval[i] = 0;
  }
}

// writes the CTA's accumulated deltas to the tile (CTA-collective; the
// tables are cleared again on the way)
__device__ __forceinline__ void tables_flush(const DeltaTables& t, int* M, int* Mt, int* CS, int ld, int cld) {
  __syncthreads();
  for (int i = threadIdx.x; i < (1 << t.mlg); i += blockDim.x) {
    const int k = t.mkey[i];
    if (k < 0) continue;
    const int d = t.mval[i];
    t.mkey[i] = -1;
    t.mval[i] = 0;
    if (d == 0) continue;
    const int x = k / ld, y = k - x * ld;
    atomicAdd(M + static_cast<long long>(x) * ld + y, d);
    atomicAdd(Mt + static_cast<long long>(y) * ld + x, d);
    cs_add(t, CS, x * cld + y / kChunk, d);
    cs_add(t, CS, y * cld + x / kChunk, d);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < (1 << t.clg); i += blockDim.x) {
    const int k = t.ckey[i];
    if (k < 0) continue;
    const int d = t.cval[i];
    t.ckey[i] = -1;
    t.cval[i] = 0;
    if (d) atomicAdd(CS + k, d);
  }
  __syncthreads();
}

// kDeltaDense: zero the B x B deltas and the B * cld chunk-sum deltas
__device__ __forceinline__ void dense_clear(const DeltaTables& t, int cld) {
  const int nm = t.dB * t.dB, nc = t.dB * cld;
  for (int i = threadIdx.x; i < nm; i += blockDim.x) t.mkey[i] = 0;
  for (int i = threadIdx.x; i < nc; i += blockDim.x) t.ckey[i] = 0;
}

// kDeltaDense: writes the non-zero deltas to M, Mt and the chunk sums (whose
// layout row * cld + chunk the dense array shares) and zeroes them
// (CTA-collective)
__device__ __forceinline__ void dense_flush(const DeltaTables& t, int* M, int* Mt, int* CS, int ld, int cld) {
  __syncthreads();
  const int B = t.dB, nm = B * B, nc = B * cld;
  for (int i = threadIdx.x; i < nm; i += blockDim.x) {
    const int d = t.mkey[i];
    if (d == 0) continue;
    t.mkey[i] = 0;
    const int x = i / B, y = i - x * B;
    atomicAdd(M + static_cast<long long>(x) * ld + y, d);
    atomicAdd(Mt + static_cast<long long>(y) * ld + x, d);
  }
  for (int i = threadIdx.x; i < nc; i += blockDim.x) {
    const int d = t.ckey[i];
    if (d == 0) continue;
    t.ckey[i] = 0;
    atomicAdd(CS + i, d);
  }
}

// Applies and commits the moves of one 32-edge chunk of a batch vertex
// (warp-collective).  A chunk whose vertex did not move returns at once.
// Old blocks of batch vertices come from `from`, so part[] is committed in
// the same pass: part is read only for vertices outside [beg, end).  An
// edge between two moved vertices is applied once, from its source's
// out-list.  LDM loads move_to/from, LDP the partition.  Tile deltas go to
// the CTA's tables.
template <class LDM, class LDP>
__device__ __forceinline__ void apply_chunk(int2 ch, const GraphDev& g, int32_t* part, const int32_t* move_to,
                                            const int32_t* from, int beg, int end, const DeltaTables& t, int ld,
                                            int* M, int* Mt, int cld, int* CS, int32_t* dout, int32_t* din,
                                            int lane) {
  const int v = ch.x;
  const int s = LDM::ld(move_to + v);
  if (s < 0) return;   // warp-uniform
  const int r = LDM::ld(from + v);
  const int o0 = __ldg(g.out_ptr + v), dego = __ldg(g.out_ptr + v + 1) - o0;
  const int i0 = __ldg(g.in_ptr + v), degi = __ldg(g.in_ptr + v + 1) - i0;
  if (ch.y == 0 && lane == 0) {
    part[v] = s;
    const int ko = __ldg(g.kout + v), ki = __ldg(g.kin + v);
    atomicSub(dout + r, ko);
    atomicAdd(dout + s, ko);
    atomicSub(din + r, ki);
    atomicAdd(din + s, ki);
  }
  const unsigned span = static_cast<unsigned>(end - beg);
  const int j = ch.y * 32 + lane;
  if (j >= dego + degi) return;
  const bool is_out = j < dego;
  const int y = is_out ? __ldg(g.out_idx + o0 + j) : __ldg(g.in_idx + i0 + j - dego);
  int w = 1;
  if (is_out ? g.out_w != nullptr : g.in_w != nullptr)
    w = is_out ? __ldg(g.out_w + o0 + j) : __ldg(g.in_w + i0 + j - dego);
  const bool inb = static_cast<unsigned>(y - beg) < span;
  const int my = inb ? LDM::ld(move_to + y) : -1;
  const int oy = inb ? LDM::ld(from + y) : LDP::ld(part + y);
  if (is_out) {
    tile_add(t, M, Mt, CS, ld, cld, r, oy, -w);
    tile_add(t, M, Mt, CS, ld, cld, s, my >= 0 ? my : oy, w);
  } else if (my < 0) {
    tile_add(t, M, Mt, CS, ld, cld, oy, r, -w);
    tile_add(t, M, Mt, CS, ld, cld, oy, s, w);
  }
}

constexpr int kApplyMLg = 11;   // per-CTA delta tables of the apply kernel
constexpr int kApplyCLg = 10;

// apply + commit of one batch on the dense tile, one warp per chunk
// ([c0, c1) of g.chunks); the last CTA to finish runs the batch-end
// bookkeeping
__global__ void __launch_bounds__(kThreads) k_nodal_apply_commit(GraphDev g, int64_t c0, int64_t c1, int32_t* part,
                                                                 const int32_t* __restrict__ move_to,
                                                                 const int32_t* __restrict__ from, int beg, int end,
                                                                 int ld, int* __restrict__ M, int* __restrict__ Mt,
                                                                 int cld, int* __restrict__ CS,
                                                                 int32_t* __restrict__ dout, int32_t* __restrict__ din,
                                                                 NodalCtl* ctl, CtlArgs c) {
  __shared__ int s_mkey[1 << kApplyMLg], s_mval[1 << kApplyMLg];
  __shared__ int s_ckey[1 << kApplyCLg], s_cval[1 << kApplyCLg];
  if (ctl->done) return;   // set only by the last CTA below, after every CTA passed here
  const DeltaTables t{s_mkey, s_mval, s_ckey, s_cval, kApplyMLg, kApplyCLg};
  tables_clear(t);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t nw = static_cast<int64_t>(gridDim.x) * kWarps;
  for (int64_t q = c0 + static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5); q < c1; q += nw)
    apply_chunk<LdNC, LdPlain>(__ldg(g.chunks + q), g, part, move_to, from, beg, end, t, ld, M, Mt, cld, CS, dout,
                               din, lane);
  tables_flush(t, M, Mt, CS, ld, cld);
  if (c.active) {
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned done_ctas = atomicAdd(&ctl->apply_done, 1u);
      if (done_ctas == gridDim.x - 1) {
        __threadfence();
        ctl_batch_end(ctl, c);
        ctl->apply_done = 0;
      }
    }
  }
}

// commits the batch's moves (degrees, partition) and runs the batch-end
// bookkeeping in one launch (sorted views, which are rebuilt per batch)
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

__global__ void k_ctl_sweep_start(NodalCtl* ctl, int W, const long long* ide_q,
                                  const int* ide_n) {
  ctl_sweep_start(ctl, W, ide_q, ide_n);
}

// --- persistent nodal phase ----------------------------------------------------
constexpr int kPThreads = 768;    // one CTA per SM (80 registers a thread)
constexpr int kPWarps = kPThreads / 32;
constexpr int kUnitWarp = -2;     // work unit of one vertex with 64 < degree <= 128
constexpr int kPHubLg = 13;
constexpr int kPHubSlots = 1 << kPHubLg;  // hub table slots in shared memory; larger hub tables are global
constexpr int kDeltaGlobalMinB = 256;     // from this B the phase kernel's apply writes straight to global memory
// the proposals of the phase kernel read the tile from shared memory up to
// this B: M and Mt (B x ld each, ld = B rounded up to 4) after the first
// kSnapOff slots of the hub table's first and second arrays, chunk sums and
// degrees after those of its third
constexpr int kSnapMaxB = 88;
constexpr int kSnapOff = 256;   // >= a hub table's capacity for B <= kSnapMaxB (2 * B rounded up to a power of 2)
static_assert(kSnapOff + kSnapMaxB * ((kSnapMaxB + 3) & ~3) <= kPHubSlots, "tile copy overruns its region");
static_assert(kSnapOff + 3 * kSnapMaxB <= kPHubSlots, "degree copy overruns its region");
static_assert(2 * kSnapMaxB <= kSnapOff && kSnapMaxB <= kChunk, "hub tables or chunk sums outgrow the layout");
static_assert(kPHubSlots == kPhaseHubSlots, "hub regions are assigned for tables beyond this size");
constexpr unsigned long long kBarrierTimeoutNs = 200ull * 1000ull * 1000ull;
// dynamic shared memory: per-warp tables and lists, then the hub table
constexpr size_t kPWarpInts = 3 * kHCap + kHubDegree;
constexpr size_t kPSmemBytes = sizeof(int) * (kPWarps * kPWarpInts + 3 * kPHubSlots);

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add64(unsigned long long* p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

constexpr unsigned long long kBarDone = 1ull << 32;   // bits 32..47: done arrivals
constexpr unsigned long long kBarOvf = 1ull << 48;    // bits 48..63: overflow arrivals (mod 2^16)

// Grid-wide barrier of the persistent kernel (all CTAs are co-resident:
// cooperative launch).  ctl->bar counts arrivals over the whole launch in
// its low 32 bits; barrier number k is passed once it reaches
// k * gridDim.x (`target`, advanced here).  After __syncthreads, thread 0
// adds its arrival with release semantics (publishing the CTA's writes)
// and waits with acquire loads.  The arrival may also carry kBarDone or
// kBarOvf, which every CTA then sees in the same load; *s_ovf (if given)
// receives the overflow count.  A wait gives up after kBarrierTimeoutNs and
// sets bar_err.  Returns -1 on error (every CTA then leaves at its next
// barrier), else 1 if kBarDone is set, else 0.
// Wait limit of a grid barrier and the failure-injection switch: a CTA
// with `hold` set never arrives, so every wait of the launch runs out.
struct BarrierOpts {
  unsigned long long timeout_ns = kBarrierTimeoutNs;
  bool hold = false;
};

template <class CtlT>
__device__ __forceinline__ int grid_barrier(CtlT* ctl, unsigned* target, bool publish_done, int* s_state,
                                            bool publish_ovf = false, unsigned* s_ovf = nullptr,
                                            BarrierOpts bo = BarrierOpts{}) {
  *target += gridDim.x;
  __syncthreads();
  if (threadIdx.x == 0) {
    // a CTA told to withhold its arrival (failure injection) still waits,
    // so that every CTA leaves through the timeout below
    if (!bo.hold)
      red_release_add64(&ctl->bar, (publish_done ? 1ull + kBarDone : 1ull) + (publish_ovf ? kBarOvf : 0ull));
    const unsigned long long t0 = global_ns();
    unsigned spins = 0;
    int st;
    for (;;) {
      const unsigned long long v = ld_acquire64(&ctl->bar);
      if (static_cast<unsigned>(v) >= *target) {
        st = ((v >> 32) & 0xffffull) ? 1 : 0;
        if (s_ovf) *s_ovf = static_cast<unsigned>(v >> 48);
        break;
      }
      if ((++spins & 63u) == 0) {
        if (*reinterpret_cast<volatile int*>(&ctl->bar_err)) {
          st = -1;
          break;
        }
        if (global_ns() - t0 > bo.timeout_ns) {
          atomicExch(&ctl->bar_err, 1);
          st = -1;
          break;
        }
      }
    }
    *s_state = st;
  }
  __syncthreads();
  return *s_state;
}

// One stage's nodal phase in one cooperative launch: up to `maxitr` sweeps,
// each an entropy pass, the sweep-start bookkeeping, and for every batch a
// proposal pass (hubs first, one per CTA; then warp-per-vertex, first one
// vertex per warp of the CTAs without a hub, the rest handed out by a
// counter) and an apply pass, during which one thread runs the batch-end
// bookkeeping.  Each CTA applies the moves it accepted itself: the chunks
// of its moved work-unit vertices (listed in shared memory during the
// proposals) and of its moved hubs.  If any CTA's list overflowed (it
// announces that with its barrier arrival, so every CTA learns it from the
// same barrier load), every CTA instead scans all of the batch's edge
// chunks, skipping vertices that did not move.  Tile deltas accumulate per
// CTA as DeltaTables' mode for this B says.  Leaves when the convergence
// test sets `done`.
constexpr int kOwnCap = 1024;   // chunk entries of a CTA's own-move list

// algorithmic bytes of an applied chunk: per edge of a moved vertex its
// neighbour's id and block (8) and the two updated entries of M (16)
__device__ __forceinline__ unsigned long long apply_bytes(const NodalArgs& a, int2 ch) {
  if (__ldcg(a.move_to + ch.x) < 0) return 0;
  const int deg = (__ldg(a.out_ptr + ch.x + 1) - __ldg(a.out_ptr + ch.x)) +
                  (__ldg(a.in_ptr + ch.x + 1) - __ldg(a.in_ptr + ch.x));
  return 24ull * static_cast<unsigned long long>(max(0, min(32, deg - 32 * ch.y)));
}
// One work unit of the persistent kernels: two vertices of degree <= 64
// (a half-warp each; un.y = -1 when there is only one) or one vertex of
// degree <= 128 (the whole warp, un.y = kUnitWarp).  wtab: the warp's
// shared-memory tables.
template <class Ops>
__device__ __forceinline__ void unit_vertices(const NodalArgs& a, const Ops& ops, int2 un, uint32_t itr, int* wtab,
                                              CtaTally* tl, int lane, unsigned long long* my_bytes) {
  if (un.y == kUnitWarp) {
    group_vertex(a, ops, un.x, itr, wtab, wtab + kHCap, wtab + 2 * kHCap, wtab + 3 * kHCap, tl, Grp<32>(lane),
                 my_bytes);
  } else {
    const int h = lane >> 4;
    const int vv = h ? un.y : un.x;
    if (vv >= 0)
      group_vertex(a, ops, vv, itr, wtab + h * (kHCap / 2), wtab + kHCap + h * (kHCap / 2),
                   wtab + 2 * kHCap + h * (kHCap / 2), wtab + 3 * kHCap + h * (kHubDegree / 2), tl, Grp<16>(lane),
                   my_bytes);
  }
}

// Precision mode 3: the reference's old-state dS terms of every tile cell
// for the batch about to be proposed (grid-collective; they depend on the
// cell and its blocks' degrees only, not on the proposing vertex):
//   Trow[b, i] = M[b,i] log(M[b,i] / (d_in[i] d_out[b]))
//   Tcol[b, i] = M[i,b] log(M[i,b] / (d_out[i] d_in[b]))
// in the reference's float arithmetic (ref_term), 0 for empty cells.
__device__ __forceinline__ void ref32_tables_pass(int B, int ld, const int* M, const int* Mt, const int32_t* din,
                                                  const int32_t* dout, float* Trow, float* Tcol) {
  const long long cells = static_cast<long long>(B) * ld;
  for (long long c = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; c < cells;
       c += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int b = static_cast<int>(c / ld), i = static_cast<int>(c - static_cast<long long>(b) * ld);
    float tr = 0.0f, tc = 0.0f;
    if (i < B) {
      const int x = __ldcg(M + c), y = __ldcg(Mt + c);
      if (x) tr = ref_term(x, static_cast<long long>(__ldcg(din + i)) * __ldcg(dout + b));
      if (y) tc = ref_term(y, static_cast<long long>(__ldcg(dout + i)) * __ldcg(din + b));
    }
    __stcg(Trow + c, tr);
    __stcg(Tcol + c, tc);
  }
}

template <int P, bool kSnap>
__global__ void __launch_bounds__(kPThreads, 1) k_nodal_phase(PhaseArgs p) {
  extern __shared__ __align__(16) int dyn[];
  __shared__ CtaTally s_tally;
  __shared__ HubShared<kPWarps> sh;
  __shared__ int s_base, s_state;
  __shared__ unsigned s_ovf;
  __shared__ int2 s_own[kOwnCap];
  __shared__ int s_nown;
  using Ops = DenseOpsT<LdCG, P, std::conditional_t<kSnap, LdPlain, LdCG>>;
  NodalCtl* ctl = p.a.ctl;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int gw = blockIdx.x * kPWarps + wib;
  const int nw = gridDim.x * kPWarps;
  int* wtab = dyn + wib * kPWarpInts;
  int* htab = dyn + kPWarps * kPWarpInts;   // hub table during proposals, delta tables during apply
  // kSnap (B <= kSnapMaxB): the proposals read M, Mt, the chunk sums and the
  // block degrees from a copy in shared memory, taken at every batch start;
  // it shares the hub table's region (a hub's table then needs at most
  // kSnapOff slots per array)
  int* sM = htab + kSnapOff;
  int* sMt = htab + kPHubSlots + kSnapOff;
  int* sCS = htab + 2 * kPHubSlots + kSnapOff;
  int* sdin = sCS + kSnapMaxB;
  int* sdout = sdin + kSnapMaxB;
  DenseView vs = p.v;
  if (kSnap) {
    vs.M = sM;
    vs.Mt = sMt;
    vs.CS = sCS;
  }
  const Ops ops{vs, p.a.B};
  BarrierOpts bo;
  bo.timeout_ns = p.bar_timeout_ns ? p.bar_timeout_ns : kBarrierTimeoutNs;
  bo.hold = static_cast<int>(blockIdx.x) == p.bar_hold;
  // dense deltas in the first 2 * kPHubSlots ints, chunk-sum deltas (B <= 128: B entries) after them
  const int mode = p.a.B >= kDeltaGlobalMinB ? kDeltaGlobal
                   : (p.a.B * p.a.B <= 2 * kPHubSlots ? kDeltaDense : kDeltaHashed);
  const DeltaTables dt{htab, htab + kPHubSlots, htab + 2 * kPHubSlots, htab + 2 * kPHubSlots + kPHubSlots / 2,
                       kPHubLg, kPHubLg - 1, 0, mode, p.a.B};
  const int B = p.a.B;
  unsigned ovf_seen = 0;   // overflow count at the previous proposal barrier
  const int64_t cells = static_cast<int64_t>(B) * B;
  unsigned target = 0;
  unsigned long long my_bytes = 0;
  bool converged = false;
  for (int sw = 0; sw < p.maxitr; sw++) {
    // data term of S for this sweep (the entropy kernel's sum)
    {
      long long acc = 0;
      unsigned long long seen = 0, nz = 0;
      for (int64_t c = static_cast<int64_t>(blockIdx.x) * kPThreads + threadIdx.x; c < cells;
           c += static_cast<int64_t>(gridDim.x) * kPThreads) {
        const int i = static_cast<int>(c / B), j = static_cast<int>(c - static_cast<int64_t>(i) * B);
        const int m = __ldcg(p.v.M + static_cast<int64_t>(i) * p.v.ld + j);
        seen++;
        if (m) {
          nz++;
          acc += q32(g_term(p.a.L, m, __ldcg(p.din + j), __ldcg(p.dout + i)));
        }
      }
      // algorithmic bytes: every cell of the tile, two degrees per nonzero
      if (p.a.stats) my_bytes += 4 * seen + 8 * nz;
      acc = warp_sum_ll(acc);
      if (lane == 0 && acc) atomicAdd(&ctl->entropy_acc, static_cast<unsigned long long>(acc));
    }
    if (grid_barrier(ctl, &target, false, &s_state, false, nullptr, bo) < 0) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ctl_sweep_start(ctl, p.W, p.ide_q, p.ide_n);
      ctl->entropy_acc = 0;
    }
    if (grid_barrier(ctl, &target, false, &s_state, false, nullptr, bo) < 0) return;
    const uint32_t itr = static_cast<uint32_t>(sw);   // ctl->sweeps before this sweep started
    for (int bi = 0; bi * p.bs < p.n; bi++) {
      NodalArgs a = p.a;
      a.beg = bi * p.bs;
      a.end = a.beg + p.bs < p.n ? a.beg + p.bs : p.n;
      const int count = a.end - a.beg;
      if constexpr (P == 3) {
        if (p.a.Trow) {   // the batch's old-state terms, before anyone proposes
          ref32_tables_pass(B, p.a.tld, p.v.M, p.v.Mt, p.din, p.dout, p.a.Trow, p.a.Tcol);
          if (grid_barrier(ctl, &target, false, &s_state, false, nullptr, bo) < 0) return;
        }
      }
      if (kSnap) {
        // the tile as the previous batch left it (rows padded to ld with
        // zeros; cld = 1)
        const int n4 = B * p.v.ld / 4;
        for (int i = threadIdx.x; i < n4; i += kPThreads) {
          reinterpret_cast<int4*>(sM)[i] = __ldcg(reinterpret_cast<const int4*>(p.v.M) + i);
          reinterpret_cast<int4*>(sMt)[i] = __ldcg(reinterpret_cast<const int4*>(p.v.Mt) + i);
        }
        for (int i = threadIdx.x; i < B; i += kPThreads) {
          sCS[i] = __ldcg(p.v.CS + i);
          sdin[i] = __ldcg(p.din + i);
          sdout[i] = __ldcg(p.dout + i);
        }
        a.din = sdin;
        a.dout = sdout;
        __syncthreads();
      }
      // proposals
      if (threadIdx.x == 0) {
        s_tally = CtaTally{0, 0, 0, 0};
        s_tally.own = s_own;
        s_tally.nown = &s_nown;
        s_tally.own_cap = kOwnCap;
        s_nown = 0;
      }
      __syncthreads();
      const int hub_lo = __ldg(p.batch_hub + bi), hub_hi = __ldg(p.batch_hub + bi + 1);
      const int hcta = min(hub_hi - hub_lo, static_cast<int>(gridDim.x));
      for (int h = hub_lo + blockIdx.x; h < hub_hi; h += gridDim.x)
        hub_vertex<Ops, kPThreads>(a, ops, __ldg(p.hubs + h), itr, htab, kPHubSlots, &sh, &my_bytes);
      // work units: two vertices of degree <= 64 (a half-warp each) or one
      // of degree <= 128 (a warp)
      const int u_lo = __ldg(p.unit_ptr + bi), nun = __ldg(p.unit_ptr + bi + 1) - u_lo;
      const int first = (gridDim.x - hcta) * kPWarps;   // units handed out without the counter
      if (static_cast<int>(blockIdx.x) >= hcta) {
        const int i = (blockIdx.x - hcta) * kPWarps + wib;
        if (i < nun) unit_vertices(a, ops, __ldg(p.units + u_lo + i), itr, wtab, &s_tally, lane, &my_bytes);
      }
      // the rest in rounds of one unit per warp, kPWarps per counter step
      for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_base = first + static_cast<int>(atomicAdd(&ctl->vnext, static_cast<unsigned>(kPWarps)));
        __syncthreads();
        const int i0 = s_base;
        if (i0 >= nun) break;
        if (i0 + wib < nun) unit_vertices(a, ops, __ldg(p.units + u_lo + i0 + wib), itr, wtab, &s_tally, lane, &my_bytes);
      }
      __syncthreads();
      if (threadIdx.x == 0) tally_flush(&s_tally, ctl);
      const int nown = s_nown;
      if (grid_barrier(ctl, &target, false, &s_state, nown > kOwnCap, &s_ovf, bo) < 0) return;
      // every CTA reads the same count here: the next overflow arrivals come
      // after the next proposal pass, which no CTA starts before all passed
      // the apply barrier below
      const bool scan_all = s_ovf != ovf_seen;
      ovf_seen = s_ovf;
      if (dt.mode == kDeltaDense) dense_clear(dt, p.v.cld);
      else if (dt.mode == kDeltaHashed) tables_clear(dt);
      // apply + commit; one thread closes the batch meanwhile
      bool done = false;
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        const long long edges = (static_cast<long long>(__ldg(p.a.out_ptr + a.end)) - __ldg(p.a.out_ptr + a.beg)) +
                                (static_cast<long long>(__ldg(p.a.in_ptr + a.end)) - __ldg(p.a.in_ptr + a.beg));
        const CtlArgs ca{1, p.W, p.thr, p.model_d, p.ide_q, p.ide_n, count, edges};
        done = ctl_batch_end(ctl, ca);
        ctl->vnext = 0;
        if (scan_all) ctl->apply_scans++;
      }
      __syncthreads();
      {
        // own moves (chunk k of the CTA's list), or every chunk of the batch
        const int64_t cb = scan_all ? __ldg(p.chunk_ptr + a.beg) : 0;
        const int64_t k1 = scan_all ? __ldg(p.chunk_ptr + a.end) : nown;
        const int step = scan_all ? nw : kPWarps;
        for (int64_t k = (scan_all ? cb + gw : wib); k < k1; k += step) {
          const int2 ch = scan_all ? __ldg(p.g.chunks + k) : s_own[k];
          apply_chunk<LdCG, LdCG>(ch, p.g, p.part, a.move_to, a.from, a.beg, a.end, dt, p.v.ld, p.M, p.Mt,
                                  p.v.cld, p.CS, p.dout, p.din, lane);
          if (p.a.stats && lane == 0) my_bytes += apply_bytes(p.a, ch);
        }
      }
      // the CTA's moved hubs, whose chunks are not listed
      for (int h = hub_lo + blockIdx.x; !scan_all && h < hub_hi; h += gridDim.x) {
        const int v = __ldg(p.hubs + h);
        if (__ldcg(a.move_to + v) < 0) continue;   // CTA-uniform
        const int64_t q1 = __ldg(p.chunk_ptr + v + 1);
        for (int64_t q = __ldg(p.chunk_ptr + v) + wib; q < q1; q += kPWarps) {
          const int2 ch = __ldg(p.g.chunks + q);
          apply_chunk<LdCG, LdCG>(ch, p.g, p.part, a.move_to, a.from, a.beg, a.end, dt, p.v.ld, p.M, p.Mt,
                                  p.v.cld, p.CS, p.dout, p.din, lane);
          if (p.a.stats && lane == 0) my_bytes += apply_bytes(p.a, ch);
        }
      }
      if (dt.mode == kDeltaDense) dense_flush(dt, p.M, p.Mt, p.CS, p.v.ld, p.v.cld);
      else if (dt.mode == kDeltaHashed) tables_flush(dt, p.M, p.Mt, p.CS, p.v.ld, p.v.cld);
      const int st = grid_barrier(ctl, &target, done, &s_state, false, nullptr, bo);
      if (st < 0) return;   // a barrier failed
      if (st > 0) {         // converged
        converged = true;
        break;
      }
    }
    if (converged) break;
  }
  // the data term of the final state (the stage's description length),
  // read by the host with the control block; entropy_acc was cleared at
  // the last sweep start
  {
    long long acc = 0;
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * kPThreads + threadIdx.x; c < cells;
         c += static_cast<int64_t>(gridDim.x) * kPThreads) {
      const int i = static_cast<int>(c / B), j = static_cast<int>(c - static_cast<int64_t>(i) * B);
      const int m = __ldcg(p.v.M + static_cast<int64_t>(i) * p.v.ld + j);
      if (m) acc += q32(g_term(p.a.L, m, __ldcg(p.din + j), __ldcg(p.dout + i)));
    }
    acc = warp_sum_ll(acc);
    if (lane == 0 && acc) atomicAdd(&ctl->entropy_acc, static_cast<unsigned long long>(acc));
  }
  if (p.a.stats && my_bytes) atomicAdd(&ctl->bytes, my_bytes);
}

// --- gang of jobs: many nodal phases in one cooperative launch ---------------
// first index j with pref[j + 1] > x (pref ascending, pref[0] = 0, x < pref[K])
__device__ __forceinline__ int find_job(const long long* pref, int K, long long x) {
  int lo = 0, hi = K;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (pref[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// writes the deltas of the gang's jobs (key = job << 24 | index) to their
// tiles (CTA-collective; tables cleared on the way)
__device__ __forceinline__ void gang_tables_flush(const DeltaTables& t, const PhaseArgs* __restrict__ jobs) {
  __syncthreads();
  for (int i = threadIdx.x; i < (1 << t.mlg); i += blockDim.x) {
    const int k = t.mkey[i];
    if (k < 0) continue;
    const int d = t.mval[i];
    t.mkey[i] = -1;
    t.mval[i] = 0;
    if (d == 0) continue;
    const int j = k >> 24, idx = k & 0xffffff;
    const PhaseArgs& p = jobs[j];
    const int ld = p.v.ld, cld = p.v.cld;
    const int x = idx / ld, y = idx - x * ld;
    atomicAdd(p.M + static_cast<long long>(x) * ld + y, d);
    atomicAdd(p.Mt + static_cast<long long>(y) * ld + x, d);
    DeltaTables tj = t;
    tj.tag = j << 24;
    cs_add(tj, p.CS, x * cld + y / kChunk, d);
    cs_add(tj, p.CS, y * cld + x / kChunk, d);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < (1 << t.clg); i += blockDim.x) {
    const int k = t.ckey[i];
    if (k < 0) continue;
    const int d = t.cval[i];
    t.ckey[i] = -1;
    t.cval[i] = 0;
    if (d) atomicAdd(jobs[k >> 24].CS + (k & 0xffffff), d);
  }
  __syncthreads();
}

// out[0] = 0, out[j + 1] = v_0 + ... + v_j over the gang's jobs, where
// thread j holds v_j (0 for j >= K); CTA-collective, K <= kGangMax = 64
__device__ __forceinline__ void job_prefix(long long v, long long* tmp, long long* out) {
  if (threadIdx.x < kGangMax) tmp[threadIdx.x] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    const int l = threadIdx.x;
    const long long a = warp_incl_scan_ll(tmp[l], l);
    const long long ta = __shfl_sync(0xffffffffu, a, 31);
    const long long b = warp_incl_scan_ll(tmp[l + 32], l) + ta;
    out[l + 1] = a;
    out[l + 33] = b;
    if (l == 0) out[0] = 0;
  }
  __syncthreads();
}

// The nodal phases of K jobs (each at some stage of its own solve, dense
// tile, B <= 4096) in one cooperative launch.  Every round advances each
// unfinished job by one batch: jobs that start a sweep get their entropy
// pass and sweep-start bookkeeping first; then the proposals of all jobs'
// current batches (hubs one per CTA, then work units) share the grid, and
// so do their apply passes, while one thread per job closes its batch.  A
// job leaves the gang when its convergence test fires or its sweep budget
// is spent; the launch ends with the last job.  The arithmetic per job is
// that of k_nodal_phase (same device functions, same order of the integer
// sums' terms is irrelevant), so each job's result equals its solo solve.
template <int P>
__global__ void __launch_bounds__(kPThreads, 1) k_nodal_gang(const PhaseArgs* __restrict__ jobs, int K, GangCtl* gc,
                                                             int exit_below) {
  extern __shared__ __align__(16) int dyn[];
  __shared__ CtaTally s_tally[kGangMax];
  __shared__ HubShared<kPWarps> sh;
  __shared__ int s_bi[kGangMax], s_sw[kGangMax], s_act[kGangMax], s_nb[kGangMax];
  __shared__ int s_fin[kGangMax];   // finished in the last round: its final data term is due
  __shared__ long long s_hp[kGangMax + 1], s_up[kGangMax + 1], s_cp[kGangMax + 1], s_tmp[kGangMax];
  __shared__ int s_base, s_state;
  __shared__ unsigned s_ovf;
  __shared__ int2 s_own[kOwnCap];   // {v, job << 16 | chunk} of the CTA's accepted work-unit moves
  __shared__ int s_nown;
  unsigned ovf_seen = 0;
  using Ops = DenseOpsT<LdCG, P>;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int gw = blockIdx.x * kPWarps + wib;
  const int nw = gridDim.x * kPWarps;
  int* wtab = dyn + wib * kPWarpInts;
  int* htab = dyn + kPWarps * kPWarpInts;
  const DeltaTables dt{htab, htab + kPHubSlots, htab + 2 * kPHubSlots, htab + 2 * kPHubSlots + kPHubSlots / 2,
                       kPHubLg, kPHubLg - 1};
  unsigned target = 0;
  unsigned long long unused_bytes = 0;
  // a job may resume where an earlier launch left it: at batch gang_batch
  // of the sweep it had started (ctl->sweeps counts started sweeps)
  if (threadIdx.x < K) {
    const PhaseArgs& p = jobs[threadIdx.x];
    const int gb = __ldcg(&p.a.ctl->gang_batch);
    const int started = static_cast<int>(__ldcg(&p.a.ctl->sweeps));
    const int done = __ldcg(&p.a.ctl->done);
    s_bi[threadIdx.x] = gb;
    s_sw[threadIdx.x] = gb > 0 ? started - 1 : started;
    s_act[threadIdx.x] = !done && s_sw[threadIdx.x] < p.maxitr ? 1 : 0;
    s_nb[threadIdx.x] = (p.n + p.bs - 1) / p.bs;
    s_fin[threadIdx.x] = 0;
  }
  __syncthreads();

  for (;;) {
    __syncthreads();
    const bool mine = threadIdx.x < K && s_act[threadIdx.x];
    const int count = __syncthreads_count(mine);
    const int fin = __syncthreads_or(threadIdx.x < K && s_fin[threadIdx.x]);
    // no job left, or enough are done: the rest resume in the next launch
    const bool leaving = count == 0 || count < exit_below;
    const int start = leaving ? 0 : __syncthreads_or(mine && s_bi[threadIdx.x] == 0);
    if (start || fin) {
      // data term of S: at the sweep start of the jobs that begin one, and
      // of the final state of those that finished (read by the host)
      {
        long long cells = 0;
        if ((start && mine && s_bi[threadIdx.x] == 0) || (threadIdx.x < K && s_fin[threadIdx.x])) {
          const long long B = jobs[threadIdx.x].a.B;
          cells = B * B;
        }
        job_prefix(cells, s_tmp, s_cp);
      }
      const long long total = s_cp[K];
      long long acc = 0;
      int cj = -1;
      for (long long c = static_cast<long long>(blockIdx.x) * kPThreads + threadIdx.x; c < total;
           c += static_cast<long long>(gridDim.x) * kPThreads) {
        const int j = find_job(s_cp, K, c);
        if (j != cj) {
          if (cj >= 0 && acc) atomicAdd(&jobs[cj].a.ctl->entropy_acc, static_cast<unsigned long long>(acc));
          acc = 0;
          cj = j;
        }
        const PhaseArgs& p = jobs[j];
        const long long cc = c - s_cp[j];
        const int B = p.a.B;
        const int i = static_cast<int>(cc / B), jj = static_cast<int>(cc - static_cast<long long>(i) * B);
        const int m = __ldcg(p.v.M + static_cast<long long>(i) * p.v.ld + jj);
        if (m) acc += q32(g_term(p.a.L, m, __ldcg(p.din + jj), __ldcg(p.dout + i)));
      }
      if (cj >= 0 && acc) atomicAdd(&jobs[cj].a.ctl->entropy_acc, static_cast<unsigned long long>(acc));
      __syncthreads();
      if (threadIdx.x < K) s_fin[threadIdx.x] = 0;
      if (start) {
        if (grid_barrier(gc, &target, false, &s_state) < 0) return;
        if (blockIdx.x == 0 && threadIdx.x < K && s_act[threadIdx.x] && s_bi[threadIdx.x] == 0) {
          const PhaseArgs& p = jobs[threadIdx.x];
          ctl_sweep_start(p.a.ctl, p.W, p.ide_q, p.ide_n);
          p.a.ctl->entropy_acc = 0;
        }
        if (grid_barrier(gc, &target, false, &s_state) < 0) return;
      }
    }
    if (leaving) break;
    if constexpr (P == 3) {
      // precision 3: the old-state term tables of every unfinished job's
      // batch (as the single-job kernel's ref32_tables_pass), before anyone
      // proposes
      {
        long long cells = 0;
        if (mine && jobs[threadIdx.x].a.Trow) cells = static_cast<long long>(jobs[threadIdx.x].a.B) * jobs[threadIdx.x].a.tld;
        job_prefix(cells, s_tmp, s_cp);
      }
      const long long total = s_cp[K];
      if (total > 0) {
        for (long long c = static_cast<long long>(blockIdx.x) * kPThreads + threadIdx.x; c < total;
             c += static_cast<long long>(gridDim.x) * kPThreads) {
          const int j = find_job(s_cp, K, c);
          const PhaseArgs& p = jobs[j];
          const long long cc = c - s_cp[j];
          const int ld = p.a.tld, B = p.a.B;
          const int b = static_cast<int>(cc / ld), i = static_cast<int>(cc - static_cast<long long>(b) * ld);
          float tr = 0.0f, tc = 0.0f;
          if (i < B) {
            const int x = __ldcg(p.v.M + cc), y = __ldcg(p.v.Mt + cc);
            if (x) tr = ref_term(x, static_cast<long long>(__ldcg(p.din + i)) * __ldcg(p.dout + b));
            if (y) tc = ref_term(y, static_cast<long long>(__ldcg(p.dout + i)) * __ldcg(p.din + b));
          }
          __stcg(p.a.Trow + cc, tr);
          __stcg(p.a.Tcol + cc, tc);
        }
        if (grid_barrier(gc, &target, false, &s_state) < 0) return;
      }
    }
    // proposals of every unfinished job's current batch
    if (threadIdx.x < K) {
      s_tally[threadIdx.x] = CtaTally{0, 0, 0, 0};
      s_tally[threadIdx.x].own = s_own;
      s_tally[threadIdx.x].nown = &s_nown;
      s_tally[threadIdx.x].own_cap = kOwnCap;
      s_tally[threadIdx.x].own_tag = threadIdx.x << 16;
    }
    if (threadIdx.x == 0) s_nown = 0;
    {
      long long nh = 0, nu = 0;
      if (mine) {
        const PhaseArgs& p = jobs[threadIdx.x];
        const int b = s_bi[threadIdx.x];
        nh = __ldg(p.batch_hub + b + 1) - __ldg(p.batch_hub + b);
        nu = __ldg(p.unit_ptr + b + 1) - __ldg(p.unit_ptr + b);
      }
      job_prefix(nh, s_tmp, s_hp);
      job_prefix(nu, s_tmp, s_up);
    }
    const int H = static_cast<int>(s_hp[K]);
    const int U = static_cast<int>(s_up[K]);
    for (int h = blockIdx.x; h < H; h += gridDim.x) {
      const int j = find_job(s_hp, K, h);
      const PhaseArgs& p = jobs[j];
      const int v = __ldg(p.hubs + __ldg(p.batch_hub + s_bi[j]) + (h - static_cast<int>(s_hp[j])));
      hub_vertex<Ops, kPThreads>(p.a, Ops{p.v, p.a.B}, v, static_cast<uint32_t>(s_sw[j]), htab, kPHubSlots, &sh,
                                 &unused_bytes);
    }
    auto run_unit = [&](int u) {
      const int j = find_job(s_up, K, u);
      const PhaseArgs& p = jobs[j];
      const int2 un = __ldg(p.units + __ldg(p.unit_ptr + s_bi[j]) + (u - static_cast<int>(s_up[j])));
      unit_vertices(p.a, Ops{p.v, p.a.B}, un, static_cast<uint32_t>(s_sw[j]), wtab, &s_tally[j], lane,
                    &unused_bytes);
    };
    const int hcta = min(H, static_cast<int>(gridDim.x));
    const int first = (gridDim.x - hcta) * kPWarps;
    if (static_cast<int>(blockIdx.x) >= hcta) {
      const int i = (blockIdx.x - hcta) * kPWarps + wib;
      if (i < U) run_unit(i);
    }
    for (;;) {
      __syncthreads();
      if (threadIdx.x == 0) s_base = first + static_cast<int>(atomicAdd(&gc->vnext, static_cast<unsigned>(kPWarps)));
      __syncthreads();
      const int i0 = s_base;
      if (i0 >= U) break;
      if (i0 + wib < U) run_unit(i0 + wib);
    }
    __syncthreads();
    if (threadIdx.x < K && s_act[threadIdx.x]) tally_flush(&s_tally[threadIdx.x], jobs[threadIdx.x].a.ctl);
    const int nown = s_nown;
    if (grid_barrier(gc, &target, false, &s_state, nown > kOwnCap, &s_ovf) < 0) return;
    // as in k_nodal_phase: every CTA reads the same overflow count here
    const bool scan_all = s_ovf != ovf_seen;
    ovf_seen = s_ovf;
    // apply + commit of every job's batch; one thread per job closes it.
    // Each CTA applies the moves it accepted (its listed work-unit chunks
    // and its moved hubs), or, after an overflow anywhere, every CTA takes
    // its share of all jobs' batch chunks.
    if (blockIdx.x == 0) {
      if (threadIdx.x < K && s_act[threadIdx.x]) {
        const PhaseArgs& p = jobs[threadIdx.x];
        const int beg = s_bi[threadIdx.x] * p.bs, end = min(p.n, beg + p.bs);
        const long long edges = (static_cast<long long>(__ldg(p.a.out_ptr + end)) - __ldg(p.a.out_ptr + beg)) +
                                (static_cast<long long>(__ldg(p.a.in_ptr + end)) - __ldg(p.a.in_ptr + beg));
        const CtlArgs ca{1, p.W, p.thr, p.model_d, p.ide_q, p.ide_n, end - beg, edges};
        ctl_batch_end(p.a.ctl, ca);
      }
      if (threadIdx.x == 0) gc->vnext = 0;
    }
    tables_clear(dt);
    if (scan_all) {
      long long c = 0;
      if (mine) {
        const PhaseArgs& p = jobs[threadIdx.x];
        const int beg = s_bi[threadIdx.x] * p.bs, end = min(p.n, beg + p.bs);
        c = __ldg(p.chunk_ptr + end) - __ldg(p.chunk_ptr + beg);
      }
      job_prefix(c, s_tmp, s_cp);
      const long long C = s_cp[K];
      for (long long q = gw; q < C; q += nw) {
        const int j = find_job(s_cp, K, q);
        const PhaseArgs& p = jobs[j];
        const int beg = s_bi[j] * p.bs, end = min(p.n, beg + p.bs);
        const int2 ch = __ldg(p.g.chunks + __ldg(p.chunk_ptr + beg) + (q - s_cp[j]));
        DeltaTables tj = dt;
        tj.tag = j << 24;
        apply_chunk<LdCG, LdCG>(ch, p.g, p.part, p.a.move_to, p.a.from, beg, end, tj, p.v.ld, p.M, p.Mt,
                                p.v.cld, p.CS, p.dout, p.din, lane);
      }
    } else {
      __syncthreads();
      for (int i = wib; i < nown; i += kPWarps) {
        const int2 e = s_own[i];
        const int j = e.y >> 16;
        const PhaseArgs& p = jobs[j];
        const int beg = s_bi[j] * p.bs, end = min(p.n, beg + p.bs);
        DeltaTables tj = dt;
        tj.tag = j << 24;
        apply_chunk<LdCG, LdCG>(make_int2(e.x, e.y & 0xffff), p.g, p.part, p.a.move_to, p.a.from, beg, end, tj,
                                p.v.ld, p.M, p.Mt, p.v.cld, p.CS, p.dout, p.din, lane);
      }
      for (int h = blockIdx.x; h < H; h += gridDim.x) {   // the hubs this CTA proposed for
        const int j = find_job(s_hp, K, h);
        const PhaseArgs& p = jobs[j];
        const int v = __ldg(p.hubs + __ldg(p.batch_hub + s_bi[j]) + (h - static_cast<int>(s_hp[j])));
        if (__ldcg(p.a.move_to + v) < 0) continue;   // CTA-uniform
        const int beg = s_bi[j] * p.bs, end = min(p.n, beg + p.bs);
        DeltaTables tj = dt;
        tj.tag = j << 24;
        const int64_t q1 = __ldg(p.chunk_ptr + v + 1);
        for (int64_t q = __ldg(p.chunk_ptr + v) + wib; q < q1; q += kPWarps)
          apply_chunk<LdCG, LdCG>(__ldg(p.g.chunks + q), p.g, p.part, p.a.move_to, p.a.from, beg, end, tj, p.v.ld,
                                  p.M, p.Mt, p.v.cld, p.CS, p.dout, p.din, lane);
      }
    }
    gang_tables_flush(dt, jobs);
    if (grid_barrier(gc, &target, false, &s_state) < 0) return;
    // advance every job by one batch
    if (threadIdx.x < K && s_act[threadIdx.x]) {
      const int j = threadIdx.x;
      const PhaseArgs& p = jobs[j];
      const int done = *reinterpret_cast<volatile int*>(&p.a.ctl->done);
      if (++s_bi[j] == s_nb[j]) {
        s_bi[j] = 0;
        s_sw[j]++;
      }
      if (done || s_sw[j] >= p.maxitr) {
        s_act[j] = 0;
        s_fin[j] = 1;
      }
    }
  }
  // where each job stands: finished, or the batch to resume at
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x < K) {
    const int j = threadIdx.x;
    gc->finished[j] = s_act[j] ? 0 : 1;
    jobs[j].a.ctl->gang_batch = s_act[j] ? s_bi[j] : 0;
  }
}

// the hub CTAs run on a second stream, concurrently with the warp kernel
template <class Ops>
void launch_propose(const NodalArgs& a, Ops ops, const HubList& hubs, const StreamPair& sp) {
  const int count = a.end - a.beg;
  if (count <= 0) return;
  const bool has_hubs = hubs.hi > hubs.lo;
  const bool fork = has_hubs && sp.side != sp.main;   // hubs overlap the warp kernel on the side stream
  if (fork) {
    USAP_CUDA(cudaEventRecord(sp.fork, sp.main));
    USAP_CUDA(cudaStreamWaitEvent(sp.side, sp.fork, 0));
  }
  if (has_hubs) {
    const size_t smem = sizeof(int) * 3 * static_cast<size_t>(hubs.smem_cap);
    k_nodal_propose_hub<Ops><<<hubs.hi - hubs.lo, kHubThreads, smem, sp.side>>>(a, ops, hubs.ids, hubs.lo,
                                                                                hubs.hi, hubs.smem_cap);
    USAP_LAUNCHED();
  }
  int blocks = (count + kWarps - 1) / kWarps;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_nodal_propose<Ops><<<blocks, kThreads, 0, sp.main>>>(a, ops);
  USAP_LAUNCHED();
  if (fork) {
    USAP_CUDA(cudaEventRecord(sp.join, sp.side));
    USAP_CUDA(cudaStreamWaitEvent(sp.main, sp.join, 0));
  }
}

}  // namespace

namespace {
int g_phase_grid[64];
int g_gang_grid[64];
}

// dynamic shared memory limits, set once per device, and the grid of the
// persistent kernel (CTAs per SM that fit x SMs; 0 if the device cannot
// run it cooperatively)
void nodal_configure(int device) {
  static std::once_flag once[64];
  if (device < 0 || device >= 64) return;
  std::call_once(once[device], [device] {
    const int smem = static_cast<int>(sizeof(int) * 3 * kHubSmemSlots);
    const int psmem = static_cast<int>(kPSmemBytes);
    int coop = 0, sms = 0;
    USAP_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
    USAP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    // one grid for every precision mode: the fewest co-resident CTAs
    int per_phase = 1 << 30, per_gang = 1 << 30;
    auto configure = [&](auto tag) {
      constexpr int P = decltype(tag)::value;
      USAP_CUDA(cudaFuncSetAttribute(k_nodal_propose_hub<DenseOpsT<LdNC, P>>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      USAP_CUDA(cudaFuncSetAttribute(k_nodal_propose_hub<SortedOpsT<P>>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      USAP_CUDA(cudaFuncSetAttribute(k_nodal_phase<P, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, psmem));
      USAP_CUDA(cudaFuncSetAttribute(k_nodal_phase<P, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, psmem));
      USAP_CUDA(cudaFuncSetAttribute(k_nodal_gang<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, psmem));
      int a = 0, a2 = 0, b = 0;
      USAP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_nodal_phase<P, false>, kPThreads, kPSmemBytes));
      USAP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a2, k_nodal_phase<P, true>, kPThreads, kPSmemBytes));
      USAP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_nodal_gang<P>, kPThreads, kPSmemBytes));
      per_phase = std::min(per_phase, std::min(a, a2));
      per_gang = std::min(per_gang, b);
    };
    configure(std::integral_constant<int, 0>{});
    configure(std::integral_constant<int, 1>{});
    configure(std::integral_constant<int, 2>{});
    configure(std::integral_constant<int, 3>{});
    g_phase_grid[device] = coop ? per_phase * sms : 0;
    g_gang_grid[device] = coop ? per_gang * sms : 0;
  });
}

int nodal_phase_grid(int device) {
  if (device < 0 || device >= 64) return 0;
  nodal_configure(device);
  return g_phase_grid[device];
}

int nodal_gang_grid(int device) {
  if (device < 0 || device >= 64) return 0;
  nodal_configure(device);
  return g_gang_grid[device];
}

// the apply pass keys a tile cell as x * ld + y in 31 bits
int nodal_phase_max_blocks() { return 32768; }

// the cooperative kernels of precision mode `prec` (0, 1, 2, 3)
static const void* gang_kernel(int prec) {
  if (prec == 1) return reinterpret_cast<const void*>(k_nodal_gang<1>);
  if (prec == 2) return reinterpret_cast<const void*>(k_nodal_gang<2>);
  if (prec == 3) return reinterpret_cast<const void*>(k_nodal_gang<3>);
  return reinterpret_cast<const void*>(k_nodal_gang<0>);
}

// snap: the variant that copies the tile into shared memory (B <= kSnapMaxB)
static const void* phase_kernel(int prec, bool snap) {
  if (snap) {
    if (prec == 1) return reinterpret_cast<const void*>(k_nodal_phase<1, true>);
    if (prec == 2) return reinterpret_cast<const void*>(k_nodal_phase<2, true>);
    if (prec == 3) return reinterpret_cast<const void*>(k_nodal_phase<3, true>);
    return reinterpret_cast<const void*>(k_nodal_phase<0, true>);
  }
  if (prec == 1) return reinterpret_cast<const void*>(k_nodal_phase<1, false>);
  if (prec == 2) return reinterpret_cast<const void*>(k_nodal_phase<2, false>);
  if (prec == 3) return reinterpret_cast<const void*>(k_nodal_phase<3, false>);
  return reinterpret_cast<const void*>(k_nodal_phase<0, false>);
}

void launch_nodal_gang(const PhaseArgs* jobs_dev, int K, GangCtl* gc, int exit_below, int grid, int prec,
                       cudaStream_t st) {
  const PhaseArgs* j = jobs_dev;
  int k = K;
  GangCtl* c = gc;
  int e = exit_below;
  void* kargs[] = {&j, &k, &c, &e};
  const void* fn = gang_kernel(prec);
  USAP_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kPThreads), kargs, kPSmemBytes, st));
  USAP_LAUNCHED();
}

void launch_nodal_phase(const PhaseArgs& p, int grid, cudaStream_t st) {
  PhaseArgs args = p;
  void* kargs[] = {&args};
  const void* fn = phase_kernel(p.a.prec, p.a.B <= kSnapMaxB);
  USAP_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kPThreads), kargs, kPSmemBytes, st));
  USAP_LAUNCHED();
}

void launch_nodal_propose_dense(const NodalArgs& a, DenseView v, const HubList& hubs,
                                const StreamPair& sp) {
  if (a.prec == 1) launch_propose(a, DenseOpsT<LdNC, 1>{v, a.B}, hubs, sp);
  else if (a.prec == 2) launch_propose(a, DenseOpsT<LdNC, 2>{v, a.B}, hubs, sp);
  else if (a.prec == 3) launch_propose(a, DenseOpsT<LdNC, 3>{v, a.B}, hubs, sp);
  else launch_propose(a, DenseOps{v, a.B}, hubs, sp);
}

void launch_nodal_propose_sorted(const NodalArgs& a, SortedView v, const HubList& hubs,
                                 const StreamPair& sp) {
  if (a.prec == 1) launch_propose(a, SortedOpsT<1>{v, a.B}, hubs, sp);
  else if (a.prec == 2) launch_propose(a, SortedOpsT<2>{v, a.B}, hubs, sp);
  else if (a.prec == 3) launch_propose(a, SortedOpsT<3>{v, a.B}, hubs, sp);
  else launch_propose(a, SortedOps{v, a.B}, hubs, sp);
}

void launch_merge_propose_dense(DenseView v, const MergeArgs& a, cudaStream_t st) {
  long long items = static_cast<long long>(a.B) * a.K;
  long long blocks = (items + kWarps - 1) / kWarps;
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  if (a.prec == 1) k_merge_propose_dense<1><<<static_cast<int>(blocks), kThreads, 0, st>>>(v, a);
  else if (a.prec == 2) k_merge_propose_dense<2><<<static_cast<int>(blocks), kThreads, 0, st>>>(v, a);
  else k_merge_propose_dense<0><<<static_cast<int>(blocks), kThreads, 0, st>>>(v, a);
  USAP_LAUNCHED();
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

void launch_nodal_apply_commit_dense(const GraphDev& g, int32_t* part, const int32_t* move_to,
                                     const int32_t* from, int beg, int end, int64_t c0, int64_t c1,
                                     int ld, int* M, int* Mt, int cld, int* CS, int32_t* dout,
                                     int32_t* din, NodalCtl* ctl, const CtlArgs& c, cudaStream_t st) {
  const int64_t items = c1 - c0;
  if (items <= 0) return;
  int64_t blocks = (items + kWarps - 1) / kWarps;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_nodal_apply_commit<<<static_cast<int>(blocks), kThreads, 0, st>>>(g, c0, c1, part, move_to, from, beg, end, ld,
                                                                      M, Mt, cld, CS, dout, din, ctl, c);
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

void launch_ctl_sweep_start(NodalCtl* ctl, int W, const long long* ide_q,
                            const int* ide_n, cudaStream_t st) {
  k_ctl_sweep_start<<<1, 1, 0, st>>>(ctl, W, ide_q, ide_n);
  USAP_LAUNCHED();
}


}  // namespace usap
