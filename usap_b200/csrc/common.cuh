// Shared device/host arithmetic of the SBP path.
//
// The replay contract (identical on the CPU oracle and on the GPU):
//  * Philox4x32-10 draws keyed by the seed, counter (item, sub, stage, tag);
//  * integer inverse-CDF draws t = (u * total) >> 32;
//  * entropy terms x*log(x/(a*b)) in FP64 from a table of log(k) for
//    integers k, each rounded to a Q32 fixed-point integer, so that sums are
//    exact and the result does not depend on summation order (warp
//    reductions and atomics are free to reorder them).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace usap {

constexpr uint32_t kTagMerge = 0x4D455247u;  // 'MERG'
constexpr uint32_t kTagNodal = 0x4E4F4441u;  // 'NODA'
constexpr double kQ32 = 4294967296.0;
constexpr long long kNearQ = 4;              // |dS| <= 1e-9 in Q32 units

struct Draws {
  uint32_t x0, x1, x2, x3;
};

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
// easy as 1, 2, 3", SC'11).
__host__ __device__ __forceinline__ Draws philox(uint32_t c0, uint32_t c1, uint32_t c2,
                                                 uint32_t c3, uint64_t seed) {
  uint32_t k0 = static_cast<uint32_t>(seed), k1 = static_cast<uint32_t>(seed >> 32);
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
  for (int round = 0; round < 10; round++) {
    if (round) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
#ifdef __CUDA_ARCH__
    uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
    uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
    uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
    uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
    uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
#endif
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  return Draws{c0, c1, c2, c3};
}

__host__ __device__ __forceinline__ uint32_t draw_below(uint32_t u, long long n) {
  return static_cast<uint32_t>((static_cast<uint64_t>(u) * static_cast<uint64_t>(n)) >> 32);
}

// x <= B / (d_a[u] + B) with x = u / 2^32, exactly
__host__ __device__ __forceinline__ bool accept_uniform(uint32_t u, long long da, long long B) {
  return static_cast<uint64_t>(u) * static_cast<uint64_t>(da + B) <=
         (static_cast<uint64_t>(B) << 32);
}

// the uniform block draw of the merge proposal, r skipped
__host__ __device__ __forceinline__ int skip_r(int i, int r, int B) {
  if (i == r) i++;
  if (i == B) i = 0;
  return i;
}

#ifdef __CUDACC__
// --- FP64 entropy terms, rounded as written (no contraction) -------------
// g(x, din, dout) = x * ((L[x] - L[din]) - L[dout]) = x log(x / (din*dout))
__device__ __forceinline__ double g_term(const double* __restrict__ L, long long x,
                                         long long din_arg, long long dout_arg) {
  if (x == 0) return 0.0;
  double t = __dsub_rn(__dsub_rn(__ldg(L + x), __ldg(L + din_arg)), __ldg(L + dout_arg));
  return __dmul_rn(static_cast<double>(x), t);
}

// n * (L[a_new] - L[a_old]): entries a move leaves unchanged
__device__ __forceinline__ double coef_term(const double* __restrict__ L, long long n,
                                            long long a_new, long long a_old) {
  if (n == 0) return 0.0;
  return __dmul_rn(static_cast<double>(n), __dsub_rn(__ldg(L + a_new), __ldg(L + a_old)));
}

// h(x, y) = x L[x] + y L[y] - (x+y) L[x+y]: two rows merging
__device__ __forceinline__ double h_term(const double* __restrict__ L, long long x, long long y) {
  double a = __dmul_rn(static_cast<double>(x), __ldg(L + x));
  double b = __dmul_rn(static_cast<double>(y), __ldg(L + y));
  double c = __dmul_rn(static_cast<double>(x + y), __ldg(L + x + y));
  return __dsub_rn(__dadd_rn(a, b), c);
}

__device__ __forceinline__ long long q32(double t) {
  return __double2ll_rn(__dmul_rn(t, kQ32));
}

// --- warp helpers ------------------------------------------------------------
__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += n;
  }
  return v;
}

__device__ __forceinline__ long long warp_incl_scan_ll(long long v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    long long n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += n;
  }
  return v;
}

// first index j in [lo, hi) with a[j] > key (a non-decreasing), hi if none
__device__ __forceinline__ int upper_bound_i(const int* __restrict__ a, int lo, int hi, long long key) {
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (static_cast<long long>(__ldg(a + mid)) > key) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// position of key in sorted a[lo, hi), -1 if absent
__device__ __forceinline__ int find_sorted(const int* __restrict__ a, int lo, int hi, int key) {
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    int v = __ldg(a + mid);
    if (v == key) return mid;
    if (v < key) lo = mid + 1;
    else hi = mid;
  }
  return -1;
}
#endif

}  // namespace usap
