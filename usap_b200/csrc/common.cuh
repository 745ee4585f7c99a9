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

// statistics of precision modes 1 and 2 (FP32 dS beside the exact FP64 value):
// evaluations, decisions whose sign differs, the largest and the summed
// |dS_fp32 - dS_fp64|
struct F32Tally {
  unsigned long long evals, flips, err_max;   // err_max: bits of a non-negative double
  double err_sum;
};

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

// --- FP32 evaluation of the same terms (precision modes 1 and 2) --------
// Only single-precision operations, each rounded to nearest as written.
// Values are float pairs (hi, lo) worth hi + lo, |lo| <= ulp(hi) / 2.  The
// log table is held as such pairs too: hi = log k rounded to float, lo = the
// remainder rounded to float.
//  * mode 1: every term in pair arithmetic (Dekker / Knuth error-free
//    transformations: TwoSum, and TwoProduct by fused multiply-add), about
//    44 significant bits;
//  * mode 2: every term in plain float from the hi parts; only the sum is
//    compensated.
// Terms are accumulated in pairs in both modes.
struct FF {
  float hi, lo;
};

// a + b = s + e exactly (TwoSum; needs no ordering of a, b)
__device__ __forceinline__ FF two_sum(float a, float b) {
  const float s = __fadd_rn(a, b);
  const float z = __fsub_rn(s, a);
  return FF{s, __fadd_rn(__fsub_rn(a, __fsub_rn(s, z)), __fsub_rn(b, z))};
}

// pair sum; the result does not depend on the operands' order, so every
// lane of a butterfly reduction ends with the same value
__device__ __forceinline__ FF ff_add(FF a, FF b) {
  const FF s = two_sum(a.hi, b.hi);
  return two_sum(s.hi, __fadd_rn(s.lo, __fadd_rn(a.lo, b.lo)));
}

__device__ __forceinline__ FF ff_neg(FF a) { return FF{-a.hi, -a.lo}; }
__device__ __forceinline__ FF ff_sub(FF a, FF b) { return ff_add(a, ff_neg(b)); }

// the integer x (|x| < 2^48) times a pair: x = xh + xl in floats, xh * d.hi
// split exactly by a fused multiply-add, the cross terms added to the error
__device__ __forceinline__ FF ff_mul_ll(FF d, long long x) {
  const float xh = __ll2float_rn(x);
  const float xl = __ll2float_rn(x - __float2ll_rn(xh));
  const float p = __fmul_rn(xh, d.hi);
  float e = __fmaf_rn(xh, d.hi, -p);
  e = __fadd_rn(e, __fadd_rn(__fmul_rn(xh, d.lo), __fmul_rn(xl, d.hi)));
  return two_sum(p, e);
}

// the exact value hi + lo (at most 48 significant bits, so exact in FP64)
__device__ __forceinline__ double ff_value(FF a) {
  return __dadd_rn(static_cast<double>(a.hi), static_cast<double>(a.lo));
}

__device__ __forceinline__ FF ld_ff(const float2* __restrict__ T, long long k) {
  const float2 v = __ldg(T + k);
  return FF{v.x, v.y};
}

// x * ((L[x] - L[d1]) - L[d2]) from loaded table pairs
template <int P>
__device__ __forceinline__ FF g_ff(long long x, FF Lx, FF L1, FF L2) {
  if (x == 0) return FF{0.0f, 0.0f};
  if constexpr (P == 1) return ff_mul_ll(ff_sub(ff_sub(Lx, L1), L2), x);
  return FF{__fmul_rn(__ll2float_rn(x), __fsub_rn(__fsub_rn(Lx.hi, L1.hi), L2.hi)), 0.0f};
}

template <int P>
__device__ __forceinline__ FF g_term_ff(const float2* __restrict__ T, long long x, long long din_arg,
                                        long long dout_arg) {
  if (x == 0) return FF{0.0f, 0.0f};
  return g_ff<P>(x, ld_ff(T, x), ld_ff(T, din_arg), ld_ff(T, dout_arg));
}

// n * (L[a_new] - L[a_old])
template <int P>
__device__ __forceinline__ FF coef_ff(long long n, FF Lnew, FF Lold) {
  if (n == 0) return FF{0.0f, 0.0f};
  if constexpr (P == 1) return ff_mul_ll(ff_sub(Lnew, Lold), n);
  return FF{__fmul_rn(__ll2float_rn(n), __fsub_rn(Lnew.hi, Lold.hi)), 0.0f};
}

// x L[x] + y L[y] - (x+y) L[x+y]
template <int P>
__device__ __forceinline__ FF h_term_ff(const float2* __restrict__ T, long long x, long long y) {
  const FF Lx = ld_ff(T, x), Ly = ld_ff(T, y), Lxy = ld_ff(T, x + y);
  if constexpr (P == 1) return ff_sub(ff_add(ff_mul_ll(Lx, x), ff_mul_ll(Ly, y)), ff_mul_ll(Lxy, x + y));
  const float a = __fmul_rn(__ll2float_rn(x), Lx.hi);
  const float b = __fmul_rn(__ll2float_rn(y), Ly.hi);
  const float c = __fmul_rn(__ll2float_rn(x + y), Lxy.hi);
  return FF{__fsub_rn(__fadd_rn(a, b), c), 0.0f};
}

// --- precision mode 3: the reference's own float arithmetic --------------
// The float-pair terms above exist for modes 1 and 2; mode 3 reproduces the
// reference's single-precision dS instead.
template <int P>
constexpr bool kPairTerms = (P == 1 || P == 2);

// log(x) rounded to float, evaluated in double with IEEE +, -, * and fused
// multiply-add only, in the same steps as the oracle's og_log_f32, so host
// and device agree bit for bit.  x = m * 2^e with m in [sqrt(1/2), sqrt(2));
// k = 128 (m - 1) rounded half up picks r_k = round(1024 / (1 + k/128)) / 1024 and
// L_k = -log(r_k) from ref_log_table.inc (written by ref_log_table.py);
// u = m r_k - 1 is exact (|u| < 0.0066) and
//   log x = e ln 2 + L_k + log1p(u),  log1p(u) = u - u^2/2 + ... - u^8/8
// (the next term is below 3e-21).  The double result is within a few units
// of 1e-16 of log x, so it rounds to the correctly rounded float except
// when log x lies that close to a rounding boundary.
static __device__ const double2 kRefLogTab[] = {
#include "ref_log_table.inc"
};
constexpr int kRefLogK0 = 38;   // table index of k = 0

__device__ __forceinline__ float ref_logf(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? __int_as_float(0xff800000) : __int_as_float(0x7fc00000);
  const unsigned u = __float_as_uint(x);
  if (u >= 0x7f800000u) return x;   // +inf
  int e = static_cast<int>(u >> 23);
  unsigned frac = u & 0x7fffffu;
  if (e == 0) {   // subnormal: shift the leading one into the hidden bit
    const int sh = __clz(static_cast<int>(frac)) - 8;
    frac = (frac << sh) & 0x7fffffu;
    e = 1 - sh;
  }
  e -= 127;
  // m = 1 + frac / 2^23, halved above sqrt(2) (frac >= 0x3504F4); k from the
  // bits: round(frac / 2^16), or round(frac / 2^17) - 64 after halving
  unsigned long long mbits;
  int k;
  if (frac >= 0x3504F4u) {
    e += 1;
    mbits = (1022ull << 52) | (static_cast<unsigned long long>(frac) << 29);
    k = static_cast<int>((frac + 0x10000u) >> 17) - 64;
  } else {
    mbits = (1023ull << 52) | (static_cast<unsigned long long>(frac) << 29);
    k = static_cast<int>((frac + 0x8000u) >> 16);
  }
  const double m = __longlong_as_double(static_cast<long long>(mbits));
  const double2 t = __ldg(kRefLogTab + kRefLogK0 + k);
  const double w = __dsub_rn(__dmul_rn(m, t.x), 1.0);
  double q = -1.0 / 8.0;
  q = __fma_rn(q, w, 1.0 / 7.0);
  q = __fma_rn(q, w, -1.0 / 6.0);
  q = __fma_rn(q, w, 1.0 / 5.0);
  q = __fma_rn(q, w, -1.0 / 4.0);
  q = __fma_rn(q, w, 1.0 / 3.0);
  q = __fma_rn(q, w, -1.0 / 2.0);
  const double l1p = __fma_rn(__dmul_rn(w, w), q, w);
  // e as a double without a conversion instruction: 2^52 + 2^51 + e, minus the offset
  const double ed = __dsub_rn(__longlong_as_double(0x4338000000000000ll + e), 6755399441055744.0);
  const double hi = __fma_rn(ed, 0.69314718055994530942, t.y);
  return __double2float_rn(__dadd_rn(hi, l1p));
}

// ref_logf for x > 0 (+inf included) without branches: the same operations
// on the same values, the special cases chosen by selects, so that several
// evaluations can be interleaved by the compiler.
__device__ __forceinline__ float ref_logf_pos(float x) {
  const unsigned u = __float_as_uint(x);
  int e = static_cast<int>(u >> 23);
  unsigned frac = u & 0x7fffffu;
  const bool sub = e == 0;   // subnormal: shift the leading one into the hidden bit
  const int sh = sub ? __clz(static_cast<int>(frac)) - 8 : 0;
  frac = (frac << sh) & 0x7fffffu;
  e = (sub ? 1 - sh : e) - 127;
  const bool half = frac >= 0x3504F4u;
  e += half ? 1 : 0;
  const unsigned long long mbits = ((half ? 1022ull : 1023ull) << 52) | (static_cast<unsigned long long>(frac) << 29);
  const int k = half ? static_cast<int>((frac + 0x10000u) >> 17) - 64 : static_cast<int>((frac + 0x8000u) >> 16);
  const double m = __longlong_as_double(static_cast<long long>(mbits));
  const double2 t = __ldg(kRefLogTab + kRefLogK0 + (u >= 0x7f800000u ? 0 : k));
  const double w = __dsub_rn(__dmul_rn(m, t.x), 1.0);
  double q = -1.0 / 8.0;
  q = __fma_rn(q, w, 1.0 / 7.0);
  q = __fma_rn(q, w, -1.0 / 6.0);
  q = __fma_rn(q, w, 1.0 / 5.0);
  q = __fma_rn(q, w, -1.0 / 4.0);
  q = __fma_rn(q, w, 1.0 / 3.0);
  q = __fma_rn(q, w, -1.0 / 2.0);
  const double l1p = __fma_rn(__dmul_rn(w, w), q, w);
  const double ed = __dsub_rn(__longlong_as_double(0x4338000000000000ll + e), 6755399441055744.0);
  const double hi = __fma_rn(ed, 0.69314718055994530942, t.y);
  const float r = __double2float_rn(__dadd_rn(hi, l1p));
  return u >= 0x7f800000u ? x : r;   // +inf
}

// ref_term(x, prod) where x != 0, else 0, without branches (x, prod >= 0)
__device__ __forceinline__ float ref_term_nz(int x, long long prod) {
  const float xf = __int2float_rn(x ? x : 1);
  const float t = __fmul_rn(xf, ref_logf_pos(__fdiv_rn(xf, __ll2float_rn(x ? prod : 1))));
  return x ? t : 0.0f;
}

// one term of the reference's dS: count * log((float)count / (float)prod),
// the long product converted to float, a float division, a float product
__device__ __forceinline__ float ref_term(int x, long long prod) {
  const float xf = __int2float_rn(x);
  return __fmul_rn(xf, ref_logf(__fdiv_rn(xf, __ll2float_rn(prod))));
}

// |dS_fp32 - dS_fp64| of one evaluation; f is the FP32 pair's value, the
// FP64 value is the exact sum acc / 2^32
__device__ __forceinline__ double f32_err(double f, long long acc) {
  return fabs(__dsub_rn(f, __dmul_rn(static_cast<double>(acc), 1.0 / kQ32)));
}

__device__ __forceinline__ void f32_tally(F32Tally* t, double f, long long acc) {
  const double err = f32_err(f, acc);
  atomicAdd(&t->evals, 1ull);
  if ((acc < 0) != (f < 0.0)) atomicAdd(&t->flips, 1ull);
  atomicMax(&t->err_max, static_cast<unsigned long long>(__double_as_longlong(err)));
  atomicAdd(&t->err_sum, err);
}

__device__ __forceinline__ void f32_tally_flush(const F32Tally* t, F32Tally* dst) {
  if (!t->evals) return;
  atomicAdd(&dst->evals, t->evals);
  if (t->flips) atomicAdd(&dst->flips, t->flips);
  atomicMax(&dst->err_max, t->err_max);
  atomicAdd(&dst->err_sum, t->err_sum);
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
