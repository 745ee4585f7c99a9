// usap_entropy_static: the description length of a partition computed in a
// fixed, file-scope device scratch array, with no allocation of any kind.
//
// Some callers cannot allocate when they need the score: a host framework
// whose own allocator has already reserved the device memory it may use
// (a cudaMalloc of ours would fail or push it past its budget), and a
// latency-sensitive loop that cannot take the device-wide synchronisation
// that cudaMalloc/cudaFree imply.  For them this entry point reads
// device-resident edges and block ids and writes the Q32 value to a device
// pointer, in the caller's stream order, using only the array below.
//
// The score is the one usap_op_entropy returns (model term of
// _compute_overall_entropy, graph_parallel.hpp:1314-1316, minus the data term
// summed over the dense block matrix, :1297-1312), term for term: the same
// glibc log table, the same rounding of each term and an order-independent
// int64 sum, so the two agree exactly.
#include <cstdint>
#include <cmath>
#include <climits>
#include <mutex>

#include "../../include/usap.h"
#include "common.cuh"
#include "engine.h"
#include "job.h"

namespace usap {
namespace {

constexpr int kStaticMaxBlocks = USAP_STATIC_MAX_BLOCKS;
constexpr int64_t kStaticMaxWeight = USAP_STATIC_MAX_WEIGHT;
constexpr int kStaticMaxDevices = 64;
constexpr int kThreads = 256;

constexpr size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// regions of the scratch array
constexpr size_t kLogOff = 0;                                                // L[0..W]
constexpr size_t kMOff = align256(kLogOff + sizeof(double) * (kStaticMaxWeight + 1));
constexpr size_t kDoutOff = align256(kMOff + sizeof(int32_t) * kStaticMaxBlocks * kStaticMaxBlocks);
constexpr size_t kDinOff = align256(kDoutOff + sizeof(int32_t) * kStaticMaxBlocks);
constexpr size_t kCtrOff = align256(kDinOff + sizeof(int32_t) * kStaticMaxBlocks);

struct StaticCounters {
  unsigned long long acc;    // data term, Q32, two's complement
  unsigned long long wsum;   // total edge weight seen
  int bad;                   // an input failed a device-side check
};

constexpr size_t kScratchBytes = align256(kCtrOff + sizeof(StaticCounters));

// One array per device, shared by every call on that device.  The log table
// at its head is written once at set-up; the rest is cleared by each call.
static __device__ __align__(256) unsigned char g_static_scratch[kScratchBytes];

struct StaticView {
  const double* L;
  int32_t* M;        // B x B, row stride B
  int32_t* dout;
  int32_t* din;
  StaticCounters* ctr;
};

StaticView view_of(unsigned char* base) {
  return StaticView{reinterpret_cast<const double*>(base + kLogOff),
                    reinterpret_cast<int32_t*>(base + kMOff),
                    reinterpret_cast<int32_t*>(base + kDoutOff),
                    reinterpret_cast<int32_t*>(base + kDinOff),
                    reinterpret_cast<StaticCounters*>(base + kCtrOff)};
}

__global__ void k_static_clear(StaticView v, int B) {
  const int64_t cells = static_cast<int64_t>(B) * B;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += stride) {
    v.M[c] = 0;
    if (c < B) {
      v.dout[c] = 0;
      v.din[c] = 0;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    v.ctr->acc = 0;
    v.ctr->wsum = 0;
    v.ctr->bad = 0;
  }
}

// block matrix and degrees from the edge list; ids outside [0, n) or
// [0, B) and negative weights are recorded, not followed
__global__ void k_static_build(StaticView v, const int32_t* __restrict__ src,
                               const int32_t* __restrict__ dst, const int32_t* __restrict__ w,
                               int64_t e, int32_t n, const int32_t* __restrict__ part, int B) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  long long wt = 0;
  bool bad = false;
  if (i < e) {
    const int32_t a = __ldg(src + i), b = __ldg(dst + i);
    wt = w ? __ldg(w + i) : 1;
    if (a < 0 || a >= n || b < 0 || b >= n || wt < 0) {
      bad = true;
    } else {
      const int32_t r = __ldg(part + a), s = __ldg(part + b);
      if (r < 0 || r >= B || s < 0 || s >= B) {
        bad = true;
      } else if (wt > 0) {
        atomicAdd(v.M + static_cast<int64_t>(r) * B + s, static_cast<int32_t>(wt));
        atomicAdd(v.dout + r, static_cast<int32_t>(wt));
        atomicAdd(v.din + s, static_cast<int32_t>(wt));
      }
    }
    if (bad) wt = 0;
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&v.ctr->bad, 1);
  wt = warp_sum_ll(wt);
  if ((threadIdx.x & 31) == 0 && wt) atomicAdd(&v.ctr->wsum, static_cast<unsigned long long>(wt));
}

// data term over the B x B cells; a count or degree outside the log table
// is recorded instead of read
__global__ void k_static_entropy(StaticView v, int B) {
  long long part = 0;
  bool bad = false;
  const int64_t cells = static_cast<int64_t>(B) * B;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += stride) {
    const int m = v.M[c];
    if (!m) continue;
    const int i = static_cast<int>(c / B), j = static_cast<int>(c - static_cast<int64_t>(i) * B);
    const int di = v.din[j], dr = v.dout[i];
    if (m < 0 || m > kStaticMaxWeight || di <= 0 || di > kStaticMaxWeight || dr <= 0 ||
        dr > kStaticMaxWeight) {
      bad = true;
      continue;
    }
    part += q32(g_term(v.L, m, di, dr));
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&v.ctr->bad, 1);
  part = warp_sum_ll(part);
  if ((threadIdx.x & 31) == 0 && part) atomicAdd(&v.ctr->acc, static_cast<unsigned long long>(part));
}

__global__ void k_static_finish(StaticView v, long long model_q, int64_t* S_q) {
  const StaticCounters c = *v.ctr;
  const bool bad = c.bad || c.wsum > static_cast<unsigned long long>(kStaticMaxWeight);
  // model term (saturated on the host) plus data term, saturated
  const long long b = -static_cast<long long>(c.acc);
  long long r = static_cast<long long>(static_cast<unsigned long long>(model_q) + static_cast<unsigned long long>(b));
  if ((model_q > 0 && b > 0 && r < 0) || (model_q < 0 && b < 0 && r >= 0)) r = model_q > 0 ? LLONG_MAX : LLONG_MIN;
  *S_q = bad ? static_cast<int64_t>(LLONG_MIN) : r;
}

int grid_of(int64_t work) {
  const int64_t g = (work + kThreads - 1) / kThreads;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(g, 148 * 16)));
}

std::mutex g_setup_mu;
unsigned char* g_scratch_ptr[kStaticMaxDevices] = {};

// Once per device, with that device current: the address of the array and
// the log table in its first region.  Copies go through a stack buffer.
unsigned char* scratch_for(int dev) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (g_scratch_ptr[dev]) return g_scratch_ptr[dev];
  void* ptr = nullptr;
  USAP_CUDA(cudaGetSymbolAddress(&ptr, g_static_scratch));
  unsigned char* base = static_cast<unsigned char*>(ptr);
  constexpr int64_t kChunk = 4096;
  double buf[kChunk];
  for (int64_t k0 = 0; k0 <= kStaticMaxWeight; k0 += kChunk) {
    const int64_t k1 = std::min<int64_t>(kStaticMaxWeight + 1, k0 + kChunk);
    for (int64_t k = k0; k < k1; k++) buf[k - k0] = k == 0 ? -INFINITY : std::log(static_cast<double>(k));
    USAP_CUDA(cudaMemcpy(base + kLogOff + sizeof(double) * k0, buf, sizeof(double) * (k1 - k0),
                         cudaMemcpyHostToDevice));
  }
  // a copy from pageable memory may return before it lands; the first call's
  // kernels can run on a non-blocking stream, so wait for the table here
  USAP_CUDA(cudaDeviceSynchronize());
  g_scratch_ptr[dev] = base;
  return base;
}

void entropy_static(const int32_t* src, const int32_t* dst, const int32_t* weight, int64_t e,
                    int32_t n, const int32_t* part, int32_t B, int64_t* S_q, cudaStream_t st) {
  if (!src || !dst || !part || !S_q) throw Error(USAP_ERR_INVALID, "null device pointer");
  if (n < 1 || e < 1) throw Error(USAP_ERR_INVALID, "need n >= 1 and e >= 1");
  if (B < 1) throw Error(USAP_ERR_INVALID, "need B >= 1");
  if (B > kStaticMaxBlocks)
    throw Error(USAP_ERR_LIMIT, "B = " + std::to_string(B) + " exceeds the static scratch limit of " +
                                    std::to_string(kStaticMaxBlocks) + " blocks");
  if (e > kStaticMaxWeight)
    throw Error(USAP_ERR_LIMIT, "e = " + std::to_string(e) + " exceeds the static scratch limit of " +
                                    std::to_string(kStaticMaxWeight) + " edges");
  int dev = -1;
  USAP_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kStaticMaxDevices) throw Error(USAP_ERR_INVALID, "device index out of range");
  int major = 0;
  USAP_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  if (major != 10) throw Error(USAP_ERR_NO_DEVICE, "current device is not sm_100 class");
  const StaticView v = view_of(scratch_for(dev));
  const long long model_q = q32_host(model_S(n, e, B));
  const int64_t cells = static_cast<int64_t>(B) * B;
  k_static_clear<<<grid_of(cells), kThreads, 0, st>>>(v, B);
  USAP_LAUNCHED();
  k_static_build<<<static_cast<unsigned>((e + kThreads - 1) / kThreads), kThreads, 0, st>>>(
      v, src, dst, weight, e, n, part, B);
  USAP_LAUNCHED();
  k_static_entropy<<<grid_of(cells), kThreads, 0, st>>>(v, B);
  USAP_LAUNCHED();
  k_static_finish<<<1, 1, 0, st>>>(v, model_q, S_q);
  USAP_LAUNCHED();
}

}  // namespace
}  // namespace usap

extern "C" usap_status usap_entropy_static(const int32_t* src, const int32_t* dst,
                                           const int32_t* weight, int64_t e, int32_t n,
                                           const int32_t* part, int32_t B, int64_t* S_q,
                                           void* stream) {
  return usap::call_guarded([&] {
    usap::entropy_static(src, dst, weight, e, n, part, B, S_q, static_cast<cudaStream_t>(stream));
  });
}
