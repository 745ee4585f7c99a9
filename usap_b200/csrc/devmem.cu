// Device memory and host tables shared by all jobs of the process.
//
// Device buffers come from the device's stream-ordered memory pool with its
// release threshold raised, so memory freed by one job stays reserved and
// the next job's allocations (a one-shot usap_partition call creates and
// destroys a job) are served from the pool instead of the driver.
// The FP64 log table log(k) is computed once per process on the host (glibc
// log, the values both the GPU path and the oracle read) and grown on demand.
#include <algorithm>
#include <cmath>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/usap.h"
#include "engine.h"

namespace usap {

namespace {
constexpr int kMaxDevices = 64;
std::once_flag g_pool_once[kMaxDevices];
std::mutex g_log_mu;
std::shared_ptr<const std::vector<double>> g_log;
}  // namespace

void pool_configure(int device) {
  if (device < 0 || device >= kMaxDevices) return;
  std::call_once(g_pool_once[device], [device] {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) return;
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  });
}

void pool_reserve(int device, int64_t bytes) {
  if (bytes <= 0) return;
  pool_configure(device);
  size_t free_b = 0, total_b = 0;
  USAP_CUDA(cudaMemGetInfo(&free_b, &total_b));
  bytes = std::min<int64_t>(bytes, static_cast<int64_t>(0.5 * static_cast<double>(free_b)));
  cudaStream_t st = nullptr;
  USAP_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  void* p = nullptr;
  if (cudaMallocAsync(&p, static_cast<size_t>(bytes), st) == cudaSuccess) cudaFreeAsync(p, st);
  cudaGetLastError();   // a reservation that does not fit is not an error
  USAP_CUDA(cudaStreamSynchronize(st));
  USAP_CUDA(cudaStreamDestroy(st));
}

void* dev_alloc(size_t bytes, cudaStream_t st) {
  void* p = nullptr;
  USAP_CUDA(cudaMallocAsync(&p, bytes ? bytes : 16, st));
  return p;
}

void dev_free(void* p, cudaStream_t st) {
  if (p) cudaFreeAsync(p, st);
}

DeviceLogTable::~DeviceLogTable() {
  if (L) cudaFree(L);
  if (L2) cudaFree(L2);
}

namespace {
std::mutex g_dlog_mu[kMaxDevices];
std::shared_ptr<const DeviceLogTable> g_dlog[kMaxDevices];
}  // namespace

std::shared_ptr<const DeviceLogTable> device_log_table(int device, int64_t max_k, int64_t* uploaded) {
  if (uploaded) *uploaded = 0;
  if (device < 0 || device >= kMaxDevices) throw Error(USAP_ERR_INVALID, "device index out of range");
  std::lock_guard<std::mutex> lk(g_dlog_mu[device]);
  std::shared_ptr<const DeviceLogTable>& cur = g_dlog[device];
  if (cur && cur->size > max_k) return cur;
  // grow geometrically so that a stream of slightly larger graphs uploads rarely
  const int64_t size = std::max<int64_t>(max_k + 1, cur ? 2 * cur->size : max_k + 1);
  const std::shared_ptr<const std::vector<double>> host = log_table(size - 1);
  auto t = std::make_shared<DeviceLogTable>();
  USAP_CUDA(cudaSetDevice(device));
  USAP_CUDA(cudaMalloc(reinterpret_cast<void**>(&t->L), sizeof(double) * size));
  USAP_CUDA(cudaMalloc(reinterpret_cast<void**>(&t->L2), sizeof(float2) * size));
  t->size = size;
  cudaStream_t st = nullptr;
  USAP_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  USAP_CUDA(cudaMemcpyAsync(t->L, host->data(), sizeof(double) * size, cudaMemcpyHostToDevice, st));
  launch_log_pairs(t->L, t->L2, size, st);
  USAP_CUDA(cudaStreamSynchronize(st));   // ready for every stream before anyone gets it
  USAP_CUDA(cudaStreamDestroy(st));
  if (uploaded) *uploaded = static_cast<int64_t>(sizeof(double) * size);
  cur = t;
  return cur;
}

std::shared_ptr<const std::vector<double>> log_table(int64_t max_k) {
  std::lock_guard<std::mutex> lk(g_log_mu);
  if (!g_log || static_cast<int64_t>(g_log->size()) <= max_k) {
    auto t = std::make_shared<std::vector<double>>();
    size_t old = g_log ? g_log->size() : 0;
    t->resize(static_cast<size_t>(max_k) + 1);
    if (old) std::copy(g_log->begin(), g_log->end(), t->begin());
    if (old == 0) {
      (*t)[0] = -INFINITY;
      old = 1;
    }
    for (size_t k = old; k < t->size(); k++) (*t)[k] = std::log(static_cast<double>(k));
    g_log = t;
  }
  return g_log;
}

}  // namespace usap
