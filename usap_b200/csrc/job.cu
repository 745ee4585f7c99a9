// Host orchestration of one partitioning job (Graph_P::partition,
// graph_parallel.hpp:322-512): initial blocks, then stages of
// merge phase -> merge application -> batched nodal sweeps -> description
// length -> golden-section step, until the bracket closes.  All phases run
// on the device; the host keeps the golden-section bracket (three partition
// slots resident in HBM, swapped by index) and reads back one control block
// per sweep.
#include "job.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <cub/cub.cuh>

namespace usap {

// device buffers of a job come from the retained stream-ordered pool
template <class T>
void dalloc_on(T** p, size_t count, cudaStream_t st) {
  *p = static_cast<T*>(dev_alloc(sizeof(T) * (count > 0 ? count : 1), st));
}
template <class T>
void dfree_on(T*& p, cudaStream_t st) {
  dev_free(p, st);
  p = nullptr;
}
#define dalloc(pp, count) dalloc_on((pp), static_cast<size_t>(count), st_)
#define dfree(p) dfree_on((p), st_)

LaunchCount& launch_count() {
  static thread_local LaunchCount c;
  return c;
}

void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
  if (e == cudaSuccess) return;
  int code = (e == cudaErrorMemoryAllocation) ? USAP_ERR_OOM : USAP_ERR_CUDA;
  throw Error(code, std::string(what) + ": " + cudaGetErrorString(e) + " (" + file + ":" +
                        std::to_string(line) + ")");
}

namespace {


inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

int hash_lg(int deg) {
  int lg = 5;
  while ((1 << lg) < 2 * deg) lg++;
  return lg;
}

}  // namespace

int32_t reduce_blocks(int32_t B, float rate) {
  return static_cast<int32_t>(static_cast<float>(B) * rate);
}

double model_S(int64_t n, int64_t e, int32_t B) {
  double x = static_cast<double>(B) * static_cast<double>(B) / static_cast<double>(e);
  return static_cast<double>(e) * (1.0 + x) * std::log(1.0 + x) - x * std::log(x) +
         static_cast<double>(n) * std::log(static_cast<double>(B));
}

long long q32_host(double t) {
  const double x = t * 4294967296.0;
  if (x >= 9223372036854775807.0) return LLONG_MAX;
  if (x <= -9223372036854775807.0) return LLONG_MIN;
  return std::llrint(x);
}

long long add_sat(long long a, long long b) {
  long long r;
  if (__builtin_add_overflow(a, b, &r)) return a > 0 ? LLONG_MAX : LLONG_MIN;
  return r;
}

bool Golden::step(int32_t B, double S, int64_t S_q, int32_t cur_slot, float rate, int32_t* restore_slot,
                  int32_t* btm) {
  GoldenPoint cur{B, S, S_q, true, cur_slot};
  if (!med.finite || cur.S <= med.S) {
    if (med.B > cur.B) large = med;
    else small = med;
    med = cur;
  } else {
    if (med.B > cur.B) small = cur;
    else large = cur;
  }
  *restore_slot = -1;
  *btm = 0;
  if (!small.finite) {
    *restore_slot = med.slot;
    *btm = reduce_blocks(med.B, rate);
    return *btm == 0;
  }
  // the reference would continue from an empty default state when the
  // bracket has no upper end; the search stops at med
  if (!large.finite) return true;
  if (large.B - small.B == 2) return true;
  if ((large.B - med.B) >= (med.B - small.B)) {
    int32_t next_B = med.B + static_cast<int32_t>(std::round((large.B - med.B) * 0.618));
    *restore_slot = large.slot;
    *btm = large.B - next_B;
  } else {
    int32_t next_B = small.B + static_cast<int32_t>(std::round((med.B - small.B) * 0.618));
    *restore_slot = med.slot;
    *btm = med.B - next_B;
  }
  return false;
}

Job::Job(int device) : device_(device) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    throw Error(USAP_ERR_NO_DEVICE, "no CUDA device available");
  if (device < 0 || device >= count) throw Error(USAP_ERR_INVALID, "device index out of range");
  USAP_CUDA(cudaSetDevice(device));
  int major = 0;
  USAP_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
  if (major < 10) {
    cudaDeviceProp prop;
    USAP_CUDA(cudaGetDeviceProperties(&prop, device));
    throw Error(USAP_ERR_NO_DEVICE, std::string("device is not sm_100 class: ") + prop.name);
  }
  pool_configure(device);
  USAP_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
  USAP_CUDA(cudaStreamCreateWithFlags(&st_side_, cudaStreamNonBlocking));
  USAP_CUDA(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
  USAP_CUDA(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
  USAP_CUDA(cudaEventCreateWithFlags(&ev_wait_, cudaEventDisableTiming | cudaEventBlockingSync));
  nodal_configure(device);
  USAP_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h_ctl_), sizeof(NodalCtl)));
  USAP_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h_ring_), 2 * sizeof(NodalCtl)));
  for (auto& e : ev_sweep_) USAP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  dalloc(&ctl_, 1);
  dalloc(&f32d_, 2);
}

Job::~Job() {
  cudaSetDevice(device_);
  free_state();
  free_graph();
  dfree(ctl_);
  dfree(f32d_);
  if (st_) cudaStreamSynchronize(st_);
  if (h_ctl_) cudaFreeHost(h_ctl_);
  if (h_ring_) cudaFreeHost(h_ring_);
  for (auto e : ev_sweep_)
    if (e) cudaEventDestroy(e);
  for (auto e : ev_pool_) cudaEventDestroy(e);
  if (ev_fork_) cudaEventDestroy(ev_fork_);
  if (ev_join_) cudaEventDestroy(ev_join_);
  if (ev_wait_) cudaEventDestroy(ev_wait_);
  if (st_side_) cudaStreamDestroy(st_side_);
  if (st_) cudaStreamDestroy(st_);
}

// waits for the job's stream; with blocking waits the host thread sleeps
// instead of spinning, so many concurrent jobs can share the host cores
void Job::wait() {
  if (blocking_wait_) {
    USAP_CUDA(cudaEventRecord(ev_wait_, st_));
    USAP_CUDA(cudaEventSynchronize(ev_wait_));
  } else {
    USAP_CUDA(cudaStreamSynchronize(st_));
  }
}

void Job::free_graph() {
  dfree(hkey_); dfree(hwo_); dfree(hwi_);
  gr_.reset();
  hg_ = nullptr;
  g_ = GraphDev{};
}

void Job::free_vertex_state() {
  for (auto& s : slots_) dfree(s);
  dfree(move_to_); dfree(from_);
  dfree(rp_s_); dfree(rp_n_); dfree(rp_q_); dfree(rp_f_);
  ncap_ = 0;
}

void Job::free_state() {
  free_vertex_state();
  dfree(dout_); dfree(din_); dfree(batch_hub_); dfree(unit_ptr_); dfree(units_);
  batch_hub_bs_ = 0;
  batch_hub_cap_ = 0;
  units_cap_ = 0;
  dfree(M_); dfree(Mt_); dfree(CS_);
  dfree(Trow_); dfree(Tcol_);
  tcap_ = 0;
  sb_.release(st_);
  dfree(prop_s_); dfree(prop_q_); dfree(prop_x_); dfree(prop_f_); dfree(best_s_); dfree(best_q_); dfree(best_x_);
  dfree(skeys_); dfree(skeys_alt_); dfree(sidx_); dfree(sidx_alt_);
  dfree(union_work_); dfree(root_); dfree(present_); dfree(newlabel_); dfree(merged_dev_);
  dfree(cub_tmp_);
  cub_bytes_ = 0;
  dfree(ide_q_); dfree(ide_n_);
  bcap_ = kcap_ = dcap_ = icap_ = 0;
}

// --- graph load -----------------------------------------------------------------
std::shared_ptr<GraphResident> load_graph(int device, const usap_graph& in, HostGraph* pre) {
  USAP_CUDA(cudaSetDevice(device));
  HostGraph h;
  int64_t wtot = 0;
  if (pre) {
    h = std::move(*pre);
    wtot = h.wtot;
  } else {
  if (in.e <= 0 || !in.src || !in.dst) throw Error(USAP_ERR_INVALID, "graph needs at least one edge");
  if (in.e >= (1ll << 30)) throw Error(USAP_ERR_LIMIT, "more than 2^30 edges");
  h.e = in.e;
  const int32_t base = in.one_based ? 1 : 0;
  h.src.resize(in.e);
  h.dst.resize(in.e);
  int64_t maxsrc = -1, maxid = -1;
  {
    // converted and checked in slices on host threads
    const int T = in.e < (1 << 17) ? 1 : std::max(1, std::min<int>(16, static_cast<int>(std::thread::hardware_concurrency())));
    std::vector<int64_t> ms(T, -1), mi(T, -1), bad(T, -1);
    auto work = [&](int t) {
      const int64_t i0 = in.e * t / T, i1 = in.e * (t + 1) / T;
      int64_t lms = -1, lmi = -1;
      for (int64_t i = i0; i < i1; i++) {
        const int64_t a = static_cast<int64_t>(in.src[i]) - base, b = static_cast<int64_t>(in.dst[i]) - base;
        if ((a < 0 || b < 0) && bad[t] < 0) bad[t] = i;
        lms = std::max(lms, a);
        lmi = std::max(lmi, std::max(a, b));
        h.src[i] = static_cast<int32_t>(a);
        h.dst[i] = static_cast<int32_t>(b);
      }
      ms[t] = lms;
      mi[t] = lmi;
    };
    std::vector<std::thread> th;
    for (int t = 1; t < T; t++) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
    for (int t = 0; t < T; t++) {
      if (bad[t] >= 0) throw Error(USAP_ERR_INVALID, "negative vertex id at edge " + std::to_string(bad[t]));
      maxsrc = std::max(maxsrc, ms[t]);
      maxid = std::max(maxid, mi[t]);
    }
  }
  h.n = in.n > 0 ? in.n : static_cast<int32_t>(maxsrc + 1);
  if (maxid >= h.n)
    throw Error(USAP_ERR_INVALID, "vertex id " + std::to_string(maxid) + " >= n = " + std::to_string(h.n));
  h.unit = true;
  if (in.weight) {
    h.w.resize(in.e);
    for (int64_t i = 0; i < in.e; i++) {
      if (in.weight[i] <= 0) throw Error(USAP_ERR_INVALID, "edge weights must be positive");
      h.w[i] = in.weight[i];
      wtot += in.weight[i];
      if (in.weight[i] != 1) h.unit = false;
    }
    if (h.unit) h.w.clear();
  } else {
    wtot = in.e;
  }
  if (wtot >= (1ll << 24)) throw Error(USAP_ERR_LIMIT, "total edge weight must be below 2^24");
  h.wtot = wtot;
  }
  const int32_t n = h.n;
  if (!h.csr_built) build_csr(h);
  scc_prepare(h);
  // per-vertex global hash regions for degrees beyond the shared-memory table
  std::vector<int64_t> hi_off(n, -1);
  std::vector<int32_t> hubs;
  int64_t hi_slots = 0;
  for (int32_t v = 0; v < n; v++) {
    int deg = (h.out_ptr[v + 1] - h.out_ptr[v]) + (h.in_ptr[v + 1] - h.in_ptr[v]);
    if (deg > kHubDegree) {
      hubs.push_back(v);
      int cap = 1 << hash_lg(deg);
      if (cap > kPhaseHubSlots) {   // beyond the smaller shared-memory table of the two kernels
        hi_off[v] = hi_slots;
        hi_slots += cap;
      }
    }
  }

  auto gr = std::make_shared<GraphResident>(device);
  // the first solve's initial blocks, on a host thread while the graph
  // uploads (the CSR buffers keep their addresses when h moves into gr)
  {
    gr->scc_part.resize(n);
    const int32_t* tp = h.transpose_is_in ? h.in_ptr.data() : h.tptr.data();
    const int32_t* ti = h.transpose_is_in ? h.in_idx.data() : h.tidx.data();
    gr->scc_b = std::async(std::launch::async, scc_arrays, n, h.e, h.out_ptr.data(), h.out_idx.data(), tp, ti,
                           kDefaultDfsDepth, gr->scc_part.data());
  }
  cudaStream_t st_ = gr->st;
  cudaEvent_t e0, e1;
  USAP_CUDA(cudaEventCreate(&e0));
  USAP_CUDA(cudaEventCreate(&e1));
  USAP_CUDA(cudaEventRecord(e0, st_));
  GraphDev g;
  g.n = n;
  g.e = h.e;
  g.wtot = wtot;
  g.unit = h.unit;
  long long up_bytes = 0;
  auto up = [&](int32_t** d, const std::vector<int32_t>& v) {
    dalloc(d, v.size());
    if (!v.empty())
      USAP_CUDA(cudaMemcpyAsync(*d, v.data(), sizeof(int32_t) * v.size(), cudaMemcpyHostToDevice, st_));
    up_bytes += static_cast<long long>(sizeof(int32_t) * v.size());
  };
  up(&g.src, h.src);
  up(&g.dst, h.dst);
  if (!h.unit) {
    up(&g.w, h.w);
    up(&g.out_w, h.out_w);
    up(&g.in_w, h.in_w);
  }
  up(&g.out_ptr, h.out_ptr);
  up(&g.out_idx, h.out_idx);
  up(&g.in_ptr, h.in_ptr);
  up(&g.in_idx, h.in_idx);
  up(&g.kout, h.kout);
  up(&g.kin, h.kin);
  {
    h.chunk_ptr.assign(static_cast<size_t>(n) + 1, 0);
    for (int32_t v = 0; v < n; v++) {
      const int64_t deg = (h.out_ptr[v + 1] - h.out_ptr[v]) + (h.in_ptr[v + 1] - h.in_ptr[v]);
      h.chunk_ptr[v + 1] = h.chunk_ptr[v] + std::max<int64_t>(1, (deg + 31) / 32);
    }
    g.nchunks = h.chunk_ptr[n];
    std::vector<int32_t> ch(2 * static_cast<size_t>(g.nchunks));
    for (int32_t v = 0; v < n; v++)
      for (int64_t q = h.chunk_ptr[v]; q < h.chunk_ptr[v + 1]; q++) {
        ch[2 * q] = v;
        ch[2 * q + 1] = static_cast<int32_t>(q - h.chunk_ptr[v]);
      }
    int32_t* d = nullptr;
    up(&d, ch);
    g.chunks = reinterpret_cast<int2*>(d);
    dalloc(&g.chunk_ptr, h.chunk_ptr.size());
    USAP_CUDA(cudaMemcpyAsync(g.chunk_ptr, h.chunk_ptr.data(), sizeof(int64_t) * h.chunk_ptr.size(),
                              cudaMemcpyHostToDevice, st_));
    up_bytes += static_cast<long long>(sizeof(int64_t) * h.chunk_ptr.size());
  }
  int64_t log_bytes = 0;
  gr->logs = device_log_table(device, wtot, &log_bytes);
  g.logk = gr->logs->L;
  g.logk2 = gr->logs->L2;
  dalloc(&g.hi_off, n);
  USAP_CUDA(cudaMemcpyAsync(g.hi_off, hi_off.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, st_));
  up_bytes += static_cast<long long>(log_bytes + sizeof(int64_t) * n +
                                     sizeof(int32_t) * hubs.size());
  g.hi_slots = hi_slots;
  dalloc(&gr->hubs_dev, hubs.size());
  if (!hubs.empty())
    USAP_CUDA(cudaMemcpyAsync(gr->hubs_dev, hubs.data(), sizeof(int32_t) * hubs.size(), cudaMemcpyHostToDevice, st_));
  USAP_CUDA(cudaEventRecord(e1, st_));
  USAP_CUDA(cudaStreamSynchronize(st_));
  float ms = 0;
  USAP_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  gr->h2d_ms = ms;
  gr->h2d_bytes = up_bytes;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  gr->g = g;
  gr->hg = std::move(h);
  gr->hub_ids = std::move(hubs);
  return gr;
}

bool GraphResident::take_initial_blocks(int32_t* B, std::vector<int32_t>* part) {
  std::lock_guard<std::mutex> lk(scc_mu);
  if (!scc_b.valid()) return false;
  *B = scc_b.get();
  part->swap(scc_part);
  return true;
}

GraphResident::GraphResident(int dev) : device(dev) {
  pool_configure(dev);
  USAP_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
}

GraphResident::~GraphResident() {
  if (scc_b.valid()) scc_b.wait();   // the host thread reads hg
  cudaSetDevice(device);
  cudaStream_t st_ = st;
  dfree(g.src); dfree(g.dst); dfree(g.w);
  dfree(g.out_ptr); dfree(g.out_idx); dfree(g.out_w);
  dfree(g.in_ptr); dfree(g.in_idx); dfree(g.in_w);
  dfree(g.chunks); dfree(g.chunk_ptr);
  dfree(g.kout); dfree(g.kin);   // the log tables belong to the device (logs)
  dfree(g.hi_off);
  dfree(hubs_dev);
  if (st) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
}

void Job::load(const usap_graph& in) {
  USAP_CUDA(cudaSetDevice(device_));
  attach(load_graph(device_, in));
}

void Job::load_host(HostGraph&& h) {
  USAP_CUDA(cudaSetDevice(device_));
  const usap_graph none{};
  attach(load_graph(device_, none, &h));
}

void Job::attach(std::shared_ptr<GraphResident> gr) {
  USAP_CUDA(cudaSetDevice(device_));
  const bool other = gr_ != gr;
  if (other) {
    // buffers stay allocated across graphs (allocating while other solves
    // run on the device is slow); only those that no longer fit are
    // replaced, and the caches built for the previous graph are dropped
    USAP_CUDA(cudaStreamSynchronize(st_));
    if (gr->hg.n > ncap_) free_vertex_state();
    batch_hub_bs_ = 0;
  }
  gr_ = std::move(gr);
  hg_ = &gr_->hg;
  g_ = gr_->g;
  if (!hkey_ || g_.hi_slots > hcap_) {
    dfree(hkey_); dfree(hwo_); dfree(hwi_);
    hcap_ = std::max<int64_t>(g_.hi_slots, 1);
    dalloc(&hkey_, hcap_);
    dalloc(&hwo_, hcap_);
    dalloc(&hwi_, hcap_);
  }
  if (other && move_to_) USAP_CUDA(cudaMemsetAsync(move_to_, 0xff, sizeof(int32_t) * hg_->n, st_));
  g_.hkey = hkey_;
  g_.hwo = hwo_;
  g_.hwi = hwi_;
}



HubList Job::hubs_for(int32_t beg, int32_t end, int32_t B) const {
  HubList hl;
  const std::vector<int32_t>& hub_ids = gr_->hub_ids;
  hl.ids = gr_->hubs_dev;
  hl.lo = static_cast<int>(std::lower_bound(hub_ids.begin(), hub_ids.end(), beg) - hub_ids.begin());
  hl.hi = static_cast<int>(std::lower_bound(hub_ids.begin(), hub_ids.end(), end) - hub_ids.begin());
  int cap = 32;
  for (int i = hl.lo; i < hl.hi; i++) {
    const int32_t v = hub_ids[i];
    int deg = (hg_->out_ptr[v + 1] - hg_->out_ptr[v]) + (hg_->in_ptr[v + 1] - hg_->in_ptr[v]);
    int c = 1 << hash_lg(std::min(deg, B));
    cap = std::max(cap, c);
  }
  hl.smem_cap = std::min(cap, kHubSmemSlots);
  return hl;
}

void Job::ensure_capacity(int32_t B, int32_t K, int32_t dense_max, int32_t maxitr) {
  const int32_t n = hg_->n;
  bool fresh = slots_[0] == nullptr;
  if (fresh) {
    for (auto& s : slots_) dalloc(&s, n);
    dalloc(&move_to_, n);
    USAP_CUDA(cudaMemsetAsync(move_to_, 0xff, sizeof(int32_t) * n, st_));
    dalloc(&from_, n);
    dalloc(&rp_s_, n);
    dalloc(&rp_n_, n);
    dalloc(&rp_q_, n);
    dalloc(&rp_f_, n);
    ncap_ = n;
  }
  // the sorted views hold a slot per edge: grow them for a larger graph
  if (bcap_ > 0) sb_.reserve(hg_->e, bcap_, st_);
  if (B > bcap_) {
    dfree(dout_); dfree(din_); dfree(best_s_); dfree(best_q_); dfree(best_x_);
    dfree(skeys_); dfree(skeys_alt_); dfree(sidx_); dfree(sidx_alt_);
    dfree(union_work_); dfree(root_); dfree(present_); dfree(newlabel_); dfree(merged_dev_);
    dalloc(&dout_, B);
    dalloc(&din_, B);
    dalloc(&best_s_, B);
    dalloc(&best_q_, B);
    dalloc(&best_x_, B);
    dalloc(&skeys_, B);
    dalloc(&skeys_alt_, B);
    dalloc(&sidx_, B);
    dalloc(&sidx_alt_, B);
    dalloc(&union_work_, 8ll * B);
    dalloc(&root_, B);
    dalloc(&present_, B);
    dalloc(&newlabel_, B);
    dalloc(&merged_dev_, 1);
    dfree(cub_tmp_);
    size_t b1 = 0, b2 = 0;
    USAP_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b1, skeys_, skeys_alt_, sidx_, sidx_alt_, B));
    USAP_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b2, present_, newlabel_, B));
    cub_bytes_ = std::max(b1, b2);
    cub_tmp_ = dev_alloc(cub_bytes_, st_);
    sb_.reserve(hg_->e, B, st_);
    bcap_ = B;
    kcap_ = 0;
  }
  if (static_cast<int64_t>(B) * K > static_cast<int64_t>(bcap_) * kcap_) {
    dfree(prop_s_);
    dfree(prop_q_);
    dfree(prop_x_);
    dfree(prop_f_);
    dalloc(&prop_s_, static_cast<size_t>(bcap_) * K);
    dalloc(&prop_q_, static_cast<size_t>(bcap_) * K);
    dalloc(&prop_x_, static_cast<size_t>(bcap_) * K);
    dalloc(&prop_f_, static_cast<size_t>(bcap_) * K);
    kcap_ = K;
  }
  int32_t dneed = std::min(B, dense_max);
  int32_t ld = (dneed + 3) & ~3;
  if (ld > dcap_) {
    dfree(M_);
    dfree(Mt_);
    dfree(CS_);
    dalloc(&M_, static_cast<size_t>(ld) * ld);
    dalloc(&Mt_, static_cast<size_t>(ld) * ld);
    const int cld = (ld + 127) / 128;
    dalloc(&CS_, static_cast<size_t>(ld) * cld);
    dcap_ = ld;
  }
  if (maxitr > icap_) {
    dfree(ide_q_);
    dfree(ide_n_);
    dalloc(&ide_q_, maxitr);
    dalloc(&ide_n_, maxitr);
    icap_ = maxitr;
  }
}

// --- phases ---------------------------------------------------------------------
void Job::prepare_nodal_blocks(const int32_t* part, int32_t B, bool dense) {
  launch_degrees(g_, part, B, dout_, din_, st_);
  if (dense) {
    ld_ = (B + 3) & ~3;
    cld_ = (B + 127) / 128;
    launch_dense_build(g_, part, B, ld_, M_, Mt_, st_);
    launch_chunk_sums(B, dense_view(), CS_, st_);
  } else {
    sb_.build(g_, part, B, false, true, st_);
  }
}

void Job::merge_phase(const int32_t* part, int32_t B, int32_t K, uint32_t stage, uint64_t seed, bool dense) {
  // dense: the tile (and its chunk sums) the nodal phase uses, else sorted views
  if (dense) {
    prepare_nodal_blocks(part, B, true);
  } else {
    launch_degrees(g_, part, B, dout_, din_, st_);
    sb_.build(g_, part, B, true, true, st_);
  }
  MergeArgs a;
  a.L = g_.logk;
  a.B = B;
  a.K = K;
  a.stage = stage;
  a.seed = seed;
  a.dout = dout_;
  a.din = din_;
  a.prop_s = prop_s_;
  a.prop_q = prop_q_;
  a.L2 = g_.logk2;
  const int mp = merge_prec();
  a.prec = mp;
  a.prop_x = mp ? prop_x_ : nullptr;
  a.prop_f = mp ? prop_f_ : nullptr;
  a.f32 = mp ? f32d_ : nullptr;
  if (dense) launch_merge_propose_dense(dense_view(), a, st_);
  else launch_merge_propose(g_, sb_.view(), a, st_);
  launch_merge_argmin(B, K, prop_s_, prop_q_, a.prop_x, best_s_, best_q_, mp ? best_x_ : nullptr, a.f32, st_);
}

int32_t Job::merge_apply(int32_t* part, int32_t B, int32_t btm) {
  launch_merge_sort_keys(B, best_q_, skeys_, sidx_, st_);
  size_t bytes = cub_bytes_;
  USAP_CUB(cub::DeviceRadixSort::SortPairs(cub_tmp_, bytes, skeys_, skeys_alt_, sidx_, sidx_alt_, B, 0,
                                           64, st_));
  launch_merge_union(B, sidx_alt_, best_s_, btm, union_work_, root_, merged_dev_, st_);
  launch_merge_relabel(hg_->n, B, part, root_, present_, newlabel_, cub_tmp_, cub_bytes_, st_);
  int32_t merged = 0;
  USAP_CUDA(cudaMemcpyAsync(&h_ctl_->itr, merged_dev_, sizeof(int32_t), cudaMemcpyDeviceToHost, st_));
  wait();
  merged = h_ctl_->itr;
  return merged;
}

void Job::entropy_launch(const int32_t* part, int32_t B, bool dense) {
  USAP_CUDA(cudaMemsetAsync(&ctl_->entropy_acc, 0, sizeof(unsigned long long), st_));
  if (dense) {
    launch_entropy_dense(g_, dense_view(), B, dout_, din_, &ctl_->entropy_acc, st_);
  } else {
    launch_entropy_sorted(g_, sb_.view(), sb_.nnz_dev(), sb_.max_nnz(), sb_.rowof(), dout_, din_,
                          &ctl_->entropy_acc, st_);
  }
}

NodalArgs Job::nodal_args(int32_t* part, int32_t B, int32_t beg, int32_t end, uint32_t stage, uint64_t seed,
                          int stats) const {
  NodalArgs a;
  a.out_ptr = g_.out_ptr;
  a.out_idx = g_.out_idx;
  a.out_w = g_.out_w;
  a.in_ptr = g_.in_ptr;
  a.in_idx = g_.in_idx;
  a.in_w = g_.in_w;
  a.kout = g_.kout;
  a.kin = g_.kin;
  a.L = g_.logk;
  a.unit = g_.unit ? 1 : 0;
  a.part = part;
  a.B = B;
  a.dout = dout_;
  a.din = din_;
  a.beg = beg;
  a.end = end;
  a.stage = stage;
  a.seed = seed;
  a.move_to = move_to_;
  a.from = from_;
  a.prop_s = nullptr;
  a.prop_q = nullptr;
  a.prop_ninf = nullptr;
  a.prop_f = nullptr;
  a.ctl = ctl_;
  a.hi_off = g_.hi_off;
  a.hkey = g_.hkey;
  a.hwo = g_.hwo;
  a.hwi = g_.hwi;
  a.stats = stats;
  a.prec = prec_;
  a.shadow = prec_ != 3 || shadow_ || stats == 2 ? 1 : 0;
  a.L2 = g_.logk2;
  a.Trow = nullptr;
  a.Tcol = nullptr;
  a.tld = 0;
  if (stats == 2) {   // replay: per-vertex proposals
    a.prop_s = rp_s_;
    a.prop_q = rp_q_;
    a.prop_ninf = rp_n_;
    a.prop_f = rp_f_;
  }
  return a;
}

void Job::nodal_batch(int32_t* part, int32_t B, bool dense, int32_t beg, int32_t end, uint32_t stage,
                      uint64_t seed, bool first_of_sweep, int stats, const CtlArgs& ctl_args) {
  if (!dense && !first_of_sweep) sb_.build(g_, part, B, false, true, st_);
  const NodalArgs a = nodal_args(part, B, beg, end, stage, seed, stats);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (stats == 1) {
    while (ev_pool_.size() < ev_used_ + 2) {
      cudaEvent_t e;
      USAP_CUDA(cudaEventCreate(&e));
      ev_pool_.push_back(e);
    }
    e0 = ev_pool_[ev_used_++];
    e1 = ev_pool_[ev_used_++];
    USAP_CUDA(cudaEventRecord(e0, st_));
  }
  const HubList hubs = hubs_for(beg, end, B);
  if (dense) launch_nodal_propose_dense(a, dense_view(), hubs, streams());
  else launch_nodal_propose_sorted(a, sb_.view(), hubs, streams());
  if (stats == 1) USAP_CUDA(cudaEventRecord(e1, st_));
  if (dense) {
    launch_nodal_apply_commit_dense(g_, part, move_to_, from_, beg, end, hg_->chunk_ptr[beg],
                                    hg_->chunk_ptr[end], ld_, M_, Mt_, cld_, CS_, dout_, din_, ctl_,
                                    ctl_args, st_);
  } else {
    launch_nodal_commit(g_, part, move_to_, beg, end, 1, dout_, din_, ctl_, ctl_args, st_);
  }
}

float Job::nodal_phase(int32_t* part, int32_t B, uint32_t stage, uint64_t seed, int W, double thr,
                       double model_d, int32_t maxitr, int stats, int grid, bool timed) {
  const int32_t n = hg_->n;
  const int32_t nb = (n + bs_ - 1) / bs_;
  if (batch_hub_bs_ != bs_) {   // first hub of each batch, for this batch size
    const std::vector<int32_t>& hub_ids = gr_->hub_ids;
    std::vector<int32_t> bh(static_cast<size_t>(nb) + 1);
    for (int32_t b = 0; b <= nb; b++) {
      const int32_t v = static_cast<int32_t>(std::min<int64_t>(static_cast<int64_t>(b) * bs_, n));
      bh[b] = static_cast<int32_t>(std::lower_bound(hub_ids.begin(), hub_ids.end(), v) - hub_ids.begin());
    }
    // work units: pairs of vertices of degree <= 64 (half-warps), single
    // vertices of degree <= 128 (warps); hubs are proposed by whole CTAs
    std::vector<int32_t> up(static_cast<size_t>(nb) + 1, 0);
    std::vector<int32_t> un;
    un.reserve(2 * static_cast<size_t>(n));
    std::vector<int32_t> mid;
    for (int32_t b = 0; b < nb; b++) {
      const int32_t beg = b * bs_, end = std::min(n, beg + bs_);
      int32_t pending = -1;
      mid.clear();
      for (int32_t v = beg; v < end; v++) {
        const int64_t deg = (hg_->out_ptr[v + 1] - hg_->out_ptr[v]) + (hg_->in_ptr[v + 1] - hg_->in_ptr[v]);
        if (deg > kHubDegree) continue;
        if (deg > kHubDegree / 2) {
          mid.push_back(v);
        } else if (pending < 0) {
          pending = v;
        } else {
          un.push_back(pending);
          un.push_back(v);
          pending = -1;
        }
      }
      if (pending >= 0) {
        un.push_back(pending);
        un.push_back(-1);
      }
      for (int32_t v : mid) {
        un.push_back(v);
        un.push_back(-2);
      }
      up[b + 1] = static_cast<int32_t>(un.size() / 2);
    }
    if (batch_hub_cap_ < nb + 1) {
      dfree(batch_hub_);
      dfree(unit_ptr_);
      dalloc(&batch_hub_, nb + 1);
      dalloc(&unit_ptr_, nb + 1);
      batch_hub_cap_ = nb + 1;
    }
    if (units_cap_ < std::max<size_t>(un.size(), 2)) {
      dfree(units_);
      units_cap_ = std::max<size_t>(un.size(), 2);
      int32_t* ua = nullptr;
      dalloc(&ua, units_cap_);
      units_ = reinterpret_cast<int2*>(ua);
    }
    int32_t* ud = reinterpret_cast<int32_t*>(units_);
    USAP_CUDA(cudaMemcpyAsync(batch_hub_, bh.data(), sizeof(int32_t) * bh.size(), cudaMemcpyHostToDevice, st_));
    USAP_CUDA(cudaMemcpyAsync(unit_ptr_, up.data(), sizeof(int32_t) * up.size(), cudaMemcpyHostToDevice, st_));
    if (!un.empty())
      USAP_CUDA(cudaMemcpyAsync(ud, un.data(), sizeof(int32_t) * un.size(), cudaMemcpyHostToDevice, st_));
    wait();
    batch_hub_bs_ = bs_;
  }
  PhaseArgs pa;
  pa.a = nodal_args(part, B, 0, 0, stage, seed, stats);
  pa.v = dense_view();
  pa.g = g_;
  pa.part = part;
  pa.dout = dout_;
  pa.din = din_;
  pa.M = M_;
  pa.Mt = Mt_;
  pa.CS = CS_;
  pa.hubs = gr_->hubs_dev;
  pa.batch_hub = batch_hub_;
  pa.units = units_;
  pa.unit_ptr = unit_ptr_;
  pa.chunk_ptr = g_.chunk_ptr;
  pa.n = n;
  pa.bs = bs_;
  pa.maxitr = maxitr;
  pa.W = W;
  pa.thr = thr;
  pa.model_d = model_d;
  pa.ide_q = ide_q_;
  pa.ide_n = ide_n_;
  pa.bar_timeout_ns = bar_test_timeout_ns_;
  pa.bar_hold = bar_test_hold_;
  bar_test_hold_ = -1;   // one launch only
  bar_test_timeout_ns_ = 0;
  // precision mode 3: the old-state term tables of the persistent kernels,
  // single-job and gang (B <= kRefTabMaxB; above it the per-cell tables
  // cost more than the proposals' own evaluation)
  if (prec_ == 3 && B <= kRefTabMaxB) {
    const size_t cells = static_cast<size_t>(ld_) * ld_;
    if (cells > tcap_) {
      dfree(Trow_);
      dfree(Tcol_);
      dalloc(&Trow_, cells);
      dalloc(&Tcol_, cells);
      tcap_ = cells;
    }
    pa.a.Trow = Trow_;
    pa.a.Tcol = Tcol_;
    pa.a.tld = ld_;
  }
  if (gang_ && !timed) {
    gang_->run(pa, st_);
    USAP_CUDA(cudaMemcpyAsync(h_ctl_, ctl_, sizeof(NodalCtl), cudaMemcpyDeviceToHost, st_));
    wait();
    return 0.0f;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (timed) {
    while (ev_pool_.size() < ev_used_ + 2) {
      cudaEvent_t e;
      USAP_CUDA(cudaEventCreate(&e));
      ev_pool_.push_back(e);
    }
    e0 = ev_pool_[ev_used_];
    e1 = ev_pool_[ev_used_ + 1];
    USAP_CUDA(cudaEventRecord(e0, st_));
  }
  launch_nodal_phase(pa, grid, st_);
  if (timed) USAP_CUDA(cudaEventRecord(e1, st_));
  USAP_CUDA(cudaMemcpyAsync(h_ctl_, ctl_, sizeof(NodalCtl), cudaMemcpyDeviceToHost, st_));
  wait();
  if (h_ctl_->bar_err) throw Error(USAP_ERR_INTERNAL, "persistent nodal kernel: a grid barrier timed out");
  float ms = 0;
  if (timed) USAP_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  return ms;
}

void Job::enqueue_sweep(int32_t* part, int32_t B, bool dense, uint32_t stage, uint64_t seed, int W,
                        double thr, double model_d, int stats) {
  const int32_t n = hg_->n;
  if (!dense) sb_.build(g_, part, B, false, true, st_);
  entropy_launch(part, B, dense);
  launch_ctl_sweep_start(ctl_, W, ide_q_, ide_n_, st_);
  for (int32_t beg = 0; beg < n; beg += bs_) {
    const int32_t end = beg + bs_ < n ? beg + bs_ : n;
    const long long edges = (static_cast<long long>(hg_->out_ptr[end]) - hg_->out_ptr[beg]) +
                            (static_cast<long long>(hg_->in_ptr[end]) - hg_->in_ptr[beg]);
    const CtlArgs ca{1, W, thr, model_d, ide_q_, ide_n_, end - beg, edges};
    nodal_batch(part, B, dense, beg, end, stage, seed, beg == 0, stats, ca);
  }
}

void Job::emit_trace(int kind, int stage, int itr, int beg, int32_t B, const int32_t* part, bool dense,
                     long long S_q, int S_ninf, long long cum_q, int cum_ninf, long long moves) {
  const int32_t n = hg_->n;
  std::vector<int32_t> hp(n), hdo(B), hdi(B);
  USAP_CUDA(cudaMemcpyAsync(hp.data(), part, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st_));
  USAP_CUDA(cudaMemcpyAsync(hdo.data(), dout_, sizeof(int32_t) * B, cudaMemcpyDeviceToHost, st_));
  USAP_CUDA(cudaMemcpyAsync(hdi.data(), din_, sizeof(int32_t) * B, cudaMemcpyDeviceToHost, st_));
  uint64_t hM = 0;
  if (dense) {
    std::vector<int32_t> hm(static_cast<size_t>(ld_) * B);
    USAP_CUDA(cudaMemcpyAsync(hm.data(), M_, sizeof(int32_t) * hm.size(), cudaMemcpyDeviceToHost, st_));
    wait();
    for (int32_t i = 0; i < B; i++)
      for (int32_t j = 0; j < B; j++) {
        int32_t m = hm[static_cast<size_t>(i) * ld_ + j];
        if (m) hM += mix64(mix64((static_cast<uint64_t>(i) << 32) | static_cast<uint32_t>(j)) ^ static_cast<uint64_t>(m));
      }
  } else {
    sb_.build(g_, part, B, false, false, st_);
    SortedView v = sb_.view();
    int nnz = 0;
    USAP_CUDA(cudaMemcpyAsync(&nnz, sb_.nnz_dev(), sizeof(int), cudaMemcpyDeviceToHost, st_));
    wait();
    std::vector<int32_t> rp(B + 1), col(nnz), val(nnz);
    USAP_CUDA(cudaMemcpyAsync(rp.data(), v.rowptr, sizeof(int32_t) * (B + 1), cudaMemcpyDeviceToHost, st_));
    USAP_CUDA(cudaMemcpyAsync(col.data(), v.col, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, st_));
    USAP_CUDA(cudaMemcpyAsync(val.data(), v.val, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, st_));
    wait();
    for (int32_t i = 0; i < B; i++)
      for (int32_t p = rp[i]; p < rp[i + 1]; p++)
        if (val[p]) hM += mix64(mix64((static_cast<uint64_t>(i) << 32) | static_cast<uint32_t>(col[p])) ^ static_cast<uint64_t>(val[p]));
  }
  uint64_t hpart = 1469598103934665603ull;
  for (int32_t v = 0; v < n; v++) {
    hpart ^= static_cast<uint32_t>(hp[v]);
    hpart *= 1099511628211ull;
  }
  uint64_t hdeg = 0;
  for (int32_t i = 0; i < B; i++)
    hdeg += mix64(mix64(static_cast<uint64_t>(i)) ^ ((static_cast<uint64_t>(hdo[i]) << 32) ^ static_cast<uint64_t>(hdi[i])));
  usap_trace_event ev;
  std::memset(&ev, 0, sizeof(ev));
  ev.kind = kind;
  ev.stage = stage;
  ev.itr = itr;
  ev.batch_beg = beg;
  ev.B = B;
  ev.S_q = S_q;
  ev.S_ninf = S_ninf;
  ev.cum_q = cum_q;
  ev.cum_ninf = cum_ninf;
  ev.moves = moves;
  ev.h_part = hpart;
  ev.h_M = hM;
  ev.h_deg = hdeg;
  trace_(trace_user_, &ev);
}

// --- the whole solve ------------------------------------------------------------
void Job::partition(const usap_params& p, int32_t* out_assign, usap_result* res, const int32_t* init) {
  if (!loaded()) throw Error(USAP_ERR_STATE, "no graph loaded");
  USAP_CUDA(cudaSetDevice(device_));
  if (p.num_agg_proposals_per_block < 1) throw Error(USAP_ERR_INVALID, "num_agg_proposals_per_block must be >= 1");
  if (p.max_num_nodal_itr < 0) throw Error(USAP_ERR_INVALID, "max_num_nodal_itr must be >= 0");
  if (p.num_batch_nodal_update < 1) throw Error(USAP_ERR_INVALID, "num_batch_nodal_update must be >= 1");
  if (p.delta_entropy_moving_avg_window < 1) throw Error(USAP_ERR_INVALID, "moving average window must be >= 1");
  if (!(p.num_block_reduction_rate > 0.0f && p.num_block_reduction_rate < 1.0f))
    throw Error(USAP_ERR_INVALID, "num_block_reduction_rate must be in (0, 1)");
  if (p.precision < 0 || p.precision > 3) throw Error(USAP_ERR_INVALID, "precision must be 0, 1, 2 or 3");
  const int dense_max = effective_dense_max(p);
  auto t_start = std::chrono::steady_clock::now();
  std::memset(res, 0, sizeof(*res));
  const int32_t n = hg_->n;
  const int32_t K = p.num_agg_proposals_per_block;
  const int32_t W = p.delta_entropy_moving_avg_window;
  const int32_t maxitr = p.max_num_nodal_itr;
  bs_ = n / p.num_batch_nodal_update;
  if (bs_ < 1) bs_ = 1;
  const int stats = p.stats ? 1 : 0;
  const bool use_graphs = p.sweep_graphs != 0 && !stats;
  trace_mask_ = p.trace_kinds ? p.trace_kinds : 7;
  ev_used_ = 0;
  const LaunchCount lc0 = launch_count();
  long long d2h = 0;
  prec_ = p.precision;
  shadow_ = p.fp64_shadow != 0;
  F32Tally nodal32{0, 0, 0, 0.0};   // summed over the stages' nodal phases
  if (prec_) USAP_CUDA(cudaMemsetAsync(f32d_, 0, 2 * sizeof(F32Tally), st_));

  // initial blocks: the host's depth-limited DFS on the transpose (the
  // reference's), one block per vertex, or the device's matching stand-in
  std::vector<int32_t> part0(n);
  int32_t B;
  int32_t* dpart0 = nullptr;
  if (!init && p.init_mode == 2) {
    dpart0 = static_cast<int32_t*>(dev_alloc(sizeof(int32_t) * n, st_));
    B = device_initial_blocks(g_, dpart0, st_, nullptr);
  } else if (init) {
    B = compact_labels(init, n, part0.data());
  } else if (p.init_mode == 1) {
    for (int32_t v = 0; v < n; v++) part0[v] = v;
    B = n;
  } else if (p.dfs_depth != kDefaultDfsDepth || !gr_->take_initial_blocks(&B, &part0)) {
    B = scc_host(*hg_, p.dfs_depth, part0.data());
  }
  ensure_capacity(B, K, dense_max, std::max(maxitr, 1));
  int32_t work = 0;
  if (dpart0) {
    USAP_CUDA(cudaMemcpyAsync(slots_[work], dpart0, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st_));
    dev_free(dpart0, st_);
  } else {
    USAP_CUDA(cudaMemcpyAsync(slots_[work], part0.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st_));
  }
  wait();
  auto t_init = std::chrono::steady_clock::now();
  res->ms_init = std::chrono::duration<double, std::milli>(t_init - t_start).count();

  res->B_init = B;
  int32_t btm = reduce_blocks(B, p.num_block_reduction_rate);
  Golden gs;
  uint32_t stage = 0;
  const uint64_t seed = p.seed;
  double ms_merge = 0, ms_nodal = 0;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> kernel_events;
  for (;;) {
    if (stage > 100000u) throw Error(USAP_ERR_INTERNAL, "golden-section search did not close");
    int32_t* part = slots_[work];
    auto tm0 = std::chrono::steady_clock::now();
    // merge phase and its application
    // the dense merge scans whole rows (K B^2 reads): below 4096 blocks it
    // beats rebuilding the sorted views, above it does not
    merge_phase(part, B, K, stage, seed, B <= std::min(dense_max, kDenseMergeMax));
    int32_t merged = merge_apply(part, B, btm);
    if (merge_prec()) launch_order_flips(B, sidx_alt_, best_x_, &f32d_[1].flips, st_);
    d2h += sizeof(int32_t);
    if (merged < btm) res->merge_shortfall += btm - merged;
    B -= merged;
    auto tm1 = std::chrono::steady_clock::now();
    ms_merge += std::chrono::duration<double, std::milli>(tm1 - tm0).count();

    // batched nodal sweeps
    const bool dense = B <= dense_max;
    prepare_nodal_blocks(part, B, dense);
    if (trace_on(1)) emit_trace(1, stage, 0, 0, B, part, dense, 0, 0, 0, 0, 0);
    USAP_CUDA(cudaMemsetAsync(ctl_, 0, sizeof(NodalCtl), st_));
    USAP_CUDA(cudaMemsetAsync(ide_q_, 0, sizeof(long long) * std::max(maxitr, 1), st_));
    USAP_CUDA(cudaMemsetAsync(ide_n_, 0, sizeof(int) * std::max(maxitr, 1), st_));
    const bool isf = gs.large.finite && gs.med.finite && gs.small.finite;
    const double thr = isf ? p.delta_entropy_threshold2 : p.delta_entropy_threshold1;
    const double model_d = model_S(n, hg_->e, B);
    trace_prev_moves_ = 0;
    const bool phase_ok = dense && !use_graphs && maxitr > 0 && B <= nodal_phase_max_blocks() && !trace_on(2);
    // the gang's delta-table keys pack (job, cell) into 31 bits: B <= 4096
    const bool in_gang = gang_ != nullptr && phase_ok && !stats && B <= 4096;
    const int pgrid = phase_ok && (p.persistent || in_gang) ? nodal_phase_grid(device_) : 0;
    const int pctas = p.persistent_ctas > 0 ? std::min(pgrid, static_cast<int>(p.persistent_ctas)) : pgrid;
    if (pgrid > 0) {
      const float ms = nodal_phase(part, B, stage, seed, W, thr, model_d, maxitr, stats, pctas, stats != 0);
      d2h += sizeof(NodalCtl);
      if (stats) {
        res->ms_nodal_kernel += ms;
        res->nodal_kernel_launches++;
      }
    } else if (!trace_on(2)) {
      // the host keeps one sweep in flight ahead of the one it checks (a
      // sweep queued after convergence returns at once); with sweep_graphs
      // the sweep is recorded once per stage and replayed as a CUDA graph
      cudaGraph_t graph = nullptr;
      cudaGraphExec_t exec = nullptr;
      LaunchCount per_sweep;
      if (maxitr > 0 && use_graphs) {
        const LaunchCount before = launch_count();
        USAP_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
        enqueue_sweep(part, B, dense, stage, seed, W, thr, model_d, 0);
        USAP_CUDA(cudaStreamEndCapture(st_, &graph));
        USAP_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        per_sweep.kernels = launch_count().kernels - before.kernels;
        per_sweep.cub = launch_count().cub - before.cub;
      }
      int32_t launched = 0;
      const size_t ev_mark = ev_used_;
      auto launch_one = [&] {
        if (exec) USAP_CUDA(cudaGraphLaunch(exec, st_));
        else enqueue_sweep(part, B, dense, stage, seed, W, thr, model_d, stats);
        USAP_CUDA(cudaMemcpyAsync(h_ring_ + (launched & 1), ctl_, sizeof(NodalCtl), cudaMemcpyDeviceToHost, st_));
        USAP_CUDA(cudaEventRecord(ev_sweep_[launched & 1], st_));
        launched++;
        d2h += sizeof(NodalCtl);
      };
      // an instrumented solve does not run ahead, so that no queued no-op
      // sweep enters the kernel timings
      const bool ahead = !stats;
      if (maxitr > 0) launch_one();
      for (int32_t itr = 0; itr < maxitr; itr++) {
        if (ahead && itr + 1 < maxitr) launch_one();
        USAP_CUDA(cudaEventSynchronize(ev_sweep_[itr & 1]));
        if (h_ring_[itr & 1].done) break;
        if (!ahead && itr + 1 < maxitr) launch_one();
      }
      wait();
      if (launched > 0) *h_ctl_ = h_ring_[(launched - 1) & 1];
      else std::memset(h_ctl_, 0, sizeof(NodalCtl));
      if (exec) cudaGraphExecDestroy(exec);
      if (graph) cudaGraphDestroy(graph);
      if (exec) {
        res->sweep_graph_launches += launched;
        if (launched > 1) {   // recorded once, executed `launched` times
          launch_count().kernels += per_sweep.kernels * (launched - 1);
          launch_count().cub += per_sweep.cub * (launched - 1);
        }
      }
      if (stats) {
        for (size_t i = ev_mark; i + 1 < ev_used_; i += 2) {
          float ms = 0;
          USAP_CUDA(cudaEventElapsedTime(&ms, ev_pool_[i], ev_pool_[i + 1]));
          res->ms_nodal_kernel += ms;
          res->nodal_kernel_launches++;
        }
        ev_used_ = ev_mark;
      }
    } else {
      for (int32_t itr = 0; itr < maxitr; itr++) {
        size_t ev_mark = ev_used_;
        {
          if (!dense) sb_.build(g_, part, B, false, true, st_);
          entropy_launch(part, B, dense);
          launch_ctl_sweep_start(ctl_, W, ide_q_, ide_n_, st_);
          for (int32_t beg = 0; beg < n; beg += bs_) {
            const int32_t end = beg + bs_ < n ? beg + bs_ : n;
            const long long edges = (static_cast<long long>(hg_->out_ptr[end]) - hg_->out_ptr[beg]) +
                                    (static_cast<long long>(hg_->in_ptr[end]) - hg_->in_ptr[beg]);
            const CtlArgs ca{1, W, thr, model_d, ide_q_, ide_n_, end - beg, edges};
            nodal_batch(part, B, dense, beg, end, stage, seed, beg == 0, stats, ca);
            USAP_CUDA(cudaMemcpyAsync(h_ctl_, ctl_, sizeof(NodalCtl), cudaMemcpyDeviceToHost, st_));
            wait();
            NodalCtl c = *h_ctl_;
            emit_trace(2, stage, itr, beg, B, part, dense, c.S_q, c.S_ninf, static_cast<long long>(c.cum_q),
                       c.cum_ninf, static_cast<long long>(c.moves) - trace_prev_moves_);
            trace_prev_moves_ = static_cast<long long>(c.moves);
            if (c.done) break;
          }
        }
        USAP_CUDA(cudaMemcpyAsync(h_ctl_, ctl_, sizeof(NodalCtl), cudaMemcpyDeviceToHost, st_));
        wait();
        d2h += sizeof(NodalCtl);
        if (stats) {
          for (size_t i = ev_mark; i + 1 < ev_used_; i += 2) {
            float ms = 0;
            USAP_CUDA(cudaEventElapsedTime(&ms, ev_pool_[i], ev_pool_[i + 1]));
            res->ms_nodal_kernel += ms;
            res->nodal_kernel_launches++;
          }
          ev_used_ = ev_mark;
        }
        if (h_ctl_->done) break;
      }
    }
    // the control block was read after the last sweep
    res->sweeps += static_cast<int64_t>(h_ctl_->sweeps);
    res->batches += static_cast<int64_t>(h_ctl_->batches);
    res->nodal_proposals += static_cast<int64_t>(h_ctl_->proposals);
    res->nodal_moves += static_cast<int64_t>(h_ctl_->moves);
    res->near_threshold += static_cast<int64_t>(h_ctl_->near);
    res->apply_scans += static_cast<int64_t>(h_ctl_->apply_scans);
    if (prec_) {
      const F32Tally& t = h_ctl_->f32;
      nodal32.evals += t.evals;
      nodal32.flips += t.flips;
      nodal32.err_max = std::max(nodal32.err_max, t.err_max);   // bits of non-negative doubles order as integers
      nodal32.err_sum += t.err_sum;
    }
    res->edge_visits += static_cast<int64_t>(h_ctl_->edge_visits);
    res->nodal_kernel_bytes += static_cast<double>(h_ctl_->bytes);
    // description length of the finished stage: the cooperative kernels
    // computed its data term at the end of the phase
    long long data_fin = -static_cast<long long>(h_ctl_->entropy_acc);
    if (pgrid <= 0) {
      if (!dense) sb_.build(g_, part, B, false, true, st_);
      entropy_launch(part, B, dense);
      USAP_CUDA(cudaMemcpyAsync(h_ctl_, ctl_, sizeof(NodalCtl), cudaMemcpyDeviceToHost, st_));
      wait();
      data_fin = -static_cast<long long>(h_ctl_->entropy_acc);
      d2h += sizeof(NodalCtl);
    }
    const double S_fin = desc_length(model_d, data_fin);
    const long long S_fin_q = add_sat(q32_host(model_d), data_fin);
    auto tn1 = std::chrono::steady_clock::now();
    ms_nodal += std::chrono::duration<double, std::milli>(tn1 - tm1).count();
    if (trace_on(3)) emit_trace(3, stage, static_cast<int>(h_ctl_->sweeps), 0, B, part, dense, S_fin_q, 0, 0, 0, 0);
    res->stages++;
    stage++;

    int32_t restore = -1;
    bool done = gs.step(B, S_fin, S_fin_q, work, p.num_block_reduction_rate, &restore, &btm);
    if (done) {
      auto td0 = std::chrono::steady_clock::now();
      if (out_assign)
        USAP_CUDA(cudaMemcpyAsync(out_assign, slots_[gs.med.slot], sizeof(int32_t) * n,
                                  cudaMemcpyDeviceToHost, st_));
      wait();
      auto td1 = std::chrono::steady_clock::now();
      res->ms_d2h = std::chrono::duration<double, std::milli>(td1 - td0).count();
      if (out_assign) d2h += static_cast<long long>(sizeof(int32_t)) * n;
      res->B = gs.med.B;
      last_part_ = slots_[gs.med.slot];
      res->S_q = gs.med.S_q;
      res->S = gs.med.S;
      break;
    }
    // continue from a bracket point: copy it into a slot outside the bracket
    bool used[4] = {false, false, false, false};
    for (const GoldenPoint* gp : {&gs.large, &gs.med, &gs.small})
      if (gp->finite) used[gp->slot] = true;
    int32_t next = -1;
    for (int i = 0; i < 4; i++)
      if (!used[i]) {
        next = i;
        break;
      }
    if (next < 0 || restore < 0) throw Error(USAP_ERR_INTERNAL, "golden-section slot bookkeeping");
    USAP_CUDA(cudaMemcpyAsync(slots_[next], slots_[restore], sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st_));
    B = restore == gs.large.slot ? gs.large.B : gs.med.B;
    work = next;
  }
  if (prec_) {
    F32Tally m[2];
    USAP_CUDA(cudaMemcpyAsync(m, f32d_, sizeof(m), cudaMemcpyDeviceToHost, st_));
    wait();
    d2h += sizeof(m);
    auto as_double = [](unsigned long long bits) {
      double d;
      std::memcpy(&d, &bits, sizeof(d));
      return d;
    };
    res->fp32_nodal_evals = static_cast<int64_t>(nodal32.evals);
    res->fp32_nodal_flips = static_cast<int64_t>(nodal32.flips);
    res->fp32_merge_evals = static_cast<int64_t>(m[0].evals);
    res->fp32_merge_flips = static_cast<int64_t>(m[0].flips);
    res->fp32_order_flips = static_cast<int64_t>(m[1].flips);
    res->fp32_flip_rate = nodal32.evals ? static_cast<double>(nodal32.flips) / static_cast<double>(nodal32.evals) : 0.0;
    res->fp32_err_max = std::max(as_double(nodal32.err_max), as_double(m[0].err_max));
    res->fp32_err_mean = nodal32.evals ? nodal32.err_sum / static_cast<double>(nodal32.evals) : 0.0;
  }
  res->ms_merge = ms_merge;
  res->ms_nodal = ms_nodal;
  res->kernel_launches = launch_count().kernels - lc0.kernels;
  res->cub_calls = launch_count().cub - lc0.cub;
  res->h2d_bytes = static_cast<long long>(sizeof(int32_t)) * n;   // initial partition
  res->d2h_bytes = d2h;
  res->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
}

// labels renumbered 0..B-1 in ascending order of their values (the
// oracle's og_compact_labels); returns B
int32_t compact_labels(const int32_t* init, int32_t n, int32_t* part) {
  int32_t mx = -1;
  for (int32_t v = 0; v < n; v++) {
    if (init[v] < 0) throw Error(USAP_ERR_INVALID, "initial block labels must be >= 0");
    mx = std::max(mx, init[v]);
  }
  if (static_cast<int64_t>(mx) <= 4ll * n + 1024) {
    std::vector<int32_t> map(static_cast<size_t>(mx) + 1, -1);
    for (int32_t v = 0; v < n; v++) map[init[v]] = 0;
    int32_t B = 0;
    for (auto& m : map)
      if (m == 0) m = B++;
    for (int32_t v = 0; v < n; v++) part[v] = map[init[v]];
    return B;
  }
  std::vector<int32_t> u(init, init + n);
  std::sort(u.begin(), u.end());
  u.erase(std::unique(u.begin(), u.end()), u.end());
  for (int32_t v = 0; v < n; v++)
    part[v] = static_cast<int32_t>(std::lower_bound(u.begin(), u.end(), init[v]) - u.begin());
  return static_cast<int32_t>(u.size());
}

void Job::add_edges(const usap_graph& d) {
  if (!loaded()) throw Error(USAP_ERR_STATE, "no graph loaded");
  if (!d.src || !d.dst || d.e <= 0) throw Error(USAP_ERR_INVALID, "no edges to add");
  const HostGraph& h = *hg_;
  const int32_t base = d.one_based ? 1 : 0;
  int64_t n = std::max<int64_t>(h.n, d.n);
  for (int64_t i = 0; i < d.e; i++) n = std::max<int64_t>(n, static_cast<int64_t>(d.src[i]) - base + 1);
  if (n > INT32_MAX) throw Error(USAP_ERR_LIMIT, "more than 2^31 - 1 vertices");
  const int64_t e = h.e + d.e;
  std::vector<int32_t> src(e), dst(e), w;
  std::copy(h.src.begin(), h.src.end(), src.begin());
  std::copy(h.dst.begin(), h.dst.end(), dst.begin());
  for (int64_t i = 0; i < d.e; i++) {
    src[h.e + i] = d.src[i] - base;
    dst[h.e + i] = d.dst[i] - base;
  }
  bool unit = h.unit && !d.weight;
  if (d.weight)
    for (int64_t i = 0; i < d.e; i++) unit = unit && d.weight[i] == 1;
  if (!unit) {
    w.assign(e, 1);
    if (!h.unit) std::copy(h.w.begin(), h.w.end(), w.begin());
    if (d.weight) std::copy(d.weight, d.weight + d.e, w.begin() + h.e);
  }
  usap_graph g{};
  g.n = static_cast<int32_t>(n);
  g.e = e;
  g.src = src.data();
  g.dst = dst.data();
  g.weight = unit ? nullptr : w.data();
  g.one_based = 0;
  load(g);
}

// scores of the last solve's partition, evaluated where it lies in HBM
void Job::evaluate_last(const int32_t* truth, usap_scores* out) {
  if (!loaded() || !last_part_) throw Error(USAP_ERR_STATE, "no solve to evaluate");
  USAP_CUDA(cudaSetDevice(device_));
  const int32_t n = hg_->n;
  int32_t* t = nullptr;
  dalloc(&t, n);
  USAP_CUDA(cudaMemcpyAsync(t, truth, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st_));
  USAP_CUDA(cudaStreamSynchronize(st_));
  try {
    evaluate_device(t, last_part_, n, device_, out);
  } catch (...) {
    dfree(t);
    throw;
  }
  dfree(t);
}

// --- phase-level operations -------------------------------------------------------
int32_t Job::op_scc(int32_t depth, int32_t* part) {
  if (!loaded()) throw Error(USAP_ERR_STATE, "no graph loaded");
  return scc_host(*hg_, depth, part);
}

void Job::op_build(const int32_t* part, int32_t B, int32_t dense_max, int32_t* M, int32_t* dout,
                   int32_t* din) {
  if (!loaded()) throw Error(USAP_ERR_STATE, "no graph loaded");
  USAP_CUDA(cudaSetDevice(device_));
  ensure_capacity(B, 1, dense_max, 1);
  const int32_t n = hg_->n;
  USAP_CUDA(cudaMemcpyAsync(slots_[0], part, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st_));
  const bool dense = B <= dense_max;
  prepare_nodal_blocks(slots_[0], B, dense);
  USAP_CUDA(cudaMemcpyAsync(dout, dout_, sizeof(int32_t) * B, cudaMemcpyDeviceToHost, st_));
  USAP_CUDA(cudaMemcpyAsync(din, din_, sizeof(int32_t) * B, cudaMemcpyDeviceToHost, st_));
  if (M) {
    if (dense) {
      USAP_CUDA(cudaMemcpy2DAsync(M, sizeof(int32_t) * B, M_, sizeof(int32_t) * ld_, sizeof(int32_t) * B, B,
                                  cudaMemcpyDeviceToHost, st_));
      USAP_CUDA(cudaStreamSynchronize(st_));
    } else {
      SortedView v = sb_.view();
      int nnz = 0;
      USAP_CUDA(cudaMemcpyAsync(&nnz, sb_.nnz_dev(), sizeof(int), cudaMemcpyDeviceToHost, st_));
      USAP_CUDA(cudaStreamSynchronize(st_));
      std::vector<int32_t> rp(B + 1), col(nnz), val(nnz);
      USAP_CUDA(cudaMemcpyAsync(rp.data(), v.rowptr, sizeof(int32_t) * (B + 1), cudaMemcpyDeviceToHost, st_));
      USAP_CUDA(cudaMemcpyAsync(col.data(), v.col, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, st_));
      USAP_CUDA(cudaMemcpyAsync(val.data(), v.val, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, st_));
      USAP_CUDA(cudaStreamSynchronize(st_));
      std::memset(M, 0, sizeof(int32_t) * static_cast<size_t>(B) * B);
      for (int32_t i = 0; i < B; i++)
        for (int32_t q = rp[i]; q < rp[i + 1]; q++) M[static_cast<size_t>(i) * B + col[q]] = val[q];
    }
  }
  USAP_CUDA(cudaStreamSynchronize(st_));
}

int64_t Job::op_entropy(const int32_t* part, int32_t B, int32_t dense_max) {
  if (!loaded()) throw Error(USAP_ERR_STATE, "no graph loaded");
  USAP_CUDA(cudaSetDevice(device_));
  ensure_capacity(B, 1, dense_max, 1);
  USAP_CUDA(cudaMemcpyAsync(slots_[0], part, sizeof(int32_t) * hg_->n, cudaMemcpyHostToDevice, st_));
  const bool dense = B <= dense_max;
  prepare_nodal_blocks(slots_[0], B, dense);
  entropy_launch(slots_[0], B, dense);
  USAP_CUDA(cudaMemcpyAsync(h_ctl_, ctl_, sizeof(NodalCtl), cudaMemcpyDeviceToHost, st_));
  USAP_CUDA(cudaStreamSynchronize(st_));
  return add_sat(q32_host(model_S(hg_->n, hg_->e, B)), -static_cast<long long>(h_ctl_->entropy_acc));
}

void Job::op_merge_phase(const int32_t* part, int32_t B, int32_t K, int32_t stage, uint64_t seed,
                         int32_t* best_s, int64_t* best_q, int32_t* prop_s, int64_t* prop_q, int prec,
                         double* prop_f, int64_t* flips, int32_t dense_max) {
  if (!loaded()) throw Error(USAP_ERR_STATE, "no graph loaded");
  if (K < 1) throw Error(USAP_ERR_INVALID, "K must be >= 1");
  USAP_CUDA(cudaSetDevice(device_));
  ensure_capacity(B, K, dense_max, 1);
  if (prec < 0 || prec > 3) throw Error(USAP_ERR_INVALID, "precision must be 0, 1, 2 or 3");
  prec_ = prec;
  if (prec_) USAP_CUDA(cudaMemsetAsync(f32d_, 0, 2 * sizeof(F32Tally), st_));
  USAP_CUDA(cudaMemcpyAsync(slots_[0], part, sizeof(int32_t) * hg_->n, cudaMemcpyHostToDevice, st_));
  merge_phase(slots_[0], B, K, static_cast<uint32_t>(stage), seed, B <= std::min(dense_max, kDenseMergeMax));
  const size_t nk = static_cast<size_t>(B) * K;
  USAP_CUDA(cudaMemcpyAsync(best_s, best_s_, sizeof(int32_t) * B, cudaMemcpyDeviceToHost, st_));
  USAP_CUDA(cudaMemcpyAsync(best_q, best_q_, sizeof(int64_t) * B, cudaMemcpyDeviceToHost, st_));
  if (prop_s) USAP_CUDA(cudaMemcpyAsync(prop_s, prop_s_, sizeof(int32_t) * nk, cudaMemcpyDeviceToHost, st_));
  if (prop_q)
    USAP_CUDA(cudaMemcpyAsync(prop_q, merge_prec() ? prop_x_ : prop_q_, sizeof(int64_t) * nk, cudaMemcpyDeviceToHost, st_));
  if (merge_prec() && prop_f) USAP_CUDA(cudaMemcpyAsync(prop_f, prop_f_, sizeof(double) * nk, cudaMemcpyDeviceToHost, st_));
  F32Tally m{0, 0, 0, 0.0};
  if (merge_prec()) USAP_CUDA(cudaMemcpyAsync(&m, f32d_, sizeof(m), cudaMemcpyDeviceToHost, st_));
  USAP_CUDA(cudaStreamSynchronize(st_));
  if (flips) *flips = static_cast<int64_t>(m.flips);
  prec_ = 0;
}

void Job::op_merge_apply(int32_t* part, int32_t B, const int32_t* best_s, const int64_t* best_q,
                         int32_t btm, int32_t* B_new, int32_t* merged) {
  if (!loaded()) throw Error(USAP_ERR_STATE, "no graph loaded");
  USAP_CUDA(cudaSetDevice(device_));
  for (int32_t i = 0; i < B; i++)
    if (best_s[i] < 0 || best_s[i] >= B) throw Error(USAP_ERR_INVALID, "best merge target out of range");
  ensure_capacity(B, 1, 1, 1);
  USAP_CUDA(cudaMemcpyAsync(slots_[0], part, sizeof(int32_t) * hg_->n, cudaMemcpyHostToDevice, st_));
  USAP_CUDA(cudaMemcpyAsync(best_s_, best_s, sizeof(int32_t) * B, cudaMemcpyHostToDevice, st_));
  USAP_CUDA(cudaMemcpyAsync(best_q_, best_q, sizeof(int64_t) * B, cudaMemcpyHostToDevice, st_));
  int32_t m = merge_apply(slots_[0], B, btm);
  USAP_CUDA(cudaMemcpyAsync(part, slots_[0], sizeof(int32_t) * hg_->n, cudaMemcpyDeviceToHost, st_));
  USAP_CUDA(cudaStreamSynchronize(st_));
  *merged = m;
  *B_new = B - m;
}

void Job::op_nodal_batch(int32_t* part, int32_t B, int32_t dense_max, int32_t beg, int32_t end,
                         int32_t itr, int32_t stage, uint64_t seed, int32_t* prop_s, int64_t* prop_q,
                         int32_t* prop_ninf, int64_t* cum_q, int32_t* cum_ninf, int64_t* moves, int prec,
                         double* prop_f, int64_t* flips) {
  if (!loaded()) throw Error(USAP_ERR_STATE, "no graph loaded");
  if (beg < 0 || end > hg_->n || beg > end) throw Error(USAP_ERR_INVALID, "batch range out of bounds");
  USAP_CUDA(cudaSetDevice(device_));
  if (prec < 0 || prec > 3) throw Error(USAP_ERR_INVALID, "precision must be 0, 1, 2 or 3");
  prec_ = prec;
  ensure_capacity(B, 1, dense_max, 1);
  USAP_CUDA(cudaMemcpyAsync(slots_[0], part, sizeof(int32_t) * hg_->n, cudaMemcpyHostToDevice, st_));
  const bool dense = B <= dense_max;
  prepare_nodal_blocks(slots_[0], B, dense);
  USAP_CUDA(cudaMemsetAsync(ctl_, 0, sizeof(NodalCtl), st_));
  h_ctl_->itr = itr;
  USAP_CUDA(cudaMemcpyAsync(&ctl_->itr, &h_ctl_->itr, sizeof(int), cudaMemcpyHostToDevice, st_));
  const CtlArgs ca{0, 1, 0.0, 0.0, ide_q_, ide_n_, 0, 0};
  nodal_batch(slots_[0], B, dense, beg, end, static_cast<uint32_t>(stage), seed, true, 2, ca);
  const int32_t cnt = end - beg;
  USAP_CUDA(cudaMemcpyAsync(part, slots_[0], sizeof(int32_t) * hg_->n, cudaMemcpyDeviceToHost, st_));
  if (prop_s) USAP_CUDA(cudaMemcpyAsync(prop_s, rp_s_, sizeof(int32_t) * cnt, cudaMemcpyDeviceToHost, st_));
  if (prop_q) USAP_CUDA(cudaMemcpyAsync(prop_q, rp_q_, sizeof(int64_t) * cnt, cudaMemcpyDeviceToHost, st_));
  if (prop_ninf) USAP_CUDA(cudaMemcpyAsync(prop_ninf, rp_n_, sizeof(int32_t) * cnt, cudaMemcpyDeviceToHost, st_));
  if (prec_ && prop_f) USAP_CUDA(cudaMemcpyAsync(prop_f, rp_f_, sizeof(double) * cnt, cudaMemcpyDeviceToHost, st_));
  USAP_CUDA(cudaMemcpyAsync(h_ctl_, ctl_, sizeof(NodalCtl), cudaMemcpyDeviceToHost, st_));
  USAP_CUDA(cudaStreamSynchronize(st_));
  prec_ = 0;
  if (cum_q) *cum_q = static_cast<int64_t>(h_ctl_->cum_q);
  if (cum_ninf) *cum_ninf = h_ctl_->cum_ninf;
  if (moves) *moves = static_cast<int64_t>(h_ctl_->moves);
  if (flips) *flips = static_cast<int64_t>(h_ctl_->f32.flips);
}

}  // namespace usap
