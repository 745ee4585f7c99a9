// Edge-list ingest on the device: the text of a reference-format .tsv file
// (load_graph_from_tsv, graph_parallel.hpp:251-317; one edge per line,
// "from<TAB>to<TAB>weight", 1-based ids) is copied to the GPU once and parsed
// there: newline positions by per-block counts and a scan, then one thread
// per line.  Each field is read as the reference reads it: the text up to
// the next tab, leading whitespace skipped, the digits that follow (std::stoul;
// std::stof for the weight, whose value is then truncated to an integer as
// the reference's cast to the integer weight type does).  A line with no
// second tab gets the whole line as its weight field (the reference's
// find('\t') returns npos and npos + 1 wraps to 0), i.e. the weight equals
// the source id.  A line that std::stoul would reject (no digits, an empty
// line) is an error naming the line.  The parsed edges come back in file
// order for the host-side adjacency build, which the host-side initial
// blocks need anyway.
#include <cub/cub.cuh>

#include <climits>
#include <string>
#include <vector>

#include "job.h"

namespace usap {

namespace {

constexpr int kThreads = 256;
constexpr int kBytesPerThread = 16;
constexpr int kChunk = kThreads * kBytesPerThread;   // bytes per block

struct TsvStatus {
  unsigned long long bad;   // (line << 3) | kind of the first malformed line, all ones if none; kind
                            // 1: a field without digits, 2: id 0, 3: weight not positive, 4: value too large
  int max_src, max_id;
  int nonunit;
};

__global__ void k_tsv_count(const char* __restrict__ text, int64_t len, int* __restrict__ counts) {
  const int64_t base = blockIdx.x * static_cast<int64_t>(kChunk) + threadIdx.x * static_cast<int64_t>(kBytesPerThread);
  int c = 0;
  for (int k = 0; k < kBytesPerThread; k++) {
    const int64_t i = base + k;
    if (i < len && text[i] == '\n') c++;
  }
  typedef cub::BlockReduce<int, kThreads> Reduce;
  __shared__ typename Reduce::TempStorage tmp;
  const int total = Reduce(tmp).Sum(c);
  if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

// newline positions in order: block offsets from the scan of the counts
__global__ void k_tsv_positions(const char* __restrict__ text, int64_t len, const int* __restrict__ offsets,
                                int64_t* __restrict__ nl) {
  const int64_t base = blockIdx.x * static_cast<int64_t>(kChunk) + threadIdx.x * static_cast<int64_t>(kBytesPerThread);
  int c = 0;
  for (int k = 0; k < kBytesPerThread; k++) {
    const int64_t i = base + k;
    if (i < len && text[i] == '\n') c++;
  }
  typedef cub::BlockScan<int, kThreads> Scan;
  __shared__ typename Scan::TempStorage tmp;
  int before = 0;
  Scan(tmp).ExclusiveSum(c, before);
  int64_t o = offsets[blockIdx.x] + before;
  for (int k = 0; k < kBytesPerThread; k++) {
    const int64_t i = base + k;
    if (i < len && text[i] == '\n') nl[o++] = i;
  }
}

__device__ __forceinline__ bool is_space(char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f' || c == '\v';
}

// std::stoul of text[b, e): leading whitespace, optional '+', digits; false
// when there are no digits; *big when the value exceeds 2^31 - 1
__device__ bool parse_ul(const char* t, int64_t b, int64_t e, long long* v, bool* big) {
  while (b < e && is_space(t[b])) b++;
  if (b < e && t[b] == '+') b++;
  long long x = 0;
  bool any = false;
  while (b < e && t[b] >= '0' && t[b] <= '9') {
    any = true;
    if (x < (1ll << 40)) x = x * 10 + (t[b] - '0');
    b++;
  }
  *big = x > INT_MAX;
  *v = x;
  return any;
}

// the integer part of std::stof of text[b, e) (digits, an optional
// fraction, no exponent); false without digits
__device__ bool parse_weight(const char* t, int64_t b, int64_t e, long long* v, bool* big, bool* neg) {
  while (b < e && is_space(t[b])) b++;
  *neg = false;
  if (b < e && (t[b] == '+' || t[b] == '-')) {
    *neg = t[b] == '-';
    b++;
  }
  long long x = 0;
  bool any = false;
  while (b < e && t[b] >= '0' && t[b] <= '9') {
    any = true;
    if (x < (1ll << 40)) x = x * 10 + (t[b] - '0');
    b++;
  }
  if (b < e && t[b] == '.') {
    b++;
    while (b < e && t[b] >= '0' && t[b] <= '9') {
      any = true;
      b++;
    }
  }
  *big = x > INT_MAX;
  *v = x;
  return any;
}

__device__ __forceinline__ int64_t find_tab(const char* t, int64_t b, int64_t e) {
  while (b < e && t[b] != '\t') b++;
  return b;   // e when there is none
}

__global__ void k_tsv_parse(const char* __restrict__ text, int64_t len, const int64_t* __restrict__ nl, int64_t lines,
                            int32_t* __restrict__ src, int32_t* __restrict__ dst, int32_t* __restrict__ w,
                            TsvStatus* st) {
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < lines;
       k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = k == 0 ? 0 : nl[k - 1] + 1;
    const int64_t e = nl[k];   // the last line ends at len (an appended entry)
    int kind = 0;
    long long a = 0, c = 0, x = 0;
    bool big1 = false, big2 = false, big3 = false, neg = false;
    const int64_t t1 = find_tab(text, b, e);
    if (!parse_ul(text, b, t1, &a, &big1)) kind = 1;
    // no tab: the reference's next field starts at npos + 1 = 0, the line start
    const int64_t s2 = t1 < e ? t1 + 1 : b;
    const int64_t t2 = find_tab(text, s2, e);
    if (!kind && !parse_ul(text, s2, t2, &c, &big2)) kind = 1;
    // weight field: after the second tab, or the whole line when there is none
    const int64_t s3 = t2 < e ? t2 + 1 : b;
    const int64_t t3 = t2 < e ? find_tab(text, s3, e) : e;
    if (!kind && !parse_weight(text, s3, t3, &x, &big3, &neg)) kind = 1;
    if (!kind && (big1 || big2 || big3)) kind = 4;
    if (!kind && (a == 0 || c == 0)) kind = 2;
    if (!kind && (neg || x <= 0)) kind = 3;
    if (kind) {
      atomicMin(&st->bad, (static_cast<unsigned long long>(k) << 3) | static_cast<unsigned long long>(kind));
      continue;
    }
    src[k] = static_cast<int32_t>(a - 1);
    dst[k] = static_cast<int32_t>(c - 1);
    w[k] = static_cast<int32_t>(x);
    atomicMax(&st->max_src, static_cast<int>(a));
    atomicMax(&st->max_id, static_cast<int>(a > c ? a : c));
    if (x != 1) st->nonunit = 1;
  }
}

}  // namespace

TsvEdges parse_tsv_device(int device, const char* text, int64_t len, int32_t n, HostGraph* graph) {
  if (!text || len < 0) throw Error(USAP_ERR_INVALID, "null text");
  // line counts and offsets are int32: at most 2^31 - 1 bytes of text
  if (len > static_cast<int64_t>(INT_MAX)) throw Error(USAP_ERR_LIMIT, "tsv text above 2^31 - 1 bytes");
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
  TsvEdges out;
  if (len == 0) return out;
  char* d_text = static_cast<char*>(alloc(static_cast<size_t>(len)));
  USAP_CUDA(cudaMemcpyAsync(d_text, text, static_cast<size_t>(len), cudaMemcpyHostToDevice, st));
  const int blocks = static_cast<int>((len + kChunk - 1) / kChunk);
  int* counts = static_cast<int*>(alloc(sizeof(int) * (blocks + 1)));
  int* offsets = static_cast<int*>(alloc(sizeof(int) * (blocks + 1)));
  k_tsv_count<<<blocks, kThreads, 0, st>>>(d_text, len, counts);
  USAP_LAUNCHED();
  USAP_CUDA(cudaMemsetAsync(counts + blocks, 0, sizeof(int), st));
  size_t tmp_bytes = 0;
  USAP_CUB(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, counts, offsets, blocks + 1, st));
  void* tmp = alloc(tmp_bytes);
  USAP_CUB(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, counts, offsets, blocks + 1, st));
  int newlines = 0;
  char last = 0;
  USAP_CUDA(cudaMemcpyAsync(&newlines, offsets + blocks, sizeof(int), cudaMemcpyDeviceToHost, st));
  USAP_CUDA(cudaMemcpyAsync(&last, d_text + len - 1, 1, cudaMemcpyDeviceToHost, st));
  USAP_CUDA(cudaStreamSynchronize(st));
  // lines: one per newline, plus the text after the last newline
  const int64_t lines = newlines + (last != '\n' ? 1 : 0);
  if (lines == 0) return out;
  int64_t* nl = static_cast<int64_t*>(alloc(sizeof(int64_t) * (lines + 1)));
  k_tsv_positions<<<blocks, kThreads, 0, st>>>(d_text, len, offsets, nl);
  USAP_LAUNCHED();
  if (last != '\n') {
    const int64_t end = len;
    USAP_CUDA(cudaMemcpyAsync(nl + lines - 1, &end, sizeof(int64_t), cudaMemcpyHostToDevice, st));
  }
  int32_t* dv = static_cast<int32_t*>(alloc(sizeof(int32_t) * 3 * lines));
  TsvStatus* ds = static_cast<TsvStatus*>(alloc(sizeof(TsvStatus)));
  const TsvStatus init{~0ull, 0, 0, 0};
  USAP_CUDA(cudaMemcpyAsync(ds, &init, sizeof(init), cudaMemcpyHostToDevice, st));
  int64_t pb = (lines + kThreads - 1) / kThreads;
  if (pb > 148 * 16) pb = 148 * 16;
  k_tsv_parse<<<static_cast<int>(pb), kThreads, 0, st>>>(d_text, len, nl, lines, dv, dv + lines, dv + 2 * lines, ds);
  USAP_LAUNCHED();
  TsvStatus hs{};
  USAP_CUDA(cudaMemcpyAsync(&hs, ds, sizeof(hs), cudaMemcpyDeviceToHost, st));
  USAP_CUDA(cudaStreamSynchronize(st));
  if (hs.bad != ~0ull) {
    static const char* what[] = {"", "a field without digits", "vertex id 0 (ids are 1-based)",
                                 "a weight that is not positive", "a value above 2^31 - 1"};
    const int kind = static_cast<int>(hs.bad & 7);
    throw Error(USAP_ERR_INVALID, "tsv line " + std::to_string(static_cast<int64_t>(hs.bad >> 3) + 1) + ": " +
                                      what[kind >= 1 && kind <= 4 ? kind : 1]);
  }
  out.src.resize(lines);
  out.dst.resize(lines);
  USAP_CUDA(cudaMemcpyAsync(out.src.data(), dv, sizeof(int32_t) * lines, cudaMemcpyDeviceToHost, st));
  USAP_CUDA(cudaMemcpyAsync(out.dst.data(), dv + lines, sizeof(int32_t) * lines, cudaMemcpyDeviceToHost, st));
  if (hs.nonunit) {
    out.w.resize(lines);
    USAP_CUDA(cudaMemcpyAsync(out.w.data(), dv + 2 * lines, sizeof(int32_t) * lines, cudaMemcpyDeviceToHost, st));
  }
  USAP_CUDA(cudaStreamSynchronize(st));
  out.max_src = hs.max_src;
  out.max_id = hs.max_id;
  if (graph) {
    // the graph of load_graph_from_tsv: N = the largest source id (:276),
    // or the caller's n; adjacency lists built here, on the device copy
    HostGraph& h = *graph;
    h.n = n > 0 ? n : out.max_src;
    if (out.max_id > h.n)
      throw Error(USAP_ERR_INVALID, "vertex id " + std::to_string(out.max_id - 1) + " >= n = " + std::to_string(h.n));
    if (lines >= (1ll << 30)) throw Error(USAP_ERR_LIMIT, "more than 2^30 edges");
    h.e = lines;
    h.unit = !hs.nonunit;
    h.wtot = 0;
    for (int32_t x : out.w) h.wtot += x;
    if (h.unit) h.wtot = lines;
    if (h.wtot >= (1ll << 24)) throw Error(USAP_ERR_LIMIT, "total edge weight must be below 2^24");
    h.src = out.src;
    h.dst = out.dst;
    h.w = out.w;
    build_csr_device(dv, dv + lines, dv + 2 * lines, h, st, alloc);
  }
  return out;
}

}  // namespace usap
