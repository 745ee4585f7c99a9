// Device state of one partitioning job and the launchers of its kernels.
//
// HBM layout (one job):
//   graph   edge list src/dst[/w] (file order), CSR out/in (int32 offsets,
//           file order inside each list), weighted degrees, log table
//           log(k) for k <= total weight (FP64);
//   state   four partition buffers (working + golden-section bracket),
//           block degrees dout/din;
//   blocks  either a dense int32 tile M and its transpose Mt (row stride
//           ld = B rounded up to 4) when B <= dense_max, or sorted sparse
//           views rebuilt from the edge list: CSR of M (row = source
//           block), CSC of M, and the symmetric rows M[u,:]+M[:,u] with
//           inclusive cumulative counts for block-order sampling;
//   merge   K proposals per block, best target/dS, union-find scratch;
//   nodal   per-vertex move target (-1 = stay), control block.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>

#include "common.cuh"
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace usap {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

void cuda_check(cudaError_t e, const char* what, const char* file, int line);
#define USAP_CUDA(x) ::usap::cuda_check((x), #x, __FILE__, __LINE__)

// runs f, turning an exception into a status and the calling thread's
// last-error message, as every extern "C" entry point does
int call_guarded(const std::function<void()>& f);

// launches of this library's own kernels and of CUB primitives on the
// calling thread (reported per solve)
struct LaunchCount {
  long long kernels = 0;
  long long cub = 0;
};
LaunchCount& launch_count();
// after each kernel launch of this library: error check + count
#define USAP_LAUNCHED()                          \
  do {                                           \
    USAP_CUDA(cudaGetLastError());               \
    ::usap::launch_count().kernels++;            \
  } while (0)
#define USAP_CUB(x)                              \
  do {                                           \
    USAP_CUDA(x);                                \
    ::usap::launch_count().cub++;                \
  } while (0)

// Vertices whose degree exceeds kHubDegree are proposed by a whole CTA;
// its neighbour-block hash holds up to kHubSmemSlots entries in shared
// memory (3 ints per slot), larger ones use the vertex's global region.
constexpr int kHubDegree = 128;
constexpr int kHubSmemSlots = 16384;
// the persistent kernels' hub table (shared memory): hubs whose table is
// larger get a region of global memory, so those kernels take any B
constexpr int kPhaseHubSlots = 8192;

// process-wide device memory pool and host tables (devmem.cu)
void pool_configure(int device);
// grows the device's memory pool to hold `bytes` (allocated and freed once,
// then kept by the pool), so that later allocations are served from it
void pool_reserve(int device, int64_t bytes);
void* dev_alloc(size_t bytes, cudaStream_t st);
void dev_free(void* p, cudaStream_t st);
std::shared_ptr<const std::vector<double>> log_table(int64_t max_k);

// The same table on a device, as FP64 values and as float pairs (the FP32
// precision modes), for k < size.  One per device for the process: graphs
// share it, and it is replaced by a larger one when a graph needs more
// entries (holders keep the table they were given alive).
struct DeviceLogTable {
  double* L = nullptr;
  float2* L2 = nullptr;
  int64_t size = 0;
  ~DeviceLogTable();
};
// the device's table with at least max_k + 1 entries; *uploaded = bytes
// copied to the device by this call (0 when the current table was enough)
std::shared_ptr<const DeviceLogTable> device_log_table(int device, int64_t max_k, int64_t* uploaded);

// Dense block matrix view: M[x*ld + y], transposed copy Mt[y*ld + x], and
// per-row chunk sums CS[u*cld + c] of M[u,i]+M[i,u] over blocks
// i in [128c, 128c+128).
struct DenseView {
  const int* M;
  const int* Mt;
  int ld;
  const int* CS;
  int cld;
};

// hub vertices of one batch: ids[lo, hi), hash capacity in shared memory
struct HubList {
  const int32_t* ids;
  int lo, hi;
  int smem_cap;
};

// main stream plus a side stream for kernels that overlap it
struct StreamPair {
  cudaStream_t main, side;
  cudaEvent_t fork, join;
};

// batch-end bookkeeping, run by the commit kernel (active = 1); the sweep
// index comes from the control block
struct CtlArgs {
  int active;
  int W;
  double thr;
  double model_d;      // model term of S; the convergence test uses model_d + S_q / 2^32
  long long* ide_q;
  int* ide_n;
  long long batch_vertices, batch_edges;
};

// Sorted sparse view built from the edge list.
struct SortedView {
  const int* rowptr;  // [B+1]
  const int* col;     // [nnz] column (target block) of each M entry, row-major sorted
  const int* val;
  const int* colptr;  // [B+1] CSC of M (may be null when not built)
  const int* row;
  const int* cval;
  const int* symptr;  // [B+1] rows of M[u,:]+M[:,u]
  const int* symcol;
  const int* symcum;  // global inclusive cumulative count
};

// Control block of a nodal phase, resident on the device so that batches
// and sweeps can be queued without host round trips.
struct NodalCtl {
  int done;          // convergence reached: later batch kernels return at once
  int S_ninf;
  int cum_ninf;
  int itr;           // index of the current sweep (set by the sweep-start kernel)
  long long S_q;     // data term of the running description length (Q32); S = model + S_q / 2^32
  unsigned long long cum_q;   // accepted dS of the current sweep (Q32, two's complement)
  unsigned long long moves;   // accepted moves (whole phase)
  unsigned long long near;    // proposals with |dS| <= 1e-9
  unsigned long long proposals;
  unsigned long long edge_visits;
  unsigned long long batches;
  unsigned long long sweeps;
  double mean;       // moving average of the previous sweeps' dS
  unsigned long long entropy_acc;  // data term accumulator of the entropy kernel
  unsigned long long bytes;        // algorithmic bytes of the nodal kernel (stats)
  unsigned int apply_done;         // CTAs of the apply kernel that have finished
  // persistent kernel: grid barrier (arrivals, generation, timeout flag)
  // and the counter that hands out a batch's vertices
  unsigned long long bar;   // arrivals (low 32 bits), convergence (bits 32-47) and move-list overflow (bits 48-63) arrivals
  int bar_err;
  unsigned int vnext;
  int gang_batch;           // gang launches: next batch of the current sweep (0: a new sweep starts)
  F32Tally f32;             // precision mode 1: FP32 decisions against the FP64 values
  unsigned long long apply_scans;   // persistent kernel: batches applied by scanning all chunks (a CTA's move list overflowed)
};

struct GraphDev {
  int32_t n = 0;
  int64_t e = 0;
  int64_t wtot = 0;
  bool unit = true;
  int32_t *src = nullptr, *dst = nullptr, *w = nullptr;
  int32_t *out_ptr = nullptr, *out_idx = nullptr, *out_w = nullptr;
  int32_t *in_ptr = nullptr, *in_idx = nullptr, *in_w = nullptr;
  // 32-edge chunks of every vertex's out- then in-list, (vertex, chunk index)
  // in vertex order; a vertex without edges has one empty chunk
  int2* chunks = nullptr;
  int64_t nchunks = 0;
  int64_t* chunk_ptr = nullptr;   // first chunk of each vertex (n + 1)
  int32_t *kout = nullptr, *kin = nullptr;
  double* logk = nullptr;
  float2* logk2 = nullptr;   // the same table as float pairs (hi, lo) for the FP32 precision modes
  // per-vertex global hash region for vertices too large for shared memory
  int64_t* hi_off = nullptr;
  int64_t hi_slots = 0;
  int32_t *hkey = nullptr, *hwo = nullptr, *hwi = nullptr;
};

// Arguments of the nodal proposal kernel.
struct NodalArgs {
  const int32_t *out_ptr, *out_idx, *out_w, *in_ptr, *in_idx, *in_w, *kout, *kin;
  const double* L;
  int unit;
  const int32_t* part;
  int B;
  const int32_t *dout, *din;
  int beg, end;
  uint32_t stage;    // the sweep index is read from ctl->itr
  uint64_t seed;
  int32_t* move_to;       // per batch vertex: the accepted target, or -1
  int32_t* from;          // per batch vertex: its block at the batch start
  int32_t* prop_s;        // optional, [end-beg]
  long long* prop_q;
  int32_t* prop_ninf;
  double* prop_f;         // optional: FP32 dS, the float pair's exact value (precision modes 1, 2)
  NodalCtl* ctl;
  const int64_t* hi_off;
  int32_t *hkey, *hwo, *hwi;
  int stats;
  int prec;               // precision mode: 0 FP64; 1, 2 decide on the FP32 dS; 3 the reference's float dS
  int shadow;             // precision 3: also evaluate the exact FP64 dS (flip counts, replay)
  const float2* L2;       // the log table as float pairs (precision modes 1, 2)
  // precision mode 3, persistent kernel: the reference's old-state terms of
  // every tile cell, recomputed at each batch start (null: computed per
  // proposal); row b, column i at b * tld + i
  float* Trow;            // M[b,i] log(M[b,i] / (d_in[i] d_out[b]))
  float* Tcol;            // M[i,b] log(M[i,b] / (d_out[i] d_in[b]))
  int tld;
};

struct MergeArgs {
  const double* L;
  const float2* L2;  // the log table as float pairs
  int prec;          // precision mode
  int B, K;
  uint32_t stage;
  uint64_t seed;
  const int32_t *dout, *din;
  int32_t* prop_s;   // [B*K]
  long long* prop_q; // the merge key: exact FP64 dS in Q32, or in precision modes 1, 2 the FP32 dS in Q32
  // precision modes 1, 2 only: the exact FP64 dS (Q32), the FP32 dS, the statistics
  long long* prop_x;
  double* prop_f;
  F32Tally* f32;
};

// Arguments of the persistent nodal-phase kernel (dense tile only).
struct PhaseArgs {
  NodalArgs a;              // beg / end are set per batch inside the kernel
  DenseView v;
  GraphDev g;
  int32_t *part, *dout, *din;
  int *M, *Mt, *CS;         // the tile behind `v`, written by the apply pass
  const int32_t* hubs;      // hub vertex ids, ascending
  const int32_t* batch_hub; // first hub of each batch (batches + 1 entries)
  const int2* units;        // per batch: vertex pairs of degree <= 64, or (v, -2) for 64 < degree <= 128
  const int32_t* unit_ptr;  // first unit of each batch (batches + 1 entries)
  const int64_t* chunk_ptr;
  int n, bs, maxitr, W;
  double thr;
  double model_d;           // model term of S for this stage's B
  long long* ide_q;
  int* ide_n;
  unsigned long long bar_timeout_ns;  // wait limit of the grid barriers (0: 200 ms)
  int bar_hold;             // failure injection: this CTA never arrives at a barrier (-1: none)
};

// Control block of a gang launch (several jobs' nodal phases at once).
constexpr int kGangMax = 64;
struct GangCtl {
  unsigned long long bar;   // grid barrier arrivals
  int bar_err;
  unsigned int vnext;       // work units handed out by the counter
  int finished[kGangMax];   // 1: the job's nodal phase is complete; 0: resume it in a later launch
};

// --- launchers (kernels_*.cu) -------------------------------------------------
void launch_dense_build(const GraphDev& g, const int32_t* part, int B, int ld, int* M, int* Mt,
                        cudaStream_t st);
void launch_degrees(const GraphDev& g, const int32_t* part, int B, int32_t* dout, int32_t* din,
                    cudaStream_t st);
void launch_log_pairs(const double* L, float2* T, int64_t n, cudaStream_t st);
void launch_entropy_dense(const GraphDev& g, DenseView v, int B, const int32_t* dout,
                          const int32_t* din, unsigned long long* acc, cudaStream_t st);
void launch_entropy_sorted(const GraphDev& g, SortedView v, const int* nnz_dev, int64_t max_nnz,
                           const int32_t* rowof, const int32_t* dout, const int32_t* din,
                           unsigned long long* acc, cudaStream_t st);

void launch_merge_propose(const GraphDev& g, SortedView v, const MergeArgs& a, cudaStream_t st);
// the same on the dense tile (B <= dense_max; M, Mt and the chunk sums current)
void launch_merge_propose_dense(DenseView v, const MergeArgs& a, cudaStream_t st);
// prop_x / best_x / f32: precision modes 1, 2 only (else null)
void launch_merge_argmin(int B, int K, const int32_t* prop_s, const long long* prop_q, const long long* prop_x,
                         int32_t* best_s, long long* best_q, long long* best_x, F32Tally* f32, cudaStream_t st);
void launch_order_flips(int B, const int32_t* order, const long long* best_x, unsigned long long* count,
                        cudaStream_t st);
void launch_merge_union(int B, const int32_t* order, const int32_t* best_s, int btm,
                        int32_t* work, int32_t* root, int32_t* merged, cudaStream_t st);
void launch_merge_relabel(int n, int B, int32_t* part, const int32_t* root, int32_t* present,
                          int32_t* newlabel, void* cub_tmp, size_t cub_bytes, cudaStream_t st);

void nodal_configure(int device);
// grid of the persistent nodal kernel on `device` (0: not available)
int nodal_phase_grid(int device);
int nodal_gang_grid(int device);
// largest B whose hub tables fit the persistent kernel's shared memory
int nodal_phase_max_blocks();
void launch_nodal_phase(const PhaseArgs& p, int grid, cudaStream_t st);
// nodal phases of K <= kGangMax jobs (PhaseArgs array in device memory)
// (the launch ends once fewer than exit_below jobs are unfinished)
// (prec: every job's precision mode)
void launch_nodal_gang(const PhaseArgs* jobs_dev, int K, GangCtl* gc, int exit_below, int grid, int prec,
                       cudaStream_t st);
void launch_nodal_propose_dense(const NodalArgs& a, DenseView v, const HubList& hubs,
                                const StreamPair& sp);
void launch_nodal_propose_sorted(const NodalArgs& a, SortedView v, const HubList& hubs,
                                 const StreamPair& sp);
void launch_chunk_sums(int B, DenseView v, int* CS, cudaStream_t st);
// applies and commits the moves of batch [beg, end) on the dense tile
// (chunks [c0, c1) of GraphDev::chunks); runs the batch-end bookkeeping
void launch_nodal_apply_commit_dense(const GraphDev& g, int32_t* part, const int32_t* move_to,
                                     const int32_t* from, int beg, int end, int64_t c0, int64_t c1,
                                     int ld, int* M, int* Mt, int cld, int* CS, int32_t* dout,
                                     int32_t* din, NodalCtl* ctl, const CtlArgs& c, cudaStream_t st);
void launch_nodal_commit(const GraphDev& g, int32_t* part, int32_t* move_to, int beg, int end,
                         int update_degrees, int32_t* dout, int32_t* din, NodalCtl* ctl,
                         const CtlArgs& c, cudaStream_t st);
void launch_ctl_sweep_start(NodalCtl* ctl, int W, const long long* ide_q,
                            const int* ide_n, cudaStream_t st);
void launch_merge_sort_keys(int B, const long long* best_q, unsigned long long* keys, int32_t* idx,
                            cudaStream_t st);

// Sort-based construction of the sparse views (CUB radix sort).
class SortedBuilder {
 public:
  void reserve(int64_t e, int bmax, cudaStream_t st);
  void release(cudaStream_t st);
  // builds row view (+ optional CSC) and symmetric rows for partition `part`
  void build(const GraphDev& g, const int32_t* part, int B, bool with_csc, bool with_sym,
             cudaStream_t st);
  SortedView view() const;
  const int* nnz_dev() const { return nnz_; }
  const int32_t* rowof() const { return rowof_; }
  int64_t max_nnz() const { return e_; }

 private:
  void sort_reduce(int64_t count, int B, int kind, cudaStream_t st);
  int64_t e_ = 0;
  int bmax_ = 0;
  unsigned long long *keys_ = nullptr, *keys_alt_ = nullptr, *ukeys_ = nullptr;
  int *vals_ = nullptr, *vals_alt_ = nullptr, *uvals_ = nullptr;
  int *nruns_ = nullptr;  // [3]: nnz of row view, CSC, sym
  int *nnz_ = nullptr;
  int *rowptr_ = nullptr, *col_ = nullptr, *val_ = nullptr, *rowof_ = nullptr;
  int *colptr_ = nullptr, *crow_ = nullptr, *cval_ = nullptr;
  int *symptr_ = nullptr, *symcol_ = nullptr, *symcum_ = nullptr;
  void* tmp_ = nullptr;
  size_t tmp_bytes_ = 0;
  bool has_csc_ = false;
};

}  // namespace usap
