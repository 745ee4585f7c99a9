// One partitioning job: a graph resident in HBM plus the state of a solve.
#pragma once

#include <chrono>
#include <functional>
#include <future>
#include <memory>
#include <condition_variable>
#include <mutex>
#include <string>
#include <cstdint>
#include <vector>

#include "../../include/usap.h"
#include "engine.h"

namespace usap {

// upper estimate of the device memory one solve holds (server.cpp)
int64_t solve_footprint_bytes(int64_t n, int64_t e, int64_t dense_max, bool weighted, bool float_ds);
// the largest B held as a dense tile: the caller's dense_max, or by default
// 4096 (exact and FP32 modes) and 16384 with the float nodal dS, whose
// proposals read whole rows (on sorted views that is a binary search per
// block); 16384 blocks is a 2 GB tile pair
inline int32_t effective_dense_max(const usap_params& p) {
  return p.dense_max > 0 ? p.dense_max : (p.precision == 3 ? 16384 : 4096);
}

struct HostGraph {
  int32_t n = 0;
  int64_t e = 0;
  int64_t wtot = 0;
  bool unit = true;
  std::vector<int32_t> src, dst, w;
  std::vector<int32_t> out_ptr, out_idx, out_w, in_ptr, in_idx, in_w, kout, kin;
  // in-lists ordered by source vertex id (the transpose _scc builds,
  // graph_parallel.hpp:518-523), prepared once at load
  std::vector<int32_t> tptr, tidx;
  // the edge list was ordered by source: the in-lists are that transpose
  // already, and tptr/tidx stay empty
  bool transpose_is_in = false;
  // first 32-edge chunk of each vertex (n + 1 entries; GraphDev::chunks)
  std::vector<int64_t> chunk_ptr;
  // the out/in lists and weighted degrees are filled already (built on the
  // device from a parsed TSV, build_csr_device)
  bool csr_built = false;
};

// _scc + _dfs_itr (graph_parallel.hpp:514-603), host side; scc_prepare
// builds the transpose it walks (once per graph)
void scc_prepare(HostGraph& g);
// out- and in-lists (and weighted degrees) from h.src/dst/w in file order
void build_csr(HostGraph& h);
int32_t scc_arrays(int32_t n, int64_t e, const int32_t* optr, const int32_t* oidx, const int32_t* tptr,
                   const int32_t* tidx, int32_t dfs_depth, int32_t* part);
int32_t scc_host(const HostGraph& g, int32_t dfs_depth, int32_t* part);

// host evaluation (evaluate.hpp:18-266 scores + NMI + Hungarian accuracy)
void evaluate_host(const int32_t* truth, const int32_t* given, int64_t n, usap_scores* out);
// labels renumbered 0..B-1 in ascending order of their values; returns B
int32_t compact_labels(const int32_t* init, int32_t n, int32_t* part);

// edges parsed on the device from the text of a reference-format .tsv
// file (kernels_tsv.cu): 0-based ids in file order, weights empty when all
// are 1; max_src is the reference's N
struct TsvEdges {
  std::vector<int32_t> src, dst, w;
  int32_t max_src = 0, max_id = 0;
};
// With `graph` given, the parsed edges (0-based, n = the given n or else the
// largest source id) and their out/in lists, built on the device by
// build_csr_device, are also returned there.
TsvEdges parse_tsv_device(int device, const char* text, int64_t len, int32_t n = 0, HostGraph* graph = nullptr);
// out/in lists and weighted degrees of h's edges (h.n, h.e, h.src, h.unit
// set) from the same edges in device memory (kernels_csr.cu); alloc
// returns stream-ordered device memory freed by the caller
void build_csr_device(const int32_t* d_src, const int32_t* d_dst, const int32_t* d_w, HostGraph& h,
                      cudaStream_t st, const std::function<void*(size_t)>& alloc);
void scan_exclusive_i32(const int32_t* in, int64_t m, int32_t* out, cudaStream_t st,
                        const std::function<void*(size_t)>& alloc);
// initial blocks on the device (init_mode 2, kernels_init.cu): compact
// labels of n vertices into part (device), returns B; *rounds: matching rounds
int32_t device_initial_blocks(const GraphDev& g, int32_t* part, cudaStream_t st, int* rounds);

// the same scores from device arrays on `device` (kernels_eval.cu)
void evaluate_device(const int32_t* truth, const int32_t* given, int64_t n, int device, usap_scores* out);

// _prepare_for_partition_next (graph_parallel.hpp:1322-1365) on slot ids
struct GoldenPoint {
  int32_t B = 0;
  double S = 0.0;      // description length (model term + Q32 data term)
  int64_t S_q = 0;     // the same in Q32, saturated beyond +-2^31
  bool finite = false;
  int32_t slot = -1;
};

struct Golden {
  GoldenPoint large, med, small;
  // returns true when the search is over (answer: med)
  bool step(int32_t B, double S, int64_t S_q, int32_t cur_slot, float rate, int32_t* restore_slot,
            int32_t* btm);
};

int32_t reduce_blocks(int32_t B, float rate);   // (size_t)_P.B * rate, :340
double model_S(int64_t n, int64_t e, int32_t B);   // :1314-1316
// t in Q32, saturated to the int64 range (|t| >= 2^31 saturates)
long long q32_host(double t);
// a + b in int64, saturated
long long add_sat(long long a, long long b);
// description length from the model term and the Q32 data term, in the
// order both the kernels and the oracle evaluate it
inline double desc_length(double model, long long data_q) {
  return model + static_cast<double>(data_q) / 4294967296.0;
}

// A graph loaded into HBM (CSR, edge list, log table, hub list); read-only
// once loaded and shared by every job that solves it.  Its device arrays
// are allocated and released on its own stream.
// largest B whose merge phase reads the dense tile (row scans, K B^2 reads)
constexpr int32_t kDenseMergeMax = 4096;

// the reference's default DFS depth (graph_parallel.hpp:51)
constexpr int32_t kDefaultDfsDepth = 20;

struct GraphResident {
  explicit GraphResident(int device);
  ~GraphResident();
  GraphResident(const GraphResident&) = delete;
  GraphResident& operator=(const GraphResident&) = delete;
  // the initial blocks for the default DFS depth, computed on a host thread
  // while the graph uploads; the first solve takes them (later solves
  // compute their own).  True with B and part filled when they were there.
  bool take_initial_blocks(int32_t* B, std::vector<int32_t>* part);
  int device;
  cudaStream_t st = nullptr;
  std::mutex scc_mu;
  std::future<int32_t> scc_b;          // B of scc_part, once the host thread is done
  std::vector<int32_t> scc_part;
  std::shared_ptr<const DeviceLogTable> logs;   // log k for k <= the total edge weight
  HostGraph hg;
  GraphDev g;                      // hkey/hwo/hwi belong to the jobs
  std::vector<int32_t> hub_ids;    // vertices of degree > kHubDegree, ascending
  int32_t* hubs_dev = nullptr;
  double h2d_ms = 0;
  long long h2d_bytes = 0;
};

// Graph_P constructor / load_graph_from_tsv (graph_parallel.hpp:251-317)
// (pre: a graph whose edges and lists are already on the host, e.g. from
// parse_tsv_device; `in` is then ignored)
std::shared_ptr<GraphResident> load_graph(int device, const usap_graph& in, HostGraph* pre = nullptr);

// Runs the dense nodal phases of concurrent solves together in single
// cooperative launches (k_nodal_gang); see gang.cpp.
class NodalGang {
 public:
  explicit NodalGang(int device);
  ~NodalGang();
  NodalGang(const NodalGang&) = delete;
  NodalGang& operator=(const NodalGang&) = delete;
  // a solve starts / ends: a launch waits for every solve in progress to
  // reach its nodal phase (or for kGangWait)
  void enter();
  void leave();
  // runs this nodal phase in the next gang launch, after the work queued on
  // job_stream; returns when it is done
  void run(const PhaseArgs& pa, cudaStream_t job_stream);
  long long launches() const { return launches_; }
  long long phases() const { return jobs_run_; }
  double ms() const { return ms_; }

 private:
  struct Pending {
    PhaseArgs pa;
    cudaEvent_t ready = nullptr;
    std::chrono::steady_clock::time_point since;
    bool done = false;
    bool waited = false;
    std::string error;
  };
  bool ready_to_launch() const;
  void launch(const std::vector<Pending*>& batch);
  int device_;
  int grid_ = 0;
  std::mutex mu_;
  std::condition_variable cv_;
  std::vector<Pending*> pending_;
  int live_ = 0;
  bool busy_ = false;
  cudaStream_t st_ = nullptr;
  PhaseArgs* h_jobs_ = nullptr;
  PhaseArgs* d_jobs_ = nullptr;
  GangCtl* h_ctl_ = nullptr;
  GangCtl* d_ctl_ = nullptr;
  long long launches_ = 0, jobs_run_ = 0;
  double ms_ = 0.0;
  std::chrono::steady_clock::time_point last_end_{};
};

class Job {
 public:
  explicit Job(int device);
  ~Job();
  Job(const Job&) = delete;
  Job& operator=(const Job&) = delete;

  void load(const usap_graph& g);
  // a graph whose adjacency lists are built already (parse_tsv_device)
  void load_host(HostGraph&& h);
  // solve a graph that is already resident (shared with other jobs)
  void attach(std::shared_ptr<GraphResident> gr);
  bool loaded() const { return hg_ != nullptr; }
  const HostGraph& host_graph() const {
    static const HostGraph empty;
    return hg_ ? *hg_ : empty;
  }
  const std::shared_ptr<GraphResident>& graph() const { return gr_; }
  // host threads sleep (instead of spinning) while waiting for the device
  void set_blocking_wait(bool on) { blocking_wait_ = on; }
  // dense nodal phases go to this gang instead of a launch of their own
  void set_gang(NodalGang* g) { gang_ = g; }
  void set_trace(usap_trace_fn fn, void* user) {
    trace_ = fn;
    trace_user_ = user;
  }
  // failure injection for tests: the next cooperative nodal-phase launch
  // has CTA `hold` withhold its barrier arrivals and waits limited to
  // timeout_ns, so the launch ends with USAP_ERR_INTERNAL
  void arm_barrier_test(int hold, unsigned long long timeout_ns) {
    bar_test_hold_ = hold;
    bar_test_timeout_ns_ = timeout_ns;
  }
  // init (n labels >= 0, renumbered 0..B-1 in ascending order) replaces
  // the SCC pass as the initial partition when given
  void partition(const usap_params& p, int32_t* out_assign, usap_result* res, const int32_t* init = nullptr);
  // streaming input: the resident graph becomes its edges followed by
  // these, with n grown to cover them
  void add_edges(const usap_graph& delta);
  // bf::evaluate scores of the last partition() result against truth (host
  // array of n labels), computed on the device where the result lies
  void evaluate_last(const int32_t* truth, usap_scores* out);
  // drops the graph (its device memory is freed when no job holds it);
  // the solver state stays allocated for the next graph
  void detach() { free_graph(); }
  int device() const { return device_; }

  // phase-level operations on host buffers
  int32_t op_scc(int32_t depth, int32_t* part);
  void op_build(const int32_t* part, int32_t B, int32_t dense_max, int32_t* M, int32_t* dout,
                int32_t* din);
  int64_t op_entropy(const int32_t* part, int32_t B, int32_t dense_max);
  // prec: precision mode (1, 2: prop_q then gets the exact values,
  // prop_f the FP32 ones, *flips the blocks whose FP32 choice differs)
  void op_merge_phase(const int32_t* part, int32_t B, int32_t K, int32_t stage, uint64_t seed,
                      int32_t* best_s, int64_t* best_q, int32_t* prop_s, int64_t* prop_q, int prec = 0,
                      double* prop_f = nullptr, int64_t* flips = nullptr, int32_t dense_max = 1);
  void op_merge_apply(int32_t* part, int32_t B, const int32_t* best_s, const int64_t* best_q,
                      int32_t btm, int32_t* B_new, int32_t* merged);
  void op_nodal_batch(int32_t* part, int32_t B, int32_t dense_max, int32_t beg, int32_t end,
                      int32_t itr, int32_t stage, uint64_t seed, int32_t* prop_s, int64_t* prop_q,
                      int32_t* prop_ninf, int64_t* cum_q, int32_t* cum_ninf, int64_t* moves, int prec = 0,
                      double* prop_f = nullptr, int64_t* flips = nullptr);

  double last_h2d_ms() const { return gr_ ? gr_->h2d_ms : 0.0; }
  long long last_h2d_bytes() const { return gr_ ? gr_->h2d_bytes : 0; }

 private:
  void free_graph();
  void free_state();
  void free_vertex_state();   // buffers sized by the number of vertices
  void ensure_capacity(int32_t B, int32_t K, int32_t dense_max, int32_t maxitr);
  // block structures for a nodal phase / batch
  void prepare_nodal_blocks(const int32_t* part, int32_t B, bool dense);
  void merge_phase(const int32_t* part, int32_t B, int32_t K, uint32_t stage, uint64_t seed, bool dense);
  int32_t merge_apply(int32_t* part, int32_t B, int32_t btm);
  void entropy_launch(const int32_t* part, int32_t B, bool dense);
  void nodal_batch(int32_t* part, int32_t B, bool dense, int32_t beg, int32_t end, uint32_t stage,
                   uint64_t seed, bool first_of_sweep, int stats, const CtlArgs& ctl_args);
  NodalArgs nodal_args(int32_t* part, int32_t B, int32_t beg, int32_t end, uint32_t stage, uint64_t seed,
                       int stats) const;
  // a stage's whole nodal phase in one persistent launch (dense tile);
  // returns the kernel's duration in ms when `timed`
  float nodal_phase(int32_t* part, int32_t B, uint32_t stage, uint64_t seed, int W, double thr,
                    double model_d, int32_t maxitr, int stats, int grid, bool timed);
  // one nodal sweep (entropy, sweep start, every batch), launched directly
  // or recorded into a CUDA graph
  void enqueue_sweep(int32_t* part, int32_t B, bool dense, uint32_t stage, uint64_t seed, int W,
                     double thr, double model_d, int stats);
  void emit_trace(int kind, int stage, int itr, int beg, int32_t B, const int32_t* part,
                  bool dense, long long S_q, int S_ninf, long long cum_q, int cum_ninf,
                  long long moves);
  DenseView dense_view() const { return DenseView{M_, Mt_, ld_, CS_, cld_}; }
  HubList hubs_for(int32_t beg, int32_t end, int32_t B) const;

  StreamPair streams() const { return StreamPair{st_, st_side_, ev_fork_, ev_join_}; }

  int device_;
  cudaStream_t st_ = nullptr;
  cudaStream_t st_side_ = nullptr;   // hub CTAs overlap the warp kernel here
  cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
  cudaEvent_t ev_wait_ = nullptr;
  cudaEvent_t ev_sweep_[2] = {nullptr, nullptr};   // sweep done + control copied
  NodalCtl* h_ring_ = nullptr;                     // pinned, two control copies
  bool blocking_wait_ = false;
  NodalGang* gang_ = nullptr;
  void wait();
  std::shared_ptr<GraphResident> gr_;
  const HostGraph* hg_ = nullptr;
  GraphDev g_;                       // the graph's arrays + this job's hub scratch
  int32_t *hkey_ = nullptr, *hwo_ = nullptr, *hwi_ = nullptr;
  // state
  int32_t bcap_ = 0, kcap_ = 0, dcap_ = 0, icap_ = 0;
  int32_t ncap_ = 0;          // vertices the per-vertex buffers hold
  int64_t hcap_ = 0;          // hub scratch slots
  size_t units_cap_ = 0;      // ints of units_
  int32_t bs_ = 1;   // nodal batch size of the current solve
  int bar_test_hold_ = -1;                 // arm_barrier_test
  unsigned long long bar_test_timeout_ns_ = 0;
  int32_t* slots_[4] = {nullptr, nullptr, nullptr, nullptr};
  int32_t* move_to_ = nullptr;
  int32_t* from_ = nullptr;
  const int32_t* last_part_ = nullptr;   // slot holding the last solve's result
  int32_t* batch_hub_ = nullptr;     // first hub of each batch of size bs_
  int32_t* unit_ptr_ = nullptr;      // first work unit of each batch
  int2* units_ = nullptr;            // work units of the persistent kernel
  int32_t batch_hub_bs_ = 0;
  int32_t batch_hub_cap_ = 0;
  int32_t *dout_ = nullptr, *din_ = nullptr;
  int *M_ = nullptr, *Mt_ = nullptr, *CS_ = nullptr;
  // precision mode 3: old-state term tables of the persistent kernel (ld_ x ld_ floats each)
  static constexpr int32_t kRefTabMaxB = 4096;
  float *Trow_ = nullptr, *Tcol_ = nullptr;
  size_t tcap_ = 0;
  int ld_ = 0, cld_ = 0;
  SortedBuilder sb_;
  int32_t* prop_s_ = nullptr;
  long long* prop_q_ = nullptr;
  long long* prop_x_ = nullptr;   // precision modes 1, 2: exact merge dS beside the FP32 key in prop_q_
  double* prop_f_ = nullptr;
  int32_t* best_s_ = nullptr;
  long long* best_q_ = nullptr;
  long long* best_x_ = nullptr;
  // precision mode of the current solve; with modes 1, 2: [0] merge
  // proposals, [1].flips merge-order inversions
  int prec_ = 0;
  bool shadow_ = false;   // precision 3: evaluate the exact FP64 dS beside the float one
  // the merge phase's mode: mode 3 changes only the nodal dS (the
  // reference's float merge dS does not move its solve) and keeps merges exact
  int merge_prec() const { return prec_ == 3 ? 0 : prec_; }
  F32Tally* f32d_ = nullptr;
  unsigned long long *skeys_ = nullptr, *skeys_alt_ = nullptr;
  int32_t *sidx_ = nullptr, *sidx_alt_ = nullptr;
  int32_t *union_work_ = nullptr, *root_ = nullptr, *present_ = nullptr, *newlabel_ = nullptr;
  int32_t* merged_dev_ = nullptr;
  void* cub_tmp_ = nullptr;
  size_t cub_bytes_ = 0;
  NodalCtl* ctl_ = nullptr;
  NodalCtl* h_ctl_ = nullptr;   // pinned
  long long* ide_q_ = nullptr;
  int* ide_n_ = nullptr;
  int32_t *rp_s_ = nullptr, *rp_n_ = nullptr;   // replay proposal buffers [n]
  long long* rp_q_ = nullptr;
  double* rp_f_ = nullptr;
  // stats
  std::vector<cudaEvent_t> ev_pool_;
  size_t ev_used_ = 0;
  // trace
  usap_trace_fn trace_ = nullptr;
  void* trace_user_ = nullptr;
  long long trace_prev_moves_ = 0;
  int trace_mask_ = 7;
  bool trace_on(int kind) const { return trace_ && (trace_mask_ >> (kind - 1) & 1); }
};

}  // namespace usap
