/* usap-b200: C ABI of the B200 stochastic block partitioning path.
 *
 * Drop-in boundary for uSAP's entry point (chih-chun-chang/uSAP):
 *   directed edge list in -> block assignment (+ evaluation scores) out.
 * The reference exposes it as a header-only C++ class,
 *   sgp::Graph_P<W>(FileName, num_threads)   include/graph_parallel.hpp:61-78
 *   public parameters                         include/graph_parallel.hpp:40-52
 *   void partition()                          include/graph_parallel.hpp:59, :322-512
 *   const std::vector<size_t>& get_partitions()  include/graph_parallel.hpp:58
 *   num_nodes(), num_edges()                  include/graph_parallel.hpp:56-57
 * and scores through bf::evaluate(truth, given)   include/evaluate.hpp:18-266.
 * include/usap/graph_p.hpp wraps this ABI in a class of that shape.
 *
 * Conventions: plain pointers and sizes, caller-owned buffers, int32 ids.
 * Every call returns a usap_status (0 = ok, negative = error) and never
 * exits the process (the reference calls std::exit on bad input files,
 * graph_parallel.hpp:254-257); usap_last_error() gives a message for the
 * calling thread.  One usap_ctx serves one caller at a time; different
 * contexts may be used from different threads.
 */
#ifndef USAP_H
#define USAP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t usap_status;
#define USAP_OK 0
#define USAP_ERR_INVALID (-1)   /* bad argument or graph */
#define USAP_ERR_CUDA (-2)      /* CUDA runtime error */
#define USAP_ERR_OOM (-3)       /* device or host allocation failed */
#define USAP_ERR_LIMIT (-4)     /* input beyond a documented size limit */
#define USAP_ERR_NO_DEVICE (-5) /* no usable sm_100 device */
#define USAP_ERR_INTERNAL (-6)
#define USAP_ERR_STATE (-7)     /* call out of order (e.g. no graph loaded) */

/* A directed graph.  Edges are kept in the given order: a vertex's out- and
 * in-neighbour lists are in edge order, as the reference builds them from
 * the file (graph_parallel.hpp:285-290).  n = 0 takes the number of
 * vertices from the largest source id, as the reference does
 * (graph_parallel.hpp:276).  weight = NULL means unit weights (weights must
 * be positive).  Limits: n < 2^31, total weight < 2^24. */
typedef struct usap_graph {
  int32_t n;
  int64_t e;
  const int32_t* src;
  const int32_t* dst;
  const int32_t* weight;
  int32_t one_based;  /* 1: ids are 1-based like the reference's TSV files */
} usap_graph;

/* Parameters: the first group mirrors Graph_P's public members with the
 * reference defaults (graph_parallel.hpp:40-52); `beta`, `verbose` and
 * `t_block_num` are accepted and, as in the reference, not used. */
typedef struct usap_params {
  int32_t beta;                             /* 3 */
  int32_t block_size;                       /* 1024 (the reference's dense/sparse switch) */
  int32_t num_agg_proposals_per_block;      /* 10 */
  float num_block_reduction_rate;           /* 0.5 */
  int32_t max_num_nodal_itr;                /* 100 */
  int32_t num_batch_nodal_update;           /* 4 */
  double delta_entropy_threshold1;          /* 5e-4 */
  double delta_entropy_threshold2;          /* 1e-4 */
  int32_t delta_entropy_moving_avg_window;  /* 3 */
  int32_t verbose;                          /* 0 */
  int32_t dfs_depth;                        /* 20 */
  int32_t t_block_num;                      /* 20 */
  /* B200 build */
  uint64_t seed;       /* Philox key of every proposal draw */
  int32_t init_mode;   /* 0: SCC/DFS initial blocks on the host (the reference's, exact);
                          1: one block per vertex; 2: a device stand-in for the SCC pass
                          (the cells of a multi-source breadth-first search from one
                          vertex in eight; different blocks of the same kind, no host pass) */
  int32_t dense_max;   /* dense int32 tile for B <= dense_max, sorted views above; 0 (default):
                          16384 with precision 3 (its proposals read whole tile rows), else 4096 */
  int32_t device;      /* CUDA device for usap_partition (ignored by contexts) */
  int32_t stats;       /* 1: per-kernel CUDA-event timings and algorithmic byte counts */
  int32_t trace_kinds; /* trace events to emit: bit k-1 for kind k; 0 = all kinds */
  int32_t sweep_graphs;/* 1: record each stage's nodal sweep as a CUDA graph and replay it */
  int32_t persistent;  /* 1 (default): run each stage's nodal phase as one cooperative kernel
                          when the tile is dense and B <= 4096; 0: one launch per batch.
                          usap_batch_partition always uses per-batch launches. */
  int32_t persistent_ctas; /* CTAs of the cooperative kernel (one per SM); 0 = every SM */
  int32_t precision;   /* 3 (default): the reference's float nodal dS, below.
                          0: every dS term in FP64, rounded to Q32 and summed exactly.
                          1 and 2: dS also evaluated with single-precision operations only, and
                          the nodal accept and merge choices taken on that value; the exact FP64
                          value is computed beside it to count flipped decisions
                          (usap_result.fp32_*).  1: compensated FP32 -- the log table held as
                          float pairs (hi + lo), every term and sum in float-pair arithmetic
                          (TwoSum, TwoProduct by fused multiply-add), about 44 bits.  2: plain
                          FP32 terms from the rounded log table, compensated sums only (loses
                          accuracy on large counts; kept to measure that).  The description
                          length, the golden-section comparisons and the convergence test stay
                          FP64 in every mode.
                          3 (default): the reference's own single-precision nodal dS
                          (graph_parallel.hpp:1066-1215): every term count * logf((float)count /
                          (float)(d_a * d_b)) in float, added to one float accumulator in the
                          reference's term order over all B blocks; accept iff it is < 0, and the
                          accepted float values are what the convergence test sums (:428-444),
                          as in the reference.  Merges stay exact.  The rounding noise of that
                          O(B) float sum is part of the reference's behaviour: with it the solve
                          ends at the reference's block counts and NMI, where exact arithmetic
                          (mode 0, or the reference itself compiled with double) ends at fewer
                          blocks on large graphs.  usap_result.fp32_* compare it with the exact
                          value. */
  int32_t fp64_shadow; /* precision 3 only: 1 = also evaluate the exact FP64 value of every nodal
                          dS beside the float one and report the flipped decisions and errors in
                          usap_result.fp32_*; 0 (default) = skip that evaluation (it decides
                          nothing in precision 3) and leave fp32_* at 0.  The other precisions
                          always evaluate it. */
} usap_params;

typedef struct usap_result {
  int32_t B;               /* number of blocks of the returned partition */
  int32_t stages;          /* merge + nodal phases run */
  double S;                /* description length of the result: model term + data term */
  int64_t S_q;             /* the same in Q32 fixed point, saturated beyond +-2^31 */
  int64_t sweeps, batches;
  int64_t nodal_proposals, nodal_moves;
  int64_t near_threshold;  /* nodal proposals with |dS| <= 1e-9 (the deciding value: exact, or
                              the float dS in precision 3) */
  int64_t merge_shortfall; /* merges the merge order could not supply */
  int64_t edge_visits;     /* sum over proposing vertices of in+out degree */
  double ms_total, ms_init, ms_merge, ms_nodal, ms_h2d, ms_d2h;
  double ms_nodal_kernel;  /* stats: summed time of the nodal proposal kernel */
  int64_t nodal_kernel_launches;
  double nodal_kernel_bytes;  /* stats: algorithmic bytes of those launches */
  int64_t kernel_launches;    /* launches of this library's kernels during the call */
  int64_t cub_calls;          /* CUB sort/scan/reduce calls during the call */
  int64_t h2d_bytes, d2h_bytes;  /* host<->device traffic of the call */
  int64_t sweep_graph_launches;  /* nodal sweeps replayed from a captured CUDA graph */
  /* precision 1, 2 or 3: the FP32 values and decisions against the FP64
   * values of the same evaluations (zero with precision = 0) */
  int64_t fp32_nodal_evals;  /* nodal dS evaluations with a finite FP64 value */
  int64_t fp32_nodal_flips;  /* ... whose FP32 accept decision differs from FP64's */
  int64_t fp32_merge_evals;  /* merge proposals */
  int64_t fp32_merge_flips;  /* blocks whose chosen merge target differs from FP64's choice */
  int64_t fp32_order_flips;  /* adjacent pairs of the merge order that FP64 ranks the other way */
  double fp32_flip_rate;     /* fp32_nodal_flips / fp32_nodal_evals */
  double fp32_err_max;       /* largest |dS_fp32 - dS_fp64| over nodal and merge evaluations */
  double fp32_err_mean;      /* mean |dS_fp32 - dS_fp64| over nodal evaluations */
  int64_t apply_scans;       /* nodal batches of the cooperative kernel whose moves were applied by
                                scanning all of the batch's edges (a CTA accepted more moves than its
                                shared-memory list holds) instead of each CTA's own list */
  int64_t B_init;            /* blocks of the initial partition (before the first merge phase) */
} usap_result;

typedef struct usap_scores {
  double accuracy;               /* optimal block matching (Hungarian); NaN if too many blocks */
  double rand_index, adjusted_rand_index, adjusted_rand_index_exact;
  double pairwise_recall, pairwise_precision;
  double h_truth, h_given, h_truth_given, h_given_truth, mi;
  double nmi, nmi_sqrt;          /* 2 MI / (H_t + H_g), MI / sqrt(H_t H_g) */
  double missed_info, erroneous_info;
  int64_t n, b_truth, b_given;
} usap_scores;

/* Trace events for replay harnesses: one after each merge application
 * (kind 1), each nodal batch (kind 2) and each finished stage (kind 3),
 * with checksums of the partition, of M's non-zeros and of the degrees.
 * itr: the sweep of a batch (kind 2), the sweeps the stage ran (kind 3). */
typedef struct usap_trace_event {
  int32_t kind, stage, itr, batch_beg, B;
  int64_t S_q;     /* kind 2: data term of the running S (Q32; S = model term + S_q / 2^32);
                      kind 3: S in Q32, saturated beyond +-2^31 */
  int32_t S_ninf;
  int64_t cum_q;
  int32_t cum_ninf;
  int64_t moves;
  uint64_t h_part, h_M, h_deg;
} usap_trace_event;
typedef void (*usap_trace_fn)(void* user, const usap_trace_event* ev);

typedef struct usap_ctx usap_ctx;

/* --- basics ------------------------------------------------------------- */
const char* usap_version(void);
const char* usap_last_error(void);
void usap_params_default(usap_params* p);

/* One-shot solve: Graph_P(file) + partition() + get_partitions()
 * (graph_parallel.hpp:61-78, :322-512, :58).  out_assign[n] receives the
 * 0-based block of every vertex. */
usap_status usap_partition(const usap_graph* g, const usap_params* p, int32_t* out_assign,
                           usap_result* out);

/* Scores of bf::evaluate (evaluate.hpp:18-266) plus NMI, returned instead of
 * printed.  Labels are 0-based; truth label -1 marks unknown vertices. */
usap_status usap_evaluate(const int32_t* truth, const int32_t* given, int64_t n,
                          usap_scores* out);
/* The same scores from DEVICE arrays (n labels each, on `device`): the
 * contingency table, pair counts and information sums are computed on the
 * GPU, the block matching of `accuracy` on the host.  Bit-identical to
 * usap_evaluate: both form the scores from exact integer pair counts and
 * information terms summed in fixed point (2^-50).  USAP_ERR_LIMIT above
 * 2^26 table cells (truth blocks x given blocks). */
usap_status usap_evaluate_device(const int32_t* truth, const int32_t* given, int64_t n,
                                 int32_t device, usap_scores* out);

/* --- resident contexts: the graph stays in HBM across solves ------------- */
usap_status usap_ctx_create(int32_t device, usap_ctx** out);
usap_status usap_ctx_destroy(usap_ctx* ctx);
/* Graph_P constructor / load_graph_from_tsv (graph_parallel.hpp:251-317) */
usap_status usap_ctx_load(usap_ctx* ctx, const usap_graph* g);
usap_status usap_ctx_num_nodes(usap_ctx* ctx, int32_t* n, int64_t* e);
/* load_graph_from_tsv (graph_parallel.hpp:251-317) from the bytes of the
 * .tsv file (`len` bytes, host memory): the text is parsed on the device,
 * one line per edge, fields read as the reference reads them (stoul, stof
 * truncated to an integer weight; a line with no second tab takes its
 * source id as its weight, as the reference's npos arithmetic does).
 * n = 0: N = the largest source id, as in the reference.  A malformed line
 * (a field without digits, id 0, weight not positive, a value above
 * 2^31 - 1) is USAP_ERR_INVALID naming the line. */
usap_status usap_ctx_load_tsv(usap_ctx* ctx, const char* text, int64_t len, int32_t n);
/* --- streaming input (no counterpart in the reference, whose README lists
 * streaming graphs as future work, README.md:47-49) ------------------------
 * usap_ctx_add_edges appends an edge batch to the resident graph: the edge
 * list becomes the current one followed by these edges (file order), n
 * grows to max(current n, g->n, largest source id + 1).
 * usap_ctx_partition_from is partition() started from init[n] (block labels
 * >= 0, renumbered 0..B-1 in ascending order) instead of the SCC pass
 * (graph_parallel.hpp:338-342): pass the previous stage's result extended
 * with labels for the new vertices to continue a partition as edges arrive. */
usap_status usap_ctx_add_edges(usap_ctx* ctx, const usap_graph* g);
usap_status usap_ctx_partition_from(usap_ctx* ctx, const usap_params* p, const int32_t* init,
                                    int32_t* out_assign, usap_result* out);
/* Scores of the context's last partition result against truth (host array
 * of n labels), evaluated on the device where that result lies (the
 * partition itself is not copied back). */
usap_status usap_ctx_evaluate(usap_ctx* ctx, const int32_t* truth, usap_scores* out);
/* partition() on the loaded graph; out_assign may be NULL */
usap_status usap_ctx_partition(usap_ctx* ctx, const usap_params* p, int32_t* out_assign,
                               usap_result* out);
usap_status usap_ctx_set_trace(usap_ctx* ctx, usap_trace_fn fn, void* user);
/* The resident graph's adjacency (graph_parallel.hpp:285-290, insertion order
 * = file order inside each list): out_ptr/in_ptr n + 1 entries, out_idx,
 * in_idx, out_w, in_w e entries (weights 1 for an unweighted graph), kout,
 * kin the weighted degrees (n).  Any pointer may be NULL.  A graph loaded
 * with usap_ctx_load_tsv has these lists built on the device. */
usap_status usap_ctx_adjacency(usap_ctx* ctx, int32_t* out_ptr, int32_t* out_idx, int32_t* out_w,
                               int32_t* in_ptr, int32_t* in_idx, int32_t* in_w, int32_t* kout, int32_t* kin);
/* Failure injection for tests (no counterpart in the reference): in the next
 * cooperative nodal-phase launch of this context, CTA `hold_cta` never
 * arrives at its grid barriers and every barrier wait gives up after
 * timeout_ns (> 0; at most 10 s), so that solve returns USAP_ERR_INTERNAL
 * ("a grid barrier timed out").  One launch only; the context stays usable. */
usap_status usap_ctx_test_barrier_timeout(usap_ctx* ctx, int32_t hold_cta, int64_t timeout_ns);

/* --- batched form: many independent jobs on one GPU ---------------------- */
/* One job solves graphs[graph] with its own Philox seed (several jobs on the
 * same graph are independent chains).  Graphs are loaded once and shared.
 * Jobs run concurrently, each on its own stream driven by one of `workers`
 * host threads (0 = automatic: 64); their kernels overlap on the GPU, and
 * their dense nodal phases (B <= 4096) run together in cooperative "gang"
 * launches that advance every waiting job by one batch a round.  Every
 * job's result equals the result of solving it alone with the same seed. */
typedef struct usap_batch_job {
  int32_t graph;        /* index into graphs[] */
  uint64_t seed;        /* Philox seed of this chain */
  int32_t* out_assign;  /* caller buffer of that graph's n entries, or NULL */
  usap_result result;   /* filled by the call */
  usap_status status;   /* per-job status */
} usap_batch_job;

typedef struct usap_batch_stats {
  double ms_total;      /* wall time of the whole call */
  double ms_load;       /* loading the graphs */
  int32_t workers;
  int64_t kernel_launches;
  int64_t gang_launches;  /* cooperative launches that ran several jobs' nodal phases */
  int64_t gang_phases;    /* job nodal phases (or resumed parts of them) in those launches */
  double ms_gang;         /* wall time of those launches */
} usap_batch_stats;

usap_status usap_batch_partition(const usap_graph* graphs, int32_t ngraphs, const usap_params* p,
                                 usap_batch_job* jobs, int32_t njobs, int32_t workers,
                                 int32_t device, usap_batch_stats* stats);

/* --- phase-level replay operations (host buffers in and out) ------------- */
/* _scc (graph_parallel.hpp:514-603) */
usap_status usap_op_scc(usap_ctx* ctx, int32_t dfs_depth, int32_t* part, int32_t* B);
/* _initialize_edge_counts (:703-759): M (B*B row-major, may be NULL) and degrees */
usap_status usap_op_build(usap_ctx* ctx, const int32_t* part, int32_t B, int32_t dense_max,
                          int32_t* M, int32_t* dout, int32_t* din);
/* _compute_overall_entropy (:1281-1319), Q32, saturated beyond +-2^31 (reached
 * when B is near N: the model term grows like B^2 log(B^2/E)) */
usap_status usap_op_entropy(usap_ctx* ctx, const int32_t* part, int32_t B, int32_t dense_max,
                            int64_t* S_q);
/* block_merge task (:349-368): K proposals per block; prop_* may be NULL */
usap_status usap_op_merge_phase(usap_ctx* ctx, const int32_t* part, int32_t B, int32_t K,
                                int32_t stage, uint64_t seed, int32_t* best_s, int64_t* best_q,
                                int32_t* prop_s, int64_t* prop_q);
/* _carry_out_best_merges (:1225-1279); part is updated in place */
usap_status usap_op_merge_apply(usap_ctx* ctx, int32_t* part, int32_t B, const int32_t* best_s,
                                const int64_t* best_q, int32_t b_to_merge, int32_t* B_new,
                                int32_t* merged);
/* nodal_move + update tasks for one batch [beg, end) (:397-443); part is
 * updated in place; prop_* (end-beg entries) may be NULL */
usap_status usap_op_nodal_batch(usap_ctx* ctx, int32_t* part, int32_t B, int32_t dense_max,
                                int32_t beg, int32_t end, int32_t itr, int32_t stage,
                                uint64_t seed, int32_t* prop_s, int64_t* prop_q,
                                int32_t* prop_ninf, int64_t* cum_q, int32_t* cum_ninf,
                                int64_t* moves);
/* The same two operations in a given precision mode (usap_params.precision;
 * no counterpart in the reference, whose dS is single precision throughout),
 * on the path a solve takes at this B: the merge phase reads the dense tile
 * when B <= 4096 (the plain usap_op_merge_phase always uses sorted views).
 * In modes 1 and 2, dS is evaluated in FP32 beside the exact FP64 value and
 * decisions are taken on the FP32 value: prop_q gets the exact FP64 values
 * (Q32) and prop_f the FP32 ones (the float pair's value hi + lo, which is
 * exact in a double); best_q is the merge key, the chosen proposal's FP32
 * value in Q32; *flips counts the blocks whose chosen merge
 * target, or the batch vertices whose accept decision, differs from the
 * FP64 path's on the same state.  Mode 0 is the plain operation. */
usap_status usap_op_merge_phase_prec(usap_ctx* ctx, const int32_t* part, int32_t B, int32_t K,
                                     int32_t stage, uint64_t seed, int32_t precision, int32_t* best_s,
                                     int64_t* best_q, int32_t* prop_s, int64_t* prop_q, double* prop_f,
                                     int64_t* flips);
usap_status usap_op_nodal_batch_prec(usap_ctx* ctx, int32_t* part, int32_t B, int32_t dense_max,
                                     int32_t beg, int32_t end, int32_t itr, int32_t stage,
                                     uint64_t seed, int32_t precision, int32_t* prop_s, int64_t* prop_q,
                                     double* prop_f, int32_t* prop_ninf, int64_t* cum_q, int32_t* cum_ninf,
                                     int64_t* moves, int64_t* flips);

/* --- served form: a partition service on one GPU --------------------------
 * The reference has no service; this replaces a caller running Graph_P
 * objects on its own threads.  usap_server_submit copies the edge list and
 * returns a ticket at once; worker threads (each with its own streams and
 * solver state) take requests in arrival order whenever a worker is free
 * and the request's device-memory footprint fits in what running requests
 * leave of the budget, so requests that arrive while others run start as
 * soon as a slot and memory free up and their kernels overlap on the GPU.
 * out_assign must stay valid until the request is taken with poll or
 * wait.  A request's result is the same as usap_partition's for the same
 * graph and parameters (the cooperative nodal kernel is not used, since it
 * would hold every SM). */
typedef struct usap_server usap_server;
typedef struct usap_server_config {
  int32_t device;
  int32_t workers;        /* concurrent requests (0: min(32, 2 x host threads)) */
  int64_t memory_budget;  /* bytes of device memory for admitted requests (0: 80% of free) */
  int32_t reserved[4];
} usap_server_config;
typedef struct usap_server_timing {
  double ms_queued;   /* submit to start */
  double ms_running;  /* start to finish */
  double ms_latency;  /* submit to finish */
} usap_server_timing;
typedef struct usap_server_stats {
  int32_t queued, running, workers, peak_running;
  int64_t completed, failed;
  int64_t admitted_bytes, peak_admitted_bytes, memory_budget;
} usap_server_stats;
void usap_server_config_default(usap_server_config* c);
usap_status usap_server_create(const usap_server_config* cfg, usap_server** out);
/* finishes every submitted request first */
void usap_server_destroy(usap_server* s);
/* USAP_ERR_LIMIT when the request alone exceeds the memory budget */
usap_status usap_server_submit(usap_server* s, const usap_graph* g, const usap_params* p,
                               int32_t* out_assign, int64_t* ticket);
/* *done = 0: still queued or running.  *done = 1: finished and forgotten;
 * the call returns the request's own status (and message). */
usap_status usap_server_poll(usap_server* s, int64_t ticket, int32_t* done, usap_result* result,
                             usap_server_timing* timing);
usap_status usap_server_wait(usap_server* s, int64_t ticket, usap_result* result,
                             usap_server_timing* timing);
usap_status usap_server_get_stats(usap_server* s, usap_server_stats* out);

/* --- allocation-free scoring (no counterpart in the reference) ----------- */
/* The reference has no such entry point: it exists for callers that cannot
 * allocate device memory at the moment they need a score (a host whose own
 * allocator already owns the memory budget, or a loop that cannot take the
 * device-wide synchronisation of cudaMalloc/cudaFree).
 *
 * Same value as usap_op_entropy (Q32 description length of `part`, model
 * term minus data term), but every pointer is a DEVICE pointer on the
 * current device: src/dst (e entries, 0-based, in [0, n)), weight (NULL for
 * unit weights), part (n entries in [0, B)) and the output S_q (one int64).
 * The kernels run on `stream` (a cudaStream_t; NULL = default stream) and
 * the result is ready in stream order; the call does not wait for it.
 *
 * Nothing is allocated: the work uses one fixed scratch array per device
 * inside this library.  Limits: 1 <= B <= USAP_STATIC_MAX_BLOCKS and
 * e <= USAP_STATIC_MAX_WEIGHT (USAP_ERR_LIMIT beyond them); the total edge
 * weight must also be <= USAP_STATIC_MAX_WEIGHT.  Inputs that fail the
 * device-side checks (an id out of range, a negative weight, too much total
 * weight) make *S_q = INT64_MIN.
 *
 * The first call on a device does a one-time set-up on the calling thread
 * (locates the array and fills its log table, with synchronous copies):
 * make that first call before any stream capture.  Every call on a device
 * shares the one array: calls that overlap in time (on different streams,
 * or from different threads without ordering) race and give wrong results. */
#define USAP_STATIC_MAX_BLOCKS 1024
#define USAP_STATIC_MAX_WEIGHT 1048576
usap_status usap_entropy_static(const int32_t* src, const int32_t* dst, const int32_t* weight,
                                int64_t e, int32_t n, const int32_t* part, int32_t B,
                                int64_t* S_q, void* stream);

#ifdef __cplusplus
}
#endif
#endif
