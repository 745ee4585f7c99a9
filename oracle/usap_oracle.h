/* Oracle: a plain-C restatement of uSAP's stochastic block
 * partitioning path (include/graph_parallel.hpp of chih-chun-chang/uSAP).
 *
 * TEST INFRASTRUCTURE ONLY.  It is what the CUDA path is compared
 * against; it is never part of the product path.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 *
 * It follows the reference's control flow and arithmetic rules, with the
 * replay contract that makes two implementations comparable bit for bit:
 *
 *  - Random draws: Philox4x32-10 (Salmon et al., SC'11) keyed by the seed,
 *    counter (item, sub, stage, tag).  Discrete draws are integer
 *    inverse-CDF: t = (u * total) >> 32, pick the first index whose
 *    inclusive cumulative weight exceeds t, in the order the reference lists
 *    its candidates (block-id order for blocks; out-list then in-list for a
 *    vertex's neighbours).  The "x <= B/(d_a[u]+B)" test is the exact
 *    integer comparison u*(d_a[u]+B) <= B<<32.
 *  - Entropy terms x*log(x/(a*b)) are evaluated in FP64 from a table of
 *    log(k) for integers k (log(0) = -inf) and each term is rounded to a
 *    fixed-point integer with 32 fraction bits (Q32) before summation, so
 *    sums are exact and independent of order.
 *  - Block-merge order ties are broken by block index (the reference's
 *    std::sort at graph_parallel.hpp:1230 is unstable).
 */
#ifndef USAP_ORACLE_H
#define USAP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OG_Q32_SCALE 4294967296.0

/* FP32 terms of precision mode 1 (float-pair terms) or 2 (plain float
 * terms), summed in double with compensation: value = s + c; abs = sum of
 * |term|; n = number of non-zero terms */
typedef struct {
  double s, c, abs;
  int64_t n;
  int32_t mode;
} og_fsum;

typedef struct {
  int32_t n;
  int64_t e;
  int32_t *src, *dst, *w;          /* edge list, file order, 0-based */
  int64_t *out_ptr, *in_ptr;        /* CSR offsets [n+1] */
  int32_t *out_idx, *out_w;         /* out-neighbours in file order */
  int32_t *in_idx, *in_w;           /* in-neighbours in file order */
  int64_t *kout, *kin;              /* weighted out/in degree per vertex */
  int64_t wtot;                     /* total edge weight */
  double *logk;                     /* logk[k] = log(k), k in [0, wtot] */
} og_graph;

typedef struct {
  int32_t B;
  int64_t *M;      /* dense B*B, row = source block */
  int64_t *dout, *din;
} og_blocks;

typedef struct {
  int32_t num_agg_proposals_per_block;   /* K, graph_parallel.hpp:43 */
  float num_block_reduction_rate;        /* graph_parallel.hpp:44 */
  int32_t max_num_nodal_itr;             /* graph_parallel.hpp:45 */
  int32_t num_batch_nodal_update;        /* graph_parallel.hpp:46 */
  double delta_entropy_threshold1;       /* graph_parallel.hpp:47 */
  double delta_entropy_threshold2;       /* graph_parallel.hpp:48 */
  int32_t delta_entropy_moving_avg_window;/* graph_parallel.hpp:49 */
  int32_t dfs_depth;                     /* graph_parallel.hpp:51 */
  uint64_t seed;
  int32_t init_mode;                     /* 0: SCC (reference), 1: identity */
  int32_t precision;                     /* 3 (default): the reference's float nodal dS; 0: exact Q32 dS */
} og_params;

typedef struct {
  int32_t kind;      /* 1 merge applied, 2 batch end, 3 stage end */
  int32_t stage, itr;
  int32_t batch_beg;
  int32_t B;
  int64_t S_q;       /* batch end: data term of the running S (Q32); stage end: S in
                        Q32, saturated beyond +-2^31 */
  int32_t S_ninf;
  int64_t cum_q;
  int32_t cum_ninf;
  int64_t moves;     /* accepted moves in the batch */
  uint64_t h_part, h_M, h_deg;
} og_trace_event;

typedef void (*og_trace_fn)(void* user, const og_trace_event* ev);

typedef struct {
  int32_t B;
  int64_t S_q;       /* Q32, saturated beyond +-2^31 */
  double S;          /* model term + data term */
  int32_t stages;
  int64_t sweeps, batches;
  int64_t nodal_proposals, nodal_moves, near_threshold, merge_shortfall;
} og_result;

typedef struct {
  double rand_index, adjusted_rand_index, pairwise_recall, pairwise_precision;
  double h_truth, h_given, h_truth_given, h_given_truth, mi, nmi, nmi_sqrt;
  double missed_info, erroneous_info;
  double adjusted_rand_index_exact;
  int64_t n, b_truth, b_given;
} og_scores;

/* --- RNG contract ------------------------------------------------------ */
void og_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
uint32_t og_draw_below(uint32_t u, int64_t n);
int og_accept_uniform(uint32_t u, int64_t da, int64_t B);

/* --- graph --------------------------------------------------------------- */
int og_graph_init(og_graph* g, int32_t n, int64_t e, const int32_t* src,
                  const int32_t* dst, const int32_t* w);
void og_graph_free(og_graph* g);

/* --- building blocks ------------------------------------------------------ */
int32_t og_scc(const og_graph* g, int32_t dfs_depth, int32_t* part);
int og_blocks_alloc(og_blocks* b, int32_t B);
void og_blocks_free(og_blocks* b);
void og_build(const og_graph* g, const int32_t* part, og_blocks* b);
int64_t og_quantize(double t);   /* saturated to the int64 range */
int64_t og_add_sat(int64_t a, int64_t b);
/* description length = model term + data term: S = model + data_q / 2^32 */
double og_desc_length(double model, int64_t data_q);
int64_t og_data_q(const og_graph* g, const og_blocks* b);   /* -(sum of Q32 terms) */
double og_model_S(int64_t n, int64_t e, int32_t B);
int64_t og_entropy_q(const og_graph* g, const og_blocks* b);
int64_t og_merge_dq(const og_graph* g, const og_blocks* b, int32_t r, int32_t s);
int64_t og_nodal_dq(const og_graph* g, const int32_t* part, const og_blocks* b,
                    int32_t v, int32_t s, int32_t* neg_inf);
/* the same dS with the FP32 terms of precision mode 1 summed into *f */
int64_t og_merge_dq_f32(const og_graph* g, const og_blocks* b, int32_t r, int32_t s, int32_t mode,
                        og_fsum* f);
int64_t og_nodal_dq_f32(const og_graph* g, const int32_t* part, const og_blocks* b,
                        int32_t v, int32_t s, int32_t mode, int32_t* neg_inf, og_fsum* f);
double og_fsum_value(const og_fsum* f);
/* precision mode 3: log rounded to float (own evaluation, bit-identical on
 * the CUDA path) and the reference's float nodal dS in its term order */
float og_log_f32(float x);
float og_nodal_ds_ref32(const og_graph* g, const int32_t* part, const og_blocks* b, int32_t v,
                        int32_t s);
int32_t og_merge_propose(const og_graph* g, const og_blocks* b, int32_t r, int32_t k,
                         int32_t stage, uint64_t seed);
int32_t og_nodal_propose(const og_graph* g, const int32_t* part, const og_blocks* b,
                         int32_t v, int32_t itr, int32_t stage, uint64_t seed);
void og_merge_phase(const og_graph* g, const og_blocks* b, int32_t K, int32_t stage,
                    uint64_t seed, int32_t* best_s, int64_t* best_q);
int32_t og_merge_apply(int32_t n, int32_t* part, int32_t B, const int32_t* best_s,
                       const int64_t* best_q, int32_t b_to_merge, int32_t* merged);
/* One nodal batch [beg, end) against the snapshot (part, b).  Writes the
 * proposal per vertex (-1 if none), its dS_q and acceptance; applies the
 * accepted moves to part and rebuilds b.  Returns the number of moves and
 * adds the accepted dS to *cum_q / *cum_ninf. */
int64_t og_nodal_batch(const og_graph* g, int32_t* part, og_blocks* b, int32_t beg,
                       int32_t end, int32_t itr, int32_t stage, uint64_t seed,
                       int32_t* prop_s, int64_t* prop_q, int32_t* prop_ninf,
                       int64_t* cum_q, int32_t* cum_ninf, int64_t* near_threshold);
int64_t og_nodal_batch_p(const og_graph* g, int32_t* part, og_blocks* b, int32_t beg,
                         int32_t end, int32_t itr, int32_t stage, uint64_t seed, int32_t precision,
                         int32_t* prop_s, int64_t* prop_q, int32_t* prop_ninf, float* prop_f,
                         int64_t* cum_q, int32_t* cum_ninf, int64_t* near_threshold);

/* --- golden-section search over B (host-side in the product) ------------- */
typedef struct { int32_t B; double S; int64_t S_q; int32_t finite; int32_t slot; } og_gpoint;
typedef struct { og_gpoint large, med, small; } og_golden;
void og_golden_init(og_golden* gs);
int og_golden_step(og_golden* gs, int32_t B, double S, int64_t S_q, int32_t cur_slot, float rate,
                   int32_t* restore_slot, int32_t* btm, int32_t* free_slot);

/* --- whole solve ---------------------------------------------------------- */
void og_params_default(og_params* p);
int og_partition(const og_graph* g, const og_params* p, int32_t* part_out,
                 og_result* res, og_trace_fn trace, void* user);
/* the same from a given initial partition (labels >= 0, renumbered 0..B-1
 * in ascending order) instead of the SCC pass */
int og_partition_from(const og_graph* g, const og_params* p, const int32_t* init, int32_t* part_out,
                      og_result* res, og_trace_fn trace, void* user);
int32_t og_compact_labels(const int32_t* init, int32_t n, int32_t* part);

/* --- checksums used by traces (order independent where noted) ----------- */
uint64_t og_hash_part(const int32_t* part, int32_t n);
uint64_t og_hash_blocks(const og_blocks* b, uint64_t* h_deg);

/* --- evaluation ----------------------------------------------------------- */
int og_evaluate(const int32_t* truth, const int32_t* given, int64_t n, og_scores* s);

#ifdef __cplusplus
}
#endif
#endif
