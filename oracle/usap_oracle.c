/* Oracle: plain-C restatement of uSAP's SBP path (see usap_oracle.h).
 * TEST INFRASTRUCTURE ONLY: what the CUDA path is compared against, never shipped.
 * Every function cites the reference lines it restates
 * (include/graph_parallel.hpp unless noted).  Compile with
 * -ffp-contract=off: terms must round exactly as written.
 */
#include "usap_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define OG_TAG_MERGE 0x4D455247u /* 'MERG' */
#define OG_TAG_NODAL 0x4E4F4441u /* 'NODA' */
#define OG_NEAR_Q 4              /* |dS| <= 1e-9 in Q32 units */

/* ------------------------------------------------------------------------ */
/* A parallel loop over [0, n) on host threads (items handed out in chunks by
 * an atomic counter).  Used only where the reference itself runs items in
 * parallel from one snapshot (a batch's nodal proposals, a merge phase's
 * blocks); every result is written per item or summed as integers, so the
 * outcome does not depend on the thread count.  OG_THREADS overrides the
 * thread count (1: sequential).                                            */
typedef void (*og_item_fn)(void* ctx, int32_t item, int32_t worker);
typedef struct {
  og_item_fn fn;
  void* ctx;
  int32_t n, chunk, worker;
  atomic_int* next;
} og_pf_arg;

static void* og_pf_run(void* p) {
  og_pf_arg* a = (og_pf_arg*)p;
  for (;;) {
    int32_t i0 = atomic_fetch_add(a->next, a->chunk);
    if (i0 >= a->n) break;
    int32_t i1 = i0 + a->chunk < a->n ? i0 + a->chunk : a->n;
    for (int32_t i = i0; i < i1; i++) a->fn(a->ctx, i, a->worker);
  }
  return NULL;
}

#define OG_MAX_WORKERS 64
static int32_t og_workers(void) {
  const char* e = getenv("OG_THREADS");
  long t = e ? atol(e) : sysconf(_SC_NPROCESSORS_ONLN);
  if (t < 1) t = 1;
  if (t > OG_MAX_WORKERS) t = OG_MAX_WORKERS;
  return (int32_t)t;
}

static void og_parallel_for(int32_t n, og_item_fn fn, void* ctx) {
  int32_t nt = og_workers();
  if (nt > n / 8) nt = n / 8 > 0 ? n / 8 : 1;
  atomic_int next = 0;
  og_pf_arg args[OG_MAX_WORKERS];
  pthread_t th[OG_MAX_WORKERS];
  for (int32_t t = 0; t < nt; t++)
    args[t] = (og_pf_arg){fn, ctx, n, 8, t, &next};
  int32_t started = 0;
  for (int32_t t = 1; t < nt; t++)
    if (pthread_create(&th[t], NULL, og_pf_run, &args[t]) == 0) started = t;
    else break;
  og_pf_run(&args[0]);
  for (int32_t t = 1; t <= started; t++) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).                         */
static inline void og_mulhilo(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

void og_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int round = 0; round < 10; round++) {
    if (round > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint32_t hi0, lo0, hi1, lo1;
    og_mulhilo(0xD2511F53u, c0, &hi0, &lo0);
    og_mulhilo(0xCD9E8D57u, c2, &hi1, &lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static void og_draws(uint64_t seed, uint32_t item, uint32_t sub, uint32_t stage,
                     uint32_t tag, uint32_t out[4]) {
  uint32_t ctr[4] = {item, sub, stage, tag};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  og_philox4x32_10(ctr, key, out);
}

uint32_t og_draw_below(uint32_t u, int64_t n) {
  return (uint32_t)(((uint64_t)u * (uint64_t)n) >> 32);
}

/* x <= B / (d_a[u] + B) with x = u / 2^32 (graph_parallel.hpp:817, :1037) */
int og_accept_uniform(uint32_t u, int64_t da, int64_t B) {
  return (uint64_t)u * (uint64_t)(da + B) <= ((uint64_t)B << 32);
}

/* ------------------------------------------------------------------------ */
/* Graph: adjacency in file order (load_graph_from_tsv, :251-317).           */
int og_graph_init(og_graph* g, int32_t n, int64_t e, const int32_t* src,
                  const int32_t* dst, const int32_t* w) {
  memset(g, 0, sizeof(*g));
  g->n = n;
  g->e = e;
  size_t E = (size_t)e;
  g->src = malloc(sizeof(int32_t) * (E ? E : 1));
  g->dst = malloc(sizeof(int32_t) * (E ? E : 1));
  g->w = malloc(sizeof(int32_t) * (E ? E : 1));
  g->out_ptr = calloc((size_t)n + 1, sizeof(int64_t));
  g->in_ptr = calloc((size_t)n + 1, sizeof(int64_t));
  g->out_idx = malloc(sizeof(int32_t) * (E ? E : 1));
  g->out_w = malloc(sizeof(int32_t) * (E ? E : 1));
  g->in_idx = malloc(sizeof(int32_t) * (E ? E : 1));
  g->in_w = malloc(sizeof(int32_t) * (E ? E : 1));
  g->kout = calloc((size_t)n + 1, sizeof(int64_t));
  g->kin = calloc((size_t)n + 1, sizeof(int64_t));
  if (!g->src || !g->dst || !g->w || !g->out_ptr || !g->in_ptr || !g->out_idx ||
      !g->out_w || !g->in_idx || !g->in_w || !g->kout || !g->kin) {
    og_graph_free(g);
    return -1;
  }
  int64_t wtot = 0;
  for (size_t i = 0; i < E; i++) {
    int32_t a = src[i], b = dst[i], ww = w ? w[i] : 1;
    if (a < 0 || a >= n || b < 0 || b >= n || ww <= 0) {
      og_graph_free(g);
      return -2;
    }
    g->src[i] = a;
    g->dst[i] = b;
    g->w[i] = ww;
    g->out_ptr[a + 1]++;
    g->in_ptr[b + 1]++;
    g->kout[a] += ww;
    g->kin[b] += ww;
    wtot += ww;
  }
  for (int32_t v = 0; v < n; v++) {
    g->out_ptr[v + 1] += g->out_ptr[v];
    g->in_ptr[v + 1] += g->in_ptr[v];
  }
  int64_t* fo = malloc(sizeof(int64_t) * ((size_t)n + 1));
  int64_t* fi = malloc(sizeof(int64_t) * ((size_t)n + 1));
  memcpy(fo, g->out_ptr, sizeof(int64_t) * ((size_t)n + 1));
  memcpy(fi, g->in_ptr, sizeof(int64_t) * ((size_t)n + 1));
  for (size_t i = 0; i < E; i++) {  /* stable: file order within each list */
    int64_t po = fo[g->src[i]]++;
    g->out_idx[po] = g->dst[i];
    g->out_w[po] = g->w[i];
    int64_t pi = fi[g->dst[i]]++;
    g->in_idx[pi] = g->src[i];
    g->in_w[pi] = g->w[i];
  }
  free(fo);
  free(fi);
  g->wtot = wtot;
  g->logk = malloc(sizeof(double) * ((size_t)wtot + 1));
  if (!g->logk) {
    og_graph_free(g);
    return -1;
  }
  g->logk[0] = -INFINITY;
  for (int64_t k = 1; k <= wtot; k++) g->logk[k] = log((double)k);
  return 0;
}

void og_graph_free(og_graph* g) {
  free(g->src); free(g->dst); free(g->w);
  free(g->out_ptr); free(g->in_ptr);
  free(g->out_idx); free(g->out_w); free(g->in_idx); free(g->in_w);
  free(g->kout); free(g->kin); free(g->logk);
  memset(g, 0, sizeof(*g));
}

/* ------------------------------------------------------------------------ */
/* Initial partition: _scc (:514-556) after _dfs_itr (:573-603).             */
typedef struct { int32_t* a; size_t n, cap; } og_stack;
static int og_push(og_stack* s, int32_t v) {
  if (s->n == s->cap) {
    size_t nc = s->cap ? s->cap * 2 : 1024;
    int32_t* na = realloc(s->a, nc * sizeof(int32_t));
    if (!na) return -1;
    s->a = na;
    s->cap = nc;
  }
  s->a[s->n++] = v;
  return 0;
}

int32_t og_scc(const og_graph* g, int32_t dfs_depth, int32_t* part) {
  int32_t n = g->n;
  og_stack fin = {0}, st = {0}, st2 = {0};
  uint8_t* color = calloc((size_t)n + 1, 1);
  /* iterative DFS on the out-graph, finish order onto `fin` (:573-603) */
  for (int32_t v0 = 0; v0 < n; v0++) {
    if (color[v0] != 0) continue;
    og_push(&st, v0);
    while (st.n) {
      int32_t v = st.a[st.n - 1];
      if (color[v] != 0) {
        st.n--;
        if (color[v] == 1) {
          og_push(&fin, v);
          color[v] = 2;
        }
      } else {
        color[v] = 1;
        for (int64_t p = g->out_ptr[v]; p < g->out_ptr[v + 1]; p++) {
          int32_t t = g->out_idx[p];
          if (color[t] == 0) og_push(&st, t);
        }
      }
    }
  }
  /* transpose lists ordered by source vertex id (:518-523) */
  int64_t* tptr = calloc((size_t)n + 1, sizeof(int64_t));
  int32_t* tidx = malloc(sizeof(int32_t) * (g->e ? (size_t)g->e : 1));
  for (int32_t i = 0; i < n; i++)
    for (int64_t p = g->out_ptr[i]; p < g->out_ptr[i + 1]; p++) tptr[g->out_idx[p] + 1]++;
  for (int32_t v = 0; v < n; v++) tptr[v + 1] += tptr[v];
  int64_t* fill = malloc(sizeof(int64_t) * ((size_t)n + 1));
  memcpy(fill, tptr, sizeof(int64_t) * ((size_t)n + 1));
  for (int32_t i = 0; i < n; i++)
    for (int64_t p = g->out_ptr[i]; p < g->out_ptr[i + 1]; p++) tidx[fill[g->out_idx[p]]++] = i;
  free(fill);
  /* depth-limited DFS on the transpose, one block per root (:525-554) */
  uint8_t* visited = calloc((size_t)n + 1, 1);
  for (int32_t v = 0; v < n; v++) part[v] = -1;
  int32_t b = 0;
  while (fin.n) {
    int32_t v = fin.a[--fin.n];
    if (visited[v]) continue;
    int32_t i = 0;
    st2.n = 0;
    og_push(&st2, v);
    while (st2.n && i < dfs_depth) {
      int32_t ni = st2.a[--st2.n];
      if (!visited[ni]) {
        visited[ni] = 1;
        part[ni] = b;
        i++;
        for (int64_t p = tptr[ni]; p < tptr[ni + 1]; p++) {
          int32_t t = tidx[p];
          if (!visited[t]) og_push(&st2, t);
        }
      }
    }
    b++;
  }
  free(color); free(visited); free(tptr); free(tidx);
  free(fin.a); free(st.a); free(st2.a);
  return b;
}

/* ------------------------------------------------------------------------ */
/* Interblock counts M and block degrees: _initialize_edge_counts (:703-759) */
int og_blocks_alloc(og_blocks* b, int32_t B) {
  b->B = B;
  size_t bb = (size_t)B * (size_t)B;
  b->M = calloc(bb ? bb : 1, sizeof(int64_t));
  b->dout = calloc((size_t)B + 1, sizeof(int64_t));
  b->din = calloc((size_t)B + 1, sizeof(int64_t));
  return (b->M && b->dout && b->din) ? 0 : -1;
}

void og_blocks_free(og_blocks* b) {
  free(b->M); free(b->dout); free(b->din);
  memset(b, 0, sizeof(*b));
}

void og_build(const og_graph* g, const int32_t* part, og_blocks* b) {
  int32_t B = b->B;
  memset(b->M, 0, sizeof(int64_t) * (size_t)B * (size_t)B);
  memset(b->dout, 0, sizeof(int64_t) * (size_t)B);
  memset(b->din, 0, sizeof(int64_t) * (size_t)B);
  for (int32_t v = 0; v < g->n; v++) {
    int32_t k1 = part[v];
    for (int64_t p = g->out_ptr[v]; p < g->out_ptr[v + 1]; p++) {
      int32_t k2 = part[g->out_idx[p]];
      b->M[(size_t)k1 * B + k2] += g->out_w[p];
    }
  }
  for (int32_t i = 0; i < B; i++)
    for (int32_t j = 0; j < B; j++) {
      int64_t m = b->M[(size_t)i * B + j];
      b->dout[i] += m;
      b->din[j] += m;
    }
}

/* ------------------------------------------------------------------------ */
/* Entropy terms.  The reference writes each as x*log(x/(a*b)) with x an
 * interblock count and a, b block degrees.  Here log is read from the
 * integer log table and every term is quantised to Q32 on its own.        */
int64_t og_quantize(double t) {
  double x = t * OG_Q32_SCALE;
  if (x >= 9223372036854775807.0) return INT64_MAX;
  if (x <= -9223372036854775807.0) return INT64_MIN;
  return llrint(x);
}

int64_t og_add_sat(int64_t a, int64_t b) {
  int64_t r;
  if (__builtin_add_overflow(a, b, &r)) return a > 0 ? INT64_MAX : INT64_MIN;
  return r;
}

double og_desc_length(double model, int64_t data_q) { return model + (double)data_q / OG_Q32_SCALE; }

static inline double og_g(const double* L, int64_t x, int64_t din_arg, int64_t dout_arg) {
  if (x == 0) return 0.0;
  return (double)x * ((L[x] - L[din_arg]) - L[dout_arg]);
}

static inline double og_coef(const double* L, int64_t n, int64_t a_new, int64_t a_old) {
  if (n == 0) return 0.0;
  return (double)n * (L[a_new] - L[a_old]);
}

static inline double og_h(const double* L, int64_t x, int64_t y) {
  double a = (double)x * L[x];
  double b = (double)y * L[y];
  double c = (double)(x + y) * L[x + y];
  return (a + b) - c;
}

/* ------------------------------------------------------------------------ */
/* Precision modes 1 and 2 of the CUDA path evaluate the same terms with
 * single-precision operations only (C float arithmetic, no contraction):
 *  - mode 1: float pairs (hi, lo) worth hi + lo, the log table held as
 *    pairs (hi = log k rounded to float, lo = the remainder rounded), every
 *    term in pair arithmetic built from Knuth's TwoSum and a TwoProduct by
 *    fused multiply-add;
 *  - mode 2: plain float terms from the rounded log values.
 * The terms are summed here in double with Neumaier's compensation, which
 * is exact enough to be the reference for the CUDA path's FP32 pair sums;
 * `abs` and `n` give the error bound's scale (sum of |term|) and the number
 * of terms.                                                                */
typedef struct { float hi, lo; } og_ff;

static inline og_ff og_two_sum(float a, float b) {
  float s = a + b;
  float z = s - a;
  og_ff r = {s, (a - (s - z)) + (b - z)};
  return r;
}

static inline og_ff og_ff_add(og_ff a, og_ff b) {
  og_ff s = og_two_sum(a.hi, b.hi);
  return og_two_sum(s.hi, s.lo + (a.lo + b.lo));
}

static inline og_ff og_ff_neg(og_ff a) { og_ff r = {-a.hi, -a.lo}; return r; }
static inline og_ff og_ff_sub(og_ff a, og_ff b) { return og_ff_add(a, og_ff_neg(b)); }

static inline og_ff og_ff_mul_ll(og_ff d, int64_t x) {
  float xh = (float)x;
  float xl = (float)(x - (int64_t)xh);
  float p = xh * d.hi;
  float e = fmaf(xh, d.hi, -p);
  e = e + (xh * d.lo + xl * d.hi);
  return og_two_sum(p, e);
}

static inline og_ff og_ff_log(const double* L, int64_t k) {
  double x = L[k];
  float hi = (float)x;
  og_ff r = {hi, isinf(x) ? 0.0f : (float)(x - (double)hi)};
  return r;
}

static const og_ff og_ff_zero = {0.0f, 0.0f};

static inline og_ff og_g32(const double* L, int mode, int64_t x, int64_t din_arg, int64_t dout_arg) {
  if (x == 0) return og_ff_zero;
  og_ff a = og_ff_log(L, x), b = og_ff_log(L, din_arg), c = og_ff_log(L, dout_arg);
  if (mode == 1) return og_ff_mul_ll(og_ff_sub(og_ff_sub(a, b), c), x);
  og_ff r = {(float)x * ((a.hi - b.hi) - c.hi), 0.0f};
  return r;
}

static inline og_ff og_coef32(const double* L, int mode, int64_t n, int64_t a_new, int64_t a_old) {
  if (n == 0) return og_ff_zero;
  og_ff a = og_ff_log(L, a_new), b = og_ff_log(L, a_old);
  if (mode == 1) return og_ff_mul_ll(og_ff_sub(a, b), n);
  og_ff r = {(float)n * (a.hi - b.hi), 0.0f};
  return r;
}

static inline og_ff og_h32(const double* L, int mode, int64_t x, int64_t y) {
  og_ff lx = og_ff_log(L, x), ly = og_ff_log(L, y), lxy = og_ff_log(L, x + y);
  if (mode == 1)
    return og_ff_sub(og_ff_add(og_ff_mul_ll(lx, x), og_ff_mul_ll(ly, y)), og_ff_mul_ll(lxy, x + y));
  float a = (float)x * lx.hi;
  float b = (float)y * ly.hi;
  float c = (float)(x + y) * lxy.hi;
  og_ff r = {(a + b) - c, 0.0f};
  return r;
}

static inline void og_fadd(og_fsum* f, og_ff t) {
  double x = (double)t.hi + (double)t.lo;   /* exact */
  if (x == 0.0) return;
  double s = f->s + x;
  if (fabs(f->s) >= fabs(x)) f->c += (f->s - s) + x;
  else f->c += (x - s) + f->s;
  f->s = s;
  f->abs += fabs(x);
  f->n++;
}

double og_fsum_value(const og_fsum* f) { return f->s + f->c; }

/* model term of _compute_overall_entropy (:1314-1316), evaluated in FP64;
 * the reference's precedence (x*log(x) not scaled by E) is kept */
double og_model_S(int64_t n, int64_t e, int32_t B) {
  double x = (double)B * (double)B / (double)e;
  return (double)e * (1.0 + x) * log(1.0 + x) - x * log(x) + (double)n * log((double)B);
}

/* S = model + data, data = -sum M log(M/(dout*din)) (:1281-1319) */
int64_t og_data_q(const og_graph* g, const og_blocks* b) {
  const double* L = g->logk;
  int32_t B = b->B;
  int64_t data = 0;
  for (int32_t i = 0; i < B; i++)
    for (int32_t j = 0; j < B; j++) {
      int64_t m = b->M[(size_t)i * B + j];
      if (m != 0) data += og_quantize(og_g(L, m, b->din[j], b->dout[i]));
    }
  return -data;
}

/* S in Q32: model term (saturated) + data term, saturated */
int64_t og_entropy_q(const og_graph* g, const og_blocks* b) {
  return og_add_sat(og_quantize(og_model_S(g->n, g->e, b->B)), og_data_q(g, b));
}

/* ------------------------------------------------------------------------ */
/* Block-merge dS of merging r into s (:867-987).  The O(B) sums of the
 * reference are regrouped: for rows i not in {r,s},
 *   g(M_ri,din_i,dout_r) + g(M_si,din_i,dout_s) - g(M_ri+M_si,din_i,dout_s')
 *   = h(M_ri,M_si) + M_ri (L[dout_s'] - L[dout_r]) + M_si (L[dout_s'] - L[dout_s])
 * with h(x,y) = xL[x] + yL[y] - (x+y)L[x+y], which vanishes unless both
 * counts are non-zero; columns likewise.                                   */
static int64_t og_merge_dq_impl(const og_graph* g, const og_blocks* b, int32_t r, int32_t s, og_fsum* f) {
  const int FM = f ? f->mode : 0;
  const double* L = g->logk;
  int32_t B = b->B;
  const int64_t* M = b->M;
  int64_t dr_out = b->dout[r], dr_in = b->din[r];
  int64_t ds_out = b->dout[s], ds_in = b->din[s];
  int64_t ds_out_new = ds_out + dr_out;  /* k_out of r is its row sum */
  int64_t ds_in_new = ds_in + dr_in;
  int64_t Mrr = M[(size_t)r * B + r], Mrs = M[(size_t)r * B + s];
  int64_t Msr = M[(size_t)s * B + r], Mss = M[(size_t)s * B + s];
  int64_t acc = 0;
  acc += og_quantize(og_g(L, Mrr, dr_in, dr_out));
  acc += og_quantize(og_g(L, Mrs, ds_in, dr_out));
  acc += og_quantize(og_g(L, Msr, dr_in, ds_out));
  acc += og_quantize(og_g(L, Mss, ds_in, ds_out));
  acc -= og_quantize(og_g(L, Mrr + Mrs + Msr + Mss, ds_in_new, ds_out_new));
  if (f) og_fadd(f, og_g32(L, FM, Mrr, dr_in, dr_out));
  if (f) og_fadd(f, og_g32(L, FM, Mrs, ds_in, dr_out));
  if (f) og_fadd(f, og_g32(L, FM, Msr, dr_in, ds_out));
  if (f) og_fadd(f, og_g32(L, FM, Mss, ds_in, ds_out));
  if (f) og_fadd(f, og_ff_neg(og_g32(L, FM, Mrr + Mrs + Msr + Mss, ds_in_new, ds_out_new)));
  for (int32_t i = 0; i < B; i++) {
    if (i == r || i == s) continue;
    int64_t x = M[(size_t)r * B + i], y = M[(size_t)s * B + i];
    if (x > 0 && y > 0) {
      acc += og_quantize(og_h(L, x, y));
      if (f) og_fadd(f, og_h32(L, FM, x, y));
    }
    x = M[(size_t)i * B + r];
    y = M[(size_t)i * B + s];
    if (x > 0 && y > 0) {
      acc += og_quantize(og_h(L, x, y));
      if (f) og_fadd(f, og_h32(L, FM, x, y));
    }
  }
  int64_t Ar, As, Cr, Cs;
  if (s != r) {
    Ar = dr_out - Mrr - Mrs;
    As = ds_out - Msr - Mss;
    Cr = dr_in - Mrr - Msr;
    Cs = ds_in - Mrs - Mss;
  } else {
    Ar = As = dr_out - Mrr;
    Cr = Cs = dr_in - Mrr;
  }
  acc += og_quantize(og_coef(L, Ar, ds_out_new, dr_out));
  acc += og_quantize(og_coef(L, As, ds_out_new, ds_out));
  acc += og_quantize(og_coef(L, Cr, ds_in_new, dr_in));
  acc += og_quantize(og_coef(L, Cs, ds_in_new, ds_in));
  if (f) og_fadd(f, og_coef32(L, FM, Ar, ds_out_new, dr_out));
  if (f) og_fadd(f, og_coef32(L, FM, As, ds_out_new, ds_out));
  if (f) og_fadd(f, og_coef32(L, FM, Cr, ds_in_new, dr_in));
  if (f) og_fadd(f, og_coef32(L, FM, Cs, ds_in_new, ds_in));
  return acc;
}

int64_t og_merge_dq(const og_graph* g, const og_blocks* b, int32_t r, int32_t s) {
  return og_merge_dq_impl(g, b, r, s, NULL);
}

int64_t og_merge_dq_f32(const og_graph* g, const og_blocks* b, int32_t r, int32_t s, int32_t mode, og_fsum* f) {
  f->s = f->c = f->abs = 0.0;
  f->n = 0;
  f->mode = mode;
  return og_merge_dq_impl(g, b, r, s, f);
}

/* ------------------------------------------------------------------------ */
/* Nodal dS of moving v from r = part[v] to s (:1066-1215), including the
 * reference's rule that in-edges from blocks r and s do not adjust the 2x2
 * row entries (the adjustment is commented out at :1135-1142) and that the
 * column sums skip i in {r, s}.  The O(B) sums are regrouped: entries a
 * move leaves unchanged contribute count * (L[new degree] - L[old degree]),
 * with the counts known exactly from the block degrees.  A new-state term
 * with a zero degree is +inf, as log(x/0) is in the reference; dS is then
 * -inf and *neg_inf is set.                                               */
static int64_t og_nodal_dq_impl(const og_graph* g, const int32_t* part, const og_blocks* b,
                                int32_t v, int32_t s, int32_t* neg_inf, og_fsum* f) {
  const int FM = f ? f->mode : 0;
  const double* L = g->logk;
  int32_t B = b->B;
  const int64_t* M = b->M;
  int32_t r = part[v];
  *neg_inf = 0;
  if (r == s) return 0;
  int64_t* wo = calloc((size_t)B, sizeof(int64_t));
  int64_t* wi = calloc((size_t)B, sizeof(int64_t));
  uint8_t* seen = calloc((size_t)B, 1);
  int32_t* list = malloc(sizeof(int32_t) * (size_t)(g->out_ptr[v + 1] - g->out_ptr[v] +
                                                     g->in_ptr[v + 1] - g->in_ptr[v] + 1));
  int32_t nl = 0;
  for (int64_t p = g->out_ptr[v]; p < g->out_ptr[v + 1]; p++) {
    int32_t bb = part[g->out_idx[p]];
    if (!seen[bb]) { seen[bb] = 1; list[nl++] = bb; }
    wo[bb] += g->out_w[p];
  }
  for (int64_t p = g->in_ptr[v]; p < g->in_ptr[v + 1]; p++) {
    int32_t bb = part[g->in_idx[p]];
    if (!seen[bb]) { seen[bb] = 1; list[nl++] = bb; }
    wi[bb] += g->in_w[p];
  }
  int64_t kout = g->kout[v], kin = g->kin[v];
  int64_t dr_out = b->dout[r], dr_in = b->din[r], ds_out = b->dout[s], ds_in = b->din[s];
  int64_t dr_out_n = dr_out - kout, ds_out_n = ds_out + kout;
  int64_t dr_in_n = dr_in - kin, ds_in_n = ds_in + kin;
  int64_t Rr = M[(size_t)r * B + r], Rs = M[(size_t)r * B + s];
  int64_t Sr = M[(size_t)s * B + r], Ss = M[(size_t)s * B + s];
  int64_t acc = 0, sumXR = 0, sumXS = 0, sumYR = 0, sumYS = 0;
  for (int32_t t = 0; t < nl; t++) {
    int32_t bb = list[t];
    if (bb == r || bb == s) continue;
    if (wo[bb] > 0) {
      int64_t R = M[(size_t)r * B + bb], S = M[(size_t)s * B + bb], dinb = b->din[bb];
      acc += og_quantize(og_g(L, R, dinb, dr_out));
      acc += og_quantize(og_g(L, S, dinb, ds_out));
      acc -= og_quantize(og_g(L, R - wo[bb], dinb, dr_out_n));
      acc -= og_quantize(og_g(L, S + wo[bb], dinb, ds_out_n));
      if (f) og_fadd(f, og_g32(L, FM, R, dinb, dr_out));
      if (f) og_fadd(f, og_g32(L, FM, S, dinb, ds_out));
      if (f) og_fadd(f, og_ff_neg(og_g32(L, FM, R - wo[bb], dinb, dr_out_n)));
      if (f) og_fadd(f, og_ff_neg(og_g32(L, FM, S + wo[bb], dinb, ds_out_n)));
      sumXR += R;
      sumXS += S;
    }
    if (wi[bb] > 0) {
      int64_t Rc = M[(size_t)bb * B + r], Sc = M[(size_t)bb * B + s], doutb = b->dout[bb];
      acc += og_quantize(og_g(L, Rc, dr_in, doutb));
      acc += og_quantize(og_g(L, Sc, ds_in, doutb));
      acc -= og_quantize(og_g(L, Rc - wi[bb], dr_in_n, doutb));
      acc -= og_quantize(og_g(L, Sc + wi[bb], ds_in_n, doutb));
      if (f) og_fadd(f, og_g32(L, FM, Rc, dr_in, doutb));
      if (f) og_fadd(f, og_g32(L, FM, Sc, ds_in, doutb));
      if (f) og_fadd(f, og_ff_neg(og_g32(L, FM, Rc - wi[bb], dr_in_n, doutb)));
      if (f) og_fadd(f, og_ff_neg(og_g32(L, FM, Sc + wi[bb], ds_in_n, doutb)));
      sumYR += Rc;
      sumYS += Sc;
    }
  }
  int64_t wor = wo[r], wos = wo[s];
  acc += og_quantize(og_g(L, Rr, dr_in, dr_out));
  acc += og_quantize(og_g(L, Rs, ds_in, dr_out));
  acc += og_quantize(og_g(L, Sr, dr_in, ds_out));
  acc += og_quantize(og_g(L, Ss, ds_in, ds_out));
  if (f) og_fadd(f, og_g32(L, FM, Rr, dr_in, dr_out));
  if (f) og_fadd(f, og_g32(L, FM, Rs, ds_in, dr_out));
  if (f) og_fadd(f, og_g32(L, FM, Sr, dr_in, ds_out));
  if (f) og_fadd(f, og_g32(L, FM, Ss, ds_in, ds_out));
  double nt[4] = {og_g(L, Rr - wor, dr_in_n, dr_out_n), og_g(L, Rs - wos, ds_in_n, dr_out_n),
                  og_g(L, Sr + wor, dr_in_n, ds_out_n), og_g(L, Ss + wos, ds_in_n, ds_out_n)};
  og_ff nt32[4] = {og_ff_zero, og_ff_zero, og_ff_zero, og_ff_zero};
  if (f) {
    nt32[0] = og_g32(L, FM, Rr - wor, dr_in_n, dr_out_n);
    nt32[1] = og_g32(L, FM, Rs - wos, ds_in_n, dr_out_n);
    nt32[2] = og_g32(L, FM, Sr + wor, dr_in_n, ds_out_n);
    nt32[3] = og_g32(L, FM, Ss + wos, ds_in_n, ds_out_n);
  }
  for (int t = 0; t < 4; t++) {
    if (isinf(nt[t])) *neg_inf = 1;
    else {
      acc -= og_quantize(nt[t]);
      if (f) og_fadd(f, og_ff_neg(nt32[t]));
    }
  }
  acc += og_quantize(og_coef(L, dr_out - Rr - Rs - sumXR, dr_out_n, dr_out));
  acc += og_quantize(og_coef(L, ds_out - Sr - Ss - sumXS, ds_out_n, ds_out));
  acc += og_quantize(og_coef(L, dr_in - Rr - Sr - sumYR, dr_in_n, dr_in));
  acc += og_quantize(og_coef(L, ds_in - Rs - Ss - sumYS, ds_in_n, ds_in));
  if (f) og_fadd(f, og_coef32(L, FM, dr_out - Rr - Rs - sumXR, dr_out_n, dr_out));
  if (f) og_fadd(f, og_coef32(L, FM, ds_out - Sr - Ss - sumXS, ds_out_n, ds_out));
  if (f) og_fadd(f, og_coef32(L, FM, dr_in - Rr - Sr - sumYR, dr_in_n, dr_in));
  if (f) og_fadd(f, og_coef32(L, FM, ds_in - Rs - Ss - sumYS, ds_in_n, ds_in));
  free(wo); free(wi); free(seen); free(list);
  return acc;
}

int64_t og_nodal_dq(const og_graph* g, const int32_t* part, const og_blocks* b,
                    int32_t v, int32_t s, int32_t* neg_inf) {
  return og_nodal_dq_impl(g, part, b, v, s, neg_inf, NULL);
}

/* ------------------------------------------------------------------------ */
/* Precision mode 3: the reference's own single-precision nodal dS.
 *
 * The reference evaluates dS in `float` (:1066-1215): every term is
 * count * std::log((float)count / (long)(d_a * d_b)) -- the long product
 * converted to float, a float division, logf of the ratio, a float product
 * -- and the terms are added to one float accumulator in the order of its
 * loops over all B blocks.  Rounding noise of that O(B) sum decides many
 * near-zero proposals, and the reference's solve quality depends on it:
 * the reference compiled with double in place of float ends at far fewer
 * blocks on the N=50000 workload.  Mode 3 evaluates exactly that
 * expression, term order included.                                         */

/* log(x) for a float x, rounded to float.  Evaluated in double with IEEE
 * +, -, * and fma only, in the same steps as the CUDA kernels' ref_logf, so
 * both return the same bits: x = m * 2^e with m in [sqrt(1/2), sqrt(2));
 * k = 128 (m - 1) rounded half up picks r_k = round(1024 / (1 + k/128)) / 1024 and
 * L_k = -log(r_k) (usap_b200/csrc/ref_log_table.inc, written by
 * ref_log_table.py with 50-digit logs); u = m r_k - 1 is exact (|u| <
 * 0.0066), and log x = e ln 2 + L_k + log1p(u), log1p(u) by its series
 * u - u^2/2 + ... - u^8/8.  x = 0 gives -inf, x = +inf gives +inf.        */
static const double og_ref_log_tab[][2] = {
#include "../usap_b200/csrc/ref_log_table.inc"
};
#define OG_REF_LOG_K0 38

float og_log_f32(float x) {
  if (isnan(x) || x < 0.0f) return NAN;
  if (x == 0.0f) return -INFINITY;
  if (isinf(x)) return INFINITY;
  uint32_t u;
  memcpy(&u, &x, sizeof(u));
  int e = (int)((u >> 23) & 0xffu);
  uint32_t frac = u & 0x7fffffu;
  if (e == 0) {                      /* subnormal: leading one into the hidden bit */
    int sh = 0;
    while (!(frac & 0x800000u)) { frac <<= 1; sh++; }
    frac &= 0x7fffffu;
    e = 1 - sh;
  }
  e -= 127;
  /* m = 1 + frac / 2^23, halved above sqrt(2) (frac >= 0x3504F4); k =
   * 128 (m - 1) rounded half up, from the bits */
  double m = 1.0 + (double)frac * 0x1p-23;
  int k;
  if (frac >= 0x3504F4u) {
    m = m * 0.5;
    e += 1;
    k = (int)((frac + 0x10000u) >> 17) - 64;
  } else {
    k = (int)((frac + 0x8000u) >> 16);
  }
  const double* t = og_ref_log_tab[OG_REF_LOG_K0 + k];
  const double w = m * t[0] - 1.0;
  double q = -1.0 / 8.0;
  q = fma(q, w, 1.0 / 7.0);
  q = fma(q, w, -1.0 / 6.0);
  q = fma(q, w, 1.0 / 5.0);
  q = fma(q, w, -1.0 / 4.0);
  q = fma(q, w, 1.0 / 3.0);
  q = fma(q, w, -1.0 / 2.0);
  const double l1p = fma(w * w, q, w);
  const double hi = fma((double)e, 0.69314718055994530942, t[1]);
  return (float)(hi + l1p);
}

/* count * log((float)count / (float)prod), as the reference rounds it */
static inline float og_ref_term(int64_t x, int64_t prod) {
  const float xf = (float)x;
  const float ratio = xf / (float)prod;
  return xf * og_log_f32(ratio);
}

/* _propose_new_partition_nodal's dS (:1066-1215) for v moving to s, in the
 * reference's float arithmetic and term order: the old terms of rows r, s
 * and columns r, s (columns skip i in {r, s}) in block order; the deltas of
 * v's out-edges (rows) and in-edges (columns; the 2x2 row entries are not
 * adjusted for in-edges, :1135-1142); the four new 2x2 terms; the new terms
 * of rows and columns for i not in {r, s} in block order.  A term whose
 * count is 0 is skipped.  Returns 0 when s == part[v]. */
float og_nodal_ds_ref32(const og_graph* g, const int32_t* part, const og_blocks* b, int32_t v,
                        int32_t s) {
  const int32_t B = b->B, r = part[v];
  if (r == s) return 0.0f;
  const int64_t* M = b->M;
  int64_t* rr = malloc(sizeof(int64_t) * 4 * (size_t)B);
  int64_t *sr = rr + B, *rc = rr + 2 * (size_t)B, *sc = rr + 3 * (size_t)B;
  for (int32_t i = 0; i < B; i++) {
    rr[i] = M[(size_t)r * B + i];
    sr[i] = M[(size_t)s * B + i];
    rc[i] = M[(size_t)i * B + r];
    sc[i] = M[(size_t)i * B + s];
  }
  const int64_t* din = b->din;
  const int64_t* dout = b->dout;
  const int64_t kout = g->kout[v], kin = g->kin[v];
  const int64_t dor_n = dout[r] - kout, dos_n = dout[s] + kout;
  const int64_t dir_n = din[r] - kin, dis_n = din[s] + kin;
  float dS = 0.0f;
  for (int32_t i = 0; i < B; i++) {                       /* :1096-1114 */
    if (rr[i] != 0) dS = dS + og_ref_term(rr[i], din[i] * dout[r]);
    if (sr[i] != 0) dS = dS + og_ref_term(sr[i], din[i] * dout[s]);
    if (i != r && i != s) {
      if (rc[i] != 0) dS = dS + og_ref_term(rc[i], dout[i] * din[r]);
      if (sc[i] != 0) dS = dS + og_ref_term(sc[i], dout[i] * din[s]);
    }
  }
  for (int64_t p = g->out_ptr[v]; p < g->out_ptr[v + 1]; p++) {   /* :1119-1129 */
    const int32_t bb = part[g->out_idx[p]];
    rr[bb] -= g->out_w[p];
    sr[bb] += g->out_w[p];
  }
  for (int64_t p = g->in_ptr[v]; p < g->in_ptr[v + 1]; p++) {     /* :1130-1145 */
    const int32_t bb = part[g->in_idx[p]];
    rc[bb] -= g->in_w[p];
    sc[bb] += g->in_w[p];
  }
  if (rr[r] != 0) dS = dS - og_ref_term(rr[r], dir_n * dor_n);     /* :1180-1195 */
  if (rr[s] != 0) dS = dS - og_ref_term(rr[s], dis_n * dor_n);
  if (sr[r] != 0) dS = dS - og_ref_term(sr[r], dir_n * dos_n);
  if (sr[s] != 0) dS = dS - og_ref_term(sr[s], dis_n * dos_n);
  for (int32_t i = 0; i < B; i++) {                       /* :1196-1215 */
    if (i == r || i == s) continue;
    if (rr[i] != 0) dS = dS - og_ref_term(rr[i], din[i] * dor_n);
    if (sr[i] != 0) dS = dS - og_ref_term(sr[i], din[i] * dos_n);
    if (rc[i] != 0) dS = dS - og_ref_term(rc[i], dout[i] * dir_n);
    if (sc[i] != 0) dS = dS - og_ref_term(sc[i], dout[i] * dis_n);
  }
  free(rr);
  return dS;
}

/* Q32 of a float dS (-inf is flagged by the caller) */
static inline int64_t og_q32_f(float f) { return og_quantize((double)f); }

int64_t og_nodal_dq_f32(const og_graph* g, const int32_t* part, const og_blocks* b,
                        int32_t v, int32_t s, int32_t mode, int32_t* neg_inf, og_fsum* f) {
  f->s = f->c = f->abs = 0.0;
  f->n = 0;
  f->mode = mode;
  return og_nodal_dq_impl(g, part, b, v, s, neg_inf, f);
}

/* ------------------------------------------------------------------------ */
/* Proposals.                                                               */
static inline int64_t og_sym(const og_blocks* b, int32_t u, int32_t i) {
  return b->M[(size_t)u * b->B + i] + b->M[(size_t)i * b->B + u];
}

static inline int32_t og_skip_r(int32_t i, int32_t r, int32_t B) {
  if (i == r) i++;            /* :820-821 */
  if (i == B) i = 0;
  return i;
}

/* _propose_new_partition_block (:761-865): the neighbour block u is drawn
 * from M[r,:]+M[:,r]; then a uniform block (r skipped) with probability
 * B/(d_a[u]+B), else a block from M[u,:]+M[:,u] with r excluded.          */
int32_t og_merge_propose(const og_graph* g, const og_blocks* b, int32_t r, int32_t k,
                         int32_t stage, uint64_t seed) {
  int32_t B = b->B;
  uint32_t x[4];
  og_draws(seed, (uint32_t)r, (uint32_t)k, (uint32_t)stage, OG_TAG_MERGE, x);
  int64_t ka = b->dout[r] + b->din[r];
  if (ka == 0) return (int32_t)og_draw_below(x[2], B);   /* :804-807 */
  int64_t t = og_draw_below(x[0], ka), run = 0;
  int32_t u = B - 1;
  for (int32_t i = 0; i < B; i++) {
    run += og_sym(b, r, i);
    if (run > t) { u = i; break; }
  }
  int64_t dau = b->dout[u] + b->din[u];
  if (og_accept_uniform(x[1], dau, B)) return og_skip_r((int32_t)og_draw_below(x[2], B), r, B);
  int64_t wsum = dau - og_sym(b, u, r);                  /* :845-847 */
  if (wsum == 0) return og_skip_r((int32_t)og_draw_below(x[2], B), r, B);
  int64_t t2 = og_draw_below(x[2], wsum);
  run = 0;
  for (int32_t i = 0; i < B; i++) {
    if (i == r) continue;
    run += og_sym(b, u, i);
    if (run > t2) return i;
  }
  return B - 1;  /* unreachable: run reaches wsum > t2 */
}

/* _propose_new_partition_nodal (:1006-1064): a neighbour (out-list then
 * in-list, weighted) gives u; then a uniform block with probability
 * B/(d_a[u]+B), else a block from M[u,:]+M[:,u] (r included).             */
int32_t og_nodal_propose(const og_graph* g, const int32_t* part, const og_blocks* b,
                         int32_t v, int32_t itr, int32_t stage, uint64_t seed) {
  int32_t B = b->B;
  uint32_t x[4];
  og_draws(seed, (uint32_t)v, (uint32_t)itr, (uint32_t)stage, OG_TAG_NODAL, x);
  int64_t k = g->kout[v] + g->kin[v];
  if (k == 0) return (int32_t)og_draw_below(x[2], B);
  int64_t t = og_draw_below(x[0], k), run = 0;
  int32_t nbr = -1;
  for (int64_t p = g->out_ptr[v]; p < g->out_ptr[v + 1] && nbr < 0; p++) {
    run += g->out_w[p];
    if (run > t) nbr = g->out_idx[p];
  }
  for (int64_t p = g->in_ptr[v]; p < g->in_ptr[v + 1] && nbr < 0; p++) {
    run += g->in_w[p];
    if (run > t) nbr = g->in_idx[p];
  }
  int32_t u = part[nbr];
  int64_t dau = b->dout[u] + b->din[u];
  if (og_accept_uniform(x[1], dau, B)) return (int32_t)og_draw_below(x[2], B);
  int64_t t2 = og_draw_below(x[2], dau);
  run = 0;
  for (int32_t i = 0; i < B; i++) {
    run += og_sym(b, u, i);
    if (run > t2) return i;
  }
  return B - 1;  /* unreachable */
}

/* block_merge task (:349-368): K proposals per block, first strict minimum */
typedef struct {
  const og_graph* g;
  const og_blocks* b;
  int32_t K, stage;
  uint64_t seed;
  int32_t* best_s;
  int64_t* best_q;
} og_merge_task;

static void og_merge_block(void* ctx, int32_t r, int32_t worker) {
  (void)worker;
  og_merge_task* t = (og_merge_task*)ctx;
  t->best_s[r] = -1;
  t->best_q[r] = INT64_MAX;
  for (int32_t k = 0; k < t->K; k++) {
    int32_t s = og_merge_propose(t->g, t->b, r, k, t->stage, t->seed);
    int64_t q = og_merge_dq(t->g, t->b, r, s);
    if (q < t->best_q[r]) {
      t->best_q[r] = q;
      t->best_s[r] = s;
    }
  }
}

void og_merge_phase(const og_graph* g, const og_blocks* b, int32_t K, int32_t stage,
                    uint64_t seed, int32_t* best_s, int64_t* best_q) {
  og_merge_task t = {g, b, K, stage, seed, best_s, best_q};
  /* blocks are independent (the block_merge task runs them in parallel) */
  og_parallel_for(b->B, og_merge_block, &t);
}

/* _carry_out_best_merges (:1225-1279), sequential as in the reference, with
 * the sort made stable on (dS, block).  Returns the new B (B - merges);
 * *merged receives the number of merges carried out.                       */
static const int64_t* og_sort_keys;
static int og_cmp_merge(const void* a, const void* b) {
  int32_t i = *(const int32_t*)a, j = *(const int32_t*)b;
  if (og_sort_keys[i] < og_sort_keys[j]) return -1;
  if (og_sort_keys[i] > og_sort_keys[j]) return 1;
  return (i > j) - (i < j);
}

int32_t og_merge_apply(int32_t n, int32_t* part, int32_t B, const int32_t* best_s,
                       const int64_t* best_q, int32_t b_to_merge, int32_t* merged) {
  int32_t* order = malloc(sizeof(int32_t) * ((size_t)B + 1));
  int32_t* map = malloc(sizeof(int32_t) * ((size_t)B + 1));
  for (int32_t i = 0; i < B; i++) { order[i] = i; map[i] = i; }
  og_sort_keys = best_q;
  qsort(order, (size_t)B, sizeof(int32_t), og_cmp_merge);
  int32_t num = 0, counter = 0;
  while (num < b_to_merge && counter < B) {
    int32_t from = order[counter];
    int32_t to = map[best_s[from]];
    counter++;
    if (to != from) {
      for (int32_t i = 0; i < B; i++) if (map[i] == from) map[i] = to;
      for (int32_t v = 0; v < n; v++) if (part[v] == from) part[v] = to;
      num++;
    }
  }
  /* compact the labels still present, ascending (:1259-1277) */
  uint8_t* present = calloc((size_t)B + 1, 1);
  for (int32_t v = 0; v < n; v++) present[part[v]] = 1;
  int32_t next = 0;
  for (int32_t i = 0; i < B; i++) map[i] = present[i] ? next++ : -1;
  for (int32_t v = 0; v < n; v++) part[v] = map[part[v]];
  free(order); free(map); free(present);
  *merged = num;
  return B - num;
}

/* nodal_move + update tasks for one batch (:397-443).  precision 3: the
 * accept decision is the reference's float dS < 0 (-inf included), and the
 * accepted float values are what the convergence sums add (:428-430), in
 * Q32; the exact value still gives prop_q.  The near-threshold count is
 * of the deciding value: |dS| <= 1e-9 exactly, or the float dS in
 * precision 3.
 * prop_f (optional) receives the float dS of each proposal.               */
typedef struct {
  const og_graph* g;
  const int32_t* part;
  const og_blocks* b;
  int32_t beg, itr, stage, precision;
  uint64_t seed;
  int32_t *prop_s, *prop_ninf, *mv;
  int64_t* prop_q;
  float* prop_f;
  /* per worker: moves, accepted sum (Q32), near-threshold count, -inf flag */
  int64_t moves[OG_MAX_WORKERS], cq[OG_MAX_WORKERS], nnear[OG_MAX_WORKERS];
  int32_t cn[OG_MAX_WORKERS];
} og_nodal_task;

static void og_nodal_item(void* ctx, int32_t i, int32_t w) {
  og_nodal_task* t = (og_nodal_task*)ctx;
  const int32_t v = t->beg + i;
  int32_t s = og_nodal_propose(t->g, t->part, t->b, v, t->itr, t->stage, t->seed);
  int32_t ninf = 0;
  int64_t q = 0;
  float f = 0.0f;
  int32_t r = t->part[v];
  int accept = 0;
  if (s != r) {
    q = og_nodal_dq(t->g, t->part, t->b, v, s, &ninf);
    if (t->precision == 3) {
      f = og_nodal_ds_ref32(t->g, t->part, t->b, v, s);
      accept = f < 0.0f;
      if (!isinf(f) && fabs((double)f) <= 1e-9) t->nnear[w]++;
    } else {
      accept = ninf || q < 0;
      if (!ninf && (q <= OG_NEAR_Q && q >= -OG_NEAR_Q)) t->nnear[w]++;
    }
  }
  if (t->prop_s) t->prop_s[i] = (s != r) ? s : -1;
  if (t->prop_q) t->prop_q[i] = q;
  if (t->prop_ninf) t->prop_ninf[i] = ninf;
  if (t->prop_f) t->prop_f[i] = f;
  t->mv[i] = accept ? s : -1;
  if (accept) {
    t->moves[w]++;
    if (t->precision == 3) {
      if (isinf(f)) t->cn[w] = 1;
      else t->cq[w] += og_q32_f(f);
    } else if (ninf) {
      t->cn[w] = 1;
    } else {
      t->cq[w] += q;
    }
  }
}

/* one batch (:397-443): every proposal reads the batch-start state (the
 * reference runs them in parallel, so this loop does too), then the
 * accepted moves are applied and M rebuilt */
int64_t og_nodal_batch_p(const og_graph* g, int32_t* part, og_blocks* b, int32_t beg,
                         int32_t end, int32_t itr, int32_t stage, uint64_t seed, int32_t precision,
                         int32_t* prop_s, int64_t* prop_q, int32_t* prop_ninf, float* prop_f,
                         int64_t* cum_q, int32_t* cum_ninf, int64_t* near_threshold) {
  int32_t cnt = end - beg;
  og_nodal_task* t = calloc(1, sizeof(og_nodal_task));
  t->g = g; t->part = part; t->b = b; t->beg = beg; t->itr = itr; t->stage = stage;
  t->precision = precision; t->seed = seed;
  t->prop_s = prop_s; t->prop_q = prop_q; t->prop_ninf = prop_ninf; t->prop_f = prop_f;
  t->mv = malloc(sizeof(int32_t) * ((size_t)cnt + 1));
  og_parallel_for(cnt, og_nodal_item, t);
  int64_t moves = 0;
  for (int32_t w = 0; w < OG_MAX_WORKERS; w++) {
    moves += t->moves[w];
    *cum_q += t->cq[w];
    if (t->cn[w]) *cum_ninf = 1;
    if (near_threshold) *near_threshold += t->nnear[w];
  }
  for (int32_t v = beg; v < end; v++)
    if (t->mv[v - beg] >= 0) part[v] = t->mv[v - beg];
  og_build(g, part, b);
  free(t->mv);
  free(t);
  return moves;
}

int64_t og_nodal_batch(const og_graph* g, int32_t* part, og_blocks* b, int32_t beg,
                       int32_t end, int32_t itr, int32_t stage, uint64_t seed,
                       int32_t* prop_s, int64_t* prop_q, int32_t* prop_ninf,
                       int64_t* cum_q, int32_t* cum_ninf, int64_t* near_threshold) {
  return og_nodal_batch_p(g, part, b, beg, end, itr, stage, seed, 0, prop_s, prop_q, prop_ninf, NULL,
                          cum_q, cum_ninf, near_threshold);
}

/* ------------------------------------------------------------------------ */
/* Checksums for traces.                                                    */
static inline uint64_t og_mix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

uint64_t og_hash_part(const int32_t* part, int32_t n) {
  uint64_t h = 1469598103934665603ull;
  for (int32_t v = 0; v < n; v++) {
    h ^= (uint32_t)part[v];
    h *= 1099511628211ull;
  }
  return h;
}

uint64_t og_hash_blocks(const og_blocks* b, uint64_t* h_deg) {
  uint64_t h = 0, hd = 0;
  int32_t B = b->B;
  for (int32_t i = 0; i < B; i++) {
    for (int32_t j = 0; j < B; j++) {
      int64_t m = b->M[(size_t)i * B + j];
      if (m) h += og_mix(og_mix(((uint64_t)i << 32) | (uint32_t)j) ^ (uint64_t)m);
    }
    hd += og_mix(og_mix((uint64_t)i) ^ (((uint64_t)b->dout[i] << 32) ^ (uint64_t)b->din[i]));
  }
  if (h_deg) *h_deg = hd;
  return h;
}

static void og_emit(og_trace_fn trace, void* user, og_trace_event* ev, const og_graph* g,
                    const int32_t* part, const og_blocks* b) {
  if (!trace) return;
  ev->h_part = og_hash_part(part, g->n);
  ev->h_M = og_hash_blocks(b, &ev->h_deg);
  trace(user, ev);
}

/* ------------------------------------------------------------------------ */
/* Whole solve: partition() (:322-512) with the golden-section bookkeeping
 * of _prepare_for_partition_next (:1322-1365).                             */
void og_params_default(og_params* p) {
  p->num_agg_proposals_per_block = 10;
  p->num_block_reduction_rate = 0.5f;
  p->max_num_nodal_itr = 100;
  p->num_batch_nodal_update = 4;
  p->delta_entropy_threshold1 = 5e-4;
  p->delta_entropy_threshold2 = 1e-4;
  p->delta_entropy_moving_avg_window = 3;
  p->dfs_depth = 20;
  p->seed = 0;
  p->init_mode = 0;
  p->precision = 3;   /* the reference's float nodal dS, as usap_params_default */
}

static inline int32_t og_reduce(int32_t B, float rate) {
  return (int32_t)((float)B * rate);       /* (size_t)_P.B * rate, :340, :1343 */
}

void og_golden_init(og_golden* gs) { memset(gs, 0, sizeof(*gs)); }

/* _prepare_for_partition_next (:1322-1365) on slot indices: the state just
 * finished (B, S, held in buffer cur_slot) enters the bracket; on return
 * *restore_slot names the buffer to continue from (copied, so the bracket
 * keeps it), *btm the merges to do next, and *free_slot a buffer no longer
 * referenced by the bracket.  Returns 1 when the search is over (the answer
 * is gs->med).                                                             */
int og_golden_step(og_golden* gs, int32_t B, double S, int64_t S_q, int32_t cur_slot, float rate,
                   int32_t* restore_slot, int32_t* btm, int32_t* free_slot) {
  og_gpoint cur = {B, S, S_q, 1, cur_slot};
  og_gpoint* med = &gs->med;
  int32_t freed;
  if (!med->finite || cur.S <= med->S) {
    if (med->B > cur.B) { freed = gs->large.slot; gs->large = *med; }
    else { freed = gs->small.slot; gs->small = *med; }
    *med = cur;
  } else {
    if (med->B > cur.B) { freed = gs->small.slot; gs->small = cur; }
    else { freed = gs->large.slot; gs->large = cur; }
  }
  *free_slot = freed;
  *restore_slot = -1;
  *btm = 0;
  if (!gs->small.finite) {
    *restore_slot = med->slot;
    *btm = og_reduce(med->B, rate);
    return *btm == 0;
  }
  if (!gs->large.finite) {
    /* the reference continues from an empty default state here (its
       bracket has no upper end); the search stops at med instead */
    return 1;
  }
  if (gs->large.B - gs->small.B == 2) return 1;
  if ((gs->large.B - med->B) >= (med->B - gs->small.B)) {
    int32_t next_B = med->B + (int32_t)round((double)(gs->large.B - med->B) * 0.618);
    *restore_slot = gs->large.slot;
    *btm = gs->large.B - next_B;
  } else {
    int32_t next_B = gs->small.B + (int32_t)round((double)(med->B - gs->small.B) * 0.618);
    *restore_slot = med->slot;
    *btm = med->B - next_B;
  }
  return 0;
}

/* labels renumbered 0..B-1 in ascending order of their values; returns B,
   or -1 for a negative label */
int32_t og_compact_labels(const int32_t* init, int32_t n, int32_t* part) {
  int32_t mx = -1;
  for (int32_t v = 0; v < n; v++) {
    if (init[v] < 0) return -1;
    if (init[v] > mx) mx = init[v];
  }
  int32_t* map = malloc(sizeof(int32_t) * ((size_t)mx + 1));
  for (int32_t i = 0; i <= mx; i++) map[i] = -1;
  for (int32_t v = 0; v < n; v++) map[init[v]] = 0;
  int32_t B = 0;
  for (int32_t i = 0; i <= mx; i++)
    if (map[i] == 0) map[i] = B++;
  for (int32_t v = 0; v < n; v++) part[v] = map[init[v]];
  free(map);
  return B;
}

static int og_partition_impl(const og_graph* g, const og_params* p, const int32_t* init, int32_t* part_out,
                             og_result* res, og_trace_fn trace, void* user);

int og_partition(const og_graph* g, const og_params* p, int32_t* part_out,
                 og_result* res, og_trace_fn trace, void* user) {
  return og_partition_impl(g, p, NULL, part_out, res, trace, user);
}

/* the solve from a given initial partition instead of the SCC pass (the
   CUDA path's usap_ctx_partition_from; streaming input) */
int og_partition_from(const og_graph* g, const og_params* p, const int32_t* init, int32_t* part_out,
                      og_result* res, og_trace_fn trace, void* user) {
  if (!init) return -1;
  return og_partition_impl(g, p, init, part_out, res, trace, user);
}

static int og_partition_impl(const og_graph* g, const og_params* p, const int32_t* init, int32_t* part_out,
                             og_result* res, og_trace_fn trace, void* user) {
  int32_t n = g->n;
  memset(res, 0, sizeof(*res));
  if (n <= 0 || g->e <= 0) return -1;
  size_t pn = sizeof(int32_t) * (size_t)n;
  /* four partition buffers: the working state plus the three bracket
     points; slot 0 starts as the working state */
  int32_t* slots[4];
  for (int i = 0; i < 4; i++) slots[i] = malloc(pn);
  int32_t work = 0;
  int32_t* part = slots[work];
  int32_t B;
  if (init) {
    B = og_compact_labels(init, n, part);
    if (B < 0) {
      for (int i = 0; i < 4; i++) free(slots[i]);
      return -1;
    }
  } else if (p->init_mode == 1) {
    for (int32_t v = 0; v < n; v++) part[v] = v;
    B = n;
  } else {
    B = og_scc(g, p->dfs_depth, part);
  }
  int32_t Bmax = B;
  int32_t btm = og_reduce(B, p->num_block_reduction_rate);
  int32_t K = p->num_agg_proposals_per_block;
  int32_t W = p->delta_entropy_moving_avg_window;
  int32_t maxitr = p->max_num_nodal_itr;
  int32_t bs = n / p->num_batch_nodal_update;
  if (bs < 1) bs = 1;
  int32_t* best_s = malloc(sizeof(int32_t) * (size_t)Bmax);
  int64_t* best_q = malloc(sizeof(int64_t) * (size_t)Bmax);
  int64_t* ide_q = calloc((size_t)(maxitr > 0 ? maxitr : 1), sizeof(int64_t));
  int32_t* ide_n = calloc((size_t)(maxitr > 0 ? maxitr : 1), sizeof(int32_t));
  og_golden gs;
  og_golden_init(&gs);
  gs.large.slot = gs.med.slot = gs.small.slot = -1;
  og_blocks blk = {0};
  int32_t stage = 0;
  int rc = 0;
  for (;;) {
    /* merge phase on the current state */
    og_blocks_free(&blk);
    if (og_blocks_alloc(&blk, B)) { rc = -3; break; }
    og_build(g, part, &blk);
    og_merge_phase(g, &blk, K, stage, p->seed, best_s, best_q);
    int32_t merged = 0;
    B = og_merge_apply(n, part, B, best_s, best_q, btm, &merged);
    if (merged < btm) res->merge_shortfall += btm - merged;
    og_blocks_free(&blk);
    if (og_blocks_alloc(&blk, B)) { rc = -3; break; }
    og_build(g, part, &blk);
    og_trace_event ev;
    memset(&ev, 0, sizeof(ev));
    ev.kind = 1; ev.stage = stage; ev.B = B;
    og_emit(trace, user, &ev, g, part, &blk);

    /* batched nodal sweeps (:374-478) */
    memset(ide_q, 0, sizeof(int64_t) * (size_t)maxitr);
    memset(ide_n, 0, sizeof(int32_t) * (size_t)maxitr);
    int isf = gs.large.finite && gs.med.finite && gs.small.finite;
    double thr = isf ? p->delta_entropy_threshold2 : p->delta_entropy_threshold1;
    int converged = 0;
    const double model = og_model_S(n, g->e, B);
    int32_t stage_sweeps = 0;
    for (int32_t itr = 0; itr < maxitr && !converged; itr++) {
      int64_t S_q = og_data_q(g, &blk);   /* data term; S = model + S_q / 2^32 */
      int32_t S_n = 0;
      double mean = 0.0;
      if (itr >= W - 1) {
        int64_t sum = 0;
        int32_t ninf = 0;
        for (int32_t i = itr - W + 1; i < itr; i++) { sum += ide_q[i]; ninf |= ide_n[i]; }
        mean = ninf ? -INFINITY : ((double)sum / OG_Q32_SCALE) / (double)(W - 1);
      }
      int64_t cum_q = 0;
      int32_t cum_n = 0;
      res->sweeps++;
      stage_sweeps++;
      for (int32_t beg = 0; beg < n; beg += bs) {
        int32_t end = beg + bs < n ? beg + bs : n;
        int64_t mv = og_nodal_batch_p(g, part, &blk, beg, end, itr, stage, p->seed, p->precision,
                                      NULL, NULL, NULL, NULL, &cum_q, &cum_n, &res->near_threshold);
        res->batches++;
        res->nodal_proposals += end - beg;
        res->nodal_moves += mv;
        ide_q[itr] = cum_q;
        ide_n[itr] = cum_n;
        S_q += cum_q;
        S_n |= cum_n;
        memset(&ev, 0, sizeof(ev));
        ev.kind = 2; ev.stage = stage; ev.itr = itr; ev.batch_beg = beg; ev.B = B;
        ev.S_q = S_q; ev.S_ninf = S_n; ev.cum_q = cum_q; ev.cum_ninf = cum_n; ev.moves = mv;
        og_emit(trace, user, &ev, g, part, &blk);
        if (itr >= W - 1) {
          double S_d = S_n ? -INFINITY : og_desc_length(model, S_q);
          if (-mean < thr * S_d) { converged = 1; break; }
        }
      }
    }
    const int64_t data_fin = og_data_q(g, &blk);
    const double S_fin = og_desc_length(model, data_fin);
    const int64_t S_fin_q = og_add_sat(og_quantize(model), data_fin);
    memset(&ev, 0, sizeof(ev));
    ev.kind = 3; ev.stage = stage; ev.itr = stage_sweeps; ev.B = B; ev.S_q = S_fin_q;
    og_emit(trace, user, &ev, g, part, &blk);
    res->stages++;
    stage++;

    int32_t restore = -1, freed = -1;
    int done = og_golden_step(&gs, B, S_fin, S_fin_q, work, p->num_block_reduction_rate, &restore,
                              &btm, &freed);
    if (done) {
      memcpy(part_out, slots[gs.med.slot], pn);
      res->B = gs.med.B;
      res->S_q = gs.med.S_q;
      res->S = gs.med.S;
      break;
    }
    /* a buffer outside the bracket becomes the working state */
    int used[4] = {0, 0, 0, 0};
    if (gs.large.finite) used[gs.large.slot] = 1;
    if (gs.med.finite) used[gs.med.slot] = 1;
    if (gs.small.finite) used[gs.small.slot] = 1;
    work = -1;
    for (int i = 0; i < 4; i++) if (!used[i]) { work = i; break; }
    (void)freed;
    part = slots[work];
    memcpy(part, slots[restore], pn);
    B = restore == gs.large.slot ? gs.large.B : gs.med.B;
  }
  og_blocks_free(&blk);
  for (int i = 0; i < 4; i++) free(slots[i]);
  free(best_s); free(best_q); free(ide_q); free(ide_n);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* Scores of bf::evaluate (evaluate.hpp:18-266), FP64, plus NMI.            */
int og_evaluate(const int32_t* truth, const int32_t* given, int64_t n, og_scores* s) {
  memset(s, 0, sizeof(*s));
  int32_t b1 = 0, b2 = 0;
  for (int64_t i = 0; i < n; i++) {
    if (truth[i] + 1 > b1) b1 = truth[i] + 1;
    if (given[i] + 1 > b2) b2 = given[i] + 1;
  }
  if (n <= 1 || b1 <= 0 || b2 <= 0) return -1;
  int64_t* ct = calloc((size_t)b1 * (size_t)b2, sizeof(int64_t));
  int64_t* rows = calloc((size_t)b1, sizeof(int64_t));
  int64_t* cols = calloc((size_t)b2, sizeof(int64_t));
  int64_t N = 0;
  for (int64_t i = 0; i < n; i++) {
    if (truth[i] < 0) continue;
    ct[(size_t)truth[i] * b2 + given[i]]++;
    rows[truth[i]]++;
    cols[given[i]]++;
    N++;
  }
  int32_t nb1 = 0;
  for (int32_t i = 0; i < b1; i++) nb1 += rows[i] > 0;
  double pairs = (double)N * (double)(N - 1) / 2.0;
  double sq = 0, same = 0, sr = 0, sc = 0, s1 = 0, s2 = 0;
  for (size_t k = 0; k < (size_t)b1 * b2; k++) {
    double c = (double)ct[k];
    sq += c * c;
    same += c * (c - 1) / 2;
  }
  for (int32_t i = 0; i < b1; i++) { sr += (double)rows[i] * rows[i]; s1 += (double)rows[i] * (rows[i] - 1) / 2; }
  for (int32_t j = 0; j < b2; j++) { sc += (double)cols[j] * cols[j]; s2 += (double)cols[j] * (cols[j] - 1) / 2; }
  double diff = ((double)N * (double)N + sq - sc - sr) / 2.0;
  s->rand_index = (same + diff) / pairs;
  /* the reference divides the expected index in integers (size_t,
     evaluate.hpp:175-176): floor(s1*s2/pairs) */
  {
    unsigned __int128 num = (unsigned __int128)(uint64_t)s1 * (uint64_t)s2;
    uint64_t pr = (uint64_t)N * (uint64_t)(N - 1) / 2;
    double expected = (double)(uint64_t)(num / pr);
    s->adjusted_rand_index = (same - expected) / (0.5 * (s1 + s2) - expected);
    s->adjusted_rand_index_exact = (same - s1 * s2 / pairs) / (0.5 * (s1 + s2) - s1 * s2 / pairs);
  }
  s->pairwise_recall = same / s1;
  s->pairwise_precision = same / s2;
  double H1 = 0, H2 = 0, H21 = 0, H12 = 0, MI = 0, dN = (double)N;
  for (int32_t i = 0; i < b1; i++) if (rows[i]) { double p = rows[i] / dN; H1 -= p * log(p); }
  for (int32_t j = 0; j < b2; j++) if (cols[j]) { double p = cols[j] / dN; H2 -= p * log(p); }
  for (int32_t i = 0; i < b1; i++)
    for (int32_t j = 0; j < b2; j++) {
      int64_t c = ct[(size_t)i * b2 + j];
      if (!c) continue;
      double pj = c / dN, p1 = rows[i] / dN, p2 = cols[j] / dN;
      H21 -= pj * log(pj / p1);
      H12 -= pj * log(pj / p2);
      MI += pj * log(pj / (p1 * p2));
    }
  s->h_truth = H1; s->h_given = H2; s->h_given_truth = H21; s->h_truth_given = H12; s->mi = MI;
  s->nmi = (H1 + H2) > 0 ? 2.0 * MI / (H1 + H2) : 1.0;
  s->nmi_sqrt = (H1 > 0 && H2 > 0) ? MI / sqrt(H1 * H2) : 1.0;
  s->missed_info = H1 > 0 ? H12 / H1 : 0.0;
  s->erroneous_info = H2 > 0 ? H21 / H2 : 0.0;
  s->n = N; s->b_truth = nb1; s->b_given = b2;
  free(ct); free(rows); free(cols);
  return 0;
}
