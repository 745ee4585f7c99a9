// Partition scores (bf::evaluate, include/evaluate.hpp:18-266), returned
// instead of printed, computed from exact integer pair counts and
// fixed-point information sums (eval_common.h), which the device version
// (kernels_eval.cu) reproduces bit for bit.
//
// bf::evaluate permutes the contingency table's columns by a Kuhn-Munkres
// matching before scoring; the pair-counting and information scores do not
// depend on that permutation, so they are computed on the table itself.
// Two quirks of the reference are kept where they define a printed number:
// the adjusted Rand index divides its expected index in integers
// (evaluate.hpp:175-176, size_t arithmetic), and "accuracy" is the matched
// fraction of the best one-to-one block matching (the reference's matcher
// negates unsigned costs, evaluate.hpp:62-67, which makes its own figure
// unreliable; a correct Hungarian matching is used here).  The exact ARI
// is reported beside it.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <unordered_map>
#include <vector>

#include "eval_common.h"
#include "job.h"

namespace usap {

namespace {

// maximum-weight perfect matching on a square matrix (Hungarian algorithm,
// potentials form, O(n^3)); returns the matched weight
int64_t hungarian_max(const std::vector<int64_t>& w, int n) {
  const int64_t INF = std::numeric_limits<int64_t>::max() / 4;
  std::vector<int64_t> u(n + 1, 0), v(n + 1, 0), minv(n + 1);
  std::vector<int> p(n + 1, 0), way(n + 1, 0);
  std::vector<char> used(n + 1);
  for (int i = 1; i <= n; i++) {
    p[0] = i;
    int j0 = 0;
    std::fill(minv.begin(), minv.end(), INF);
    std::fill(used.begin(), used.end(), 0);
    do {
      used[j0] = 1;
      int i0 = p[j0], j1 = 0;
      int64_t delta = INF;
      for (int j = 1; j <= n; j++) {
        if (used[j]) continue;
        int64_t cur = -w[static_cast<size_t>(i0 - 1) * n + (j - 1)] - u[i0] - v[j];
        if (cur < minv[j]) {
          minv[j] = cur;
          way[j] = j0;
        }
        if (minv[j] < delta) {
          delta = minv[j];
          j1 = j;
        }
      }
      for (int j = 0; j <= n; j++) {
        if (used[j]) {
          u[p[j]] += delta;
          v[j] -= delta;
        } else {
          minv[j] -= delta;
        }
      }
      j0 = j1;
    } while (p[j0] != 0);
    do {
      int j1 = way[j0];
      p[j0] = p[j1];
      j0 = j1;
    } while (j0);
  }
  int64_t total = 0;
  for (int j = 1; j <= n; j++)
    if (p[j]) total += w[static_cast<size_t>(p[j] - 1) * n + (j - 1)];
  return total;
}

}  // namespace

void scores_from_sums(const EvalSums& e, usap_scores* s) {
  std::memset(s, 0, sizeof(*s));
  const int64_t N = e.N;
  const double dN = static_cast<double>(N);
  const double pairs = dN * static_cast<double>(N - 1) / 2.0;
  const double same = static_cast<double>(e.same), s1 = static_cast<double>(e.s1), s2 = static_cast<double>(e.s2);
  const double diff = (dN * dN + static_cast<double>(e.sq) - static_cast<double>(e.sc) - static_cast<double>(e.sr)) / 2.0;
  s->rand_index = (same + diff) / pairs;
  {
    unsigned __int128 num = static_cast<unsigned __int128>(static_cast<uint64_t>(e.s1)) * static_cast<uint64_t>(e.s2);
    uint64_t pr = static_cast<uint64_t>(N) * static_cast<uint64_t>(N - 1) / 2;
    double expected = static_cast<double>(static_cast<uint64_t>(num / pr));
    s->adjusted_rand_index = (same - expected) / (0.5 * (s1 + s2) - expected);
    double ex = s1 * s2 / pairs;
    s->adjusted_rand_index_exact = (same - ex) / (0.5 * (s1 + s2) - ex);
  }
  s->pairwise_recall = same / s1;
  s->pairwise_precision = same / s2;
  const double H1 = -static_cast<double>(e.h_truth_q) / kQ50;
  const double H2 = -static_cast<double>(e.h_given_q) / kQ50;
  const double H21 = -static_cast<double>(e.h_gt_q) / kQ50;
  const double H12 = -static_cast<double>(e.h_tg_q) / kQ50;
  const double MI = static_cast<double>(e.mi_q) / kQ50;
  s->h_truth = H1;
  s->h_given = H2;
  s->h_given_truth = H21;
  s->h_truth_given = H12;
  s->mi = MI;
  s->nmi = (H1 + H2) > 0 ? 2.0 * MI / (H1 + H2) : 1.0;
  s->nmi_sqrt = (H1 > 0 && H2 > 0) ? MI / std::sqrt(H1 * H2) : 1.0;
  s->missed_info = H1 > 0 ? H12 / H1 : 0.0;
  s->erroneous_info = H2 > 0 ? H21 / H2 : 0.0;
  s->n = N;
  s->b_truth = e.nb_truth;
  s->b_given = e.nb_given;
}

double matching_accuracy(const int64_t* table, int b1, int b2, int64_t N) {
  const int m = b1 > b2 ? b1 : b2;
  if (m > 2048) return std::nan("");
  std::vector<int64_t> w(static_cast<size_t>(m) * m, 0);
  for (int i = 0; i < b1; i++)
    for (int j = 0; j < b2; j++) w[static_cast<size_t>(i) * m + j] = table[static_cast<size_t>(i) * b2 + j];
  return static_cast<double>(hungarian_max(w, m)) / static_cast<double>(N);
}

void evaluate_host(const int32_t* truth, const int32_t* given, int64_t n, usap_scores* s) {
  std::memset(s, 0, sizeof(*s));
  int32_t b1 = 0, b2 = 0;
  for (int64_t i = 0; i < n; i++) {
    if (given[i] < 0) throw Error(USAP_ERR_INVALID, "given labels must be >= 0");
    if (truth[i] < -1) throw Error(USAP_ERR_INVALID, "truth labels must be >= -1");
    if (truth[i] + 1 > b1) b1 = truth[i] + 1;
    if (given[i] + 1 > b2) b2 = given[i] + 1;
  }
  if (n < 2 || b1 <= 0 || b2 <= 0) throw Error(USAP_ERR_INVALID, "need at least two labelled vertices");
  std::vector<int64_t> rows(b1, 0), cols(b2, 0);
  std::unordered_map<int64_t, int64_t> cells;
  int64_t N = 0;
  for (int64_t i = 0; i < n; i++) {
    if (truth[i] < 0) continue;   // -1: unknown truth (evaluate.hpp:40)
    cells[static_cast<int64_t>(truth[i]) * b2 + given[i]]++;
    rows[truth[i]]++;
    cols[given[i]]++;
    N++;
  }
  if (N < 2) throw Error(USAP_ERR_INVALID, "need at least two vertices with known truth");
  const std::shared_ptr<const std::vector<double>> Lp = log_table(N);
  const std::vector<double>& L = *Lp;
  const double dN = static_cast<double>(N), LN = L[N];
  EvalSums e{};
  e.N = N;
  for (const auto& kv : cells) {
    const int64_t c = kv.second, i = kv.first / b2, j = kv.first % b2;
    e.sq += c * c;
    e.same += c * (c - 1) / 2;
    e.h_gt_q += ev_term(c, dN, L[c], L[rows[i]]);
    e.h_tg_q += ev_term(c, dN, L[c], L[cols[j]]);
    e.mi_q += ev_mi_term(c, dN, L[c], LN, L[rows[i]], L[cols[j]]);
  }
  for (int64_t r : rows)
    if (r) {
      e.sr += r * r;
      e.s1 += r * (r - 1) / 2;
      e.nb_truth++;
      e.h_truth_q += ev_term(r, dN, L[r], LN);
    }
  for (int64_t c : cols)
    if (c) {
      e.sc += c * c;
      e.s2 += c * (c - 1) / 2;
      e.nb_given++;
      e.h_given_q += ev_term(c, dN, L[c], LN);
    }
  scores_from_sums(e, s);
  // accuracy: best one-to-one matching of truth blocks to given blocks
  const int m = b1 > b2 ? b1 : b2;
  if (m <= 2048) {
    std::vector<int64_t> t(static_cast<size_t>(b1) * b2, 0);
    for (const auto& kv : cells) t[static_cast<size_t>(kv.first)] = kv.second;
    s->accuracy = matching_accuracy(t.data(), b1, b2, N);
  } else {
    s->accuracy = std::nan("");
  }
}

}  // namespace usap
