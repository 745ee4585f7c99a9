// Partition scores (bf::evaluate, include/evaluate.hpp:18-266), returned
// instead of printed, in FP64 with exact integer pair counts.
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
#include <cmath>
#include <cstring>
#include <limits>
#include <unordered_map>
#include <vector>

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

void evaluate_host(const int32_t* truth, const int32_t* given, int64_t n, usap_scores* s) {
  std::memset(s, 0, sizeof(*s));
  int32_t b1 = 0, b2 = 0;
  for (int64_t i = 0; i < n; i++) {
    if (given[i] < 0) throw Error(USAP_ERR_INVALID, "given labels must be >= 0");
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
  const double pairs = static_cast<double>(N) * static_cast<double>(N - 1) / 2.0;
  double sq = 0, same = 0, sr = 0, sc = 0, s1 = 0, s2 = 0;
  for (const auto& kv : cells) {
    double c = static_cast<double>(kv.second);
    sq += c * c;
    same += c * (c - 1) / 2;
  }
  int32_t nb1 = 0, nb2 = 0;
  for (int64_t r : rows) {
    sr += static_cast<double>(r) * r;
    s1 += static_cast<double>(r) * (r - 1) / 2;
    nb1 += r > 0;
  }
  for (int64_t c : cols) {
    sc += static_cast<double>(c) * c;
    s2 += static_cast<double>(c) * (c - 1) / 2;
    nb2 += c > 0;
  }
  const double diff = (static_cast<double>(N) * N + sq - sc - sr) / 2.0;
  s->rand_index = (same + diff) / pairs;
  {
    unsigned __int128 num = static_cast<unsigned __int128>(static_cast<uint64_t>(s1)) * static_cast<uint64_t>(s2);
    uint64_t pr = static_cast<uint64_t>(N) * static_cast<uint64_t>(N - 1) / 2;
    double expected = static_cast<double>(static_cast<uint64_t>(num / pr));
    s->adjusted_rand_index = (same - expected) / (0.5 * (s1 + s2) - expected);
    double ex = s1 * s2 / pairs;
    s->adjusted_rand_index_exact = (same - ex) / (0.5 * (s1 + s2) - ex);
  }
  s->pairwise_recall = same / s1;
  s->pairwise_precision = same / s2;
  const double dN = static_cast<double>(N);
  double H1 = 0, H2 = 0, H21 = 0, H12 = 0, MI = 0;
  for (int64_t r : rows)
    if (r) {
      double p = r / dN;
      H1 -= p * std::log(p);
    }
  for (int64_t c : cols)
    if (c) {
      double p = c / dN;
      H2 -= p * std::log(p);
    }
  for (const auto& kv : cells) {
    int64_t i = kv.first / b2, j = kv.first % b2;
    double pj = kv.second / dN, p1 = rows[i] / dN, p2 = cols[j] / dN;
    H21 -= pj * std::log(pj / p1);
    H12 -= pj * std::log(pj / p2);
    MI += pj * std::log(pj / (p1 * p2));
  }
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
  s->b_truth = nb1;
  s->b_given = nb2;
  // accuracy: best one-to-one matching of truth blocks to given blocks
  const int m = b1 > b2 ? b1 : b2;
  if (m <= 2048) {
    std::vector<int64_t> w(static_cast<size_t>(m) * m, 0);
    for (const auto& kv : cells) {
      int64_t i = kv.first / b2, j = kv.first % b2;
      w[static_cast<size_t>(i) * m + j] = kv.second;
    }
    s->accuracy = static_cast<double>(hungarian_max(w, m)) / dN;
  } else {
    s->accuracy = std::nan("");
  }
}

}  // namespace usap
