// Canonical arithmetic of the partition scores (bf::evaluate,
// include/evaluate.hpp:18-266), shared by the host and the device versions
// so that both give the same bits.
//
// Everything is derived from the contingency table c[i][j] (truth block i,
// given block j), its row sums r[i] and column sums s[j], and N:
//  * pair counts are exact integers: sum c^2, sum c(c-1)/2 and the same
//    over rows and columns (int64; N < 2^31);
//  * every information term p log p' is evaluated in FP64 from a table of
//    log k for integers k (log of a ratio of counts is a difference of table
//    entries), each operation rounded as written, and rounded on its own to
//    a fixed-point integer with 50 fraction bits; the terms are summed in
//    int64, so the sums do not depend on the order of the cells.
// The scores are then formed on the host from these sums in one fixed order.
#pragma once

#include <cmath>
#include <cstdint>

#include "../../include/usap.h"

namespace usap {

constexpr double kQ50 = 1125899906842624.0;   // 2^50

// exact sums over the table; the *_q members are fixed-point (2^-50)
struct EvalSums {
  int64_t N;
  int64_t nb_truth, nb_given;         // non-empty rows / columns
  int64_t sq, same;                   // sum c^2, sum c(c-1)/2 over cells
  int64_t sr, s1;                     // sum r^2, sum r(r-1)/2 over rows
  int64_t sc, s2;                     // sum s^2, sum s(s-1)/2 over columns
  int64_t h_truth_q, h_given_q;       // sum (r/N)(L[r] - L[N]) over rows, same over columns
  int64_t h_gt_q, h_tg_q, mi_q;       // over cells: (c/N)(L[c] - L[r]), (c/N)(L[c] - L[s]),
                                      // (c/N)((L[c] + L[N]) - (L[r] + L[s]))
};

#if defined(__CUDA_ARCH__)
#define USAP_EV_DIV(a, b) __ddiv_rn((a), (b))
#define USAP_EV_MUL(a, b) __dmul_rn((a), (b))
#define USAP_EV_ADD(a, b) __dadd_rn((a), (b))
#define USAP_EV_SUB(a, b) __dsub_rn((a), (b))
#define USAP_EV_Q(t) __double2ll_rn(__dmul_rn((t), kQ50))
#else
#define USAP_EV_DIV(a, b) ((a) / (b))
#define USAP_EV_MUL(a, b) ((a) * (b))
#define USAP_EV_ADD(a, b) ((a) + (b))
#define USAP_EV_SUB(a, b) ((a) - (b))
#define USAP_EV_Q(t) static_cast<int64_t>(std::llrint((t) * kQ50))
#endif

// (x / N) * (La - Lb), in fixed point
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int64_t ev_term(int64_t x, double dN, double La, double Lb) {
  const double p = USAP_EV_DIV(static_cast<double>(x), dN);
  return USAP_EV_Q(USAP_EV_MUL(p, USAP_EV_SUB(La, Lb)));
}

// (c / N) * ((L[c] + L[N]) - (L[r] + L[s])), in fixed point
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int64_t ev_mi_term(int64_t c, double dN, double Lc, double LN, double Lr, double Ls) {
  const double p = USAP_EV_DIV(static_cast<double>(c), dN);
  return USAP_EV_Q(USAP_EV_MUL(p, USAP_EV_SUB(USAP_EV_ADD(Lc, LN), USAP_EV_ADD(Lr, Ls))));
}

// the scores from the sums (everything but the accuracy)
void scores_from_sums(const EvalSums& e, usap_scores* s);

// best one-to-one matching of truth blocks to given blocks on a dense
// b1 x b2 table (row-major); NaN beyond 2048 blocks a side
double matching_accuracy(const int64_t* table, int b1, int b2, int64_t N);

}  // namespace usap
