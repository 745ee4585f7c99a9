// bf::evaluate on the B200 library: a drop-in for uSAP's include/evaluate.hpp
// (evaluate.hpp:18-266).  It prints the same report lines; the scores come
// from usap_evaluate (include/usap.h), which computes them on the
// contingency table itself.  The reference rearranges that table's columns
// after its Kuhn-Munkres matching and, for tables that are not square,
// drops or duplicates columns (evaluate.hpp:93), so its printed figures
// differ from these whenever the two partitions have different block
// counts.  "Accuracy" here is the best one-to-one block matching.
// bf::evaluate_scores returns the full usap_scores (NMI included).
#pragma once

#include <cassert>
#include <cmath>
#include <cstdint>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../usap.h"

namespace bf {

template <typename V>
usap_scores evaluate_scores(const std::vector<V>& truth, const std::vector<V>& given) {
  if (truth.size() != given.size()) throw std::invalid_argument("truth and given differ in size");
  std::vector<int32_t> t(truth.size()), g(given.size());
  for (size_t i = 0; i < truth.size(); i++) {
    t[i] = static_cast<int32_t>(static_cast<int64_t>(truth[i]));
    g[i] = static_cast<int32_t>(static_cast<int64_t>(given[i]));
  }
  usap_scores s;
  if (usap_evaluate(t.data(), g.data(), static_cast<int64_t>(t.size()), &s) != USAP_OK)
    throw std::runtime_error(std::string("usap: ") + usap_last_error());
  return s;
}

template <typename V>
void evaluate(const std::vector<V>& truth, const std::vector<V>& given) {
  assert(truth.size() == given.size());
  usap_scores s = evaluate_scores(truth, given);
  std::cout << "========Partition Correctness Evaluation========\n";
  std::cout << "Number of nodes: " << given.size() << '\n';
  std::cout << "Number of partitions (truth): " << s.b_truth << "\n";
  std::cout << "Number of partitions (given): " << s.b_given << "\n";
  std::cout << "Accuracy (with optimal partition matching): " << s.accuracy << '\n';
  std::cout << '\n';
  std::cout << "Rand Index: " << s.rand_index << '\n';
  std::cout << "Adjusted Rand Index: " << s.adjusted_rand_index << '\n';
  std::cout << "Pairwise Recall: " << s.pairwise_recall << '\n';
  std::cout << "Pairwise Precision: " << s.pairwise_precision << '\n';
  std::cout << '\n';
  std::cout << "Entropy of truth partition: " << std::abs(s.h_truth) << '\n';
  std::cout << "Entropy of given partition: " << std::abs(s.h_given) << '\n';
  std::cout << "Conditional entropy of truth under given: " << std::abs(s.h_truth_given) << '\n';
  std::cout << "Conditional entropy of given under truth: " << std::abs(s.h_given_truth) << '\n';
  std::cout << "Mututal info between truth and given: " << std::abs(s.mi) << '\n';
  std::cout << "Fraction of missed info: " << std::abs(s.missed_info) << '\n';
  std::cout << "Fraction of erroneous info: " << std::abs(s.erroneous_info) << '\n';
  std::cout << "Normalized mutual info: " << s.nmi << '\n';
  std::cout << "================================================\n";
}

}  // namespace bf
