// sgp::Graph_P<W> on the B200 library: a drop-in for uSAP's
// include/graph_parallel.hpp (chih-chun-chang/uSAP) for code that uses the
// reference's public interface:
//
//   Graph_P(const std::string& FileName, size_t num_threads = 16)   :61-78
//   public parameters (same names, types and defaults)               :40-52
//   void partition()                                                 :59, :322-512
//   const std::vector<size_t>& get_partitions() const                :58
//   const size_t& num_nodes() const / num_edges() const              :56-57
//   std::vector<size_t> truePartitions                               :81
//   void load_graph_from_tsv(const std::string& FileName)            :55, :251-317
//
// The constructor reads FileName.tsv (from<TAB>to<TAB>weight, 1-based; its
// bytes are parsed on the GPU by usap_ctx_load_tsv with the reference's
// field rules) and FileName_truePartition.tsv (node<TAB>block) as the
// reference does, including N = largest source id and the three summary lines on
// stdout; an unreadable file prints "Unable to open file!" and exits, as
// the reference does (graph_parallel.hpp:254-257, :294-297).  partition()
// runs on the GPU through include/usap.h; num_threads is accepted and
// unused.  Additional members: seed, init_mode, dense_max, device, result().
// Errors from the GPU library throw std::runtime_error.
#pragma once

#include <cstdlib>
#include <fstream>
#include <iostream>
#include <iterator>
#include <stdexcept>
#include <string>
#include <vector>

#include "../usap.h"

namespace sgp {

template <typename W>
class Graph_P {
 public:
  // parameters can be set by users (reference defaults)
  int beta = 3;
  size_t block_size = 1024;
  size_t num_agg_proposals_per_block = 10;
  float num_block_reduction_rate = 0.5;
  size_t max_num_nodal_itr = 100;
  size_t num_batch_nodal_update = 4;
  float delta_entropy_threshold1 = 5e-4;
  float delta_entropy_threshold2 = 1e-4;
  size_t delta_entropy_moving_avg_window = 3;
  bool verbose = false;
  size_t dfs_depth = 20;
  size_t t_block_num = 20;
  // B200 build
  uint64_t seed = 0;
  int init_mode = 0;
  int dense_max = 0;   // 0: automatic (usap_params.dense_max)
  int device = 0;

  explicit Graph_P(const std::string& FileName, size_t num_threads = 16) {
    (void)num_threads;
    load_graph_from_tsv(FileName);
  }
  ~Graph_P() {
    if (ctx_) usap_ctx_destroy(ctx_);
  }
  Graph_P(const Graph_P&) = delete;
  Graph_P& operator=(const Graph_P&) = delete;

  void load_graph_from_tsv(const std::string& FileName) {
    std::ifstream file(FileName + ".tsv", std::ios::binary);
    if (!file.is_open()) {
      std::cerr << "Unable to open file!\n";
      std::exit(EXIT_FAILURE);
    }
    const std::string text((std::istreambuf_iterator<char>(file)), std::istreambuf_iterator<char>());
    file.close();
    if (!ctx_) check(usap_ctx_create(device, &ctx_));
    check(usap_ctx_load_tsv(ctx_, text.data(), static_cast<int64_t>(text.size()), 0));
    int32_t n = 0;
    int64_t e = 0;
    check(usap_ctx_num_nodes(ctx_, &n, &e));
    N_ = static_cast<size_t>(n);
    E_ = static_cast<size_t>(e);
    std::string line;
    std::ifstream true_file(FileName + "_truePartition.tsv");
    if (!true_file.is_open()) {
      std::cerr << "Unable to open file!\n";
      std::exit(EXIT_FAILURE);
    }
    truePartitions.clear();
    size_t b = 0;
    while (std::getline(true_file, line)) {
      size_t start = 0, tab = line.find('\t');
      start = tab + 1;
      tab = line.find('\t', start);
      size_t block = std::stoi(line.substr(start, tab - start));
      truePartitions.emplace_back(block - 1);
      if (block > b) b = block;
    }
    std::cout << "Number of nodes: " << N_ << std::endl;
    std::cout << "Number of edges: " << E_ << std::endl;
    std::cout << "NUmber of blocks:" << b << std::endl;
  }

  const size_t& num_nodes() const { return N_; }
  const size_t& num_edges() const { return E_; }
  const std::vector<size_t>& get_partitions() const { return partitions_; }

  void partition() {
    usap_params p;
    usap_params_default(&p);
    p.beta = beta;
    p.block_size = static_cast<int32_t>(block_size);
    p.num_agg_proposals_per_block = static_cast<int32_t>(num_agg_proposals_per_block);
    p.num_block_reduction_rate = num_block_reduction_rate;
    p.max_num_nodal_itr = static_cast<int32_t>(max_num_nodal_itr);
    p.num_batch_nodal_update = static_cast<int32_t>(num_batch_nodal_update);
    p.delta_entropy_threshold1 = delta_entropy_threshold1;
    p.delta_entropy_threshold2 = delta_entropy_threshold2;
    p.delta_entropy_moving_avg_window = static_cast<int32_t>(delta_entropy_moving_avg_window);
    p.verbose = verbose ? 1 : 0;
    p.dfs_depth = static_cast<int32_t>(dfs_depth);
    p.t_block_num = static_cast<int32_t>(t_block_num);
    p.seed = seed;
    p.init_mode = init_mode;
    p.dense_max = dense_max;
    std::vector<int32_t> out(N_);
    check(usap_ctx_partition(ctx_, &p, out.data(), &result_));
    partitions_.assign(out.begin(), out.end());
  }

  const usap_result& result() const { return result_; }

  // partition ground truth
  std::vector<size_t> truePartitions;

 private:
  static void check(usap_status s) {
    if (s != USAP_OK) throw std::runtime_error(std::string("usap: ") + usap_last_error());
  }
  size_t N_ = 0, E_ = 0;
  std::vector<size_t> partitions_;
  usap_ctx* ctx_ = nullptr;
  usap_result result_{};
};

}  // namespace sgp
