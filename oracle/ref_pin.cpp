// Golden-vector harness: drives the reference's own internal phases
// (uSAP include/graph_parallel.hpp, compiled unmodified against the
// Taskflow-API shim) on controlled inputs and prints what they compute, so
// the oracle's restatement can be pinned to the reference itself.
// Test infrastructure only; it is run by tests/golden/make_golden.py.
//
// Private members are reached with a `private`->`public` macro applied after
// every standard header is included.  Built twice: as shipped (float) and
// with USAP_PIN_DOUBLE, where `float` is macro-renamed to `double` in the
// reference's code so its entropy arithmetic can be compared at FP64
// precision.
//
// Protocol: argv[1] = command, argv[2] = TSV basename; numbers on stdin;
// JSON-ish lines on stdout.
#include <algorithm>
#include <cassert>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <limits>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <set>
#include <stack>
#include <string>
#include <thread>
#include <unordered_set>
#include <utility>
#include <vector>

#include <taskflow/taskflow.hpp>
#include <taskflow/algorithm/for_each.hpp>
#include <taskflow/algorithm/reduce.hpp>
#include <taskflow/algorithm/transform.hpp>
#include <evaluate.hpp>

#define private public
#ifdef USAP_PIN_DOUBLE
#define float double
#endif
#include <graph_parallel.hpp>
#undef private

using G = sgp::Graph_P<long>;

static std::vector<long> read_longs(size_t n) {
  std::vector<long> v(n);
  for (size_t i = 0; i < n; i++) {
    if (std::scanf("%ld", &v[i]) != 1) {
      std::fprintf(stderr, "short input\n");
      std::exit(4);
    }
  }
  return v;
}

static std::vector<double> read_doubles(size_t n) {
  std::vector<double> v(n);
  for (size_t i = 0; i < n; i++) {
    if (std::scanf("%lf", &v[i]) != 1) {
      std::fprintf(stderr, "short input\n");
      std::exit(4);
    }
  }
  return v;
}

// stdin: B, then N block ids; installs them as the reference's state and
// rebuilds M/degrees with the reference's own _initialize_edge_counts().
static void load_state(G& g) {
  long B = 0;
  if (std::scanf("%ld", &B) != 1) std::exit(4);
  auto part = read_longs(g._N);
  g._P.B = static_cast<size_t>(B);
  g._P.partitions.assign(part.begin(), part.end());
  g._initialize_edge_counts();
}

static void print_state(G& g) {
  size_t B = g._P.B;
  std::printf("B %zu\n", B);
  std::printf("dout");
  for (size_t i = 0; i < B; i++) std::printf(" %ld", g._P.d.out[i]);
  std::printf("\ndin");
  for (size_t i = 0; i < B; i++) std::printf(" %ld", g._P.d.in[i]);
  std::printf("\n");
  // M as (row, col, value) triples in row-major order, aggregated
  std::vector<long> row(B);
  std::printf("M");
  for (size_t i = 0; i < B; i++) {
    if (B < g.block_size) {
      for (size_t j = 0; j < B; j++) row[j] = g._P.M[i * B + j];
    } else {
      std::fill(row.begin(), row.end(), 0);
      for (const auto& [v, w] : g._P.Mrow[i]) row[v] += w;
    }
    for (size_t j = 0; j < B; j++) {
      if (row[j] != 0) std::printf(" %zu %zu %ld", i, j, row[j]);
    }
  }
  std::printf("\n");
}

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: ref_pin <cmd> <basename> [args]\n");
    return 2;
  }
  std::string cmd = argv[1];
  std::string base = argv[2];
  std::streambuf* saved = std::cout.rdbuf();
  std::ofstream devnull("/dev/null");
  std::cout.rdbuf(devnull.rdbuf());
  G g(base, 4);
  std::cout.rdbuf(saved);
  if (argc > 3) g.block_size = std::strtoul(argv[3], nullptr, 10);

  if (cmd == "scc") {
    // argv[4] = dfs_depth
    if (argc > 4) g.dfs_depth = std::strtoul(argv[4], nullptr, 10);
    g._scc();
    std::printf("B %zu\npart", g._P.B);
    for (auto b : g._P.partitions) std::printf(" %zu", b);
    std::printf("\n");
  } else if (cmd == "mbuild") {
    load_state(g);
    print_state(g);
  } else if (cmd == "entropy") {
    load_state(g);
    std::vector<long> scratch;
    auto S = g._compute_overall_entropy(scratch);
    std::printf("S %.17g\n", static_cast<double>(S));
  } else if (cmd == "merge_props") {
    // argv[4] = seed, argv[5] = proposals per block
    load_state(g);
    unsigned seed = static_cast<unsigned>(std::strtoul(argv[4], nullptr, 10));
    size_t K = std::strtoul(argv[5], nullptr, 10);
    g._merge_data.reset(g._P.B);
    std::default_random_engine gen(seed);
    std::vector<float> prob;
    auto& newM = g._pt_newM[0];
    for (size_t r = 0; r < g._P.B; r++) {
      for (size_t k = 0; k < K; k++) {
        size_t s = 0;
        float dS = 0;
        g._propose_new_partition_block(r, s, dS, prob, newM, gen);
        std::printf("%zu %zu %.17g\n", r, s, static_cast<double>(dS));
      }
    }
  } else if (cmd == "nodal_props") {
    // argv[4] = seed; every vertex proposes once against the loaded state
    load_state(g);
    unsigned seed = static_cast<unsigned>(std::strtoul(argv[4], nullptr, 10));
    std::default_random_engine gen(seed);
    std::vector<float> prob;
    std::vector<size_t> nbrs;
    auto& newM = g._pt_newM[0];
    int moves = 0;
    float dsum = 0;
    std::vector<std::pair<size_t, long>> upd;
    for (size_t ni = 0; ni < g._N; ni++) {
      size_t r = g._P.partitions[ni];
      size_t s = r;
      float dS = 0, H = 1;
      size_t before = upd.size();
      g._propose_new_partition_nodal(r, ni, s, dS, H, nbrs, prob, newM, gen, moves, dsum, upd);
      std::printf("%zu %zu %zu %.17g %d\n", ni, r, s, static_cast<double>(dS),
                  upd.size() > before ? 1 : 0);
    }
  } else if (cmd == "carry") {
    // stdin after the state: B_to_merge, then B best targets, then B dS values
    load_state(g);
    long btm = 0;
    if (std::scanf("%ld", &btm) != 1) return 4;
    g._merge_data.reset(g._P.B);
    auto best = read_longs(g._P.B);
    auto dS = read_doubles(g._P.B);
    for (size_t i = 0; i < g._P.B; i++) {
      g._merge_data.best_merge_for_each_block[i] = static_cast<size_t>(best[i]);
      g._merge_data.dS_for_each_block[i] = static_cast<float>(dS[i]);
    }
    g._P.B_to_merge = static_cast<size_t>(btm);
    g._carry_out_best_merges();
    std::printf("B %zu\npart", g._P.B);
    for (auto b : g._P.partitions) std::printf(" %zu", b);
    std::printf("\n");
  } else if (cmd == "golden") {
    // stdin: count, then (B, S) pairs fed one by one as the state after a
    // nodal phase; prints the bracket and the next B_to_merge after each.
    long count = 0;
    if (std::scanf("%ld", &count) != 1) return 4;
    g._P.partitions.assign(g._N, 0);
    for (long i = 0; i < count; i++) {
      long B = 0;
      double S = 0;
      if (std::scanf("%ld %lf", &B, &S) != 2) return 4;
      g._P.B = static_cast<size_t>(B);
      g._P.S = static_cast<float>(S);
      bool done = g._prepare_for_partition_next();
      std::printf("%d %zu %zu %zu %zu %zu\n", done ? 1 : 0, g._old.large.B, g._old.med.B,
                  g._old.small.B, g._P.B, g._P.B_to_merge);
      if (done) break;
    }
  } else if (cmd == "evaluate") {
    // stdin: N truth labels then N given labels (0-based)
    auto t = read_longs(g._N);
    auto p = read_longs(g._N);
    std::vector<size_t> truth(t.begin(), t.end()), given(p.begin(), p.end());
    bf::evaluate<size_t>(truth, given);
  } else {
    std::fprintf(stderr, "unknown command %s\n", cmd.c_str());
    return 2;
  }
  return 0;
}
