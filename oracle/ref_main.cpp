// CPU baseline driver for the reference: compiles uSAP's own
// include/graph_parallel.hpp (unmodified, against the Taskflow-API shim in
// oracle/taskflow_shim) and times Graph_P::partition() exactly as the
// reference's main.cpp:54-60 does.  Test and baseline infrastructure only.
//
// usage: ref_main <basename> <threads> <num_batch_nodal_update> [out_partition]
//   reads <basename>.tsv and <basename>_truePartition.tsv (1-based, the
//   reference's format), prints one JSON line with the solve time.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include <graph_parallel.hpp>

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: ref_main <basename> <threads> <num_batch_nodal_update> [out]\n");
    return 2;
  }
  std::string base = argv[1];
  size_t threads = std::strtoul(argv[2], nullptr, 10);
  size_t nb = std::strtoul(argv[3], nullptr, 10);

  // the loader prints node/edge counts to stdout (graph_parallel.hpp:313-315);
  // keep stdout for the JSON line
  std::streambuf* saved = std::cout.rdbuf();
  std::ofstream devnull("/dev/null");
  std::cout.rdbuf(devnull.rdbuf());
  sgp::Graph_P<long> g(base, threads);
  g.num_batch_nodal_update = nb;
  auto t0 = std::chrono::steady_clock::now();
  g.partition();
  auto t1 = std::chrono::steady_clock::now();
  std::cout.rdbuf(saved);

  const auto& p = g.get_partitions();
  size_t B = 0;
  for (auto b : p) B = b + 1 > B ? b + 1 : B;
  double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  std::printf("{\"N\": %zu, \"E\": %zu, \"threads\": %zu, \"nb\": %zu, \"ms\": %.3f, \"B\": %zu}\n",
              g.num_nodes(), g.num_edges(), threads, nb, ms, B);
  if (argc > 4) {
    std::FILE* f = std::fopen(argv[4], "w");
    if (!f) return 3;
    for (auto b : p) std::fprintf(f, "%zu\n", b);
    std::fclose(f);
  }
  return 0;
}
