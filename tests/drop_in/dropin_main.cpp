// Drives the B200 library through the reference-shaped C++ headers the way
// uSAP's main.cpp drives sgp::Graph_P and bf::evaluate: construct from a TSV
// basename, partition(), read get_partitions(), print the scores.  Used by
// tests/test_dropin.py (compile on CPU, run on a GPU).
#include <chrono>
#include <cstdio>
#include <iostream>
#include <string>

#include <usap/evaluate.hpp>
#include <usap/graph_p.hpp>

int main(int argc, char* argv[]) {
  if (argc < 3) {
    std::cerr << "usage: dropin_main <basename> <out_partition> [num_batch_nodal_update]\n";
    return 1;
  }
  sgp::Graph_P<long> g_p(argv[1]);
  if (argc > 3) g_p.num_batch_nodal_update = std::stoul(argv[3]);
  std::cout << "Partitioning..." << std::endl;
  auto t0 = std::chrono::steady_clock::now();
  g_p.partition();
  auto t1 = std::chrono::steady_clock::now();
  std::cout << "Partitioning time: "
            << std::chrono::duration_cast<std::chrono::milliseconds>(t1 - t0).count() << " ms\n";
  bf::evaluate<size_t>(g_p.truePartitions, g_p.get_partitions());
  std::FILE* f = std::fopen(argv[2], "w");
  if (!f) return 2;
  for (size_t b : g_p.get_partitions()) std::fprintf(f, "%zu\n", b);
  std::fclose(f);
  return 0;
}
