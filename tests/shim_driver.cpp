// A search_mem-style driver (the reference's bin/search_disk.cpp:118-213 with
// -DUSE_PURE_MEM, minus argparse/spdlog) written against include/gustann.hpp.
// Used by the tests to show that reference-style host code compiles and links
// against libgann.so unchanged.
//
// usage: shim_driver <uint8|float> <index> <pq_prefix> <nav_dir|-> <queries.bin> <topk> <L> <out.bin> [gpu|dram]
// gpu (default) is search_mem's -G (records in HBM); dram keeps the records in host memory.
// queries.bin: int32 nq, int32 dim, nq*dim float32; out.bin: nns, distances, found_cnt.
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "gustann.hpp"

int main(int argc, char** argv) {
  if (argc != 9 && argc != 10) {
    std::fprintf(stderr,
                 "usage: %s <uint8|float> <index> <pq_prefix> <nav_dir|-> <queries.bin> <topk> <L> <out> [gpu|dram]\n",
                 argv[0]);
    return 2;
  }
  const bool use_gpu_mem = argc == 9 || std::strcmp(argv[9], "dram") != 0;
  gustann::DataType dtype = std::strcmp(argv[1], "uint8") == 0 ? gustann::UINT8 : gustann::FLOAT;
  gustann::GustANNConfig cfg;
  cfg.index_file = argv[2];
  cfg.pq_file_prefix = argv[3];
  cfg.nav_graph_prefix = std::strcmp(argv[4], "-") == 0 ? "" : argv[4];
  const int topk = std::atoi(argv[6]), L = std::atoi(argv[7]);
  FILE* f = std::fopen(argv[5], "rb");
  if (!f) return 3;
  int nq = 0, d = 0;
  if (std::fread(&nq, 4, 1, f) != 1 || std::fread(&d, 4, 1, f) != 1) return 3;
  std::vector<float> q((size_t)nq * d);
  if (std::fread(q.data(), 4, q.size(), f) != q.size()) return 3;
  std::fclose(f);
  try {
    gustann::GustANN a(dtype);
    a.init_pure_mem(cfg, use_gpu_mem);
    std::unique_ptr<int[]> nns(new int[(size_t)nq * topk]);
    std::unique_ptr<float[]> dis(new float[(size_t)nq * topk]);
    std::unique_ptr<int[]> found(new int[nq]);
    gustann::GustANNStats stats;
    a.search(q.data(), nq, topk, L, nns.get(), dis.get(), found.get(), &stats);
    FILE* o = std::fopen(argv[8], "wb");
    std::fwrite(nns.get(), 4, (size_t)nq * topk, o);
    std::fwrite(dis.get(), 4, (size_t)nq * topk, o);
    std::fwrite(found.get(), 4, nq, o);
    std::fclose(o);
    std::printf("searched %d queries in %.6f s\n", nq, stats.run_time);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
