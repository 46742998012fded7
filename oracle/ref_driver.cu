// Checker-only C entry points over the reference GustANN all-in-GPU path.
//
// This file is compiled together with the reference's own, unmodified sources
// (src/ssd_search.cu, src/pure_mem.cu, src/pq_search.cu, src/nav_graph.cu, ...)
// by oracle/build_ref.sh into oracle/_ref/libgustann_ref.so. It is used only by
// the tests (to pin the CPU oracle and the CUDA product against the reference's
// own outputs) and by bench.py's reference arm. The product never links it.
//
// The calls mirror bin/search_disk.cpp:118-195: construct gustann::GustANN with
// the data type, init_pure_mem(config, use_gpu_mem=true) (the `-G` mode), then
// search(queries, nq, topk, ef_search, nns, distances, found_cnt, &stats).
#include <cstdint>
#include <cstdio>
#include <exception>
#include <string>

#include "ssd_search.hpp"

extern "C" {

void* gref_open(const char* index_file, const char* pq_prefix, const char* nav_dir,
                int dtype) {
  try {
    auto* g = new gustann::GustANN(dtype == 0 ? gustann::UINT8 : gustann::FLOAT);
    gustann::GustANNConfig cfg;
    cfg.index_file = index_file;
    cfg.pq_file_prefix = pq_prefix;
    cfg.nav_graph_prefix = nav_dir ? nav_dir : "";
    g->init_pure_mem(cfg, /*use_gpu_mem=*/true);
    return g;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "gref_open: %s\n", e.what());
    return nullptr;
  }
}

int gref_search(void* h, const float* q, int nq, int topk, int ef_search, int* nns,
                float* distances, int* found_cnt, double* seconds) {
  try {
    gustann::GustANNStats stats{0.0};
    static_cast<gustann::GustANN*>(h)->search(q, nq, topk, ef_search, nns, distances,
                                               found_cnt, &stats);
    if (seconds) *seconds = stats.run_time;
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "gref_search: %s\n", e.what());
    return -1;
  }
}

void gref_close(void* h) { delete static_cast<gustann::GustANN*>(h); }

}  // extern "C"
