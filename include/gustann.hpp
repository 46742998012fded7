// gustann.hpp -- C++ drop-in for the reference's host interface, over the C
// ABI of libgann.so (gann.h).
//
// Mirrors gustann::GustANN / GustANNConfig / GustANNStats / DataType of
// src/ssd_search.hpp:18-83 and src/common.hpp:22-25 for the all-in-GPU mode:
// a program written against the reference (bin/search_disk.cpp with
// -DUSE_PURE_MEM) compiles against this header and links libgann.so.
// Differences, by design:
//  * failures throw std::runtime_error carrying gann_last_error() instead of
//    exit(-1) / abort() / a bare throw (src/layout.cpp:14-17, src/common.hpp:17,
//    src/ssd_search.cu:65-66);
//  * init_pure_mem(cfg, false) -- records in pinned host memory -- is refused;
//  * init_hybrid / init_bam (SSD and BaM executors) are not part of this path.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>

#include "gann.h"

namespace gustann {

enum DataType { UINT8 = GANN_UINT8, FLOAT = GANN_FLOAT };

class GustANNConfig {
 public:
  std::string index_file;
  std::string pq_file_prefix;
  std::string nav_graph_prefix;
};

struct GustANNStats {
  double run_time;
};

class GustANN {
 public:
  explicit GustANN(DataType data_type = FLOAT) : data_type_(data_type) {}
  GustANN(const GustANN&) = delete;
  GustANN& operator=(const GustANN&) = delete;
  ~GustANN() { gann_close(h_); }

  // GustANN::init_pure_mem (src/ssd_search.cu:108-112): use_gpu_mem = true puts
  // the records in HBM (-G), false keeps them in pinned host memory read by the
  // kernels over PCIe/C2C (src/pure_mem.cu:51-66).
  void init_pure_mem(const GustANNConfig& cfg, bool use_gpu_mem) {
    gann_close(h_);
    h_ = nullptr;
    const char* nav = cfg.nav_graph_prefix.empty() ? nullptr : cfg.nav_graph_prefix.c_str();
    check(gann_open(cfg.index_file.c_str(), cfg.pq_file_prefix.c_str(), nav, data_type_,
                    use_gpu_mem ? 0 : GANN_OPEN_HOST_PAGES, &h_));
  }

  // GustANN::search (src/ssd_search.hpp:78-80): host buffers, squared L2.
  void search(const float* qdata, const int num_queries, const int topk, const int ef_search, int* nns,
              float* distances, int* found_cnt, GustANNStats* stats = nullptr) {
    double t = 0.0;
    check(gann_search(h_, qdata, num_queries, topk, ef_search, reinterpret_cast<int32_t*>(nns), distances,
                      reinterpret_cast<int32_t*>(found_cnt), &t));
    if (stats) stats->run_time = t;
  }

  gann_t* handle() const { return h_; }

 private:
  static void check(int rc) {
    if (rc != GANN_OK) throw std::runtime_error(std::string("gann: ") + gann_last_error());
  }
  DataType data_type_;
  gann_t* h_ = nullptr;
};

}  // namespace gustann
