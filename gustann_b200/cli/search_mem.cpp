// search_mem: the reference's `search_disk` driver built with USE_PURE_MEM
// (bin/search_disk.cpp:11-256), over include/gustann.hpp and libgann.
//
//   search_mem --query Q.{f,b}vecs --index X_disk.index --pq_data X_pq --data_type uint8|float
//              [--nav_graph DIR] [--ground_truth GT.ivecs] [--topk K] [--ef_search L [L ...]]
//              [--repeat|-R N] [--use-gpu-mem|-G] [--batched [--entry walk|nearest]]
//
// Same flags and meanings as the reference (search_disk.cpp:51-73): the query
// set is replicated --repeat times (default 20, :167-179); without -G the
// records stay in host memory; one L prints the first 5 x 5 results and the
// recall (:190-213), several L print an L / run time / QPS / recall table
// (:214-256). Recall@k counts result ids found among the first k ground-truth
// ids of the first (unreplicated) queries (utils.hpp:105-117). --batched runs
// the optimised form (gann_search_batch, BF16X3 tables) instead of the drop-in;
// --entry nearest starts its walks at each query's nearest pivot
// (GANN_ENTRY_NEAREST_PIVOT) instead of the pivot-graph walk.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "gustann.hpp"

namespace {

// *vecs files: per vector an int32 dimension followed by that many values.
template <class T>
std::vector<T> read_vecs(const std::string& path, size_t& d, size_t& n) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("cannot open " + path);
  std::fseek(f, 0, SEEK_END);
  const long bytes = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  int32_t dim = 0;
  if (bytes < 4 || std::fread(&dim, 4, 1, f) != 1 || dim <= 0) {
    std::fclose(f);
    throw std::runtime_error(path + ": bad vector header");
  }
  const size_t rec = 4 + sizeof(T) * (size_t)dim;
  if ((size_t)bytes % rec != 0) {
    std::fclose(f);
    throw std::runtime_error(path + ": size is not a whole number of vectors");
  }
  d = (size_t)dim;
  n = (size_t)bytes / rec;
  std::vector<T> out(n * d);
  std::fseek(f, 0, SEEK_SET);
  for (size_t i = 0; i < n; i++) {
    int32_t di = 0;
    if (std::fread(&di, 4, 1, f) != 1 || di != dim || std::fread(&out[i * d], sizeof(T), d, f) != d) {
      std::fclose(f);
      throw std::runtime_error(path + ": inconsistent vector " + std::to_string(i));
    }
  }
  std::fclose(f);
  return out;
}

double recall_at(const std::vector<int>& res, const std::vector<int32_t>& gt, size_t gt_n, size_t gt_d, int k) {
  size_t hit = 0;
  for (size_t i = 0; i < gt_n; i++) {
    const std::set<int> s(gt.begin() + i * gt_d, gt.begin() + i * gt_d + k);
    for (int j = 0; j < k; j++) hit += s.count(res[i * k + j]);
  }
  return (double)hit / ((double)gt_n * k);
}

void usage(const char* a0) {
  std::fprintf(stderr,
               "usage: %s --query Q --index I --pq_data P --data_type uint8|float [--nav_graph D]\n"
               "          [--ground_truth G] [--topk K] [--ef_search L [L ...]] [--repeat|-R N] [--use-gpu-mem|-G]\n"
               "          [--batched [--entry walk|nearest]]\n",
               a0);
}

}  // namespace

int main(int argc, char** argv) {
  std::string query, gt_file, dtype_s;
  gustann::GustANNConfig cfg;
  int topk = 100, repeat = 20;
  std::vector<int> efs;
  bool gpu_mem = false, batched = false;
  std::string entry_s;
  for (int i = 1; i < argc; i++) {
    const std::string a = argv[i];
    auto next = [&]() -> std::string {
      if (i + 1 >= argc) throw std::runtime_error("missing value after " + a);
      return argv[++i];
    };
    try {
      if (a == "--query") query = next();
      else if (a == "--index") cfg.index_file = next();
      else if (a == "--ground_truth") gt_file = next();
      else if (a == "--data_type") dtype_s = next();
      else if (a == "--topk") topk = std::stoi(next());
      else if (a == "--pq_data") cfg.pq_file_prefix = next();
      else if (a == "--nav_graph") cfg.nav_graph_prefix = next();
      else if (a == "--repeat" || a == "-R") repeat = std::stoi(next());
      else if (a == "--use-gpu-mem" || a == "-G") gpu_mem = true;
      else if (a == "--batched") batched = true;
      else if (a == "--entry") entry_s = next();
      else if (a == "--ef_search") {
        efs.push_back(std::stoi(next()));
        while (i + 1 < argc && argv[i + 1][0] != '-') efs.push_back(std::stoi(argv[++i]));
      } else {
        usage(argv[0]);
        std::fprintf(stderr, "unknown argument %s\n", a.c_str());
        return 1;
      }
    } catch (const std::exception& e) {
      usage(argv[0]);
      std::fprintf(stderr, "%s\n", e.what());
      return 1;
    }
  }
  if (query.empty() || cfg.index_file.empty() || cfg.pq_file_prefix.empty() || dtype_s.empty()) {
    usage(argv[0]);
    return 1;
  }
  if (dtype_s != "uint8" && dtype_s != "float") {
    std::fprintf(stderr, "unrecognized data type %s\n", dtype_s.c_str());
    return 1;
  }
  if (!entry_s.empty() && entry_s != "walk" && entry_s != "nearest") {
    std::fprintf(stderr, "unrecognized entry %s (walk or nearest)\n", entry_s.c_str());
    return 1;
  }
  if (!entry_s.empty() && !batched) {
    std::fprintf(stderr, "--entry applies to --batched only (the drop-in form enters by the pivot-graph walk)\n");
    return 1;
  }
  if (efs.empty()) efs.push_back(300);
  if (topk < 1 || repeat < 1) {
    std::fprintf(stderr, "topk and repeat must be >= 1\n");
    return 1;
  }
  for (int ef : efs)
    if (ef < topk) {  // search_disk.cpp:189-192 asserts ef_search >= topk
      std::fprintf(stderr, "ef_search %d is below topk %d\n", ef, topk);
      return 1;
    }
  try {
    const gustann::DataType dt = dtype_s == "uint8" ? gustann::UINT8 : gustann::FLOAT;
    size_t d = 0, nq0 = 0;
    std::vector<float> q0;
    if (dt == gustann::UINT8) {
      const std::vector<uint8_t> b = read_vecs<uint8_t>(query, d, nq0);
      q0.assign(b.begin(), b.end());
    } else {
      q0 = read_vecs<float>(query, d, nq0);
    }
    const size_t nq = nq0 * (size_t)repeat;
    std::vector<float> q(nq * d);
    for (int r = 0; r < repeat; r++) std::copy(q0.begin(), q0.end(), q.begin() + (size_t)r * nq0 * d);
    std::printf("Read %zu queries of dimension %zu (x%d)\n", nq0, d, repeat);

    std::vector<int32_t> gt;
    size_t gt_d = 0, gt_n = 0;
    if (!gt_file.empty()) gt = read_vecs<int32_t>(gt_file, gt_d, gt_n);
    if (!gt.empty() && gt_n > nq0) throw std::runtime_error("ground truth has more rows than queries");

    gustann::GustANN a(dt);
    a.init_pure_mem(cfg, gpu_mem);
    std::vector<int> nns(nq * (size_t)topk);
    std::vector<float> dis(nq * (size_t)topk);
    std::vector<int> found(nq);
    auto run = [&](int ef) -> double {
      if (!batched) {
        gustann::GustANNStats st;
        a.search(q.data(), (int)nq, topk, ef, nns.data(), dis.data(), found.data(), &st);
        return st.run_time;
      }
      double t = 0.0;
      gann_batch_opts_t o{};
      o.precision = GANN_PREC_BF16X3;  // the NULL-options default
      o.entry = entry_s == "nearest" ? GANN_ENTRY_NEAREST_PIVOT : GANN_ENTRY_NAV_WALK;
      const int rc = gann_search_batch(a.handle(), q.data(), (int)nq, nullptr, nullptr, topk, ef, &o,
                                       reinterpret_cast<int32_t*>(nns.data()), dis.data(),
                                       reinterpret_cast<int32_t*>(found.data()), &t);
      if (rc != GANN_OK) throw std::runtime_error(std::string("gann_search_batch: ") + gann_last_error());
      return t;
    };
    if (efs.size() == 1) {
      run(efs[0]);
      for (size_t i = 0; i < std::min<size_t>(5, nq); i++) {
        for (int j = 0; j < std::min(5, topk); j++)
          std::printf("%lf(%d)\t", (double)dis[i * topk + j], nns[i * topk + j]);
        std::printf("\n");
      }
      if (!gt.empty()) {
        if ((size_t)topk > gt_d) throw std::runtime_error("topk exceeds the ground-truth depth");
        const double r = recall_at(nns, gt, gt_n, gt_d, topk);
        std::printf("Recall @ %d: %lf\n", topk, r);
        std::printf("[REPORT] RECALL: %lf\n", r);
      }
    } else {
      const std::string rh = gt.empty() ? "Recall" : "Recall@" + std::to_string(topk);
      std::printf("\n%-12s %-18s %-18s %-18s\n", "L", "Run Time (s)", "QPS", rh.c_str());
      std::printf("%-12s %-18s %-18s %-18s\n", "------------", "------------------", "------------------",
                  "------------------");
      for (int ef : efs) {
        const double t = run(ef);
        const double qps = nq / t;
        if (!gt.empty() && (size_t)topk <= gt_d)
          std::printf("%-12d %-18.6f %-18.2f %-18.6f\n", ef, t, qps, recall_at(nns, gt, gt_n, gt_d, topk));
        else
          std::printf("%-12d %-18.6f %-18.2f %-18s\n", ef, t, qps, "N/A");
      }
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
