// Internal types shared by the host side and the kernels of libgann.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gann.h"

namespace gann {

constexpr int kPageSize = 4096;  // PureMemExecutor::PAGE_SIZE, src/pure_mem.hpp:25
constexpr int kPivots = 256;     // PQSearchData::num_pivots, src/pq_search.hpp:12
constexpr uint32_t kMask = 0x7fffffffu;
constexpr uint32_t kExpanded = 0x80000000u;

// Error word bits written by kernels (device -> host).
enum : uint32_t {
  kErrBadId = 1u,       // neighbour or entry id outside [0, n)
  kErrBadDegree = 2u,   // degree word larger than max_m0
  kErrHopCap = 4u,      // walk exceeded its hop limit
  kErrNavCap = 8u,      // pivot-graph walk exceeded its iteration limit
  kErrWaitLimit = 16u,  // a bounded spin-wait gave up
};

// Quotient by a divisor d >= 1 fixed at load time, for numerators in [0, 2^31):
// q = umulhi(n, m) >> s with p = 31 + ceil(log2 d), m = ceil(2^p / d), s = p - 32
// (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994). m < 2^32 because d > 2^(ceil(log2 d) - 1), and
// the rounding error n * (m d - 2^p) / (d 2^p) < 2^-ceil(log2 d) <= 1/d keeps
// floor(n m / 2^p) = floor(n / d). Record ids are below 2^31.
struct FastDiv {
  uint32_t d = 1, m = 0, s = 0;
  FastDiv() = default;
  explicit FastDiv(uint32_t div) : d(div) {
    if (d > 1) {
      uint32_t l = 0;
      while ((1ull << l) < d) l++;
      const uint32_t p = 31 + l;
      m = (uint32_t)(((1ull << p) + d - 1) / d);
      s = p - 32;
    }
  }
#ifdef __CUDACC__
  __host__ __device__
#endif
  inline uint32_t div(uint32_t n) const {
    if (d == 1) return n;
#ifdef __CUDA_ARCH__
    return __umulhi(n, m) >> s;
#else
    return (uint32_t)(((uint64_t)n * m) >> 32) >> s;
#endif
  }
};

// Host copy of the index files, parsed and checked (gann_io.cpp).
struct HostIndex {
  int dtype = 0;  // GANN_UINT8 / GANN_FLOAT
  int elt = 1;
  int64_t n = 0, dim = 0, medoid = 0, node_len = 0, npp = 0, max_m0 = 0, data_len = 0,
          num_pages = 0;
  int pq_m = 0;
  std::vector<float> pivots;          // 256 x dim (row = pivot)
  std::vector<float> centroid;        // dim
  std::vector<int32_t> chunk_offsets; // M + 1, contiguous ranges covering [0, dim)
  bool has_nav = false;
  int nav_n = 0, nav_max_m = 0, nav_start = 0;
  std::vector<uint8_t> nav_data;   // nav_n x dim x elt
  std::vector<int32_t> nav_graph;  // nav_n x nav_max_m, -1 padded
  std::vector<int32_t> nav_map;    // nav_n
};

// Device-resident index (HBM layout).
struct DeviceIndex {
  const uint8_t* pages = nullptr;   // num_pages x 4096, the _disk.index body
  const uint8_t* codes = nullptr;   // n x M PQ codes
  const float* pivots_t = nullptr;  // dim x 256 (transposed pivots)
  const float* centroid = nullptr;  // dim
  const int32_t* chunk_off = nullptr;  // M + 1
  const uint8_t* nav_data = nullptr;   // nav_n x dim x elt
  const int32_t* nav_graph = nullptr;  // nav_n x nav_max_m
  const int32_t* nav_map = nullptr;    // nav_n
  // tensor-core table build (table_tc.cu): B operand tiles, centroid norms
  const uint8_t* tc_bpanel_hi = nullptr;  // M x 8 KB
  const uint8_t* tc_bpanel_lo = nullptr;  // M x 8 KB
  const float* tc_pnorm = nullptr;        // M x 256
  int tc_p = 0, tc_groups = 0;            // padded chunk width, chunk groups per K=16 slice
  // nearest-pivot entry (entry_tc.cu): pivot tiles of 256 x nk K=16 slices, squared norms
  const uint8_t* entry_panel = nullptr;   // entry_tiles x entry_nk x 8 KB
  const float* entry_pnorm = nullptr;     // entry_tiles x 256
  int entry_nk = 0, entry_tiles = 0;
  unsigned int* err = nullptr;            // kernel error word
  // HBM copies of hot records when the pages sit in host memory
  // (gann_cache_hot_records): rec_remap[u] = cache slot of node u, or -1.
  const int32_t* rec_remap = nullptr;     // n, or null (no cache)
  const uint8_t* rec_cache = nullptr;     // slots x rec_stride, records copied verbatim
  int64_t rec_stride = 0;
};

// Address of node u's record: its HBM copy when it is cached, else its page slot.
#ifdef __CUDACC__
__device__ __forceinline__ const uint8_t* record_at(const DeviceIndex& ix, int64_t page, int64_t slot_off,
                                                    int64_t u) {
  if (ix.rec_remap) {
    const int32_t c = __ldg(ix.rec_remap + u);
    if (c >= 0) return ix.rec_cache + (int64_t)c * ix.rec_stride;
  }
  return ix.pages + page * kPageSize + slot_off;
}
#endif

// Launch parameters of the plain search kernel (walk_plain.cu).
struct PlainParams {
  DeviceIndex ix;
  int64_t n, npp, node_len, data_len, medoid;
  int dim, max_m, M;
  int has_nav, nav_n, nav_max_m, nav_start;
  const float* queries;  // nq x dim
  int nq, L, k;
  int fma_table, fma_exact;  // FMA at pq.cuh:40 / util.cuh:37
  int32_t* nns;              // nq x k
  float* dists;              // nq x k
  int32_t* found;            // nq
  int32_t* hops;             // nq or null: hops (expanded nodes) per query
  int64_t* bytes;            // nq or null: algorithmic gathered bytes per query
  int* next_query;           // work counter, zeroed before launch
  unsigned int* err;         // error word
};

// Launch parameters of the batched search kernel (walk_batch.cu).
struct BatchParams {
  DeviceIndex ix;
  int64_t n, npp, node_len, data_len, medoid;
  int dim, max_m, M;
  int has_nav, nav_n, nav_max_m, nav_start;
  const float* queries;           // nq x dim
  int nq;
  const int* nq_dev;              // or null: the query count, read at run time (<= nq)
  const int32_t* L_per_q;         // nq or null (then L_max for all)
  const int32_t* k_per_q;         // nq or null (then k_max for all)
  int L_max, k_max;
  int hash_bits;                  // visited cache: 1 << hash_bits slots
  FastDiv npp_div;                // division by nodes per page
  int32_t* visit_count;           // or null: per-node expansion counts (gann_cache_hot_records)
  const __nv_bfloat16* tables;    // nq x M x 256 BF16 tables built for the batch, or null
  const unsigned long long* entry_keys;  // nq: nearest-pivot keys (entry_tc.cu), or null (pivot-graph walk)
  int fma;
  int32_t* nns;                   // nq x k_max
  float* dists;                   // nq x k_max
  int32_t* found;                 // nq
  int32_t* hops;                  // nq or null
  int64_t* bytes;                 // nq or null (accumulated; zeroed by the caller)
  int* next_query;                // work counter, zeroed before launch
  unsigned int* err;
};

// Visited-cache size (log2 slots) of the batched form for a list of ef_max:
// the smallest power of two >= 4 ef_max, within 2^9 .. 2^13 (the handle's tuned
// delta is added by the caller).
inline int batch_hash_bits(int ef_max) {
  int b = 9;
  while ((1 << b) < 4 * ef_max && b < 13) b++;
  return b;
}

size_t batch_smem_bytes(int M, int tab_bytes, int hash_bits, int L_max, int max_m, int W, int k_max, int dim);
cudaError_t launch_batch(const BatchParams& p, int dtype, int table_bf16, int W, int num_sms, cudaStream_t stream);

// CUDA-core tables (FP32 or BF16 storage) of a query batch, one warp per query.
cudaError_t launch_table_cc(const DeviceIndex& ix, int dim, int M, const float* queries, int nq, int fma,
                            bool bf16, void* tables, cudaStream_t stream);
cudaError_t widen_bf16(const __nv_bfloat16* in, float* out, size_t n, cudaStream_t stream);

// Host layout of the tensor-core B operand tiles and centroid norms (table_tc.cu).
bool make_tc_panels(const std::vector<float>& pivots, const std::vector<int32_t>& chunk_off, int dim,
                    std::vector<uint8_t>& hi, std::vector<uint8_t>& lo, std::vector<float>& pnorm, int& p_out,
                    int& groups_out);
size_t table_tc_smem(int M, int groups);

// BF16 PQ tables of a query batch on the tensor cores (table_tc.cu):
// tables[q][c][j] = |r_qc|^2 - 2 r_qc . P_cj + |P_cj|^2 with r = q - centroid.
cudaError_t launch_table_tc(const DeviceIndex& ix, int dim, int M, const float* queries, int nq, int split3,
                            __nv_bfloat16* tables, cudaStream_t stream, int num_sms, const int* nq_dev = nullptr);

// Nearest pivot of every query on the tensor cores (entry_tc.cu): keys[q] =
// (ordered bits of |x|^2 - 2 q.x) << 32 | pivot index, the minimum over the
// pivot file; all bits set when the file is empty.
void make_entry_panels(const std::vector<uint8_t>& data, int nav_n, int dim, int elt, std::vector<uint8_t>& panel,
                       std::vector<float>& pnorm, int& nk_out, int& ntiles_out);
size_t entry_tc_smem(int nk);
cudaError_t launch_entry_tc(const DeviceIndex& ix, int dim, const float* queries, int nq, unsigned long long* keys,
                            cudaStream_t stream, int num_sms, const int* nq_dev = nullptr);
// Pivot row (or -1) and node id (or -1) of each key; either output may be null.
cudaError_t launch_entry_ids(const DeviceIndex& ix, int nav_n, const unsigned long long* keys, int nq, int32_t* pivot,
                             int32_t* node, cudaStream_t stream);

// Per-warp shared-memory footprint of the plain kernel, in bytes.
size_t plain_smem_per_warp(int M, int L, int max_m, int k, int dim);
// Launch the plain kernel for one batch (walk_plain.cu). Returns a cudaError_t.
cudaError_t launch_plain(const PlainParams& p, int dtype, int num_sms, cudaStream_t stream);

// File readers (gann_io.cpp). Throw GannError on failure.
void read_disk_index(const std::string& path, HostIndex& hx, std::vector<uint8_t>* pages_out);
void read_pq(const std::string& prefix, HostIndex& hx, std::vector<uint8_t>& codes);
void read_nav(const std::string& dir, HostIndex& hx);

struct GannError {
  int code;
  std::string msg;
};

}  // namespace gann

struct gann_index {
  std::mutex mu;
  gann::HostIndex hx;
  gann::DeviceIndex dx;
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<void*> allocations;  // device allocations owned by the handle
  int64_t device_bytes = 0;
  uint8_t* host_pages = nullptr;   // pinned, mapped page body (GANN_OPEN_HOST_PAGES)
  int64_t host_bytes = 0;
  int64_t rec_cache_bytes = 0;     // HBM record cache (gann_cache_hot_records)
  int* d_counter = nullptr;       // work counter scratch (plain kernel)
  unsigned int* d_err = nullptr;   // kernel error word
  // per-call device buffers, grown on demand
  float* d_q = nullptr;
  int32_t* d_nns = nullptr;
  float* d_dists = nullptr;
  int32_t* d_found = nullptr;
  size_t cap_q = 0, cap_out = 0, cap_dists = 0, cap_found = 0;
  int32_t* d_kq = nullptr;           // per-query k / L uploaded by the host batch entry
  int32_t* d_lq = nullptr;
  size_t cap_kq = 0, cap_lq = 0;
  __nv_bfloat16* d_tables = nullptr; // BF16 tables of one batch (scratch)
  size_t cap_tables = 0;
  unsigned long long* d_entry = nullptr;  // nearest-pivot keys of one batch (scratch)
  size_t cap_entry = 0;
  int fma_table = 1, fma_exact = 1;
  int tuned_beam = 0;       // batched-form defaults chosen by gann_autotune (0 = built-in)
  int tuned_hash_delta = 0; // added to the L-sized visited-cache bits
};
