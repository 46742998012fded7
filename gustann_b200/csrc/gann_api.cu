// C ABI of libgann: index loading into HBM and the search entry points.
//
// gann_open   ~ GustANN::GustANN + GustANN::init_pure_mem(cfg, true)  (src/ssd_search.cu:55-112,
//               src/pure_mem.cu:27-69)
// gann_search ~ GustANN::search -> PureMemExecutor::search            (src/pure_mem.cu:71-199)
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "gann_internal.h"

namespace {

thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

struct CudaFail {
  cudaError_t e;
  const char* what;
};

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaFail{e, what};
}

template <class T>
T* dev_alloc(gann_index* h, size_t count) {
  void* p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc(&p, sizeof(T) * count);
  if (e != cudaSuccess) throw CudaFail{e, "cudaMalloc"};
  h->allocations.push_back(p);
  h->device_bytes += (int64_t)(sizeof(T) * count);
  return static_cast<T*>(p);
}

template <class T>
T* upload(gann_index* h, const std::vector<T>& v) {
  T* d = dev_alloc<T>(h, v.size());
  if (!v.empty()) ck(cudaMemcpy(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "upload");
  return d;
}

// Stream the page body of _disk.index (everything after the first 4 KB sector,
// src/pure_mem.cu:51-61) into HBM through two pinned bounce buffers.
void upload_pages(gann_index* h, const std::string& path, uint8_t* dst, int64_t bytes) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) throw gann::GannError{GANN_EIO, "cannot open " + path};
  std::unique_ptr<FILE, int (*)(FILE*)> guard(f, std::fclose);
  std::fseek(f, gann::kPageSize, SEEK_SET);
  const size_t chunk = 64u << 20;
  uint8_t* bounce[2] = {nullptr, nullptr};
  cudaEvent_t done[2];
  ck(cudaMallocHost(&bounce[0], chunk), "cudaMallocHost");
  if (cudaMallocHost(&bounce[1], chunk) != cudaSuccess) {
    cudaFreeHost(bounce[0]);
    throw CudaFail{cudaErrorMemoryAllocation, "cudaMallocHost"};
  }
  cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming);
  cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming);
  bool used[2] = {false, false};
  int64_t off = 0;
  int b = 0;
  std::string err;
  while (off < bytes) {
    size_t n = (size_t)std::min<int64_t>(chunk, bytes - off);
    if (used[b]) cudaEventSynchronize(done[b]);
    if (std::fread(bounce[b], 1, n, f) != n) {
      err = "short read of index pages: " + path;
      break;
    }
    if (cudaMemcpyAsync(dst + off, bounce[b], n, cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        cudaEventRecord(done[b], h->stream) != cudaSuccess) {
      err = "page upload failed";
      break;
    }
    used[b] = true;
    off += (int64_t)n;
    b ^= 1;
  }
  cudaStreamSynchronize(h->stream);
  cudaEventDestroy(done[0]);
  cudaEventDestroy(done[1]);
  cudaFreeHost(bounce[0]);
  cudaFreeHost(bounce[1]);
  if (!err.empty()) throw gann::GannError{GANN_EIO, err};
}

// Records-in-host-memory mode (the reference's use_gpu_mem = false,
// src/pure_mem.cu:51-66): the page body is read straight into pinned, mapped
// host memory and the kernels read records through its device alias, so every
// record fetch crosses PCIe/C2C while codes, pivots and the pivot graph stay in HBM.
uint8_t* host_pages(gann_index* h, const std::string& path, int64_t bytes) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) throw gann::GannError{GANN_EIO, "cannot open " + path};
  std::unique_ptr<FILE, int (*)(FILE*)> guard(f, std::fclose);
  std::fseek(f, gann::kPageSize, SEEK_SET);
  ck(cudaHostAlloc(reinterpret_cast<void**>(&h->host_pages), (size_t)bytes,
                   cudaHostAllocPortable | cudaHostAllocMapped),
     "cudaHostAlloc (index pages)");
  h->host_bytes = bytes;
  const size_t chunk = 256u << 20;
  for (int64_t off = 0; off < bytes;) {
    size_t n = (size_t)std::min<int64_t>(chunk, bytes - off);
    if (std::fread(h->host_pages + off, 1, n, f) != n)
      throw gann::GannError{GANN_EIO, "short read of index pages: " + path};
    off += (int64_t)n;
  }
  void* dptr = nullptr;
  ck(cudaHostGetDevicePointer(&dptr, h->host_pages, 0), "cudaHostGetDevicePointer");
  return static_cast<uint8_t*>(dptr);
}

// Load-time check of every record: degree <= max_m0 and neighbour ids in [0, n).
__global__ void validate_records(const uint8_t* pages, int64_t n, int64_t npp, int64_t node_len,
                                 int64_t data_len, int max_m, unsigned long long* bad) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t* node = pages + (u / npp) * gann::kPageSize + (u % npp) * node_len;
    const int32_t* meta = reinterpret_cast<const int32_t*>(node + data_len);
    int deg = meta[0];
    bool ok = deg >= 0 && deg <= max_m;
    for (int t = 0; ok && t < deg; t++) ok = (unsigned)meta[1 + t] < (unsigned)n;
    if (!ok) atomicAdd(bad, 1ull);
  }
}

void free_all(gann_index* h) {
  for (void* p : h->allocations) cudaFree(p);
  h->allocations.clear();
  for (void* p : {(void*)h->d_q, (void*)h->d_nns, (void*)h->d_dists, (void*)h->d_found, (void*)h->d_kq,
                  (void*)h->d_lq, (void*)h->d_tables, (void*)h->d_entry})
    if (p) cudaFree(p);
  h->d_kq = h->d_lq = nullptr;
  h->d_tables = nullptr;
  h->d_entry = nullptr;
  h->d_q = nullptr;
  h->d_nns = nullptr;
  h->d_dists = nullptr;
  h->d_found = nullptr;
  if (h->host_pages) cudaFreeHost(h->host_pages);
  h->host_pages = nullptr;
  h->host_bytes = 0;
  h->dx.rec_remap = nullptr;  // both freed with the allocations above
  h->dx.rec_cache = nullptr;
  h->dx.rec_stride = 0;
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  h->ev0 = h->ev1 = nullptr;
  h->stream = nullptr;
}

template <class T>
void grow(T*& p, size_t& cap, size_t need) {
  if (need <= cap) return;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  ck(cudaMalloc(&p, sizeof(T) * need), "cudaMalloc (search buffers)");
  cap = need;
}

int check_search_args(const gann_index* h, int nq, int topk, int ef_search) {
  if (!h) return set_error(GANN_EINVAL, "null handle");
  if (nq < 0) return set_error(GANN_EINVAL, "nq must be >= 0");
  if (topk < 1 || ef_search < 1) return set_error(GANN_EINVAL, "topk and ef_search must be >= 1");
  if (ef_search > 4096 || topk > 4096) return set_error(GANN_ERANGE, "topk and ef_search are limited to 4096");
  size_t per_warp = gann::plain_smem_per_warp(h->hx.pq_m, ef_search, (int)h->hx.max_m0, topk, (int)h->hx.dim);
  if (per_warp > 227 * 1024)
    return set_error(GANN_ERANGE, "table + lists of one query exceed the 227 KB of shared memory per CTA");
  return GANN_OK;
}

gann::PlainParams make_params(gann_index* h, const float* d_q, int nq, int topk, int ef_search, int32_t* d_nns,
                              float* d_dists, int32_t* d_found) {
  gann::PlainParams p{};
  p.ix = h->dx;
  p.n = h->hx.n;
  p.npp = h->hx.npp;
  p.node_len = h->hx.node_len;
  p.data_len = h->hx.data_len;
  p.medoid = h->hx.medoid;
  p.dim = (int)h->hx.dim;
  p.max_m = (int)h->hx.max_m0;
  p.M = h->hx.pq_m;
  p.has_nav = h->hx.has_nav;
  p.nav_n = h->hx.nav_n;
  p.nav_max_m = h->hx.nav_max_m;
  p.nav_start = h->hx.nav_start;
  p.queries = d_q;
  p.nq = nq;
  p.L = ef_search;
  p.k = topk;
  p.fma_table = h->fma_table;
  p.fma_exact = h->fma_exact;
  p.nns = d_nns;
  p.dists = d_dists;
  p.found = d_found;
  p.hops = nullptr;
  p.bytes = nullptr;
  p.next_query = h->d_counter;
  p.err = h->d_err;
  return p;
}

int kernel_error_status(unsigned int err) {
  if (!err) return GANN_OK;
  std::string m = "search kernel reported:";
  if (err & gann::kErrBadId) m += " neighbour/entry id out of range;";
  if (err & gann::kErrBadDegree) m += " degree word above max_m0;";
  if (err & gann::kErrHopCap) m += " hop limit reached;";
  if (err & gann::kErrNavCap) m += " pivot-graph iteration limit reached;";
  if (err & gann::kErrWaitLimit) m += " wait limit reached;";
  return set_error(GANN_EKERNEL, m);
}

}  // namespace

// Message slot of gann_last_error() for entry points defined in other files.
int gann_internal_set_error(int code, const char* msg) { return set_error(code, msg); }

extern "C" {

const char* gann_last_error(void) { return g_last_error.c_str(); }

int gann_open(const char* index_file, const char* pq_prefix, const char* nav_dir, int dtype, int flags,
              gann_t** out) {
  if (!out) return set_error(GANN_EINVAL, "null output handle");
  *out = nullptr;
  if (!index_file || !pq_prefix) return set_error(GANN_EINVAL, "index_file and pq_prefix are required");
  if (dtype != GANN_UINT8 && dtype != GANN_FLOAT) return set_error(GANN_EINVAL, "dtype must be GANN_UINT8 or GANN_FLOAT");
  auto h = std::make_unique<gann_index>();
  try {
    h->hx.dtype = dtype;
    h->hx.elt = dtype == GANN_UINT8 ? 1 : 4;
    gann::read_disk_index(index_file, h->hx, nullptr);
    std::vector<uint8_t> codes;
    gann::read_pq(pq_prefix, h->hx, codes);
    if ((int64_t)h->hx.pivots.size() / gann::kPivots != h->hx.dim)
      throw gann::GannError{GANN_EFORMAT, "PQ pivots dimension differs from the index dimension"};
    if (nav_dir && nav_dir[0]) gann::read_nav(nav_dir, h->hx);

    ck(cudaGetDevice(&h->device), "cudaGetDevice");
    ck(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device), "cudaDeviceGetAttribute");
    ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaEventCreate(&h->ev0), "cudaEventCreate");
    ck(cudaEventCreate(&h->ev1), "cudaEventCreate");

    const gann::HostIndex& hx = h->hx;
    uint8_t* pages = nullptr;
    if (flags & GANN_OPEN_HOST_PAGES) {
      pages = host_pages(h.get(), index_file, hx.num_pages * (int64_t)gann::kPageSize);
    } else {
      pages = dev_alloc<uint8_t>(h.get(), (size_t)hx.num_pages * gann::kPageSize);
      upload_pages(h.get(), index_file, pages, hx.num_pages * (int64_t)gann::kPageSize);
    }
    h->dx.pages = pages;
    h->dx.codes = upload(h.get(), codes);
    std::vector<float> pivots_t((size_t)hx.dim * gann::kPivots);  // pq_search.cu:86-91
    for (int i = 0; i < gann::kPivots; i++)
      for (int64_t j = 0; j < hx.dim; j++) pivots_t[j * gann::kPivots + i] = hx.pivots[i * hx.dim + j];
    h->dx.pivots_t = upload(h.get(), pivots_t);
    h->dx.centroid = upload(h.get(), hx.centroid);
    h->dx.chunk_off = upload(h.get(), hx.chunk_offsets);
    if (hx.has_nav) {
      h->dx.nav_data = upload(h.get(), hx.nav_data);
      h->dx.nav_graph = upload(h.get(), hx.nav_graph);
      h->dx.nav_map = upload(h.get(), hx.nav_map);
    }
    {  // operands of the tensor-core table build, when every chunk is at most 16 wide
      std::vector<uint8_t> bhi, blo;
      std::vector<float> pn;
      int tp = 0, tg = 0;
      if (gann::make_tc_panels(hx.pivots, hx.chunk_offsets, (int)hx.dim, bhi, blo, pn, tp, tg) &&
          gann::table_tc_smem(hx.pq_m, tg) <= 227 * 1024) {
        h->dx.tc_bpanel_hi = upload(h.get(), bhi);
        h->dx.tc_bpanel_lo = upload(h.get(), blo);
        h->dx.tc_pnorm = upload(h.get(), pn);
        h->dx.tc_p = tp;
        h->dx.tc_groups = tg;
      }
    }
    if (hx.has_nav) {  // operands of the nearest-pivot entry (entry_tc.cu), when they fit shared memory
      std::vector<uint8_t> panel;
      std::vector<float> pn;
      int nk = 0, tiles = 0;
      if (gann::entry_tc_smem((int)((hx.dim + 15) / 16)) <= 227 * 1024) {
        gann::make_entry_panels(hx.nav_data, hx.nav_n, (int)hx.dim, hx.elt, panel, pn, nk, tiles);
        h->dx.entry_panel = upload(h.get(), panel);
        h->dx.entry_pnorm = upload(h.get(), pn);
        h->dx.entry_nk = nk;
        h->dx.entry_tiles = tiles;
      }
    }
    h->d_counter = dev_alloc<int>(h.get(), 1);
    h->d_err = dev_alloc<unsigned int>(h.get(), 1);
    h->dx.err = h->d_err;
    ck(cudaMemset(h->d_err, 0, sizeof(unsigned int)), "cudaMemset");
    if (!(flags & GANN_OPEN_NO_VALIDATE)) {
      unsigned long long* bad = dev_alloc<unsigned long long>(h.get(), 1);
      ck(cudaMemsetAsync(bad, 0, sizeof(*bad), h->stream), "cudaMemset");
      validate_records<<<h->num_sms * 8, 256, 0, h->stream>>>(pages, hx.n, hx.npp, hx.node_len, hx.data_len,
                                                              (int)hx.max_m0, bad);
      ck(cudaGetLastError(), "validate launch");
      unsigned long long nbad = 0;
      ck(cudaMemcpyAsync(&nbad, bad, sizeof(nbad), cudaMemcpyDeviceToHost, h->stream), "cudaMemcpy");
      ck(cudaStreamSynchronize(h->stream), "validate");
      if (nbad)
        throw gann::GannError{GANN_EFORMAT, std::to_string(nbad) +
                                                " records have a degree above max_m0 or a neighbour id outside the index"};
    }
    ck(cudaStreamSynchronize(h->stream), "open");
  } catch (const gann::GannError& e) {
    free_all(h.get());
    return set_error(e.code, e.msg);
  } catch (const CudaFail& e) {
    free_all(h.get());
    return set_error(e.e == cudaErrorMemoryAllocation ? GANN_ENOMEM : GANN_ECUDA,
                     std::string(e.what) + ": " + cudaGetErrorString(e.e));
  } catch (const std::bad_alloc&) {
    free_all(h.get());
    return set_error(GANN_ENOMEM, "host allocation failed");
  }
  *out = h.release();
  return GANN_OK;
}

int gann_close(gann_t* h) {
  if (!h) return GANN_OK;
  {
    std::lock_guard<std::mutex> lk(h->mu);
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_all(h);
    if (prev >= 0) cudaSetDevice(prev);
  }
  delete h;
  return GANN_OK;
}

int gann_get_info(const gann_t* h, gann_info_t* out) {
  if (!h || !out) return set_error(GANN_EINVAL, "null argument");
  const gann::HostIndex& hx = h->hx;
  out->num_points = hx.n;
  out->dim = hx.dim;
  out->max_degree = hx.max_m0;
  out->medoid = hx.medoid;
  out->node_len = hx.node_len;
  out->nodes_per_page = hx.npp;
  out->num_pages = hx.num_pages;
  out->pq_chunks = hx.pq_m;
  out->dtype = hx.dtype;
  out->has_nav = hx.has_nav;
  out->nav_points = hx.nav_n;
  out->nav_max_degree = hx.nav_max_m;
  out->device = h->device;
  out->device_bytes = h->device_bytes;
  out->host_pages = h->host_pages != nullptr;
  out->host_bytes = h->host_bytes;
  return GANN_OK;
}

int gann_search_device_ex(gann_t* h, const float* d_queries, int nq, int topk, int ef_search, int32_t* d_nns,
                          float* d_distances, int32_t* d_found_cnt, int32_t* d_hops, int64_t* d_bytes,
                          void* stream) {
  int rc = check_search_args(h, nq, topk, ef_search);
  if (rc) return rc;
  if (nq == 0) return GANN_OK;
  if (!d_queries || !d_nns || !d_distances || !d_found_cnt) return set_error(GANN_EINVAL, "null buffer");
  std::lock_guard<std::mutex> lk(h->mu);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
  gann::PlainParams p = make_params(h, d_queries, nq, topk, ef_search, d_nns, d_distances, d_found_cnt);
  p.hops = d_hops;
  p.bytes = d_bytes;
  cudaError_t e = cudaMemsetAsync(h->d_counter, 0, sizeof(int), s);
  if (e == cudaSuccess) e = gann::launch_plain(p, h->hx.dtype, h->num_sms, s);
  if (e != cudaSuccess) return set_error(GANN_ECUDA, std::string("plain search launch: ") + cudaGetErrorString(e));
  return GANN_OK;
}

int gann_search_device(gann_t* h, const float* d_queries, int nq, int topk, int ef_search, int32_t* d_nns,
                       float* d_distances, int32_t* d_found_cnt, void* stream) {
  return gann_search_device_ex(h, d_queries, nq, topk, ef_search, d_nns, d_distances, d_found_cnt, nullptr,
                               nullptr, stream);
}

int gann_search(gann_t* h, const float* queries, int nq, int topk, int ef_search, int32_t* nns, float* distances,
                int32_t* found_cnt, double* run_time) {
  int rc = check_search_args(h, nq, topk, ef_search);
  if (rc) return rc;
  if (run_time) *run_time = 0.0;
  if (nq == 0) return GANN_OK;
  if (!queries || !nns || !distances || !found_cnt) return set_error(GANN_EINVAL, "null buffer");
  std::lock_guard<std::mutex> lk(h->mu);
  try {
    const size_t qn = (size_t)nq * h->hx.dim, on = (size_t)nq * topk;
    grow(h->d_q, h->cap_q, qn);
    grow(h->d_nns, h->cap_out, on);
    grow(h->d_dists, h->cap_dists, on);
    grow(h->d_found, h->cap_found, (size_t)nq);
    cudaStream_t s = h->stream;
    ck(cudaMemcpyAsync(h->d_q, queries, sizeof(float) * qn, cudaMemcpyHostToDevice, s), "query upload");
    gann::PlainParams p = make_params(h, h->d_q, nq, topk, ef_search, h->d_nns, h->d_dists, h->d_found);
    ck(cudaMemsetAsync(h->d_counter, 0, sizeof(int), s), "cudaMemset");
    ck(cudaEventRecord(h->ev0, s), "cudaEventRecord");
    ck(gann::launch_plain(p, h->hx.dtype, h->num_sms, s), "plain search launch");
    ck(cudaEventRecord(h->ev1, s), "cudaEventRecord");
    ck(cudaMemcpyAsync(nns, h->d_nns, sizeof(int32_t) * on, cudaMemcpyDeviceToHost, s), "result download");
    ck(cudaMemcpyAsync(distances, h->d_dists, sizeof(float) * on, cudaMemcpyDeviceToHost, s), "result download");
    ck(cudaMemcpyAsync(found_cnt, h->d_found, sizeof(int32_t) * nq, cudaMemcpyDeviceToHost, s), "result download");
    unsigned int err = 0;
    ck(cudaMemcpyAsync(&err, h->d_err, sizeof(err), cudaMemcpyDeviceToHost, s), "error word");
    ck(cudaStreamSynchronize(s), "search");
    if (err) {
      ck(cudaMemset(h->d_err, 0, sizeof(unsigned int)), "cudaMemset");
      return kernel_error_status(err);
    }
    float ms = 0.0f;
    ck(cudaEventElapsedTime(&ms, h->ev0, h->ev1), "cudaEventElapsedTime");
    if (run_time) *run_time = ms * 1e-3;
  } catch (const CudaFail& e) {
    return set_error(GANN_ECUDA, std::string(e.what) + ": " + cudaGetErrorString(e.e));
  }
  return GANN_OK;
}

}  // extern "C"

namespace {

cudaError_t entry_scratch(gann_t* h, int nq);

// Why a handle has no nearest-pivot operands (gann_open lays them out only for
// a pivot graph whose tiles fit shared memory: 11 K slices of 16, dim <= 176).
constexpr const char* kNoEntryPanel = "the nearest-pivot entry needs a pivot graph and dim <= 176";

// Enqueue one batched search. counter / tables: caller-owned work counter and
// BF16 table buffer (nq x M x 256) for concurrent launches; null = the handle's.
int enqueue_batch(gann_t* h, const float* d_q, int nq, const int32_t* d_k, const int32_t* d_l, int k_max,
                  int l_max, const gann_batch_opts_t* opts, int32_t* d_nns, float* d_dists, int32_t* d_found,
                  int32_t* d_hops, int64_t* d_bytes, cudaStream_t s, int* counter = nullptr,
                  __nv_bfloat16* tables = nullptr, const int* nq_dev = nullptr,
                  int32_t* visit_count = nullptr, unsigned long long* entry_keys = nullptr) {
  gann_batch_opts_t o{};
  if (opts) o = *opts;
  const int prec = opts ? o.precision : GANN_PREC_BF16X3;
  const int W = o.beam_width ? o.beam_width : (h->tuned_beam ? h->tuned_beam : 4);
  if (!(W == 1 || W == 2 || W == 4 || W == 8 || W == 16))
    return set_error(GANN_EINVAL, "beam_width must be 1, 2, 4, 8 or 16");
  if (prec < GANN_PREC_FP32 || prec > GANN_PREC_BF16_CC) return set_error(GANN_EINVAL, "unknown precision");
  if (o.entry != GANN_ENTRY_NAV_WALK && o.entry != GANN_ENTRY_NEAREST_PIVOT)
    return set_error(GANN_EINVAL, "unknown entry");
  if (o.entry == GANN_ENTRY_NEAREST_PIVOT && !h->dx.entry_panel)
    return set_error(GANN_ERANGE, kNoEntryPanel);
  const int hb = o.hash_bits ? o.hash_bits : gann::batch_hash_bits(l_max) + h->tuned_hash_delta;
  if (hb < 4 || hb > 16) return set_error(GANN_EINVAL, "hash_bits must be in 4..16");
  const bool bf16 = prec != GANN_PREC_FP32;
  const size_t smem = gann::batch_smem_bytes(h->hx.pq_m, bf16 ? 2 : 4, hb, l_max, (int)h->hx.max_m0, W, k_max,
                                             (int)h->hx.dim);
  if (smem > 227 * 1024)
    return set_error(GANN_ERANGE, "table + lists + visited cache of one query exceed 227 KB of shared memory");
  gann::BatchParams p{};
  p.ix = h->dx;
  p.n = h->hx.n;
  p.npp = h->hx.npp;
  p.node_len = h->hx.node_len;
  p.data_len = h->hx.data_len;
  p.medoid = h->hx.medoid;
  p.dim = (int)h->hx.dim;
  p.max_m = (int)h->hx.max_m0;
  p.M = h->hx.pq_m;
  p.has_nav = h->hx.has_nav;
  p.nav_n = h->hx.nav_n;
  p.nav_max_m = h->hx.nav_max_m;
  p.nav_start = h->hx.nav_start;
  p.queries = d_q;
  p.nq = nq;
  p.nq_dev = nq_dev;
  p.visit_count = visit_count;
  p.L_per_q = d_l;
  p.k_per_q = d_k;
  p.L_max = l_max;
  p.k_max = k_max;
  p.hash_bits = hb;
  p.npp_div = gann::FastDiv((uint32_t)h->hx.npp);
  p.fma = h->fma_exact;
  p.nns = d_nns;
  p.dists = d_dists;
  p.found = d_found;
  p.hops = d_hops;
  p.bytes = d_bytes;
  p.next_query = counter ? counter : h->d_counter;
  p.err = h->d_err;
  cudaError_t e = cudaSuccess;
  if ((prec == GANN_PREC_BF16 || prec == GANN_PREC_BF16X3) && !h->dx.tc_bpanel_hi)
    return set_error(GANN_ERANGE, "tensor-core tables need PQ chunks of at most 16 dimensions");
  if (prec == GANN_PREC_BF16 || prec == GANN_PREC_BF16X3) {
    const size_t need = (size_t)nq * h->hx.pq_m * gann::kPivots;
    if (!tables && need > h->cap_tables) {
      if (h->d_tables) cudaFree(h->d_tables);
      h->d_tables = nullptr;
      h->cap_tables = 0;
      e = cudaMalloc(&h->d_tables, need * sizeof(__nv_bfloat16));
      if (e != cudaSuccess) return set_error(GANN_ENOMEM, "cannot allocate the batch's BF16 tables");
      h->cap_tables = need;
    }
    __nv_bfloat16* tab = tables ? tables : h->d_tables;
    e = gann::launch_table_tc(h->dx, (int)h->hx.dim, h->hx.pq_m, d_q, nq, prec == GANN_PREC_BF16X3, tab, s,
                                h->num_sms, nq_dev);
    if (e != cudaSuccess) return set_error(GANN_ECUDA, std::string("table build: ") + cudaGetErrorString(e));
    p.tables = tab;
  }
  if (o.entry == GANN_ENTRY_NEAREST_PIVOT) {
    if (!entry_keys && entry_scratch(h, nq) != cudaSuccess)
      return set_error(GANN_ENOMEM, "cannot allocate the batch's entry keys");
    unsigned long long* keys = entry_keys ? entry_keys : h->d_entry;
    e = gann::launch_entry_tc(h->dx, (int)h->hx.dim, d_q, nq, keys, s, h->num_sms, nq_dev);
    if (e != cudaSuccess) return set_error(GANN_ECUDA, std::string("entry search: ") + cudaGetErrorString(e));
    p.entry_keys = keys;
  }
  if (d_bytes) e = cudaMemsetAsync(d_bytes, 0, sizeof(int64_t) * nq, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(p.next_query, 0, sizeof(int), s);
  if (e == cudaSuccess) e = gann::launch_batch(p, h->hx.dtype, bf16, W, h->num_sms, s);
  if (e != cudaSuccess) return set_error(GANN_ECUDA, std::string("batch search launch: ") + cudaGetErrorString(e));
  return GANN_OK;
}

// The handle's entry-key scratch, grown to nq keys.
cudaError_t entry_scratch(gann_t* h, int nq) {
  if ((size_t)nq <= h->cap_entry) return cudaSuccess;
  if (h->d_entry) cudaFree(h->d_entry);
  h->d_entry = nullptr;
  h->cap_entry = 0;
  const cudaError_t e = cudaMalloc(&h->d_entry, sizeof(unsigned long long) * (size_t)nq);
  if (e == cudaSuccess) h->cap_entry = (size_t)nq;
  return e;
}

int check_batch_args(const gann_t* h, int nq, int k_max, int l_max) {
  if (!h) return set_error(GANN_EINVAL, "null handle");
  if (nq < 0) return set_error(GANN_EINVAL, "nq must be >= 0");
  if (k_max < 1 || l_max < 1) return set_error(GANN_EINVAL, "topk_max and ef_max must be >= 1");
  if (k_max > 4096 || l_max > 4096) return set_error(GANN_ERANGE, "topk and ef_search are limited to 4096");
  return GANN_OK;
}

}  // namespace

extern "C" {

int gann_search_batch_device(gann_t* h, const float* d_queries, int nq, const int32_t* d_topk,
                             const int32_t* d_ef_search, int topk_max, int ef_max, const gann_batch_opts_t* opts,
                             int32_t* d_nns, float* d_distances, int32_t* d_found_cnt, int32_t* d_hops,
                             int64_t* d_bytes, void* stream) {
  int rc = check_batch_args(h, nq, topk_max, ef_max);
  if (rc) return rc;
  if (nq == 0) return GANN_OK;
  if (!d_queries || !d_nns || !d_distances || !d_found_cnt) return set_error(GANN_EINVAL, "null buffer");
  std::lock_guard<std::mutex> lk(h->mu);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
  return enqueue_batch(h, d_queries, nq, d_topk, d_ef_search, topk_max, ef_max, opts, d_nns, d_distances,
                       d_found_cnt, d_hops, d_bytes, s);
}

int gann_nearest_pivots(gann_t* h, const float* d_queries, int nq, int32_t* d_pivot, int32_t* d_node,
                        void* stream) {
  if (!h) return set_error(GANN_EINVAL, "null handle");
  if (nq < 0) return set_error(GANN_EINVAL, "nq must be >= 0");
  if (nq == 0) return GANN_OK;
  if (!d_queries) return set_error(GANN_EINVAL, "null buffer");
  if (!h->dx.entry_panel) return set_error(GANN_ERANGE, kNoEntryPanel);
  std::lock_guard<std::mutex> lk(h->mu);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
  if (entry_scratch(h, nq) != cudaSuccess) return set_error(GANN_ENOMEM, "cannot allocate the entry keys");
  cudaError_t e = gann::launch_entry_tc(h->dx, (int)h->hx.dim, d_queries, nq, h->d_entry, s, h->num_sms);
  if (e == cudaSuccess) e = gann::launch_entry_ids(h->dx, h->hx.nav_n, h->d_entry, nq, d_pivot, d_node, s);
  if (e != cudaSuccess) return set_error(GANN_ECUDA, std::string("nearest pivots: ") + cudaGetErrorString(e));
  return GANN_OK;
}

int gann_search_batch(gann_t* h, const float* queries, int nq, const int32_t* topk, const int32_t* ef_search,
                      int topk_max, int ef_max, const gann_batch_opts_t* opts, int32_t* nns, float* distances,
                      int32_t* found_cnt, double* run_time) {
  if (run_time) *run_time = 0.0;
  if (h && nq > 0 && topk) {
    int m = 0;
    for (int i = 0; i < nq; i++) m = topk[i] > m ? topk[i] : m;
    if (m > topk_max) return set_error(GANN_EINVAL, "a topk entry exceeds topk_max");
  }
  if (h && nq > 0 && ef_search) {
    int m = 0;
    for (int i = 0; i < nq; i++) m = ef_search[i] > m ? ef_search[i] : m;
    if (m > ef_max) return set_error(GANN_EINVAL, "an ef_search entry exceeds ef_max");
  }
  int rc = check_batch_args(h, nq, topk_max, ef_max);
  if (rc) return rc;
  if (nq == 0) return GANN_OK;
  if (!queries || !nns || !distances || !found_cnt) return set_error(GANN_EINVAL, "null buffer");
  std::lock_guard<std::mutex> lk(h->mu);
  try {
    const size_t qn = (size_t)nq * h->hx.dim, on = (size_t)nq * topk_max;
    grow(h->d_q, h->cap_q, qn);
    grow(h->d_nns, h->cap_out, on);
    grow(h->d_dists, h->cap_dists, on);
    grow(h->d_found, h->cap_found, (size_t)nq);
    cudaStream_t s = h->stream;
    ck(cudaMemcpyAsync(h->d_q, queries, sizeof(float) * qn, cudaMemcpyHostToDevice, s), "query upload");
    int32_t *dk = nullptr, *dl = nullptr;
    if (topk) {
      grow(h->d_kq, h->cap_kq, (size_t)nq);
      ck(cudaMemcpyAsync(h->d_kq, topk, sizeof(int32_t) * nq, cudaMemcpyHostToDevice, s), "topk upload");
      dk = h->d_kq;
    }
    if (ef_search) {
      grow(h->d_lq, h->cap_lq, (size_t)nq);
      ck(cudaMemcpyAsync(h->d_lq, ef_search, sizeof(int32_t) * nq, cudaMemcpyHostToDevice, s), "L upload");
      dl = h->d_lq;
    }
    ck(cudaEventRecord(h->ev0, s), "cudaEventRecord");
    rc = enqueue_batch(h, h->d_q, nq, dk, dl, topk_max, ef_max, opts, h->d_nns, h->d_dists, h->d_found, nullptr,
                       nullptr, s);
    if (rc) return rc;
    ck(cudaEventRecord(h->ev1, s), "cudaEventRecord");
    ck(cudaMemcpyAsync(nns, h->d_nns, sizeof(int32_t) * on, cudaMemcpyDeviceToHost, s), "result download");
    ck(cudaMemcpyAsync(distances, h->d_dists, sizeof(float) * on, cudaMemcpyDeviceToHost, s), "result download");
    ck(cudaMemcpyAsync(found_cnt, h->d_found, sizeof(int32_t) * nq, cudaMemcpyDeviceToHost, s), "result download");
    unsigned int err = 0;
    ck(cudaMemcpyAsync(&err, h->d_err, sizeof(err), cudaMemcpyDeviceToHost, s), "error word");
    ck(cudaStreamSynchronize(s), "batch search");
    if (err) {
      ck(cudaMemset(h->d_err, 0, sizeof(unsigned int)), "cudaMemset");
      return kernel_error_status(err);
    }
    float ms = 0.0f;
    ck(cudaEventElapsedTime(&ms, h->ev0, h->ev1), "cudaEventElapsedTime");
    if (run_time) *run_time = ms * 1e-3;
  } catch (const CudaFail& e) {
    return set_error(GANN_ECUDA, std::string(e.what) + ": " + cudaGetErrorString(e.e));
  }
  return GANN_OK;
}

}  // extern "C"

extern "C" {

int gann_pq_tables(gann_t* h, const float* queries, int nq, int precision, float* tables) {
  if (!h || nq < 0 || (nq && (!queries || !tables))) return set_error(GANN_EINVAL, "bad argument");
  if (precision < GANN_PREC_FP32 || precision > GANN_PREC_BF16_CC) return set_error(GANN_EINVAL, "unknown precision");
  if (nq == 0) return GANN_OK;
  if ((precision == GANN_PREC_BF16 || precision == GANN_PREC_BF16X3) && !h->dx.tc_bpanel_hi)
    return set_error(GANN_ERANGE, "tensor-core tables need PQ chunks of at most 16 dimensions");
  std::lock_guard<std::mutex> lk(h->mu);
  const size_t qn = (size_t)nq * h->hx.dim, tn = (size_t)nq * h->hx.pq_m * gann::kPivots;
  float* dq = nullptr;
  float* dt = nullptr;
  __nv_bfloat16* db = nullptr;
  cudaStream_t s = h->stream;
  cudaError_t e = cudaMalloc(&dq, qn * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dt, tn * sizeof(float));
  if (e == cudaSuccess && precision != GANN_PREC_FP32) e = cudaMalloc(&db, tn * sizeof(__nv_bfloat16));
  if (e == cudaSuccess) e = cudaMemcpyAsync(dq, queries, qn * sizeof(float), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    if (precision == GANN_PREC_FP32)
      e = gann::launch_table_cc(h->dx, (int)h->hx.dim, h->hx.pq_m, dq, nq, h->fma_table, false, dt, s);
    else if (precision == GANN_PREC_BF16_CC)
      e = gann::launch_table_cc(h->dx, (int)h->hx.dim, h->hx.pq_m, dq, nq, h->fma_table, true, db, s);
    else
      e = gann::launch_table_tc(h->dx, (int)h->hx.dim, h->hx.pq_m, dq, nq, precision == GANN_PREC_BF16X3, db, s,
                                  h->num_sms);
  }
  if (e == cudaSuccess && db) e = gann::widen_bf16(db, dt, tn, s);
  unsigned int err = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(tables, dt, tn * sizeof(float), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&err, h->d_err, sizeof(err), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dq);
  cudaFree(dt);
  if (db) cudaFree(db);
  if (e != cudaSuccess) return set_error(GANN_ECUDA, std::string("gann_pq_tables: ") + cudaGetErrorString(e));
  if (err) {
    cudaMemset(h->d_err, 0, sizeof(unsigned int));
    return kernel_error_status(err);
  }
  return GANN_OK;
}

int gann_autotune(gann_t* h, const float* d_queries, int nq, int topk, int ef_search, int precision,
                  gann_batch_opts_t* best, double* best_seconds) {
  int rc = check_batch_args(h, nq, topk, ef_search);
  if (rc) return rc;
  if (nq < 1 || !d_queries) return set_error(GANN_EINVAL, "autotune needs queries");
  int32_t *d_nns = nullptr, *d_found = nullptr;
  float* d_dists = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaMalloc(&d_nns, sizeof(int32_t) * (size_t)nq * topk);
  if (e == cudaSuccess) e = cudaMalloc(&d_dists, sizeof(float) * (size_t)nq * topk);
  if (e == cudaSuccess) e = cudaMalloc(&d_found, sizeof(int32_t) * (size_t)nq);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  double best_t = 1e30;
  gann_batch_opts_t best_o{};
  int best_delta = 0;
  if (e == cudaSuccess) {
    std::lock_guard<std::mutex> lk(h->mu);
    cudaStream_t s = h->stream;
    const int base_bits = gann::batch_hash_bits(ef_search);
    for (int W : {2, 4, 8, 16}) {
      for (int delta : {-3, -2, -1, 0, 1}) {  // smaller caches trade re-scoring for CTAs per SM
        gann_batch_opts_t o{};
        o.precision = precision;
        o.beam_width = W;
        o.hash_bits = base_bits + delta;
        double t = 1e30;
        bool ok = true;
        for (int rep = 0; rep < 3 && ok; rep++) {
          cudaEventRecord(e0, s);
          ok = enqueue_batch(h, d_queries, nq, nullptr, nullptr, topk, ef_search, &o, d_nns, d_dists, d_found,
                             nullptr, nullptr, s) == GANN_OK;
          cudaEventRecord(e1, s);
          float ms = 0.0f;
          if (ok) ok = cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
          if (ok && rep > 0 && ms * 1e-3 < t) t = ms * 1e-3;  // first run warms caches
        }
        if (ok && t < best_t) {
          best_t = t;
          best_o = o;
          best_delta = delta;
        }
      }
    }
    if (best_t < 1e30) {
      h->tuned_beam = best_o.beam_width;
      h->tuned_hash_delta = best_delta;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(d_nns);
  cudaFree(d_dists);
  cudaFree(d_found);
  if (e != cudaSuccess) return set_error(GANN_ECUDA, std::string("gann_autotune: ") + cudaGetErrorString(e));
  if (best_t >= 1e30) return set_error(GANN_ERANGE, "no configuration could run these sizes");
  if (best) *best = best_o;
  if (best_seconds) *best_seconds = best_t;
  return GANN_OK;
}

/* Synchronise `stream` (NULL = the handle's stream) and report any error word
 * left by kernels launched with gann_search_device; clears it. */
int gann_check(gann_t* h, void* stream) {
  if (!h) return set_error(GANN_EINVAL, "null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
  unsigned int err = 0;
  cudaError_t e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaMemcpy(&err, h->d_err, sizeof(err), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_error(GANN_ECUDA, std::string("gann_check: ") + cudaGetErrorString(e));
  if (err) {
    cudaMemset(h->d_err, 0, sizeof(unsigned int));
    return kernel_error_status(err);
  }
  return GANN_OK;
}

/* Select the FMA behaviour of the plain form at the two reference sites
 * (src/impl/pq.cuh:40 table accumulate, src/impl/util.cuh:37 exact distance).
 * Both default to 1 (fused); tests/golden pins that choice against the
 * reference's own build. */
int gann_set_fma(gann_t* h, int fma_table, int fma_exact) {
  if (!h) return set_error(GANN_EINVAL, "null handle");
  std::lock_guard<std::mutex> lk(h->mu);
  h->fma_table = fma_table ? 1 : 0;
  h->fma_exact = fma_exact ? 1 : 0;
  return GANN_OK;
}

}  // extern "C"

// A batched search on device buffers with a caller-owned counter and tables;
// the query count is read at run time from device memory when nq_dev is set
// (batch_graph.cu).
int gann_internal_enqueue_batch_dev(gann_t* h, const float* d_q, int nq, const int32_t* d_k, const int32_t* d_l,
                                    int k_max, int l_max, const gann_batch_opts_t* opts, int32_t* d_nns,
                                    float* d_dists, int32_t* d_found, cudaStream_t s, int* counter,
                                    __nv_bfloat16* tables, const int* nq_dev, unsigned long long* entry_keys) {
  return enqueue_batch(h, d_q, nq, d_k, d_l, k_max, l_max, opts, d_nns, d_dists, d_found, nullptr, nullptr, s,
                       counter, tables, nq_dev, nullptr, entry_keys);
}

extern "C" int gann_cache_hot_records(gann_t* h, const float* d_queries, int nq, int ef_search, int64_t max_bytes,
                           int64_t* cached_records) {
  if (!h) return set_error(GANN_EINVAL, "null handle");
  if (cached_records) *cached_records = 0;
  if (!h->host_pages) return set_error(GANN_EINVAL, "the records are already in HBM (open with GANN_OPEN_HOST_PAGES)");
  if (nq < 1 || !d_queries) return set_error(GANN_EINVAL, "a sample of at least one device query is needed");
  if (ef_search < 1 || ef_search > 4096) return set_error(GANN_EINVAL, "ef_search must be in 1..4096");
  if (max_bytes < 0) return set_error(GANN_EINVAL, "max_bytes must be >= 0");
  std::lock_guard<std::mutex> lk(h->mu);
  const gann::HostIndex& hx = h->hx;
  const int64_t stride = (hx.node_len + 15) / 16 * 16;
  const int64_t slots = std::min<int64_t>(hx.n, std::min<int64_t>(max_bytes / stride, INT32_MAX));
  int32_t* d_count = nullptr;
  int32_t* d_nns = nullptr;
  float* d_dists = nullptr;
  int32_t* d_found = nullptr;
  auto release = [&]() {
    for (void* p : {(void*)d_count, (void*)d_nns, (void*)d_dists, (void*)d_found})
      if (p) cudaFree(p);
  };
  auto fail = [&](int code, const std::string& m) {
    release();
    return set_error(code, m);
  };
  // 1. expansion counts of a sample batch (the batched walk, BF16 tensor-core
  //    tables where available, counting each expanded node).
  cudaError_t e = cudaMalloc(&d_count, sizeof(int32_t) * hx.n);
  if (e == cudaSuccess) e = cudaMalloc(&d_nns, sizeof(int32_t) * nq);
  if (e == cudaSuccess) e = cudaMalloc(&d_dists, sizeof(float) * nq);
  if (e == cudaSuccess) e = cudaMalloc(&d_found, sizeof(int32_t) * nq);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_count, 0, sizeof(int32_t) * hx.n, h->stream);
  if (e != cudaSuccess) return fail(GANN_ENOMEM, "record cache: sample buffers");
  gann_batch_opts_t o{};
  o.precision = h->dx.tc_bpanel_hi ? GANN_PREC_BF16 : GANN_PREC_BF16_CC;
  const int rc = enqueue_batch(h, d_queries, nq, nullptr, nullptr, 1, ef_search, &o, d_nns, d_dists, d_found,
                               nullptr, nullptr, h->stream, nullptr, nullptr, nullptr, d_count);
  if (rc != GANN_OK) return fail(rc, g_last_error);
  std::vector<int32_t> count((size_t)hx.n);
  e = cudaMemcpyAsync(count.data(), d_count, sizeof(int32_t) * hx.n, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(GANN_ECUDA, std::string("record cache: sample run: ") + cudaGetErrorString(e));
  release();
  // 2. the hottest records, most expansions first (ties by id), up to the budget
  std::vector<int32_t> ids;
  for (int64_t u = 0; u < hx.n; u++)
    if (count[u] > 0) ids.push_back((int32_t)u);
  auto hotter = [&](int32_t a, int32_t b) { return count[a] > count[b] || (count[a] == count[b] && a < b); };
  if ((int64_t)ids.size() > slots) {
    std::nth_element(ids.begin(), ids.begin() + slots, ids.end(), hotter);
    ids.resize(slots);
  }
  std::sort(ids.begin(), ids.end(), hotter);
  // 3. copy them (verbatim, from the pinned page body) and the id -> slot map to HBM
  std::vector<int32_t> remap((size_t)hx.n, -1);
  std::vector<uint8_t> cache((size_t)ids.size() * stride, 0);
  for (size_t i = 0; i < ids.size(); i++) {
    const int64_t u = ids[i];
    std::memcpy(&cache[i * stride], h->host_pages + (u / hx.npp) * gann::kPageSize + (u % hx.npp) * hx.node_len,
                (size_t)hx.node_len);
    remap[u] = (int32_t)i;
  }
  try {
    // drop an earlier cache first (its two allocations are the last ones made)
    if (h->dx.rec_remap) {
      for (const void* p : {(const void*)h->dx.rec_remap, (const void*)h->dx.rec_cache}) {
        auto it = std::find(h->allocations.begin(), h->allocations.end(), p);
        if (it != h->allocations.end()) {
          cudaFree(*it);
          h->allocations.erase(it);
        }
      }
      h->device_bytes -= (int64_t)sizeof(int32_t) * hx.n + h->rec_cache_bytes;
      h->dx.rec_remap = nullptr;
      h->dx.rec_cache = nullptr;
      h->rec_cache_bytes = 0;
    }
    if (ids.empty()) return GANN_OK;
    uint8_t* d_cache = upload(h, cache);
    int32_t* d_remap = upload(h, remap);
    h->dx.rec_cache = d_cache;
    h->dx.rec_remap = d_remap;
    h->dx.rec_stride = stride;
    h->rec_cache_bytes = (int64_t)cache.size();
  } catch (const CudaFail& ce) {
    return set_error(ce.e == cudaErrorMemoryAllocation ? GANN_ENOMEM : GANN_ECUDA,
                     std::string("record cache: ") + ce.what + ": " + cudaGetErrorString(ce.e));
  }
  if (cached_records) *cached_records = (int64_t)ids.size();
  return GANN_OK;
}
