// Batched search captured once as a CUDA graph and replayed.
//
// The graph holds the whole batch: the work-counter reset, the tensor-core
// table build, the nearest-pivot entry search when the options ask for it,
// and the persistent walk, whose CTAs pull query indices from the
// counter. Buffers are fixed at capture; the number of queries of a launch is
// read by the kernels from device memory, so one graph serves every batch size
// up to its maximum and a producer on the device or the host only has to write
// the count (and the queries) before each launch. The reference launches its
// kernels once per search call (src/pure_mem.cu:101-184) and has no counterpart.
#include <string>

#include "gann_internal.h"

int gann_internal_set_error(int code, const char* msg);
int gann_internal_enqueue_batch_dev(gann_t* h, const float* d_q, int nq, const int32_t* d_k, const int32_t* d_l,
                                    int k_max, int l_max, const gann_batch_opts_t* opts, int32_t* d_nns,
                                    float* d_dists, int32_t* d_found, cudaStream_t s, int* counter,
                                    __nv_bfloat16* tables, const int* nq_dev, unsigned long long* entry_keys);

struct gann_batch_graph {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int* counter = nullptr;
  __nv_bfloat16* tables = nullptr;
  unsigned long long* entry_keys = nullptr;  // nearest-pivot keys (GANN_ENTRY_NEAREST_PIVOT)
};

namespace {

void release(gann_batch_graph* g) {
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  if (g->counter) cudaFree(g->counter);
  if (g->tables) cudaFree(g->tables);
  if (g->entry_keys) cudaFree(g->entry_keys);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

int cuda_error(const char* what, cudaError_t e) {
  return gann_internal_set_error(e == cudaErrorMemoryAllocation ? GANN_ENOMEM : GANN_ECUDA,
                                 (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}

}  // namespace

extern "C" {

int gann_batch_graph_create(gann_t* h, int max_nq, int topk_max, int ef_max, const gann_batch_opts_t* opts,
                            const float* d_queries, const int32_t* d_topk, const int32_t* d_ef_search,
                            const int32_t* d_nq, int32_t* d_nns, float* d_distances, int32_t* d_found_cnt,
                            gann_batch_graph_t** out) {
  if (!h || !out) return gann_internal_set_error(GANN_EINVAL, "null argument");
  *out = nullptr;
  if (max_nq < 1) return gann_internal_set_error(GANN_EINVAL, "max_nq must be >= 1");
  if (topk_max < 1 || ef_max < 1) return gann_internal_set_error(GANN_EINVAL, "topk_max and ef_max must be >= 1");
  if (topk_max > 4096 || ef_max > 4096)
    return gann_internal_set_error(GANN_ERANGE, "topk and ef_search are limited to 4096");
  if (!d_queries || !d_nq || !d_nns || !d_distances || !d_found_cnt)
    return gann_internal_set_error(GANN_EINVAL, "null buffer");
  const int prec = opts ? opts->precision : GANN_PREC_BF16X3;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(h->device);
  auto* g = new gann_batch_graph();
  g->device = h->device;
  int rc = GANN_OK;
  cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&g->counter, sizeof(int));
  if (e == cudaSuccess && (prec == GANN_PREC_BF16 || prec == GANN_PREC_BF16X3))
    e = cudaMalloc(&g->tables, sizeof(__nv_bfloat16) * (size_t)max_nq * h->hx.pq_m * gann::kPivots);
  if (e == cudaSuccess && opts && opts->entry == GANN_ENTRY_NEAREST_PIVOT)
    e = cudaMalloc(&g->entry_keys, sizeof(unsigned long long) * (size_t)max_nq);
  if (e != cudaSuccess) {
    rc = cuda_error("batch graph buffers", e);
  } else {
    std::lock_guard<std::mutex> lk(h->mu);
    e = cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) {
      rc = cuda_error("stream capture", e);
    } else {
      rc = gann_internal_enqueue_batch_dev(h, d_queries, max_nq, d_topk, d_ef_search, topk_max, ef_max, opts,
                                           d_nns, d_distances, d_found_cnt, g->stream, g->counter, g->tables,
                                           d_nq, g->entry_keys);
      const cudaError_t ee = cudaStreamEndCapture(g->stream, &g->graph);
      if (rc == GANN_OK && ee != cudaSuccess) rc = cuda_error("stream capture", ee);
    }
  }
  if (rc == GANN_OK) {
    e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (e != cudaSuccess) rc = cuda_error("graph instantiate", e);
  }
  if (prev >= 0) cudaSetDevice(prev);
  if (rc != GANN_OK) {
    release(g);
    return rc;
  }
  *out = g;
  return GANN_OK;
}

int gann_batch_graph_launch(gann_batch_graph_t* g, void* stream) {
  if (!g) return gann_internal_set_error(GANN_EINVAL, "null graph");
  const cudaError_t e = cudaGraphLaunch(g->exec, stream ? static_cast<cudaStream_t>(stream) : g->stream);
  return e == cudaSuccess ? GANN_OK : cuda_error("graph launch", e);
}

int gann_batch_graph_destroy(gann_batch_graph_t* g) {
  if (!g) return GANN_OK;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(g->device);
  cudaDeviceSynchronize();  // a replay may run on a caller's stream
  release(g);
  if (prev >= 0) cudaSetDevice(prev);
  return GANN_OK;
}

}  // extern "C"
