// Batched search that allocates no device memory: gann_search_batch_noalloc.
//
// Who needs it: callers that must not call cudaMalloc while they serve
// queries -- a latency-critical serving loop, where a cudaMalloc can
// synchronise the device and take the driver's allocation lock in the middle of
// other work, and host programs whose own memory manager owns every device
// allocation after start-up. gann_search_batch_device grows its BF16 table
// buffer with cudaMalloc on a larger batch than before; this variant instead
// keeps the per-call scratch (the work counter and the BF16 tables of up to
// kNoAllocMaxQueries queries with at most kNoAllocMaxChunks PQ chunks) in the
// fixed array below.
//
// The array is part of the library image: every GPU that loads libgann holds
// its 8 MiB + 256 B until the process exits. All calls on a device share it and
// find the previous call's contents in it, so each call clears the work
// counter before its kernels run; calls whose kernels overlap on the GPU (two
// streams, or two handles on one device) race on it and must be serialised by
// the caller. Only the tensor-core precisions use the table region, so only
// they are limited to kNoAllocMaxQueries queries per call. Every call looks up
// the array's device address (cudaGetSymbolAddress, with the handle's device
// current; it allocates nothing), so an address never outlives the context it
// came from. The first call on a device may load the library's device code;
// make that first call before any stream capture.
#include <mutex>
#include <string>

#include "gann_internal.h"

namespace gann {
namespace {

constexpr int kNoAllocMaxQueries = 512;
constexpr int kNoAllocMaxChunks = 32;
constexpr size_t kNoAllocHeader = 256;  // work counter at offset 0
constexpr size_t kNoAllocBytes =
    kNoAllocHeader + (size_t)kNoAllocMaxQueries * kNoAllocMaxChunks * kPivots * sizeof(__nv_bfloat16);

static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocBytes];

// Device address of the scratch array on the current device.
cudaError_t scratch_address(void** out) { return cudaGetSymbolAddress(out, g_noalloc_scratch); }

}  // namespace
}  // namespace gann

// Defined in gann_api.cu: records a message for gann_last_error().
int gann_internal_set_error(int code, const char* msg);

extern "C" int gann_search_batch_noalloc(gann_t* h, const float* d_queries, int nq, int topk, int ef_search,
                                         const gann_batch_opts_t* opts, int32_t* d_nns, float* d_distances,
                                         int32_t* d_found_cnt, void* stream) {
  using namespace gann;
  if (!h) return gann_internal_set_error(GANN_EINVAL, "null handle");
  if (nq < 0 || topk < 1 || ef_search < 1) return gann_internal_set_error(GANN_EINVAL, "bad nq / topk / ef_search");
  if (topk > 4096 || ef_search > 4096) return gann_internal_set_error(GANN_ERANGE, "topk and ef_search are limited to 4096");
  if (nq == 0) return GANN_OK;
  if (!d_queries || !d_nns || !d_distances || !d_found_cnt) return gann_internal_set_error(GANN_EINVAL, "null buffer");
  gann_batch_opts_t o{};
  if (opts) o = *opts;
  const int prec = opts ? o.precision : GANN_PREC_BF16X3;
  std::lock_guard<std::mutex> lk(h->mu);
  // The same defaults as gann_search_batch_device: the handle's tuned beam
  // width and visited-cache delta (gann_autotune) when the options leave 0.
  const int W = o.beam_width ? o.beam_width : (h->tuned_beam ? h->tuned_beam : 4);
  if (!(W == 1 || W == 2 || W == 4 || W == 8 || W == 16))
    return gann_internal_set_error(GANN_EINVAL, "beam_width must be 1, 2, 4, 8 or 16");
  if (prec < GANN_PREC_FP32 || prec > GANN_PREC_BF16_CC) return gann_internal_set_error(GANN_EINVAL, "unknown precision");
  if (o.entry != GANN_ENTRY_NAV_WALK)
    return gann_internal_set_error(GANN_EINVAL, "gann_search_batch_noalloc enters by the pivot-graph walk only");
  const bool tc = prec == GANN_PREC_BF16 || prec == GANN_PREC_BF16X3;
  if (tc && nq > kNoAllocMaxQueries)
    return gann_internal_set_error(GANN_ERANGE,
                                   "gann_search_batch_noalloc: at most 512 queries per call with tensor-core tables");
  if (tc && h->hx.pq_m > kNoAllocMaxChunks)
    return gann_internal_set_error(GANN_ERANGE, "gann_search_batch_noalloc: at most 32 PQ chunks with tensor-core tables");
  if (tc && !h->dx.tc_bpanel_hi)
    return gann_internal_set_error(GANN_ERANGE, "tensor-core tables need PQ chunks of at most 16 dimensions");
  const int hb = o.hash_bits ? o.hash_bits : batch_hash_bits(ef_search) + h->tuned_hash_delta;
  if (hb < 4 || hb > 16) return gann_internal_set_error(GANN_EINVAL, "hash_bits must be in 4..16");
  if (batch_smem_bytes(h->hx.pq_m, tc || prec == GANN_PREC_BF16_CC ? 2 : 4, hb, ef_search, (int)h->hx.max_m0, W,
                       topk, (int)h->hx.dim) > 227 * 1024)
    return gann_internal_set_error(GANN_ERANGE, "table + lists + visited cache of one query exceed 227 KB of shared memory");

  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return gann_internal_set_error(GANN_ECUDA, "cudaGetDevice failed");
  if (prev != h->device && cudaSetDevice(h->device) != cudaSuccess)
    return gann_internal_set_error(GANN_ECUDA, "cannot make the handle's device current");
  void* base = nullptr;
  cudaError_t e = scratch_address(&base);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;
  int* counter = static_cast<int*>(base);
  __nv_bfloat16* tables = reinterpret_cast<__nv_bfloat16*>(static_cast<uint8_t*>(base) + kNoAllocHeader);
  if (e == cudaSuccess) e = cudaMemsetAsync(counter, 0, sizeof(int), s);  // the previous call left its count
  if (e == cudaSuccess && tc)
    e = launch_table_tc(h->dx, (int)h->hx.dim, h->hx.pq_m, d_queries, nq, prec == GANN_PREC_BF16X3, tables, s,
                         h->num_sms);
  if (e == cudaSuccess) {
    BatchParams p{};
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
    p.queries = d_queries;
    p.nq = nq;
    p.L_max = ef_search;
    p.k_max = topk;
    p.hash_bits = hb;
    p.npp_div = gann::FastDiv((uint32_t)h->hx.npp);
    p.tables = tc ? tables : nullptr;
    p.fma = h->fma_exact;
    p.nns = d_nns;
    p.dists = d_distances;
    p.found = d_found_cnt;
    p.next_query = counter;
    p.err = h->d_err;
    e = launch_batch(p, h->hx.dtype, prec != GANN_PREC_FP32, W, h->num_sms, s);
  }
  if (prev >= 0 && prev != h->device) cudaSetDevice(prev);
  if (e != cudaSuccess)
    return gann_internal_set_error(GANN_ECUDA, (std::string("gann_search_batch_noalloc: ") + cudaGetErrorString(e)).c_str());
  return GANN_OK;
}
