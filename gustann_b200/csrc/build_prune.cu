// RobustPrune for the index builder, on the GPU: gann_build_prune.
//
// The reference builds its graphs with DiskANN (scripts/build_diskann_index.sh:7),
// whose Vamana keeps, for each point p, candidates in order of distance and
// drops every candidate c that a kept neighbour j occludes. DiskANN is an empty
// submodule in the reference, so the builder restates the rule: with squared
// L2 distances, c is dropped when alpha * d(j, c) < d(p, c), at most R
// neighbours are kept, in distance order.
//
// One warp per row. The row's candidates (ids, -1 = none; duplicates, the point
// itself and ids outside [0, n) are dropped) and the point's own vector are
// staged in shared memory, one padded row each. Each lane scores its
// candidates against the point, the candidates are ranked by (distance, id),
// and the keep/occlude pass walks them in that order; every lane re-checks its
// own candidates against each kept one. uint8 vectors are compared with
// byte-wise |a - b| and a 4-way dot product (exact in int32), rows at an odd
// word stride so that lanes reading different rows at the same word hit
// different banks. Float vectors of a dimension divisible by 4 are compared
// as |a|^2 + |b|^2 - 2 a.b in FP32 with 16-byte shared-memory loads (rows at a
// stride of dim + 4 words, norms computed once per row); other float rows by
// their differences.
#include <cuda_runtime.h>

#include <cstdint>

#include "gann_internal.h"

namespace gann {
namespace {

constexpr int kPruneMaxK = 128;
constexpr unsigned kAll = 0xffffffffu;

struct PruneArgs {
  const uint8_t* x;  // n x dim elements of T
  int64_t n;
  int dim;
  int row_words;     // 32-bit words of one vector (uint8: ceil(dim / 4), float: dim)
  int stride;        // row stride in shared memory, in words (odd)
  const int32_t* rows;  // n_rows point ids, or null (row r is point r)
  const int32_t* cand;  // n_rows x K candidate ids
  int64_t n_rows;
  int K, R;
  float alpha;
  int wpb;           // warps per block
  int warp_words;    // shared-memory words per warp
  int vec4;          // float rows compared through norms and 16-byte loads
  int32_t* out;      // n_rows x R, -1 padded
};

// Squared L2 between two staged rows (na, nb: their squared norms, used by the
// vec4 float form only).
template <class T>
__device__ __forceinline__ float row_dist(const uint32_t* a, const uint32_t* b, int words, float na, float nb,
                                          bool vec4);

// Squared norm of a staged float row (vec4 form).
__device__ __forceinline__ float row_norm(const uint32_t* a, int words) {
  const float4* x = reinterpret_cast<const float4*>(a);
  float acc = 0.0f;
  for (int w = 0; w < words / 4; w++) {
    const float4 v = x[w];
    acc = fmaf(v.x, v.x, acc);
    acc = fmaf(v.y, v.y, acc);
    acc = fmaf(v.z, v.z, acc);
    acc = fmaf(v.w, v.w, acc);
  }
  return acc;
}

template <>
__device__ __forceinline__ float row_dist<uint8_t>(const uint32_t* a, const uint32_t* b, int words, float, float,
                                                   bool) {
  unsigned acc = 0;
  for (int w = 0; w < words; w++) {
    const unsigned d = __vabsdiffu4(a[w], b[w]);
    acc = __dp4a(d, d, acc);
  }
  return (float)acc;  // <= dim * 255^2, exact in FP32 for dim <= 258
}

template <>
__device__ __forceinline__ float row_dist<float>(const uint32_t* a, const uint32_t* b, int words, float na, float nb,
                                                 bool vec4) {
  if (vec4) {
    const float4* x = reinterpret_cast<const float4*>(a);
    const float4* y = reinterpret_cast<const float4*>(b);
    float d0 = 0.0f, d1 = 0.0f;
    int w = 0;
    for (; w + 1 < words / 4; w += 2) {
      const float4 p0 = x[w], q0 = y[w], p1 = x[w + 1], q1 = y[w + 1];
      d0 = fmaf(p0.x, q0.x, d0);
      d0 = fmaf(p0.y, q0.y, d0);
      d0 = fmaf(p0.z, q0.z, d0);
      d0 = fmaf(p0.w, q0.w, d0);
      d1 = fmaf(p1.x, q1.x, d1);
      d1 = fmaf(p1.y, q1.y, d1);
      d1 = fmaf(p1.z, q1.z, d1);
      d1 = fmaf(p1.w, q1.w, d1);
    }
    if (w < words / 4) {
      const float4 p0 = x[w], q0 = y[w];
      d0 = fmaf(p0.x, q0.x, d0);
      d0 = fmaf(p0.y, q0.y, d0);
      d0 = fmaf(p0.z, q0.z, d0);
      d0 = fmaf(p0.w, q0.w, d0);
    }
    return fmaxf(na + nb - 2.0f * (d0 + d1), 0.0f);
  }
  float acc = 0.0f;
  for (int w = 0; w < words; w++) {
    const float d = __uint_as_float(a[w]) - __uint_as_float(b[w]);
    acc = fmaf(d, d, acc);
  }
  return acc;
}

// Copy vector `id` into shared-memory row `dst` (row_words words, zero padded).
// One lane copies the whole row.
template <class T>
__device__ __forceinline__ void stage_row(const PruneArgs& a, int64_t id, uint32_t* dst) {
  const size_t bytes = (size_t)a.dim * sizeof(T);
  const uint8_t* src = a.x + (size_t)id * bytes;
  if ((bytes & 15) == 0 && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
    const uint4* s4 = reinterpret_cast<const uint4*>(src);
    for (int i = 0; i < (int)(bytes >> 4); i++) {
      const uint4 v = __ldg(s4 + i);
      dst[4 * i] = v.x;
      dst[4 * i + 1] = v.y;
      dst[4 * i + 2] = v.z;
      dst[4 * i + 3] = v.w;
    }
  } else {
    for (int w = 0; w < a.row_words; w++) {
      uint32_t v = 0;
      for (int b = 0; b < 4; b++) {
        const size_t o = (size_t)w * 4 + b;
        if (o < bytes) v |= (uint32_t)__ldg(src + o) << (8 * b);
      }
      dst[w] = v;
    }
  }
}

template <class T, int KP>
__global__ void __launch_bounds__(256) prune_kernel(PruneArgs a) {
  extern __shared__ __align__(16) uint32_t psm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * a.wpb + warp;
  if (row >= a.n_rows) return;  // the whole warp leaves together
  const int K = a.K, R = a.R;
  uint32_t* vecs = psm + (size_t)warp * a.warp_words;  // (K + 1) rows; row K is the point
  int32_t* order = reinterpret_cast<int32_t*>(vecs + (size_t)(K + 1) * a.stride);  // sorted -> slot
  float* sd = reinterpret_cast<float*>(order + kPruneMaxK);                         // sorted distances
  int32_t* sid = reinterpret_cast<int32_t*>(sd + kPruneMaxK);                       // sorted ids
  float* nrm = reinterpret_cast<float*>(sid + kPruneMaxK);                          // row norms (vec4 form)
  const bool vec4 = a.vec4 != 0;
  const int64_t p = a.rows ? (int64_t)__ldg(a.rows + row) : row;
  int32_t* out = a.out + row * R;
  if (p < 0 || p >= a.n) {  // no such point: an empty row
    for (int c = lane; c < R; c += 32) out[c] = -1;
    return;
  }
  int cid[KP];
  bool cv[KP];
#pragma unroll
  for (int t = 0; t < KP; t++) {
    const int s = lane + 32 * t;
    cid[t] = s < K ? __ldg(a.cand + row * K + s) : -1;
    cv[t] = s < K && cid[t] >= 0 && cid[t] < a.n && cid[t] != p;
  }
  // stage: lane s % 32 copies slot s (slot K = the point)
#pragma unroll
  for (int t = 0; t < KP; t++)
    if (cv[t]) stage_row<T>(a, cid[t], vecs + (size_t)(lane + 32 * t) * a.stride);
  if (lane == (K & 31)) stage_row<T>(a, p, vecs + (size_t)K * a.stride);
  __syncwarp();
  if (vec4) {
#pragma unroll
    for (int t = 0; t < KP; t++)
      if (cv[t]) nrm[lane + 32 * t] = row_norm(vecs + (size_t)(lane + 32 * t) * a.stride, a.row_words);
    if (lane == (K & 31)) nrm[K] = row_norm(vecs + (size_t)K * a.stride, a.row_words);
    __syncwarp();
  }
  const uint32_t* vp = vecs + (size_t)K * a.stride;
  const float np_ = vec4 ? nrm[K] : 0.0f;
  float d[KP];
#pragma unroll
  for (int t = 0; t < KP; t++)
    d[t] = cv[t] ? row_dist<T>(vecs + (size_t)(lane + 32 * t) * a.stride, vp, a.row_words,
                               vec4 ? nrm[lane + 32 * t] : 0.0f, np_, vec4)
                 : __int_as_float(0x7f800000);
  // rank by (distance, id, slot): a repeated id gets consecutive ranks
  int rank[KP];
#pragma unroll
  for (int t = 0; t < KP; t++) rank[t] = 0;
#pragma unroll
  for (int t2 = 0; t2 < KP; t2++) {
    for (int j = 0; j < 32; j++) {
      const float od = __shfl_sync(kAll, d[t2], j);
      const int oi = __shfl_sync(kAll, cid[t2], j);
      const bool ov = __shfl_sync(kAll, (int)cv[t2], j) != 0;
      const int os = j + 32 * t2;
#pragma unroll
      for (int t = 0; t < KP; t++) {
        const int s = lane + 32 * t;
        rank[t] += ov && (od < d[t] || (od == d[t] && (oi < cid[t] || (oi == cid[t] && os < s))));
      }
    }
  }
  int nvalid = 0;
#pragma unroll
  for (int t = 0; t < KP; t++) nvalid += __popc(__ballot_sync(kAll, cv[t]));
#pragma unroll
  for (int t = 0; t < KP; t++) {
    if (cv[t]) {
      order[rank[t]] = lane + 32 * t;
      sd[rank[t]] = d[t];
      sid[rank[t]] = cid[t];
    }
  }
  __syncwarp();
  // alive flags in sorted order; a repeated id keeps its first copy only
  bool al[KP];
#pragma unroll
  for (int t = 0; t < KP; t++) {
    const int pos = lane + 32 * t;
    al[t] = pos < nvalid && !(pos > 0 && sid[pos] == sid[pos - 1]);
  }
  int count = 0;
  for (int j = 0; j < nvalid && count < R; j++) {
    bool aj = false;
#pragma unroll
    for (int t = 0; t < KP; t++) {
      const bool v = __shfl_sync(kAll, (int)al[t], j & 31) != 0;
      if (t == (j >> 5)) aj = v;
    }
    if (!aj) continue;
    if (lane == 0) out[count] = sid[j];
    count++;
    if (count == R) break;
    const uint32_t* vj = vecs + (size_t)order[j] * a.stride;
    const float nj = vec4 ? nrm[order[j]] : 0.0f;
#pragma unroll
    for (int t = 0; t < KP; t++) {
      const int pos = lane + 32 * t;
      if (al[t] && pos > j) {
        const int oc = order[pos];
        const float djc = row_dist<T>(vj, vecs + (size_t)oc * a.stride, a.row_words, nj, vec4 ? nrm[oc] : 0.0f,
                                      vec4);
        if (a.alpha * djc < sd[pos]) al[t] = false;
      }
    }
  }
  for (int c = count + lane; c < R; c += 32) out[c] = -1;
}

template <class T, int KP>
cudaError_t launch_prune(PruneArgs a, cudaStream_t s) {
  if (!a.x || !a.cand || !a.out) return cudaErrorInvalidValue;
  const size_t per_warp = (size_t)a.warp_words * 4;
  int wpb = (int)((160 * 1024) / per_warp);
  wpb = wpb < 1 ? 1 : (wpb > 8 ? 8 : wpb);
  a.wpb = wpb;
  const size_t smem = per_warp * wpb;
  if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  auto kern = prune_kernel<T, KP>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int64_t blocks = (a.n_rows + wpb - 1) / wpb;
  if (blocks > INT32_MAX) return cudaErrorInvalidConfiguration;
  kern<<<(unsigned)blocks, wpb * 32, smem, s>>>(a);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_prune_t(const PruneArgs& a, cudaStream_t s) {
  const int kp = (a.K + 31) / 32;
  switch (kp) {
    case 1: return launch_prune<T, 1>(a, s);
    case 2: return launch_prune<T, 2>(a, s);
    case 3: return launch_prune<T, 3>(a, s);
    default: return launch_prune<T, 4>(a, s);
  }
}

}  // namespace
}  // namespace gann

int gann_internal_set_error(int code, const char* msg);

extern "C" int gann_build_prune(const void* d_x, int dtype, int64_t n, int dim, const int32_t* d_rows,
                                const int32_t* d_cand, int64_t n_rows, int K, int R, float alpha, int32_t* d_out,
                                void* stream) {
  using namespace gann;
  if (!d_x || !d_cand || !d_out || n < 1 || n > INT32_MAX || dim < 1 || n_rows < 0)
    return gann_internal_set_error(GANN_EINVAL, "gann_build_prune: bad arguments");
  if (K < 1 || K > kPruneMaxK || R < 1) return gann_internal_set_error(GANN_ERANGE, "gann_build_prune: K must be 1..128, R >= 1");
  if (dtype != GANN_UINT8 && dtype != GANN_FLOAT) return gann_internal_set_error(GANN_EINVAL, "gann_build_prune: dtype");
  if (dtype == GANN_UINT8 && dim > 258) return gann_internal_set_error(GANN_ERANGE, "gann_build_prune: uint8 dim > 258");
  if (n_rows == 0) return GANN_OK;
  PruneArgs a{};
  a.x = static_cast<const uint8_t*>(d_x);
  a.n = n;
  a.dim = dim;
  a.row_words = dtype == GANN_UINT8 ? (dim + 3) / 4 : dim;
  a.vec4 = dtype == GANN_FLOAT && dim % 4 == 0;
  a.stride = a.vec4 ? dim + 4 : (a.row_words | 1);  // 16-byte rows for the vec4 form, else an odd stride
  a.rows = d_rows;
  a.cand = d_cand;
  a.n_rows = n_rows;
  a.K = K;
  a.R = R;
  a.alpha = alpha;
  a.warp_words = (K + 1) * a.stride + 3 * kPruneMaxK + 4 * ((kPruneMaxK + 1 + 3) / 4);  // + norms; a multiple of 4
  a.out = d_out;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const cudaError_t e = dtype == GANN_UINT8 ? launch_prune_t<uint8_t>(a, s) : launch_prune_t<float>(a, s);
  if (e != cudaSuccess)
    return gann_internal_set_error(GANN_ECUDA, (std::string("gann_build_prune: ") + cudaGetErrorString(e)).c_str());
  return GANN_OK;
}
