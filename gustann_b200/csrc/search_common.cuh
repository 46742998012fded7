// Device building blocks shared by the plain and batched search kernels:
// exact distance, key order, pivot-graph entry walk, FP32 table build, ADC and
// top-k insertion, each restating the reference routine it cites.
#pragma once

#include <cuda_bf16.h>

#include "gann_internal.h"

namespace gann {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kNavL = 4;   // nav.cuh:11
constexpr int kNavR = 28;  // nav.cuh:12
constexpr int kHopCap = 1 << 20;
constexpr int kNavIterCap = 1 << 16;

__device__ __forceinline__ float inf_f() { return __int_as_float(0x7f800000); }

template <class T>
__device__ __forceinline__ float load_elem(const T* p, int i);
template <>
__device__ __forceinline__ float load_elem<uint8_t>(const uint8_t* p, int i) {
  return (float)__ldg(p + i);
}
template <>
__device__ __forceinline__ float load_elem<float>(const float* p, int i) {
  return __ldg(p + i);
}

// square_sum_32 (src/impl/util.cuh:26-46): lane-strided accumulation, then a
// __shfl_down_sync tree 16,8,4,2,1; lane 0's value is the result.
template <class T>
__device__ __forceinline__ float warp_exact(const float* q, const T* v, int dim, int lane, int fma) {
  float acc = 0.0f;
  for (int i = lane; i < dim; i += 32) {
    float d = __fsub_rn(q[i], load_elem<T>(v, i));
    acc = fma ? __fmaf_rn(d, d, acc) : __fadd_rn(acc, __fmul_rn(d, d));
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc = __fadd_rn(acc, __shfl_down_sync(kFull, acc, off));
  return __shfl_sync(kFull, acc, 0);
}

// lower_bound on the key (dist, id & 0x7fffffff), src/impl/util.cuh:166-178.
__device__ __forceinline__ int lower_bound_key(const float* dist, const uint32_t* id, int l, int r, float d,
                                               uint32_t x) {
  x &= kMask;
  while (l < r) {
    int mid = (l + r) >> 1;
    float md = dist[mid];
    if (md < d || (md == d && (id[mid] & kMask) < x))
      l = mid + 1;
    else
      r = mid;
  }
  return l;
}

__device__ __forceinline__ bool key_less(float a, uint32_t ai, float b, uint32_t bi) {
  return a < b || (a == b && (ai & kMask) < (bi & kMask));
}

// Pivot graph as the entry walk sees it.
struct NavView {
  const uint8_t* data;    // nav_n x dim x elt
  const int32_t* graph;   // nav_n x max_m, -1 padded
  const int32_t* map;     // nav_n global ids (map.txt)
  int n, max_m, start, dim, fma;
  unsigned int* err;
};

// get_entry_kernel_inner (src/impl/nav.cuh:13-135) for one query, one list
// slot per lane. Returns the pivot graph's local id, or -1 after setting an
// error bit. `gathered` accumulates the algorithmic bytes read.
template <class T>
__device__ int nav_entry(const NavView& nv, const float* q, int lane, int64_t& gathered) {
  const T* nd = reinterpret_cast<const T*>(nv.data);
  const int dim = nv.dim;
  const int64_t glen = (int64_t)nv.n * nv.max_m;
  float d0 = warp_exact<T>(q, nd + (size_t)nv.start * dim, dim, lane, nv.fma);
  const int vec_bytes = dim * (int)sizeof(T);
  gathered += vec_bytes;
  uint32_t my_id = lane == 0 ? (uint32_t)nv.start : 0xffffffffu;  // nav.cuh:50-57
  float my_d = lane == 0 ? d0 : inf_f();
  int idx = 0, iters = 0;
  while (idx != -1) {
    if (++iters > kNavIterCap) {
      if (lane == 0) atomicOr(nv.err, kErrNavCap);
      return -1;
    }
    uint32_t u = __shfl_sync(kFull, my_id, idx);  // nav.cuh:62-68
    if (lane == idx) my_id |= kExpanded;
    // 28 slots of the flat row (nav.cuh:69-72); past the array end reads as -1.
    int v = -1;
    if (lane < kNavR) {
      int64_t e = (int64_t)nv.max_m * u + lane;
      v = e < glen ? __ldg(nv.graph + e) : -1;
    }
    unsigned neg = __ballot_sync(kFull, lane < kNavR && v == -1);
    int deg = neg ? __ffs(neg) - 1 : kNavR;
    // row slots read up to and including the first -1, plus one vector per neighbour
    gathered += 4 * (deg < kNavR ? deg + 1 : kNavR) + (int64_t)deg * vec_bytes;
    for (int i = 0; i < deg; i++) {  // nav.cuh:70-81
      int vi = __shfl_sync(kFull, v, i);
      if ((unsigned)vi >= (unsigned)nv.n) {
        if (lane == 0) atomicOr(nv.err, kErrBadId);
        return -1;
      }
      float di = warp_exact<T>(q, nd + (size_t)vi * dim, dim, lane, nv.fma);
      if (lane == i + kNavL) {
        my_id = (uint32_t)vi;
        my_d = di;
      }
    }
#pragma unroll
    for (int i = 0; i < kNavL; i++) {  // nav.cuh:84-119
      uint32_t prev = __shfl_sync(kFull, my_id, i > 0 ? i - 1 : 0);
      float dist = my_d;
      int pos = lane;
      bool kill = false;
      if (lane < i)
        dist = inf_f();
      else if (i != 0 && ((my_id ^ prev) & kMask) == 0)
        kill = true;
      // Several lanes store prev|own_id to slot i-1 at once in the reference;
      // the OR of all of them is taken here.
      unsigned orv = __reduce_or_sync(kFull, kill ? my_id : 0u);
      unsigned any = __ballot_sync(kFull, kill);
      if (kill) {
        dist = inf_f();
        my_d = inf_f();
      }
      if (any && lane == i - 1) my_id = prev | orv;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        float od = __shfl_down_sync(kFull, dist, off);
        int op = __shfl_down_sync(kFull, pos, off);
        if (od < dist) {
          dist = od;
          pos = op;
        }
      }
      int bp = __shfl_sync(kFull, pos, 0);
      float di = __shfl_sync(kFull, my_d, i), dp = __shfl_sync(kFull, my_d, bp);
      uint32_t ii = __shfl_sync(kFull, my_id, i), ip = __shfl_sync(kFull, my_id, bp);
      if (i != bp && di != dp) {
        if (lane == i) {
          my_d = dp;
          my_id = ip;
        }
        if (lane == bp) {
          my_d = di;
          my_id = ii;
        }
      }
    }
    unsigned un = __ballot_sync(kFull, !(my_id & kExpanded));  // nav.cuh:120-129
    int x = un ? __ffs(un) - 1 : 32;
    idx = x < kNavL ? x : -1;
  }
  return (int)(__shfl_sync(kFull, my_id, 0) & kMask);
}

// Entry node of one query: the pivot-graph walk translated through map.txt
// (src/nav_graph.cu:104-109), or the medoid without a pivot graph
// (src/pure_mem.cu:121-123). Returns -2 on error.
template <class T>
__device__ int64_t entry_node(bool has_nav, const NavView& nv, int64_t medoid, const float* q, int lane,
                              int64_t& gathered) {
  if (!has_nav) return medoid;
  int local = nav_entry<T>(nv, q, lane, gathered);
  if (local >= nv.n) {  // an all-INF slot 0 (fewer than 4 finite candidates)
    if (lane == 0) atomicOr(nv.err, kErrBadId);
    local = -1;
  }
  return local < 0 ? -2 : (int64_t)__ldg(nv.map + local);
}

// PQ data as the table build sees it.
struct PqView {
  const float* pivots_t;    // dim x 256
  const float* centroid;    // dim
  const int32_t* chunk_off; // M + 1
  int M, dim, fma;
};

__device__ __forceinline__ void store_tab(float* t, int i, float v) { t[i] = v; }
__device__ __forceinline__ void store_tab(__nv_bfloat16* t, int i, float v) { t[i] = __float2bfloat16_rn(v); }
__device__ __forceinline__ float load_tab(const float* t, int i) { return t[i]; }
__device__ __forceinline__ float load_tab(const __nv_bfloat16* t, int i) { return __bfloat162float(t[i]); }

// PQSearchData::init_query (src/impl/pq.cuh:8-59): table[c][j] accumulates,
// over the dimensions i of chunk c in increasing order, (q_i - mu_i - P_t[i][j])^2
// in FP32 (stored as TabT). Chunks are contiguous ranges, so each (c, j) is
// accumulated in a register. Chunks are spread over `nworkers` warps; the
// caller synchronises, then calls restore_query.
template <class TabT>
__device__ void build_table(const PqView& pv, TabT* table, const float* q, int worker, int nworkers, int lane) {
  for (int c = worker; c < pv.M; c += nworkers) {
    const int b = __ldg(pv.chunk_off + c), e = __ldg(pv.chunk_off + c + 1);
    float acc[8];
#pragma unroll
    for (int t = 0; t < 8; t++) acc[t] = 0.0f;
    for (int i = b; i < e; i++) {
      const float qc = __fsub_rn(q[i], __ldg(pv.centroid + i));
      const float* pt = pv.pivots_t + (size_t)i * kPivots + lane;
#pragma unroll
      for (int t = 0; t < 8; t++) {
        float d = __fsub_rn(qc, __ldg(pt + 32 * t));
        acc[t] = pv.fma ? __fmaf_rn(d, d, acc[t]) : __fadd_rn(acc[t], __fmul_rn(d, d));
      }
    }
#pragma unroll
    for (int t = 0; t < 8; t++) store_tab(table, c * kPivots + lane + 32 * t, acc[t]);
  }
}

// q_i <- fl(fl(q_i - mu_i) + mu_i), src/impl/pq.cuh:22-24,54-56.
__device__ __forceinline__ void restore_query(const PqView& pv, float* q, int tid, int nthreads) {
  for (int i = tid; i < pv.dim; i += nthreads) {
    const float mu = __ldg(pv.centroid + i);
    q[i] = __fadd_rn(__fsub_rn(q[i], mu), mu);
  }
}

// ADC of one code (src/impl/pure_mem.cuh:302-309): sequential FP32 sum over the chunks.
template <class TabT>
__device__ __forceinline__ float adc(const TabT* table, const uint8_t* code, int M) {
  float d = 0.0f;
  if ((M & 15) == 0) {
    for (int j0 = 0; j0 < M; j0 += 16) {
      uint4 w = __ldg(reinterpret_cast<const uint4*>(code + j0));
      uint32_t words[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int b = 0; b < 16; b++) {
        uint32_t c = (words[b >> 2] >> (8 * (b & 3))) & 0xffu;
        d = __fadd_rn(d, load_tab(table, (j0 + b) * kPivots + c));
      }
    }
  } else {
    for (int j = 0; j < M; j++) d = __fadd_rn(d, load_tab(table, j * kPivots + __ldg(code + j)));
  }
  return d;
}

// adc for M == 32 from the code's two 16-byte words, loaded ahead: the same
// sequential sum in chunk order.
template <class TabT>
__device__ __forceinline__ float adc32_seq(const TabT* table, const uint4& a, const uint4& b) {
  const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
  float d = 0.0f;
#pragma unroll
  for (int j = 0; j < 32; j++) d = __fadd_rn(d, load_tab(table, j * kPivots + ((w[j >> 2] >> (8 * (j & 3))) & 0xffu)));
  return d;
}

// retset_push_32 (src/impl/util.cuh:116-163) by its result: the value goes
// after every entry with distance <= value; the list keeps at most k entries.
__device__ __forceinline__ void topk_push(float* td, int32_t* ti, int& size, int k, float value, int vid,
                                          int lane) {
  int p = 0;
  for (int base = 0; base < size; base += 32) {
    int i = base + lane;
    p += __popc(__ballot_sync(kFull, i < size && td[i] <= value));
  }
  if (p < k) {
    const int last = size < k ? size : k - 1;  // slot of the last entry after the insert
    for (int top = last - 1; top >= p; top -= 32) {
      int i = top - lane;
      bool act = i >= p;
      float dv = 0.0f;
      int32_t iv = 0;
      if (act) {
        dv = td[i];
        iv = ti[i];
      }
      __syncwarp();
      if (act) {
        td[i + 1] = dv;
        ti[i + 1] = iv;
      }
      __syncwarp();
    }
    if (lane == 0) {
      td[p] = value;
      ti[p] = vid;
    }
  }
  if (size < k) size++;
  __syncwarp();
}

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

}  // namespace gann
