// Plain search kernel: the drop-in form of the reference's all-in-GPU path.
//
// One warp per query. Each warp runs, for its query: the pivot-graph entry
// walk (src/impl/nav.cuh:13-135) and map.txt translation (src/nav_graph.cu:104-109),
// the FP32 PQ table build (src/impl/pq.cuh:8-59) into its own shared memory,
// then the beam walk (src/impl/pure_mem.cuh:243-432) with exact distances and
// top-k insertion (src/impl/util.cuh:26-46,116-163). Arithmetic is FP32 in the
// reference's order with explicit rounding intrinsics, so the result does not
// depend on the compiler's contraction choices; the two FMA sites of the
// reference (pq.cuh:40 and util.cuh:37) are runtime switches.
//
// Warps take queries from a global counter (persistent grid sized to fill the
// SMs), so queries of different length balance across the chip.
#include <climits>

#include "gann_internal.h"

namespace gann {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kNavL = 4;    // nav.cuh:11
constexpr int kNavR = 28;   // nav.cuh:12
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

// square_sum_32 (util.cuh:26-46): lane-strided accumulation, then a
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

// lower_bound on the key (dist, id & 0x7fffffff), util.cuh:166-178.
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

struct WarpSmem {
  float* table;       // M x 256
  float* q;           // dim: the query, then the restored query
  uint32_t* list_id;  // L   sorted candidate list
  float* list_d;
  uint32_t* new_id;   // max_m  neighbours of the node being expanded
  float* new_d;
  uint32_t* snew_id;  // max_m  the same, sorted
  float* snew_d;
  uint32_t* mer_id;   // L + max_m  merged list
  float* mer_d;
  int32_t* topk_id;   // k
  float* topk_d;
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__device__ WarpSmem carve(uint8_t* base, int M, int L, int max_m, int k, int dim) {
  WarpSmem s;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    uint8_t* p = base + o;
    o = align16(o + bytes);
    return p;
  };
  s.table = (float*)take(sizeof(float) * (size_t)M * kPivots);
  s.q = (float*)take(sizeof(float) * dim);
  s.list_id = (uint32_t*)take(4 * (size_t)L);
  s.list_d = (float*)take(4 * (size_t)L);
  s.new_id = (uint32_t*)take(4 * (size_t)max_m);
  s.new_d = (float*)take(4 * (size_t)max_m);
  s.snew_id = (uint32_t*)take(4 * (size_t)max_m);
  s.snew_d = (float*)take(4 * (size_t)max_m);
  s.mer_id = (uint32_t*)take(4 * (size_t)(L + max_m));
  s.mer_d = (float*)take(4 * (size_t)(L + max_m));
  s.topk_id = (int32_t*)take(4 * (size_t)k);
  s.topk_d = (float*)take(4 * (size_t)k);
  return s;
}

// get_entry_kernel_inner (nav.cuh:13-135) for one query, one slot per lane.
// Returns the pivot graph's local id, or -1 after setting an error bit.
template <class T>
__device__ int nav_entry(const PlainParams& p, const float* q, int lane, int64_t& gathered) {
  const T* nd = reinterpret_cast<const T*>(p.ix.nav_data);
  const int dim = p.dim;
  const int64_t glen = (int64_t)p.nav_n * p.nav_max_m;
  float d0 = warp_exact<T>(q, nd + (size_t)p.nav_start * dim, dim, lane, p.fma_exact);
  const int vec_bytes = dim * (int)sizeof(T);
  gathered += vec_bytes;
  uint32_t my_id = lane == 0 ? (uint32_t)p.nav_start : 0xffffffffu;  // nav.cuh:50-57
  float my_d = lane == 0 ? d0 : inf_f();
  int idx = 0, iters = 0;
  while (idx != -1) {
    if (++iters > kNavIterCap) {
      if (lane == 0) atomicOr(p.err, kErrNavCap);
      return -1;
    }
    uint32_t u = __shfl_sync(kFull, my_id, idx);  // nav.cuh:62-68
    if (lane == idx) my_id |= kExpanded;
    // 28 slots of the flat row (nav.cuh:69-72); past the array end reads as -1.
    int v = -1;
    if (lane < kNavR) {
      int64_t e = (int64_t)p.nav_max_m * u + lane;
      v = e < glen ? __ldg(p.ix.nav_graph + e) : -1;
    }
    unsigned neg = __ballot_sync(kFull, lane < kNavR && v == -1);
    int deg = neg ? __ffs(neg) - 1 : kNavR;
    // row slots read up to and including the first -1, plus one vector per neighbour
    gathered += 4 * (deg < kNavR ? deg + 1 : kNavR) + (int64_t)deg * vec_bytes;
    for (int i = 0; i < deg; i++) {  // nav.cuh:70-81
      int vi = __shfl_sync(kFull, v, i);
      if ((unsigned)vi >= (unsigned)p.nav_n) {
        if (lane == 0) atomicOr(p.err, kErrBadId);
        return -1;
      }
      float di = warp_exact<T>(q, nd + (size_t)vi * dim, dim, lane, p.fma_exact);
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

// PQSearchData::init_query (pq.cuh:8-59): table[c][j] accumulates, over the
// dimensions i of chunk c in increasing order, (q_i - mu_i - P_t[i][j])^2.
// Chunks are contiguous ranges, so each (c, j) is accumulated in a register.
// Afterwards q_i is replaced by fl(fl(q_i - mu_i) + mu_i) (pq.cuh:54-56).
__device__ void build_table(const PlainParams& p, const WarpSmem& s, int lane) {
  const int M = p.M;
  for (int c = 0; c < M; c++) {
    const int b = __ldg(p.ix.chunk_off + c), e = __ldg(p.ix.chunk_off + c + 1);
    float acc[8];
#pragma unroll
    for (int t = 0; t < 8; t++) acc[t] = 0.0f;
    for (int i = b; i < e; i++) {
      const float qc = __fsub_rn(s.q[i], __ldg(p.ix.centroid + i));
      const float* pt = p.ix.pivots_t + (size_t)i * kPivots + lane;
#pragma unroll
      for (int t = 0; t < 8; t++) {
        float d = __fsub_rn(qc, __ldg(pt + 32 * t));
        acc[t] = p.fma_table ? __fmaf_rn(d, d, acc[t]) : __fadd_rn(acc[t], __fmul_rn(d, d));
      }
    }
#pragma unroll
    for (int t = 0; t < 8; t++) s.table[c * kPivots + lane + 32 * t] = acc[t];
  }
  __syncwarp();
  for (int i = lane; i < p.dim; i += 32) {
    const float mu = __ldg(p.ix.centroid + i);
    s.q[i] = __fadd_rn(__fsub_rn(s.q[i], mu), mu);
  }
  __syncwarp();
}

// ADC of one code (pure_mem.cuh:302-309): sequential FP32 sum over the chunks.
__device__ __forceinline__ float adc(const float* table, const uint8_t* code, int M) {
  float d = 0.0f;
  if ((M & 15) == 0) {
    for (int j0 = 0; j0 < M; j0 += 16) {
      uint4 w = __ldg(reinterpret_cast<const uint4*>(code + j0));
      uint32_t words[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int b = 0; b < 16; b++) {
        uint32_t c = (words[b >> 2] >> (8 * (b & 3))) & 0xffu;
        d = __fadd_rn(d, table[(j0 + b) * kPivots + c]);
      }
    }
  } else {
    for (int j = 0; j < M; j++) d = __fadd_rn(d, table[j * kPivots + __ldg(code + j)]);
  }
  return d;
}

// retset_push_32 (util.cuh:116-163) by its result: the value goes after every
// entry with distance <= value; the list keeps at most k entries.
__device__ void topk_push(float* td, int32_t* ti, int& size, int k, float value, int vid, int lane) {
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

template <class T>
__device__ void search_query(const PlainParams& p, const WarpSmem& s, int qid, int lane) {
  const int dim = p.dim, L = p.L, k = p.k, max_m = p.max_m, M = p.M;
  const float* qg = p.queries + (size_t)qid * dim;
  for (int i = lane; i < dim; i += 32) s.q[i] = __ldg(qg + i);
  __syncwarp();

  int64_t u;
  int64_t gathered = 0;  // algorithmic bytes: records, neighbour ids, codes, pivot vectors
  if (p.has_nav) {  // pure_mem.cu:106-124
    int local = nav_entry<T>(p, s.q, lane, gathered);
    if (local >= p.nav_n) {  // an all-INF slot 0 (fewer than 4 finite candidates)
      if (lane == 0) atomicOr(p.err, kErrBadId);
      local = -1;
    }
    u = local < 0 ? -2 : (int64_t)__ldg(p.ix.nav_map + local);
  } else {
    u = p.medoid;
  }
  build_table(p, s, lane);

  int sz = 0, found = 0, hops = 0;
  while (u >= 0) {  // pure_mem.cuh:287-428
    if (u >= p.n) {
      if (lane == 0) atomicOr(p.err, kErrBadId);
      break;
    }
    if (hops >= kHopCap) {
      if (lane == 0) atomicOr(p.err, kErrHopCap);
      break;
    }
    const uint8_t* node = p.ix.pages + (u / p.npp) * kPageSize + (u % p.npp) * p.node_len;
    const int32_t* meta = reinterpret_cast<const int32_t*>(node + p.data_len);
    const int deg = __ldg(meta);
    if (deg < 0 || deg > max_m) {
      if (lane == 0) atomicOr(p.err, kErrBadDegree);
      break;
    }
    // ADC of every neighbour (pure_mem.cuh:294-310).
    bool bad = false;
    for (int t = lane; t < deg; t += 32) {
      int v = __ldg(meta + 1 + t);
      float d = inf_f();
      if ((unsigned)v < (unsigned)p.n)
        d = adc(s.table, p.ix.codes + (size_t)v * M, M);
      else
        bad = true;
      s.new_id[t] = (uint32_t)v;
      s.new_d[t] = d;
    }
    if (__any_sync(kFull, bad)) {
      if (lane == 0) atomicOr(p.err, kErrBadId);
      break;
    }
    gathered += 4 + 4 * deg + p.data_len + (int64_t)deg * M;
    __syncwarp();
    // Sort the new entries by (dist, id) -- pure_mem.cuh:314-348 sorts them by
    // merge rounds; with distinct ids any correct sort gives the same order.
    for (int t = lane; t < deg; t += 32) {
      const float d = s.new_d[t];
      const uint32_t id = s.new_id[t] & kMask;
      int r = 0;
      for (int f = 0; f < deg; f++) {
        const float fd = s.new_d[f];
        const uint32_t fi = s.new_id[f] & kMask;
        r += (fd < d) || (fd == d && (fi < id || (fi == id && f < t)));
      }
      s.snew_d[r] = d;
      s.snew_id[r] = s.new_id[t];
    }
    __syncwarp();
    // Merge into the sorted list; a new entry equal to an old one goes after
    // it (pure_mem.cuh:351-376); positions past 2L are dropped (:377).
    const int cap2 = min(sz + deg, 2 * L);
    for (int t = lane; t < deg; t += 32) {
      const float d = s.snew_d[t];
      const uint32_t id = s.snew_id[t];
      int pos = lower_bound_key(s.list_d, s.list_id, 0, sz, d, id);
      if (pos != sz && ((s.list_id[pos] ^ id) & kMask) == 0) pos++;
      pos += t;
      if (pos < cap2) {
        s.mer_d[pos] = d;
        s.mer_id[pos] = id;
      }
    }
    for (int i = lane; i < sz; i += 32) {
      const float d = s.list_d[i];
      const uint32_t id = s.list_id[i];
      int pos = lower_bound_key(s.snew_d, s.snew_id, 0, deg, d, id) + i;
      if (pos < cap2) {
        s.mer_d[pos] = d;
        s.mer_id[pos] = id;
      }
    }
    __syncwarp();
    // Drop adjacent duplicate ids, keep at most L entries and find the first
    // entry without the expanded bit (pure_mem.cuh:380-419).
    int count = 0, best = INT_MAX;
    for (int base = 0; base < cap2; base += 32) {
      const int i = base + lane;
      const bool valid = i < cap2;
      uint32_t id = 0;
      float d = 0.0f;
      bool dup = false;
      if (valid) {
        id = s.mer_id[i];
        d = s.mer_d[i];
        dup = i > 0 && ((id ^ s.mer_id[i - 1]) & kMask) == 0;
      }
      const unsigned dm = __ballot_sync(kFull, dup);
      const int pos = i - count - __popc(dm & ((1u << lane) - 1));
      const bool keep = valid && !dup;
      if (keep && pos < L) {
        s.list_id[pos] = id;
        s.list_d[pos] = d;
      }
      const unsigned um = __ballot_sync(kFull, keep && !(id & kExpanded));
      if (best == INT_MAX && um) {
        const int fl = __ffs(um) - 1;
        best = base + fl - count - __popc(dm & ((1u << fl) - 1));
      }
      count += __popc(dm);
    }
    __syncwarp();
    const int C = cap2 - count;
    // Exact distance of this node and top-k insertion (pure_mem.cuh:420-424).
    const float ed = warp_exact<T>(s.q, reinterpret_cast<const T*>(node), dim, lane, p.fma_exact);
    topk_push(s.topk_d, s.topk_id, found, k, ed, (int)u, lane);
    hops++;
    // best == INT_MAX with C < L is where the reference reads stale slots; the
    // walk stops there. With C >= L the reference stops too.
    if (best >= L) {
      u = -1;
    } else {
      u = (int64_t)s.list_id[best];
      __syncwarp();
      if (lane == 0) s.list_id[best] |= kExpanded;
      sz = C < L ? C : L;
      __syncwarp();
    }
  }
  int32_t* out_id = p.nns + (size_t)qid * k;
  float* out_d = p.dists + (size_t)qid * k;
  for (int i = lane; i < k; i += 32) {
    out_id[i] = i < found ? s.topk_id[i] : 0;
    out_d[i] = i < found ? s.topk_d[i] : 0.0f;
  }
  if (lane == 0) {
    p.found[qid] = found;
    if (p.hops) p.hops[qid] = hops;
    if (p.bytes) p.bytes[qid] = gathered;
  }
  __syncwarp();
}

template <class T>
__global__ void __launch_bounds__(256) plain_search_kernel(PlainParams p, int per_warp_bytes) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const WarpSmem s = carve(smem + (size_t)warp * per_warp_bytes, p.M, p.L, p.max_m, p.k, p.dim);
  for (;;) {
    int qid = 0;
    if (lane == 0) qid = atomicAdd(p.next_query, 1);
    qid = __shfl_sync(kFull, qid, 0);
    if (qid >= p.nq) break;
    search_query<T>(p, s, qid, lane);
  }
}

}  // namespace

size_t plain_smem_per_warp(int M, int L, int max_m, int k, int dim) {
  size_t o = 0;
  o = align16(o + sizeof(float) * (size_t)M * kPivots);
  o = align16(o + sizeof(float) * dim);
  o = align16(o + 4 * (size_t)L) ;
  o = align16(o + 4 * (size_t)L);
  for (int r = 0; r < 4; r++) o = align16(o + 4 * (size_t)max_m);
  o = align16(o + 4 * (size_t)(L + max_m));
  o = align16(o + 4 * (size_t)(L + max_m));
  o = align16(o + 4 * (size_t)k);
  o = align16(o + 4 * (size_t)k);
  return o;
}

cudaError_t launch_plain(const PlainParams& p, int dtype, int num_sms, cudaStream_t stream) {
  const size_t per_warp = plain_smem_per_warp(p.M, p.L, p.max_m, p.k, p.dim);
  const size_t kMaxBlockSmem = 227 * 1024, kSmSmem = 228 * 1024, kReserve = 1024;
  // Pick warps per CTA to maximise resident warps per SM.
  int best_w = 0, best_total = 0;
  for (int w = 1; w <= 8; w++) {
    size_t blk = per_warp * w;
    if (blk > kMaxBlockSmem) break;
    int ctas = (int)(kSmSmem / (blk + kReserve));
    if (ctas > 32 / w) ctas = 32 / w;
    if (ctas * w > best_total) {
      best_total = ctas * w;
      best_w = w;
    }
  }
  if (best_w == 0) return cudaErrorInvalidConfiguration;
  const size_t blk = per_warp * best_w;
  const int ctas_per_sm = best_total / best_w;
  int grid = num_sms * ctas_per_sm;
  const int need = (p.nq + best_w - 1) / best_w;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  cudaError_t e;
  if (dtype == GANN_UINT8) {
    e = cudaFuncSetAttribute(plain_search_kernel<uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)blk);
    if (e != cudaSuccess) return e;
    plain_search_kernel<uint8_t><<<grid, 32 * best_w, blk, stream>>>(p, (int)per_warp);
  } else {
    e = cudaFuncSetAttribute(plain_search_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)blk);
    if (e != cudaSuccess) return e;
    plain_search_kernel<float><<<grid, 32 * best_w, blk, stream>>>(p, (int)per_warp);
  }
  return cudaGetLastError();
}

}  // namespace gann
