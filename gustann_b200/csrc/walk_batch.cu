// Batched search kernel: the optimised form of the all-in-GPU path.
//
// One CTA of W warps serves one query at a time and pulls the next query from a
// device counter (persistent grid). Per query: the pivot-graph entry walk
// (src/impl/nav.cuh:13-135) on warp 0, or the nearest pivot found for the
// whole batch on the tensor cores (entry_tc.cu), while the other warps build the PQ table
// (src/impl/pq.cuh:8-59) in shared memory, FP32 or BF16 (or copy a BF16 table
// built on the tensor cores for the whole batch); then a beam walk that expands
// up to W candidates per step, one per warp (src/impl/pure_mem.cuh:243-432
// expands one):
//   * the picks of a step are the first W unexpanded list entries; each step
//     works them out for the next one from its sorted survivors before it
//     rewrites the list, so every warp's next record loads during the merge;
//   * a direct-mapped cache of the ids already scored for this query (the
//     visited filter) skips their code gather and ADC. A hit is always a node
//     the list has already considered (the entry node is listed too), and a
//     node the list has considered is rejected when it is scored again:
//     it is either still in the list (same key) or at or above the list's last
//     key, which only decreases. So the cache's contents, which depend on the
//     order of the warps' atomicExch, change the work done but never the result;
//   * new candidates are merged into the sorted list of L entries by inserting
//     the survivors only (entries below the list's last key), as in the plain
//     form, in place: only the entries from the first insertion point on move;
//   * every expanded node's exact distance goes into the top-k
//     (src/impl/util.cuh:26-46,116-163).
// L and k may differ per query.
#include <climits>

#include "search_common.cuh"

namespace gann {
namespace {

struct BatchSmem {
  float* q;
  void* table;
  uint32_t* hash;   // visited cache: one id per slot
  uint32_t* l_id;   // sorted candidate list (L), updated in place
  float* l_d;
  uint32_t* c_id;  // sorted survivors (W * max_m)
  float* c_d;      // sorted survivor distances
  uint32_t* s_id;  // survivors of the step, unsorted (W * max_m)
  float* s_d;
  int32_t* s_lb;   // insertion points, unsorted then sorted
  int32_t* s_slb;
  int32_t* sel_id;  // W
  float* sel_d;     // W exact distances
  int32_t* topk_id;
  float* topk_d;
  int* ctrl;        // [0] qid, [2] survivors, [3] entry, [4] repeated id, [5] after dedupe, [6] stop,
                    // [7] first insertion point of the step
  uint32_t* wnew;   // W * max_m: per-warp list of newly seen neighbours
};

struct BatchPlan {
  size_t off[17];
  size_t total;
  __host__ __device__ BatchPlan(int M, int tab_bytes, int H, int L, int max_m, int W, int k, int dim) {
    const size_t C = (size_t)W * max_m;
    const size_t sz[17] = {4u * (size_t)dim, (size_t)tab_bytes * M * kPivots, 4u * (size_t)H, 4u * (size_t)L,
                           4u * (size_t)L, 4 * C, 4 * C, 4 * C, 4 * C, 4 * C, 4 * C, 4u * W, 4u * W,
                           4u * (size_t)k, 4u * (size_t)k, 64, 4 * C};
    size_t o = 0;
    for (int i = 0; i < 17; i++) {
      off[i] = o;
      o = align16(o + sz[i]);
    }
    total = o;
  }
};

__device__ BatchSmem carve_batch(uint8_t* base, const BatchPlan& pl) {
  BatchSmem s;
  s.q = (float*)(base + pl.off[0]);
  s.table = base + pl.off[1];
  s.hash = (uint32_t*)(base + pl.off[2]);
  s.l_id = (uint32_t*)(base + pl.off[3]);
  s.l_d = (float*)(base + pl.off[4]);
  s.c_id = (uint32_t*)(base + pl.off[5]);
  s.c_d = (float*)(base + pl.off[6]);
  s.s_id = (uint32_t*)(base + pl.off[7]);
  s.s_d = (float*)(base + pl.off[8]);
  s.s_lb = (int32_t*)(base + pl.off[9]);
  s.s_slb = (int32_t*)(base + pl.off[10]);
  s.sel_id = (int32_t*)(base + pl.off[11]);
  s.sel_d = (float*)(base + pl.off[12]);
  s.topk_id = (int32_t*)(base + pl.off[13]);
  s.topk_d = (float*)(base + pl.off[14]);
  s.ctrl = (int*)(base + pl.off[15]);
  s.wnew = (uint32_t*)(base + pl.off[16]);
  return s;
}

__device__ __forceinline__ uint32_t hash_slot(uint32_t id, int bits) { return (id * 2654435761u) >> (32 - bits); }

constexpr int kEdgeRegs = 2;  // neighbour slots held in registers per lane (max_m <= 64 without reloads)
constexpr int kVecRegs = 4;   // vector elements held in registers per lane (dim <= 128 without reloads)

// ADC of the batched form. For M a multiple of 16 the chunks are split into
// four contiguous quarters summed in chunk order, four accumulators in flight,
// and the result is (q0 + q1) + (q2 + q3); every score of a node (the entry
// included) uses this function, so a re-score reproduces the same key. Other
// M: a sequential sum (the plain form's adc).
template <class TabT>
__device__ __forceinline__ float quarter_sum(const TabT* table, const uint8_t* code, int c0, int nc) {
  float d = 0.0f;
  for (int w = 0; w < nc; w += 4) {
    const uint32_t x = __ldg(reinterpret_cast<const uint32_t*>(code + c0 + w));
    d += load_tab(table, (c0 + w) * kPivots + (x & 0xffu));
    d += load_tab(table, (c0 + w + 1) * kPivots + ((x >> 8) & 0xffu));
    d += load_tab(table, (c0 + w + 2) * kPivots + ((x >> 16) & 0xffu));
    d += load_tab(table, (c0 + w + 3) * kPivots + (x >> 24));
  }
  return d;
}

template <class TabT>
__device__ __forceinline__ float adc_split4(const TabT* table, const uint8_t* code, int M) {
  if ((M & 15) != 0) return adc(table, code, M);
  const int q = M >> 2;
  const float s0 = quarter_sum(table, code, 0, q), s1 = quarter_sum(table, code, q, q);
  const float s2 = quarter_sum(table, code, 2 * q, q), s3 = quarter_sum(table, code, 3 * q, q);
  return (s0 + s1) + (s2 + s3);
}

// The same sum for M == 32 from the code's two 16-byte words, loaded ahead:
// quarters are words {0,1}, {2,3}, {4,5}, {6,7}, bytes in chunk order.
template <class TabT>
__device__ __forceinline__ float adc32_words(const TabT* table, const uint4& a, const uint4& b) {
  const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
  float s[4];
#pragma unroll
  for (int qq = 0; qq < 4; qq++) {
    float d = 0.0f;
#pragma unroll
    for (int t = 0; t < 2; t++) {
      const uint32_t x = w[qq * 2 + t];
      const int c = (qq * 2 + t) * 4;
      d += load_tab(table, c * kPivots + (x & 0xffu));
      d += load_tab(table, (c + 1) * kPivots + ((x >> 8) & 0xffu));
      d += load_tab(table, (c + 2) * kPivots + ((x >> 16) & 0xffu));
      d += load_tab(table, (c + 3) * kPivots + (x >> 24));
    }
    s[qq] = d;
  }
  return (s[0] + s[1]) + (s[2] + s[3]);
}

// Insert up to N (distance, id) pairs, given in push order in vd/vi[0, n),
// into the sorted top-k (td, ti, size) in one pass of one warp. Pairs with an
// infinite distance are skipped. The result equals n calls of topk_push in
// order: a new pair goes after existing entries with an equal distance, and
// after earlier new pairs with an equal distance. Lane j holds pair j; the
// others' distances come by shuffle, so no per-pair registers are held.
template <int N>
__device__ __forceinline__ void topk_push_many(float* td, int32_t* ti, int& size, int k, const float* vd,
                                               const int32_t* vi, int n, int lane) {
  const bool mine = lane < N && lane < n && vd[lane] != inf_f();
  const float my_d = mine ? vd[lane] : inf_f();
  const int32_t my_id = mine ? vi[lane] : 0;
  const unsigned vm = __ballot_sync(kFull, mine);
  const int nv = __popc(vm);
  if (nv == 0) return;
  if (size == k && !__ballot_sync(kFull, mine && my_d < td[k - 1])) return;  // full: must beat the k-th
  int pos = 0;  // final position of pair `lane`
#pragma unroll
  for (int j = 0; j < N; j++) {
    const float dj = __shfl_sync(kFull, my_d, j);
    pos += ((vm >> j) & 1u) && (dj < my_d || (dj == my_d && j < lane));
  }
  for (int base = 0; base < size; base += 32) {
    const int i = base + lane;
    const float e = i < size ? td[i] : inf_f();
#pragma unroll
    for (int j = 0; j < N; j++) {
      const float dj = __shfl_sync(kFull, my_d, j);  // every lane takes part in the shuffle
      const int c = __popc(__ballot_sync(kFull, i < size && e <= dj));
      if (lane == j) pos += c;
    }
  }
  const bool enters = mine && pos < k;
  if (__ballot_sync(kFull, enters)) {
    for (int c = (size - 1) >> 5; c >= 0; c--) {  // existing entries move up, top chunk first
      const int i = c * 32 + lane;
      const float e = i < size ? td[i] : 0.0f;
      const int32_t eid = i < size ? ti[i] : 0;
      int sh = 0;
#pragma unroll
      for (int j = 0; j < N; j++) {
        const float dj = __shfl_sync(kFull, my_d, j);
        sh += ((vm >> j) & 1u) && dj < e;
      }
      __syncwarp();
      if (i < size && i + sh < k) {
        td[i + sh] = e;
        ti[i + sh] = eid;
      }
      __syncwarp();
    }
    if (enters) {
      td[pos] = my_d;
      ti[pos] = my_id;
    }
    __syncwarp();
  }
  size = min(size + nv, k);
}

// Exact squared L2 of the node (its first kVecRegs*32 elements preloaded in
// vx, lane-strided; or, PK, a uint8 vector of dim <= 128 held as one 32-bit
// word per lane, bytes 4 lane .. 4 lane + 3). uint8 vectors with an integral
// query are summed in int32 (exact); otherwise FP32 with the reference's
// reduction (util.cuh:26-46), the PK form first moving each lane's strided
// elements into place with shuffles so the sum is the same.
template <class T, bool PK>
__device__ __forceinline__ float exact_dist(const float* q, const T* v, const float (&vx_in)[kVecRegs], uint32_t vw,
                                            int dim, int lane, bool int_query, int fma) {
  if (PK && int_query) {
    int acc = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int i = 4 * lane + j;
      if (i < dim) {
        const int d = (int)q[i] - (int)((vw >> (8 * j)) & 0xffu);
        acc += d * d;
      }
    }
    acc = __reduce_add_sync(kFull, acc);
    return (float)acc;
  }
  float vx[kVecRegs];
#pragma unroll
  for (int r = 0; r < kVecRegs; r++) {
    if (PK) {
      const uint32_t w = __shfl_sync(kFull, vw, (lane + 32 * r) >> 2);
      vx[r] = (float)((w >> (8 * (lane & 3))) & 0xffu);
    } else {
      vx[r] = vx_in[r];
    }
  }
  if (!PK && sizeof(T) == 1 && int_query) {
    int acc = 0;
#pragma unroll
    for (int r = 0; r < kVecRegs; r++) {
      const int i = lane + 32 * r;
      if (i < dim) {
        const int d = (int)q[i] - (int)vx[r];
        acc += d * d;
      }
    }
    for (int i = lane + 32 * kVecRegs; i < dim; i += 32) {
      const int d = (int)q[i] - (int)load_elem<T>(v, i);
      acc += d * d;
    }
    acc = __reduce_add_sync(kFull, acc);
    return (float)acc;
  }
  float acc = 0.0f;
#pragma unroll
  for (int r = 0; r < kVecRegs; r++) {
    const int i = lane + 32 * r;
    if (i < dim) {
      const float d = __fsub_rn(q[i], vx[r]);
      acc = fma ? __fmaf_rn(d, d, acc) : __fadd_rn(acc, __fmul_rn(d, d));
    }
  }
  for (int i = lane + 32 * kVecRegs; i < dim; i += 32) {
    const float d = __fsub_rn(q[i], load_elem<T>(v, i));
    acc = fma ? __fmaf_rn(d, d, acc) : __fadd_rn(acc, __fmul_rn(d, d));
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc = __fadd_rn(acc, __shfl_down_sync(kFull, acc, off));
  return __shfl_sync(kFull, acc, 0);
}

// Copy one query's BF16 table (M x 256 x 2 bytes, a multiple of 16) from
// global memory with 16-byte loads.
__device__ void copy_table(void* dst, const __nv_bfloat16* src, int bytes, int tid, int nthreads) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4* d = reinterpret_cast<uint4*>(dst);
  for (int i = tid; i < bytes / 16; i += nthreads) d[i] = __ldg(s + i);
}

// List entries per thread staged in registers by the in-place merge: 1,024
// entries per round for W >= 8.
__host__ __device__ constexpr int stage_per_thread(int W) { return W >= 16 ? 2 : 4; }

// The node's record as one warp holds it: degree, the first kEdgeRegs * 32
// neighbour slots and kVecRegs * 32 vector elements, loaded in one round trip.
template <class T, bool PK>
struct Record {
  int64_t u = -1;
  bool uok = false;
  const uint8_t* node = nullptr;
  const int32_t* meta = nullptr;
  int deg = 0;
  int ev[kEdgeRegs];
  float vx[kVecRegs];  // lane-strided elements (not PK)
  uint32_t vw = 0;     // PK: bytes 4 lane .. 4 lane + 3 of a uint8 vector, one 128-byte load per warp
  __device__ __forceinline__ void load(const BatchParams& p, int64_t id, int lane) {
    u = id;
    uok = id >= 0 && id < p.n;
    const uint32_t uu = uok ? (uint32_t)id : 0u;
    const uint32_t pg = p.npp_div.div(uu);
    node = record_at(p.ix, pg, (int64_t)(uu - pg * (uint32_t)p.npp) * p.node_len, uu);
    meta = reinterpret_cast<const int32_t*>(node + p.data_len);
    deg = __ldg(meta);
#pragma unroll
    for (int r = 0; r < kEdgeRegs; r++) ev[r] = lane + 32 * r < p.max_m ? __ldg(meta + 1 + lane + 32 * r) : -1;
    if (PK) {
      vw = 4 * lane < p.dim ? __ldg(reinterpret_cast<const uint32_t*>(node) + lane) : 0u;
    } else {
#pragma unroll
      for (int r = 0; r < kVecRegs; r++)
        vx[r] = lane + 32 * r < p.dim ? load_elem<T>(reinterpret_cast<const T*>(node), lane + 32 * r) : 0.0f;
    }
  }
};

// CTAs per SM each kernel is compiled for: 24 warps at up to 80 registers per
// thread (2 CTAs at 64 for W 16), or, with R64, 32 warps at 64 registers, which
// the launcher takes when that many CTAs' shared memory fits.
__host__ __device__ constexpr int min_ctas(int W, bool r64) { return r64 ? 32 / W : (W <= 8 ? 24 / W : 2); }

template <class T, class TabT, int W, bool PK, bool R64>
__global__ void __launch_bounds__(W * 32, min_ctas(W, R64)) batch_search_kernel(BatchParams p) {
  constexpr int NT = W * 32;
  constexpr int TKW = W - 1;  // warp that marks the picks and keeps the top-k
  extern __shared__ __align__(16) uint8_t smem[];
  const BatchPlan pl(p.M, (int)sizeof(TabT), 1 << p.hash_bits, p.L_max, p.max_m, W, p.k_max, p.dim);
  const BatchSmem s = carve_batch(smem, pl);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int dim = p.dim, M = p.M, H = 1 << p.hash_bits;
  const bool m32 = M == 32;
  TabT* table = reinterpret_cast<TabT*>(s.table);
  const NavView nv{p.ix.nav_data, p.ix.nav_graph, p.ix.nav_map, p.nav_n, p.nav_max_m, p.nav_start, dim, p.fma,
                   p.err};
  const PqView pv{p.ix.pivots_t, p.ix.centroid, p.ix.chunk_off, M, dim, p.fma};
  uint32_t* const list_id = s.l_id;
  float* const list_d = s.l_d;
  const int nq = p.nq_dev ? min(p.nq, *p.nq_dev) : p.nq;

  for (;;) {
    if (tid == 0) s.ctrl[0] = atomicAdd(p.next_query, 1);
    __syncthreads();
    const int qid = s.ctrl[0];
    if (qid >= nq) break;
    const int L = p.L_per_q ? min(max(__ldg(p.L_per_q + qid), 1), p.L_max) : p.L_max;
    const int k = p.k_per_q ? min(max(__ldg(p.k_per_q + qid), 1), p.k_max) : p.k_max;
    for (int i = tid; i < dim; i += NT) s.q[i] = __ldg(p.queries + (size_t)qid * dim + i);
    for (int i = tid; i < H; i += NT) s.hash[i] = 0xffffffffu;
    __syncthreads();
    int64_t gathered = 0;  // per-warp share of the algorithmic bytes
    if (warp == 0) {
      int64_t u0;
      if (p.entry_keys) {  // the nearest pivot, found for the batch on the tensor cores (entry_tc.cu)
        const uint32_t local = (uint32_t)__ldg(p.entry_keys + qid);
        if (local < (uint32_t)p.nav_n) {
          u0 = __ldg(p.ix.nav_map + local);
        } else {
          if (lane == 0) atomicOr(p.err, kErrBadId);
          u0 = -2;
        }
      } else {
        u0 = entry_node<T>(p.has_nav, nv, p.medoid, s.q, lane, gathered);
      }
      if (lane == 0) s.ctrl[3] = (int)u0;
    }
    if (p.tables) {  // BF16 tables built for the whole batch on the tensor cores
      copy_table(s.table, p.tables + (size_t)qid * M * kPivots, M * kPivots * 2, tid, NT);
    } else if (W == 1) {
      build_table(pv, table, s.q, 0, 1, lane);
    } else if (warp > 0) {
      build_table(pv, table, s.q, warp - 1, W - 1, lane);
    }
    // The exact distances use the query as given (the reference uses
    // fl(fl(q - mu) + mu), src/impl/pq.cuh:54-56; the batched form does not
    // reproduce that rounding). uint8 data with integral queries take the
    // int32 path.
    bool iq = sizeof(T) == 1;
    for (int i = tid; i < dim && iq; i += NT) iq = s.q[i] == rintf(s.q[i]) && s.q[i] >= 0.0f && s.q[i] <= 255.0f;
    const bool int_query = __syncthreads_and(iq) != 0;
    // The entry node starts the list, unexpanded, with its ADC distance; the
    // first step picks it (the reference expands it without listing it,
    // src/impl/pure_mem.cuh:285-287). Listing it makes every expanded node one
    // that the list has seen, so a later re-score of it is rejected whatever
    // the visited cache holds.
    const int u0 = s.ctrl[3];
    if (tid == 0) {
      s.ctrl[2] = 0;        // survivors of the current step
      s.ctrl[4] = 0;        // a repeated id among them
      s.ctrl[6] = 0;        // stop (hop limit)
      s.ctrl[7] = INT_MAX;  // first insertion point of the current step
      if (u0 >= 0) {
        s.hash[hash_slot((uint32_t)u0, p.hash_bits)] = (uint32_t)u0;
        list_id[0] = (uint32_t)u0;
        const uint8_t* code = p.ix.codes + (size_t)u0 * M;
        list_d[0] = m32 ? adc32_words(table, __ldg(reinterpret_cast<const uint4*>(code)),
                                      __ldg(reinterpret_cast<const uint4*>(code) + 1))
                        : adc_split4(table, code, M);
      }
    }
    __syncthreads();

    // List state, identical in every thread; top-k state in warp TKW. The
    // picks of a step (the first W unexpanded entries of the list) are known
    // when the step starts: the first step picks the entry, and each step
    // works out the next step's picks from the sorted survivors before it
    // rewrites the list, so that each warp's next record is already on its
    // way while the list is merged. Lane w of warp 0 holds the list position
    // of pick w and marks it expanded when the step starts, after the merge
    // that placed it; every comparison of the step masks the mark off, and the
    // scan for old candidates starts after the last pick, so that write
    // changes nothing the step reads before barrier (1), which orders it
    // before the merge reads the list.
    int sz = u0 >= 0 ? 1 : 0, found = 0, hops = 0;
    int npick = u0 >= 0 ? 1 : 0, last_pos = 0;
    int my_pick = 0;  // warp 0, lane w < npick: position of pick w
    Record<T, PK> rec;
    if (warp == 0 && u0 >= 0) rec.load(p, u0, lane);

    for (;;) {
      if (npick == 0 || s.ctrl[6]) break;
      if (warp == 0 && lane < npick) list_id[my_pick] |= kExpanded;
      const bool full = sz == L;
      const float tail_d = full ? list_d[L - 1] : 0.0f;
      const uint32_t tail_id = full ? list_id[L - 1] : 0u;
      // Old candidates for the next step: the first W unexpanded entries after
      // the last pick (every unexpanded entry before it is a pick). Lane t < W
      // holds candidate t; every warp holds the same.
      int noc = 0, oc_pos = INT_MAX;
      uint32_t oc_id = 0;
      for (int base = last_pos + 1; base < sz && noc < W; base += 32) {
        const int i = base + lane;
        const uint32_t id = i < sz ? list_id[i] : kExpanded;
        const bool un = !(id & kExpanded);
        const unsigned um = __ballot_sync(kFull, un);
        const int g = noc + __popc(um & ((1u << lane) - 1));  // candidate index of an unexpanded entry
#pragma unroll
        for (int t = 0; t < W; t++) {
          const unsigned sel = __ballot_sync(kFull, un && g == t);
          if (sel) {
            const int srcl = __ffs(sel) - 1;
            const uint32_t cid = __shfl_sync(kFull, id, srcl);
            if (lane == t) {
              oc_pos = base + srcl;
              oc_id = cid & kMask;
            }
          }
        }
        noc = min(W, noc + __popc(um));
      }
      // Expand: warp w expands pick w (its record was loaded when the pick was
      // made). New neighbours are scored and checked against the list here;
      // survivors (below the list's last key when it is full, not in it yet)
      // are kept unsorted.
      if (warp < npick) {
        const bool ok = rec.uok && rec.deg >= 0 && rec.deg <= p.max_m;
        int deg = rec.deg;
        if (!ok) {
          if (lane == 0) atomicOr(p.err, rec.uok ? kErrBadDegree : kErrBadId);
          deg = 0;
        }
        // Visited-cache check of every neighbour; the new ones are compacted
        // into this warp's scratch list.
        uint32_t* wnew = s.wnew + warp * p.max_m;
        int nnew = 0;
        auto check = [&](int t, int v) {
          bool fresh = false;
          if (t < deg) {
            if ((unsigned)v >= (unsigned)p.n)
              atomicOr(p.err, kErrBadId);
            else
              fresh = atomicExch(&s.hash[hash_slot((uint32_t)v, p.hash_bits)], (uint32_t)v) != (uint32_t)v;
          }
          const unsigned m = __ballot_sync(kFull, fresh);
          if (fresh) wnew[nnew + __popc(m & ((1u << lane) - 1))] = (uint32_t)v;
          nnew += __popc(m);
        };
#pragma unroll
        for (int r = 0; r < kEdgeRegs; r++) check(lane + 32 * r, rec.ev[r]);
        for (int b0 = 32 * kEdgeRegs; b0 < deg; b0 += 32)
          check(b0 + lane, b0 + lane < deg ? __ldg(rec.meta + 1 + b0 + lane) : -1);
        __syncwarp();
        // Score the new ones and keep the survivors: below the list's last key
        // when it is full, not in it yet.
        auto keep = [&](uint32_t v, float d) {
          if (full && !key_less(d, v, tail_d, tail_id)) return;
          const int lb = lower_bound_key(list_d, list_id, 0, sz, d, v);
          if (lb < sz && ((list_id[lb] ^ v) & kMask) == 0) return;
          const int slot = atomicAdd(&s.ctrl[2], 1);
          s.s_id[slot] = v;
          s.s_d[slot] = d;
          s.s_lb[slot] = lb;
          atomicMin(&s.ctrl[7], lb);
        };
        // One lane per new neighbour: all of the warp's code fetches are in
        // flight at once (for M == 32 as two 16-byte loads issued before the
        // exact distance), and no lane runs a second ADC while others idle.
        const bool has = lane < nnew;
        const uint32_t v0 = has ? wnew[lane] : 0u;
        uint4 cw0 = make_uint4(0, 0, 0, 0), cw1 = cw0;
        if (has && m32) {
          const uint4* c4 = reinterpret_cast<const uint4*>(p.ix.codes + (size_t)v0 * 32);
          cw0 = __ldg(c4);
          cw1 = __ldg(c4 + 1);
        }
        float ed = inf_f();
        if (ok)
          ed = exact_dist<T, PK>(s.q, reinterpret_cast<const T*>(rec.node), rec.vx, rec.vw, dim, lane, int_query,
                                 p.fma);
        if (has) keep(v0, m32 ? adc32_words(table, cw0, cw1) : adc_split4(table, p.ix.codes + (size_t)v0 * M, M));
        for (int i = lane + 32; i < nnew; i += 32) {
          const uint32_t v = wnew[i];
          keep(v, adc_split4(table, p.ix.codes + (size_t)v * M, M));
        }
        if (lane == 0) {
          s.sel_d[warp] = ed;
          s.sel_id[warp] = (int32_t)rec.u;
          if (p.visit_count && ok) atomicAdd(p.visit_count + rec.u, 1);
        }
        gathered += ok ? 4 + 4 * deg + p.data_len + (int64_t)nnew * M : 0;
      }
      __syncthreads();  // (1) survivors and exact distances are in
      const int nsv = s.ctrl[2];
      const int first_new = s.ctrl[7];  // INT_MAX when nothing survived
      if (warp == TKW) {  // keep the top-k
        topk_push_many<W>(s.topk_d, s.topk_id, found, k, s.sel_d, s.sel_id, npick, lane);
        hops += npick;
        if (lane == 0 && hops > kHopCap) {
          s.ctrl[6] = 1;
          atomicOr(p.err, kErrHopCap);
        }
      }
      // Rank-sort the survivors (rank = number of smaller keys, ties by slot);
      // a repeated id (a cache eviction between two lookups) raises a flag.
      // Warp TKW is busy with the top-k, so the other warps sort.
      if (W == 1 || warp != TKW) {
        constexpr int RS = W == 1 ? 32 : NT - 32;
        for (int j = tid; j < nsv; j += RS) {
          const float d = s.s_d[j];
          const uint32_t id = s.s_id[j];
          int r = 0;
          bool rep = false;
          for (int f = 0; f < nsv; f++) {
            const float fd = s.s_d[f];
            const uint32_t fi = s.s_id[f];
            const bool same = fd == d && ((fi ^ id) & kMask) == 0;
            r += key_less(fd, fi, d, id) || (same && f < j);
            rep |= same && f != j;
          }
          s.c_id[r] = id;  // sorted survivors
          s.c_d[r] = d;
          s.s_slb[r] = s.s_lb[j];
          if (rep) s.ctrl[4] = 1;
        }
      }
      // In-place merge. Entries from the first insertion point on move up:
      // old entry i goes to i + #{survivors inserted at or before i}, survivor
      // r to its insertion point + r; positions >= L drop. Each round stages
      // the top KS * NT entries still to move in registers, waits for
      // every thread, then writes; the first round's wait is barrier (2), and
      // survivors are written after the last round.
      constexpr int KS = stage_per_thread(W);
      uint32_t st_id[KS];
      float st_d[KS];
      int hi = sz;
      auto round_lo = [&]() { return min(hi, max(first_new, hi - KS * NT)); };
      auto stage = [&]() {
        const int lo = round_lo();
#pragma unroll
        for (int r = 0; r < KS; r++) {
          const int i = lo + r * NT + tid;
          if (i < hi) {
            st_id[r] = list_id[i];
            st_d[r] = list_d[i];
          }
        }
      };
      stage();
      __syncthreads();  // (2)
      uint32_t* const sid = s.c_id;
      int ns = nsv;
      const bool repeated = s.ctrl[4] != 0;
      if (repeated) {  // rare: drop repeated ids (warp 0), then share the count
        if (warp == 0) {
          int cnt = 0;
          for (int base = 0; base < nsv; base += 32) {
            const int j = base + lane;
            uint32_t id = 0;
            float d = 0.0f;
            int lb = 0;
            bool keep = false;
            if (j < nsv) {
              id = sid[j];
              d = s.c_d[j];
              lb = s.s_slb[j];
              keep = j == 0 || ((sid[j - 1] ^ id) & kMask) != 0;
            }
            const unsigned km = __ballot_sync(kFull, keep);
            __syncwarp();
            if (keep) {
              const int slot = cnt + __popc(km & ((1u << lane) - 1));
              sid[slot] = id;
              s.c_d[slot] = d;
              s.s_slb[slot] = lb;
            }
            cnt += __popc(km);
            __syncwarp();
          }
          if (lane == 0) s.ctrl[5] = cnt;
        }
        __syncthreads();
        ns = s.ctrl[5];
      }
      // Next picks: the first W of the old candidates and the first W
      // survivors by position in the merged list, below L. Lane t < W holds
      // old candidate t, lane W + r survivor r; every warp computes the same.
      {
        int mpos = INT_MAX;
        uint32_t mid = 0;
        if (lane < W && lane < noc) {
          int lo = 0, up = ns;
          while (lo < up) {
            const int md = (lo + up) >> 1;
            if (s.s_slb[md] <= oc_pos) lo = md + 1; else up = md;
          }
          mpos = oc_pos + lo;
          mid = oc_id;
        } else if (lane >= W && lane < 2 * W && lane - W < ns) {
          mpos = s.s_slb[lane - W] + (lane - W);
          mid = sid[lane - W] & kMask;
        }
        if (mpos >= L) mpos = INT_MAX;
        int rank = 0;  // among the valid entries (their positions are distinct)
#pragma unroll
        for (int j = 0; j < 2 * W; j++) rank += __shfl_sync(kFull, mpos, j) < mpos;
        const bool take = mpos != INT_MAX && rank < W;
        npick = __popc(__ballot_sync(kFull, take));
        uint32_t my_next = 0;
#pragma unroll
        for (int w = 0; w < W; w++) {
          const unsigned sel = __ballot_sync(kFull, take && rank == w);
          const int srcl = sel ? __ffs(sel) - 1 : 0;
          const int ppos = __shfl_sync(kFull, mpos, srcl);
          const uint32_t pid = __shfl_sync(kFull, mid, srcl);
          if (lane == w) my_pick = ppos;
          if (sel) last_pos = ppos;
          if (w == warp) my_next = pid;
        }
        if (warp < npick) rec.load(p, (int64_t)my_next, lane);
      }
      if (ns) {
        for (;;) {
          const int lo = round_lo();
#pragma unroll
          for (int r = 0; r < KS; r++) {
            const int i = lo + r * NT + tid;
            if (i < hi) {
              int a = 0, b = ns;
              while (a < b) {
                const int md = (a + b) >> 1;
                if (s.s_slb[md] <= i) a = md + 1; else b = md;
              }
              const int dst = i + a;
              if (dst < L) {
                list_id[dst] = st_id[r];
                list_d[dst] = st_d[r];
              }
            }
          }
          hi = lo;
          if (hi <= first_new) break;
          stage();
          __syncthreads();
        }
        // Every old entry was read before a barrier that precedes this point,
        // and survivors and old entries land on distinct positions.
        for (int r = tid; r < ns; r += NT) {
          const int dst = s.s_slb[r] + r;
          if (dst < L) {
            list_id[dst] = sid[r];
            list_d[dst] = s.c_d[r];
          }
        }
      }
      sz = min(sz + ns, L);
      // Every thread read the survivor count and the first insertion point
      // after (1); the next step adds to them only after (3), so they are
      // reset here. The repeat flag is read by every thread after (2) and set
      // again only after the next (1).
      if (tid == 0) {
        s.ctrl[2] = 0;
        s.ctrl[7] = INT_MAX;
      }
      __syncthreads();  // (3) the new list is complete
      if (tid == 0) s.ctrl[4] = 0;
    }
    // outputs (warp TKW holds the top-k bookkeeping)
    if (warp == TKW) {
      const size_t row = (size_t)qid * p.k_max;
      for (int i = lane; i < p.k_max; i += 32) {
        p.nns[row + i] = i < found ? s.topk_id[i] : 0;
        p.dists[row + i] = i < found ? s.topk_d[i] : 0.0f;
      }
      if (lane == 0) {
        p.found[qid] = found;
        if (p.hops) p.hops[qid] = hops;
      }
    }
    if (p.bytes) {
      if (lane == 0) atomicAdd(reinterpret_cast<unsigned long long*>(p.bytes + qid), (unsigned long long)gathered);
    }
    __syncthreads();
  }
}

// CTAs of `kern` that fit one SM with `smem` bytes of dynamic shared memory
// each (after setting its shared-memory limit), or -1 on an error.
template <class K>
int ctas_per_sm(K kern, int W, size_t smem) {
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return -1;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, W * 32, smem) != cudaSuccess) return -1;
  return per_sm;
}

template <class T, class TabT, int W, bool PK>
cudaError_t launch_wp(const BatchParams& p, int num_sms, cudaStream_t stream) {
  const BatchPlan pl(p.M, (int)sizeof(TabT), 1 << p.hash_bits, p.L_max, p.max_m, W, p.k_max, p.dim);
  const size_t smem = pl.total;
  if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  auto kern = batch_search_kernel<T, TabT, W, PK, false>;
  if constexpr (W == 4 || W == 8) {
    // the 64-register build, when shared memory admits all of its CTAs
    auto k64 = batch_search_kernel<T, TabT, W, PK, true>;
    const int n64 = ctas_per_sm(k64, W, smem);
    if (n64 < 0) return cudaGetLastError();
    if (n64 >= min_ctas(W, true)) kern = k64;
  }
  const int per_sm = ctas_per_sm(kern, W, smem);
  if (per_sm < 0) return cudaGetLastError();
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  int grid = num_sms * per_sm;
  if (grid > p.nq) grid = p.nq;
  kern<<<grid, W * 32, smem, stream>>>(p);
  return cudaGetLastError();
}

// uint8 vectors of dim <= 128, a multiple of 4, in 4-byte aligned records
// (every record start is then 4-byte aligned) load as one word per lane.
template <class T, class TabT, int W>
cudaError_t launch_w(const BatchParams& p, int num_sms, cudaStream_t stream) {
  const bool pk = sizeof(T) == 1 && p.dim % 4 == 0 && p.dim <= 128 && p.node_len % 4 == 0 &&
                  (p.ix.rec_stride == 0 || p.ix.rec_stride % 4 == 0);
  if (pk) return launch_wp<T, TabT, W, true>(p, num_sms, stream);
  return launch_wp<T, TabT, W, false>(p, num_sms, stream);
}

template <class T, class TabT>
cudaError_t launch_t(const BatchParams& p, int W, int num_sms, cudaStream_t stream) {
  switch (W) {
    case 1: return launch_w<T, TabT, 1>(p, num_sms, stream);
    case 2: return launch_w<T, TabT, 2>(p, num_sms, stream);
    case 4: return launch_w<T, TabT, 4>(p, num_sms, stream);
    case 8: return launch_w<T, TabT, 8>(p, num_sms, stream);
    case 16: return launch_w<T, TabT, 16>(p, num_sms, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

size_t batch_smem_bytes(int M, int tab_bytes, int hash_bits, int L_max, int max_m, int W, int k_max, int dim) {
  return BatchPlan(M, tab_bytes, 1 << hash_bits, L_max, max_m, W, k_max, dim).total;
}

cudaError_t launch_batch(const BatchParams& p, int dtype, int table_bf16, int W, int num_sms, cudaStream_t stream) {
  if (dtype == GANN_UINT8)
    return table_bf16 ? launch_t<uint8_t, __nv_bfloat16>(p, W, num_sms, stream)
                      : launch_t<uint8_t, float>(p, W, num_sms, stream);
  return table_bf16 ? launch_t<float, __nv_bfloat16>(p, W, num_sms, stream)
                    : launch_t<float, float>(p, W, num_sms, stream);
}

}  // namespace gann
