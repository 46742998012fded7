// Batched search kernel: the optimised form of the all-in-GPU path.
//
// One CTA of W warps serves one query at a time and pulls the next query from a
// device counter (persistent grid). Per query: the pivot-graph entry walk
// (src/impl/nav.cuh:13-135) on warp 0 while the other warps build the PQ table
// (src/impl/pq.cuh:8-59) in shared memory, FP32 or BF16 (or copy a BF16 table
// built on the tensor cores for the whole batch); then a beam walk that expands
// up to W candidates per step, one per warp (src/impl/pure_mem.cuh:243-432
// expands one):
//   * a direct-mapped cache of the ids already scored for this query (the
//     visited filter) skips their code gather and ADC. A hit is always a node
//     the list has already considered (the entry node is listed as expanded),
//     and a node the list has considered is rejected when it is scored again:
//     it is either still in the list (same key) or at or above the list's last
//     key, which only decreases. So the cache's contents, which depend on the
//     order of the warps' atomicExch, change the work done but never the result;
//   * new candidates are merged into the sorted list of L entries by inserting
//     the survivors only (entries below the list's last key), as in the plain form;
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
  uint32_t *la_id, *lb_id;
  float *la_d, *lb_d;
  uint32_t* c_id;  // [0, W): list positions of the picks; then the sorted survivors (W * max_m)
  float* c_d;      // sorted survivor distances
  uint32_t* s_id;  // survivors of the step, unsorted (W * max_m)
  float* s_d;
  int32_t* s_lb;   // insertion points, unsorted then sorted
  int32_t* s_slb;
  int32_t* sel_id;  // W
  float* sel_d;     // W exact distances
  int32_t* topk_id;
  float* topk_d;
  int* ctrl;        // [0] qid, [2] survivors, [3] entry, [4] repeated id, [5] after dedupe, [6] stop
  uint32_t* wnew;   // W * max_m: per-warp list of newly seen neighbours
};

struct BatchPlan {
  size_t off[19];
  size_t total;
  __host__ __device__ BatchPlan(int M, int tab_bytes, int H, int L, int max_m, int W, int k, int dim) {
    const size_t C = (size_t)W * max_m;
    const size_t sz[19] = {4u * (size_t)dim, (size_t)tab_bytes * M * kPivots, 4u * (size_t)H, 4u * (size_t)L,
                           4u * (size_t)L, 4u * (size_t)L, 4u * (size_t)L, 4 * (C + W), 4 * C, 4 * C, 4 * C,
                           4 * C, 4 * C, 4u * W, 4u * W, 4u * (size_t)k, 4u * (size_t)k, 64, 4 * C};
    size_t o = 0;
    for (int i = 0; i < 19; i++) {
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
  s.la_id = (uint32_t*)(base + pl.off[3]);
  s.la_d = (float*)(base + pl.off[4]);
  s.lb_id = (uint32_t*)(base + pl.off[5]);
  s.lb_d = (float*)(base + pl.off[6]);
  s.c_id = (uint32_t*)(base + pl.off[7]);
  s.c_d = (float*)(base + pl.off[8]);
  s.s_id = (uint32_t*)(base + pl.off[9]);
  s.s_d = (float*)(base + pl.off[10]);
  s.s_lb = (int32_t*)(base + pl.off[11]);
  s.s_slb = (int32_t*)(base + pl.off[12]);
  s.sel_id = (int32_t*)(base + pl.off[13]);
  s.sel_d = (float*)(base + pl.off[14]);
  s.topk_id = (int32_t*)(base + pl.off[15]);
  s.topk_d = (float*)(base + pl.off[16]);
  s.ctrl = (int*)(base + pl.off[17]);
  s.wnew = (uint32_t*)(base + pl.off[18]);
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

// Exact squared L2 of the node (its first kVecRegs*32 elements preloaded in
// vx, lane-strided). uint8 vectors with an integral query are summed in int32
// (exact); otherwise FP32 with the reference's reduction (util.cuh:26-46).
template <class T>
__device__ __forceinline__ float exact_dist(const float* q, const T* v, const float (&vx)[kVecRegs], int dim,
                                            int lane, bool int_query, int fma) {
  if (sizeof(T) == 1 && int_query) {
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

template <class T, class TabT, int W>
__global__ void __launch_bounds__(W * 32, (W <= 4 ? 8 : 4)) batch_search_kernel(BatchParams p) {
  extern __shared__ __align__(16) uint8_t smem[];
  const BatchPlan pl(p.M, (int)sizeof(TabT), 1 << p.hash_bits, p.L_max, p.max_m, W, p.k_max, p.dim);
  const BatchSmem s = carve_batch(smem, pl);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int dim = p.dim, M = p.M, H = 1 << p.hash_bits;
  TabT* table = reinterpret_cast<TabT*>(s.table);
  const NavView nv{p.ix.nav_data, p.ix.nav_graph, p.ix.nav_map, p.nav_n, p.nav_max_m, p.nav_start, dim, p.fma,
                   p.err};
  const PqView pv{p.ix.pivots_t, p.ix.centroid, p.ix.chunk_off, M, dim, p.fma};

  for (;;) {
    if (tid == 0) s.ctrl[0] = atomicAdd(p.next_query, 1);
    __syncthreads();
    const int qid = s.ctrl[0];
    if (qid >= p.nq) break;
    const int L = p.L_per_q ? min(max(__ldg(p.L_per_q + qid), 1), p.L_max) : p.L_max;
    const int k = p.k_per_q ? min(max(__ldg(p.k_per_q + qid), 1), p.k_max) : p.k_max;
    for (int i = tid; i < dim; i += W * 32) s.q[i] = __ldg(p.queries + (size_t)qid * dim + i);
    for (int i = tid; i < H; i += W * 32) s.hash[i] = 0xffffffffu;
    __syncthreads();
    int64_t gathered = 0;  // per-warp share of the algorithmic bytes
    if (warp == 0) {
      int64_t u0 = entry_node<T>(p.has_nav, nv, p.medoid, s.q, lane, gathered);
      if (lane == 0) s.ctrl[3] = (int)u0;
    }
    if (p.tables) {  // BF16 tables built for the whole batch on the tensor cores
      copy_table(s.table, p.tables + (size_t)qid * M * kPivots, M * kPivots * 2, tid, W * 32);
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
    for (int i = tid; i < dim && iq; i += W * 32) iq = s.q[i] == rintf(s.q[i]) && s.q[i] >= 0.0f && s.q[i] <= 255.0f;
    const bool int_query = __syncthreads_and(iq) != 0;
    // The entry node starts the list, unexpanded, with its ADC distance; the
    // first step picks it (the reference expands it without listing it,
    // src/impl/pure_mem.cuh:285-287). Listing it makes every expanded node one
    // that the list has seen, so a later re-score of it is rejected whatever
    // the visited cache holds.
    const int u0 = s.ctrl[3];
    if (tid == 0) {
      s.ctrl[2] = 0;  // survivors of the current step
      s.ctrl[4] = 0;  // a repeated id among them
      s.ctrl[6] = 0;  // stop (hop limit)
      if (u0 >= 0) {
        s.hash[hash_slot((uint32_t)u0, p.hash_bits)] = (uint32_t)u0;
        s.la_id[0] = (uint32_t)u0;
        s.la_d[0] = adc_split4(table, p.ix.codes + (size_t)u0 * M, M);
      }
    }
    __syncthreads();

    // List state, identical in every thread; top-k state in warp 0.
    int sz = u0 >= 0 ? 1 : 0, found = 0, hops = 0, scan_from = 0;
    uint32_t* list_id = s.la_id;
    float* list_d = s.la_d;
    uint32_t* out_id = s.lb_id;
    float* out_d = s.lb_d;

    for (;;) {
      // Pick: every warp finds the same first W unexpanded entries (entries
      // before scan_from are expanded and have not moved) and takes its own.
      int npick = 0, my_pos = -1;
      for (int base = scan_from; base < sz && npick < W; base += 32) {
        const int i = base + lane;
        unsigned um = __ballot_sync(kFull, i < sz && !(list_id[i] & kExpanded));
        if (base == scan_from && um == 0) scan_from = min(base + 32, sz);
        while (um && npick < W) {
          const int b = __ffs(um) - 1;
          um &= um - 1;
          if (npick == warp) my_pos = base + b;
          npick++;
        }
      }
      if (npick == 0 || s.ctrl[6]) break;
      const bool full = sz == L;
      const float tail_d = full ? list_d[L - 1] : 0.0f;
      const uint32_t tail_id = full ? list_id[L - 1] : 0u;
      // Expand: warp w expands pick w. The degree word, the neighbour slots
      // (up to max_m, inside the record) and the node's vector are loaded
      // together, so the record costs one memory round trip. New neighbours
      // are scored and checked against the list here; survivors (below the
      // list's last key when it is full, not in it yet) are kept unsorted.
      if (warp < npick) {
        const int64_t u = list_id[my_pos] & kMask;
        const bool uok = u < p.n;
        const uint8_t* node = p.ix.pages + (uok ? (u / p.npp) * kPageSize + (u % p.npp) * p.node_len : 0);
        const int32_t* meta = reinterpret_cast<const int32_t*>(node + p.data_len);
        int deg = __ldg(meta);
        int ev[kEdgeRegs];
#pragma unroll
        for (int r = 0; r < kEdgeRegs; r++) ev[r] = lane + 32 * r < p.max_m ? __ldg(meta + 1 + lane + 32 * r) : -1;
        float vx[kVecRegs];
#pragma unroll
        for (int r = 0; r < kVecRegs; r++)
          vx[r] = lane + 32 * r < dim ? load_elem<T>(reinterpret_cast<const T*>(node), lane + 32 * r) : 0.0f;
        const bool ok = uok && deg >= 0 && deg <= p.max_m;
        if (!ok) {
          if (lane == 0) atomicOr(p.err, uok ? kErrBadDegree : kErrBadId);
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
        for (int r = 0; r < kEdgeRegs; r++) check(lane + 32 * r, ev[r]);
        for (int b0 = 32 * kEdgeRegs; b0 < deg; b0 += 32)
          check(b0 + lane, b0 + lane < deg ? __ldg(meta + 1 + b0 + lane) : -1);
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
        };
        // One lane per new neighbour: all of the warp's code fetches are in
        // flight at once, and no lane runs a second ADC while others idle.
        for (int i = lane; i < nnew; i += 32) {
          const uint32_t v = wnew[i];
          keep(v, adc_split4(table, p.ix.codes + (size_t)v * M, M));
        }
        const int scored = lane == 0 ? nnew : 0;
        float ed = inf_f();
        if (ok) ed = exact_dist<T>(s.q, reinterpret_cast<const T*>(node), vx, dim, lane, int_query, p.fma);
        if (lane == 0) {
          s.sel_d[warp] = ed;
          s.sel_id[warp] = (int32_t)u;
          s.c_id[warp] = (uint32_t)my_pos;  // list position of the pick (marked below)
        }
        const int sc = __reduce_add_sync(kFull, scored);
        gathered += ok ? 4 + 4 * deg + p.data_len + (int64_t)sc * M : 0;
      }
      __syncthreads();  // (1) survivors and picks are in
      const int nsv = s.ctrl[2];
      if (warp == 0) {  // mark the picks, keep the top-k
        for (int w = 0; w < npick; w++) {
          if (lane == 0) list_id[s.c_id[w]] |= kExpanded;
          if (s.sel_d[w] != inf_f()) topk_push(s.topk_d, s.topk_id, found, k, s.sel_d[w], s.sel_id[w], lane);
          hops++;
        }
        if (lane == 0 && hops > kHopCap) {
          s.ctrl[6] = 1;
          atomicOr(p.err, kErrHopCap);
        }
      }
      // Rank-sort the survivors (rank = number of smaller keys, ties by slot);
      // a repeated id (a cache eviction between two lookups) raises a flag.
      for (int j = tid; j < nsv; j += W * 32) {
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
        s.c_id[W + r] = id;  // sorted survivors after the W pick slots
        s.c_d[r] = d;
        s.s_slb[r] = s.s_lb[j];
        if (rep) s.ctrl[4] = 1;
      }
      __syncthreads();  // (2)
      uint32_t* sid = s.c_id + W;
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
      // Move old entries and survivors into the other list buffer: old entry i
      // goes to i + #{survivors inserted at or before i}, survivor r to its
      // insertion point + r; positions >= L drop.
      const int nsz = min(sz + ns, L);
      if (ns) {
        for (int i = tid; i < sz; i += W * 32) {
          int lo = 0, hi = ns;
          while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (s.s_slb[mid] <= i) lo = mid + 1; else hi = mid;
          }
          const int dst = i + lo;
          if (dst < L) {
            out_id[dst] = list_id[i];
            out_d[dst] = list_d[i];
          }
        }
        for (int r = tid; r < ns; r += W * 32) {
          const int dst = s.s_slb[r] + r;
          if (dst < L) {
            out_id[dst] = sid[r];
            out_d[dst] = s.c_d[r];
          }
        }
        const int first_new = s.s_slb[0];
        if (first_new < scan_from) scan_from = first_new;
        uint32_t* ti = list_id;
        float* td = list_d;
        list_id = out_id;
        list_d = out_d;
        out_id = ti;
        out_d = td;
      }
      sz = nsz;
      // Every thread read the survivor count after (1); the next step adds to
      // it only after (3), so it is reset here. The repeat flag is read by every
      // thread after (2) and set again only after the next (1).
      if (tid == 0) s.ctrl[2] = 0;
      __syncthreads();  // (3) the new list is complete
      if (tid == 0) s.ctrl[4] = 0;
    }
    // outputs (warp 0 holds the top-k bookkeeping)
    if (warp == 0) {
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

template <class T, class TabT, int W>
cudaError_t launch_w(const BatchParams& p, int num_sms, cudaStream_t stream) {
  const BatchPlan pl(p.M, (int)sizeof(TabT), 1 << p.hash_bits, p.L_max, p.max_m, W, p.k_max, p.dim);
  const size_t smem = pl.total;
  if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  auto kern = batch_search_kernel<T, TabT, W>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, W * 32, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  int grid = num_sms * per_sm;
  if (grid > p.nq) grid = p.nq;
  kern<<<grid, W * 32, smem, stream>>>(p);
  return cudaGetLastError();
}

template <class T, class TabT>
cudaError_t launch_t(const BatchParams& p, int W, int num_sms, cudaStream_t stream) {
  switch (W) {
    case 1: return launch_w<T, TabT, 1>(p, num_sms, stream);
    case 2: return launch_w<T, TabT, 2>(p, num_sms, stream);
    case 4: return launch_w<T, TabT, 4>(p, num_sms, stream);
    case 8: return launch_w<T, TabT, 8>(p, num_sms, stream);
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
