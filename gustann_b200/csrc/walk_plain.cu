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

#include "search_common.cuh"

namespace gann {
namespace {

struct WarpSmem {
  float* table;       // M x 256
  float* q;           // dim: the query, then the restored query
  uint32_t* la_id;    // L   sorted candidate list (ping)
  float* la_d;
  uint32_t* lb_id;    // L   (pong)
  float* lb_d;
  uint32_t* new_id;   // max_m  neighbours of the node being expanded, then the survivors
  float* new_d;
  uint32_t* sv_id;    // max_m  surviving neighbours, sorted
  float* sv_d;
  int32_t* sv_lb;     // max_m  their insertion points in the old list
  int32_t* sv_slb;    // max_m  insertion points in sorted order
  int32_t* topk_id;   // k
  float* topk_d;
};

// Byte offsets of the arrays above inside one warp's slice (host and device).
struct SmemPlan {
  size_t off[14];
  size_t total;
  __host__ __device__ SmemPlan(int M, int L, int max_m, int k, int dim) {
    const size_t sz[14] = {sizeof(float) * (size_t)M * kPivots, sizeof(float) * (size_t)dim, 4 * (size_t)L,
                           4 * (size_t)L, 4 * (size_t)L, 4 * (size_t)L, 4 * (size_t)max_m, 4 * (size_t)max_m,
                           4 * (size_t)max_m, 4 * (size_t)max_m, 4 * (size_t)max_m, 4 * (size_t)max_m,
                           4 * (size_t)k, 4 * (size_t)k};
    size_t o = 0;
    for (int i = 0; i < 14; i++) {
      off[i] = o;
      o = align16(o + sz[i]);
    }
    total = o;
  }
};

__device__ WarpSmem carve(uint8_t* base, int M, int L, int max_m, int k, int dim) {
  const SmemPlan pl(M, L, max_m, k, dim);
  WarpSmem s;
  s.table = (float*)(base + pl.off[0]);
  s.q = (float*)(base + pl.off[1]);
  s.la_id = (uint32_t*)(base + pl.off[2]);
  s.la_d = (float*)(base + pl.off[3]);
  s.lb_id = (uint32_t*)(base + pl.off[4]);
  s.lb_d = (float*)(base + pl.off[5]);
  s.new_id = (uint32_t*)(base + pl.off[6]);
  s.new_d = (float*)(base + pl.off[7]);
  s.sv_id = (uint32_t*)(base + pl.off[8]);
  s.sv_d = (float*)(base + pl.off[9]);
  s.sv_lb = (int32_t*)(base + pl.off[10]);
  s.sv_slb = (int32_t*)(base + pl.off[11]);
  s.topk_id = (int32_t*)(base + pl.off[12]);
  s.topk_d = (float*)(base + pl.off[13]);
  return s;
}

template <class T>
__device__ void search_query(const PlainParams& p, const WarpSmem& s, int qid, int lane) {
  const int dim = p.dim, L = p.L, k = p.k, max_m = p.max_m, M = p.M;
  const float* qg = p.queries + (size_t)qid * dim;
  for (int i = lane; i < dim; i += 32) s.q[i] = __ldg(qg + i);
  __syncwarp();

  int64_t gathered = 0;  // algorithmic bytes: records, neighbour ids, codes, pivot vectors
  const NavView nv{p.ix.nav_data, p.ix.nav_graph, p.ix.nav_map, p.nav_n, p.nav_max_m, p.nav_start, dim,
                   p.fma_exact, p.err};
  int64_t u = entry_node<T>(p.has_nav, nv, p.medoid, s.q, lane, gathered);  // pure_mem.cu:106-124
  const PqView pv{p.ix.pivots_t, p.ix.centroid, p.ix.chunk_off, M, dim, p.fma_table};
  build_table(pv, s.table, s.q, 0, 1, lane);
  __syncwarp();
  restore_query(pv, s.q, lane, 32);
  __syncwarp();

  int sz = 0, found = 0, hops = 0;
  uint32_t* list_id = s.la_id;
  float* list_d = s.la_d;
  uint32_t* out_id_l = s.lb_id;
  float* out_d_l = s.lb_d;
  while (u >= 0) {  // pure_mem.cuh:287-428
    if (u >= p.n) {
      if (lane == 0) atomicOr(p.err, kErrBadId);
      break;
    }
    if (hops >= kHopCap) {
      if (lane == 0) atomicOr(p.err, kErrHopCap);
      break;
    }
    const uint8_t* node = record_at(p.ix, u / p.npp, (u % p.npp) * p.node_len, u);
    const int32_t* meta = reinterpret_cast<const int32_t*>(node + p.data_len);
    // The neighbour slots (the record holds max_m of them) load with the
    // degree word, so a hop costs one round trip for the record and one for
    // the codes.
    const int e0 = lane < max_m ? __ldg(meta + 1 + lane) : -1;
    const int e1 = lane + 32 < max_m ? __ldg(meta + 1 + lane + 32) : -1;
    const int deg = __ldg(meta);
    if (deg < 0 || deg > max_m) {
      if (lane == 0) atomicOr(p.err, kErrBadDegree);
      break;
    }
    // ADC of every neighbour (pure_mem.cuh:294-310), each a sequential FP32
    // sum in chunk order.
    bool bad = false;
    if (M == 32 && max_m <= 64) {  // both code words of both neighbours of a lane in flight at once
      const bool h0 = lane < deg, h1 = lane + 32 < deg;
      const bool ok0 = h0 && (unsigned)e0 < (unsigned)p.n, ok1 = h1 && (unsigned)e1 < (unsigned)p.n;
      bad = (h0 && !ok0) || (h1 && !ok1);
      uint4 a0 = make_uint4(0, 0, 0, 0), b0 = a0, a1 = a0, b1 = a0;
      if (ok0) {
        const uint4* c = reinterpret_cast<const uint4*>(p.ix.codes + (size_t)e0 * 32);
        a0 = __ldg(c);
        b0 = __ldg(c + 1);
      }
      if (ok1) {
        const uint4* c = reinterpret_cast<const uint4*>(p.ix.codes + (size_t)e1 * 32);
        a1 = __ldg(c);
        b1 = __ldg(c + 1);
      }
      if (h0) {
        s.new_id[lane] = (uint32_t)e0;
        s.new_d[lane] = ok0 ? adc32_seq(s.table, a0, b0) : inf_f();
      }
      if (h1) {
        s.new_id[lane + 32] = (uint32_t)e1;
        s.new_d[lane + 32] = ok1 ? adc32_seq(s.table, a1, b1) : inf_f();
      }
    } else {
      for (int t = lane; t < deg; t += 32) {
        const int v = t < 32 ? e0 : t < 64 ? e1 : __ldg(meta + 1 + t);
        float d = inf_f();
        if ((unsigned)v < (unsigned)p.n)
          d = adc(s.table, p.ix.codes + (size_t)v * M, M);
        else
          bad = true;
        s.new_id[t] = (uint32_t)v;
        s.new_d[t] = d;
      }
    }
    if (__any_sync(kFull, bad)) {
      if (lane == 0) atomicOr(p.err, kErrBadId);
      break;
    }
    gathered += 4 + 4 * deg + p.data_len + (int64_t)deg * M;
    __syncwarp();
    // Merge the new entries into the sorted list. The reference merges all of
    // them (pure_mem.cuh:314-376), cuts the result at 2L (:377), drops ids equal
    // to their predecessor (a new copy always lands right after the old one,
    // :358-360) and keeps L entries (:416). The same list results from
    // inserting only the survivors: entries whose id is not in the list yet and
    // whose key (dist, id) is below the list's last key when the list is full.
    const bool full = sz == L;
    const float tail_d = full ? list_d[L - 1] : 0.0f;
    const uint32_t tail_id = full ? list_id[L - 1] : 0u;
    int nsv = 0;
    for (int base = 0; base < deg; base += 32) {
      const int t = base + lane;
      bool keep = false;
      float d = 0.0f;
      uint32_t id = 0;
      int lb = 0;
      if (t < deg) {
        d = s.new_d[t];
        id = s.new_id[t];
        keep = !full || key_less(d, id, tail_d, tail_id);
        if (keep) {
          lb = lower_bound_key(list_d, list_id, 0, sz, d, id);
          if (lb < sz && ((list_id[lb] ^ id) & kMask) == 0) keep = false;
        }
      }
      const unsigned km = __ballot_sync(kFull, keep);
      if (keep) {
        const int slot = nsv + __popc(km & ((1u << lane) - 1));
        s.sv_id[slot] = id;  // unsorted survivors (rank-sorted below)
        s.sv_d[slot] = d;
        s.sv_lb[slot] = lb;
      }
      nsv += __popc(km);
    }
    __syncwarp();
    // Rank-sort the survivors by key into new_* (ids are distinct, so the
    // rank is the count of smaller keys); carry the insertion points along.
    for (int j = lane; j < nsv; j += 32) {
      const float d = s.sv_d[j];
      const uint32_t id = s.sv_id[j];
      int r = 0;
      for (int f = 0; f < nsv; f++) {
        const float fd = s.sv_d[f];
        const uint32_t fi = s.sv_id[f];
        r += key_less(fd, fi, d, id) || (fd == d && ((fi ^ id) & kMask) == 0 && f < j);
      }
      s.new_id[r] = id;
      s.new_d[r] = d;
      s.sv_slb[r] = s.sv_lb[j];
    }
    __syncwarp();
    // Old entry i moves to i + #{survivors with insertion point <= i};
    // survivor r (sorted) goes to its insertion point + r. Positions >= L drop.
    const int nsz = min(sz + nsv, L);
    const int32_t* slb = s.sv_slb;
    if (nsv == 0) {  // list unchanged: keep it in place
      uint32_t* ti = list_id;
      float* td = list_d;
      list_id = out_id_l;
      list_d = out_d_l;
      out_id_l = ti;
      out_d_l = td;
    }
    for (int i = lane; nsv && i < sz; i += 32) {
      int lo = 0, hi = nsv;  // upper_bound of i in the non-decreasing slb
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (slb[mid] <= i) lo = mid + 1; else hi = mid;
      }
      const int dst = i + lo;
      if (dst < L) {
        out_id_l[dst] = list_id[i];
        out_d_l[dst] = list_d[i];
      }
    }
    for (int r = lane; r < nsv; r += 32) {
      const int dst = slb[r] + r;
      if (dst < L) {
        out_id_l[dst] = s.new_id[r];
        out_d_l[dst] = s.new_d[r];
      }
    }
    __syncwarp();
    // First entry without the expanded bit (pure_mem.cuh:380-419).
    int best = INT_MAX;
    for (int base = 0; base < nsz; base += 32) {
      const int i = base + lane;
      const unsigned um = __ballot_sync(kFull, i < nsz && !(out_id_l[i] & kExpanded));
      if (um) {
        best = base + __ffs(um) - 1;
        break;
      }
    }
    // Exact distance of this node and top-k insertion (pure_mem.cuh:420-424).
    const float ed = warp_exact<T>(s.q, reinterpret_cast<const T*>(node), dim, lane, p.fma_exact);
    topk_push(s.topk_d, s.topk_id, found, k, ed, (int)u, lane);
    hops++;
    // No unexpanded entry: with a list of L entries the reference stops; with a
    // shorter list it reads stale slots, and the walk stops here.
    if (best >= L) {
      u = -1;
    } else {
      u = (int64_t)out_id_l[best];
      __syncwarp();
      if (lane == 0) out_id_l[best] |= kExpanded;
      sz = nsz;
      // swap the ping-pong lists
      uint32_t* ti = list_id;
      float* td = list_d;
      list_id = out_id_l;
      list_d = out_d_l;
      out_id_l = ti;
      out_d_l = td;
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
  return SmemPlan(M, L, max_m, k, dim).total;
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
