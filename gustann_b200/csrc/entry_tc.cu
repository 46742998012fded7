// Entry nodes of a query batch on the tensor cores: for every query, the
// nearest point of the pivot file (nav_index.data, translated by map.txt).
//
// The reference enters each walk through a greedy walk over the pivot graph
// with a beam of 4 (src/impl/nav.cuh:13-135). On data made of many tight
// clusters the beam fills with points of one cluster and the walk can stop in
// the wrong one, which the main walk then has to leave through its few long
// edges. The batched form may instead start from the exact nearest pivot
// (GANN_ENTRY_NEAREST_PIVOT). Over a batch that is a dense product:
//   |q - x|^2 = |q|^2 - 2 q.x + |x|^2,
// so D = Q X^T (queries x pivots, K = dim) runs on the tensor cores and an
// epilogue keeps, per query row, the smallest |x|^2 - 2 q.x and its pivot.
//
// Layout: the pivots are laid out once at index open in tiles of 256 pivots x
// dim, K padded to a multiple of 16, each 16-wide K slice an 8 KB UMMA
// K-major canonical tile (the layout of tc_common.cuh). One CTA of 128 threads
// takes 128 queries (thread t = query row t = TMEM lane t), writes its query
// rows as BF16 A slices, and walks a range of pivot tiles: tile i is copied
// into stage i & 1 by one bulk copy, its K slices are multiplied into TMEM
// columns [256 (i & 1), + 256) and committed to an mbarrier, and while the
// epilogue drains tile i the MMAs of tile i + 1 run and tile i + 2 is copied.
// The tile's 256 squared norms are loaded by the CTA's threads (two each)
// before they wait for the tile's MMAs and stored to norm slot i & 1, which
// the barrier after that wait publishes; the slot's previous reader (tile
// i - 2) finished before the barrier that ends iteration i - 2.
// The CTA's best (value, pivot) of each row is merged into a 64-bit key per
// query with atomicMin (order-preserving float bits, then the pivot index), so
// ties go to the lowest pivot index whatever the split.
//
// Exactness: for uint8 vectors and integral queries every product and partial
// sum is an integer below 2^24, so the BF16 operands and the FP32 accumulation
// are exact and the chosen pivot is the exact nearest. Float vectors and
// queries are rounded to BF16 (relative 2^-9 per element): the entry is then
// a pivot whose distance is within that rounding of the nearest, which is all
// an entry node needs. Every wait is bounded (kErrWaitLimit on expiry).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "search_common.cuh"
#include "tc_common.cuh"

namespace gann {
namespace {

using namespace tc;

struct EntryParams {
  const float* queries;  // nq x dim
  int nq, dim, nk, ntiles;
  const int* nq_dev;     // or null: the query count, read at run time (<= nq)
  const uint8_t* panel;  // ntiles x nk x 8 KB
  const float* pnorm;    // ntiles x 256: |x|^2, +inf past the last pivot
  unsigned long long* keys;  // nq, all bits set before the launch
  unsigned int* err;
};

// Float bits that order as unsigned integers in the float's order.
__device__ __forceinline__ uint32_t ordered_bits(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void __launch_bounds__(kTile, 1) entry_tc_kernel(EntryParams p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  // [A: nk x 4 KB][B: 2 stages x nk x 8 KB][norms: 2 slots x 1 KB][bars][tmem slot]
  const uint32_t tile_bytes = (uint32_t)p.nk * kBTileBytes;
  constexpr uint32_t kNormBytes = kN * 4;
  uint8_t* a = smem;
  uint8_t* b = a + (size_t)p.nk * kATileBytes;
  uint8_t* norms = b + 2 * (size_t)tile_bytes;
  uint64_t* bars = reinterpret_cast<uint64_t*>(norms + 2 * kNormBytes);  // [0,1] copies, [2,3] MMAs done
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 4);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int q0 = blockIdx.x * kTile;
  const int qi = q0 + tid;
  if (p.nq_dev) {  // tiles past the run-time count leave before taking tensor memory
    const int n = min(p.nq, *p.nq_dev);
    if (q0 >= n) return;
    p.nq = n;
  }
  const int per = (p.ntiles + (int)gridDim.y - 1) / (int)gridDim.y;
  const int t_begin = min(p.ntiles, (int)blockIdx.y * per);
  const int nt = min(p.ntiles, t_begin + per) - t_begin;
  if (nt <= 0) return;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < 4; i++) mbar_init(&bars[i], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // A operand: this thread's query row in BF16, zero past dim and past nq.
  for (int kk = 0; kk < p.nk; kk++) {
    for (int t = 0; t < kK; t++) {
      const int i = kk * kK + t;
      const float v = qi < p.nq && i < p.dim ? __ldg(p.queries + (size_t)qi * p.dim + i) : 0.0f;
      *reinterpret_cast<__nv_bfloat16*>(a + (size_t)kk * kATileBytes + umma_kmajor_offset(tid, t)) =
          __float2bfloat16_rn(v);
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  // Tile i of this CTA (t_begin + i) uses B stage i & 1 and TMEM columns
  // [256 (i & 1), + 256); each barrier of a stage completes once per use, so
  // use u = i >> 1 waits on parity u & 1.
  auto issue_copy = [&](int i) {
    const int st = i & 1;
    mbar_expect_tx(&bars[st], tile_bytes);
    bulk_copy_g2s(b + (size_t)st * tile_bytes, p.panel + (size_t)(t_begin + i) * tile_bytes, tile_bytes, &bars[st]);
  };
  // tid 0 only: wait for tile i's B slices, then issue its MMAs
  auto issue_mma = [&](int i) -> bool {
    const int st = i & 1;
    if (!mbar_wait(&bars[st], (uint32_t)(i >> 1) & 1u)) return false;
    tc_fence_after();
    const uint32_t d = tmem + (uint32_t)(st * kN);
    for (int kk = 0; kk < p.nk; kk++) {
      const uint64_t ad = umma_desc(smem_u32(a + (size_t)kk * kATileBytes));
      const uint64_t bd = umma_desc(smem_u32(b + (size_t)st * tile_bytes + (size_t)kk * kBTileBytes));
      umma_bf16(d, ad, bd, kk > 0 ? 1u : 0u);
    }
    umma_commit(&bars[2 + st]);
    return true;
  };
  bool ok = true;
  if (tid == 0) {
    issue_copy(0);
    if (nt > 1) issue_copy(1);
    ok = issue_mma(0);
  }
  ok = __syncthreads_and(ok);

  float best = inf_f();
  uint32_t best_j = 0xffffffffu;
  for (int i = 0; i < nt && ok; i++) {
    const int st = i & 1;
    bool mine = true;
    const float* pn = p.pnorm + (size_t)(t_begin + i) * kN;
    const float n0 = __ldg(pn + tid), n1 = __ldg(pn + kTile + tid);  // in flight during the waits below
    if (tid == 0 && i + 1 < nt) mine = issue_mma(i + 1);  // runs while this tile drains
    mine = mine && mbar_wait(&bars[2 + st], (uint32_t)(i >> 1) & 1u);
    float* ns = reinterpret_cast<float*>(norms + (size_t)st * kNormBytes);
    ns[tid] = n0;
    ns[kTile + tid] = n1;
    ok = __syncthreads_and(mine);
    if (!ok) break;
    tc_fence_after();
    if (tid == 0 && i + 2 < nt) issue_copy(i + 2);  // this stage's B slices are free: MMA i is done
    // Epilogue: row tid of D (TMEM lane tid), |x_j|^2 - 2 q.x_j over the tile's 256 pivots
    const float4* pn4 = reinterpret_cast<const float4*>(norms + (size_t)st * kNormBytes);
    const uint32_t j0 = (uint32_t)(t_begin + i) * kN;
    const uint32_t dcol = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(st * kN);
    for (int col = 0; col < kN; col += 32) {
      uint32_t r[32];
      tmem_ld32(dcol + (uint32_t)col, r);
      tmem_wait_ld();
#pragma unroll
      for (int j4 = 0; j4 < 8; j4++) {
        const float4 n4 = pn4[(col >> 2) + j4];  // the same address in every thread: a broadcast
        const float nj[4] = {n4.x, n4.y, n4.z, n4.w};
#pragma unroll
        for (int t = 0; t < 4; t++) {
          const int j = 4 * j4 + t;
          const float v = __fmaf_rn(-2.0f, __uint_as_float(r[j]), nj[t]);
          if (v < best) {  // strict: the first (lowest) pivot of equal values stays
            best = v;
            best_j = j0 + (uint32_t)(col + j);
          }
        }
      }
    }
    tc_fence_before();
    __syncthreads();  // TMEM columns of stage st are read: tile i + 2 may overwrite them
  }
  if (ok && qi < p.nq && best_j != 0xffffffffu)
    atomicMin(p.keys + qi, ((unsigned long long)ordered_bits(best) << 32) | best_j);
  if (!ok && tid == 0) {
    atomicOr(p.err, kErrWaitLimit);
    // let copies and MMAs still in flight land before the memory is released
    for (int i = 0; i < 4; i++) {
      mbar_wait(&bars[i], 0);
      mbar_wait(&bars[i], 1);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// Pivot row and node id of every key (gann_nearest_pivots).
__global__ void entry_ids_kernel(const unsigned long long* keys, int nq, const int32_t* nav_map, int nav_n,
                                 int32_t* pivot, int32_t* node, unsigned int* err) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
    const uint32_t local = (uint32_t)keys[q];
    const bool ok = local < (uint32_t)nav_n;
    if (!ok) atomicOr(err, kErrBadId);
    if (pivot) pivot[q] = ok ? (int32_t)local : -1;
    if (node) node[q] = ok ? __ldg(nav_map + local) : -1;
  }
}

}  // namespace

cudaError_t launch_entry_ids(const DeviceIndex& ix, int nav_n, const unsigned long long* keys, int nq, int32_t* pivot,
                             int32_t* node, cudaStream_t stream) {
  entry_ids_kernel<<<(nq + 255) / 256, 256, 0, stream>>>(keys, nq, ix.nav_map, nav_n, pivot, node, ix.err);
  return cudaGetLastError();
}

size_t entry_tc_smem(int nk) { return (size_t)nk * (kATileBytes + 2 * kBTileBytes) + 2 * kN * 4 + 32 + 16; }

// Host layout of the pivot tiles and their squared norms. data: nav_n x dim
// elements of elt bytes (uint8 or float32). Pivots past nav_n are zero with an
// infinite norm, so they never win.
void make_entry_panels(const std::vector<uint8_t>& data, int nav_n, int dim, int elt, std::vector<uint8_t>& panel,
                       std::vector<float>& pnorm, int& nk_out, int& ntiles_out) {
  const int nk = (dim + kK - 1) / kK;
  const int ntiles = (nav_n + kN - 1) / kN;
  nk_out = nk;
  ntiles_out = ntiles;
  const size_t tile_bytes = (size_t)nk * kBTileBytes;
  panel.assign((size_t)ntiles * tile_bytes, 0);
  pnorm.assign((size_t)ntiles * kN, INFINITY);
  for (int j = 0; j < nav_n; j++) {
    const size_t t = (size_t)(j / kN);
    const int row = j % kN;
    double nrm = 0.0;
    for (int i = 0; i < dim; i++) {
      float v;
      if (elt == 1) {
        v = (float)data[(size_t)j * dim + i];
      } else {
        std::memcpy(&v, &data[((size_t)j * dim + i) * 4], 4);
      }
      const __nv_bfloat16 h = __float2bfloat16_rn(v);
      const double hv = (double)__bfloat162float(h);
      nrm += hv * hv;
      const size_t off = t * tile_bytes + (size_t)(i / kK) * kBTileBytes + (size_t)umma_kmajor_offset(row, i % kK);
      std::memcpy(&panel[off], &h, 2);
    }
    pnorm[(size_t)j] = (float)nrm;
  }
}

cudaError_t launch_entry_tc(const DeviceIndex& ix, int dim, const float* queries, int nq, unsigned long long* keys,
                            cudaStream_t stream, int num_sms, const int* nq_dev) {
  if (!ix.entry_panel) return cudaErrorNotSupported;
  const size_t smem = entry_tc_smem(ix.entry_nk);
  if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  cudaError_t e = cudaMemsetAsync(keys, 0xff, sizeof(unsigned long long) * (size_t)nq, stream);
  if (e != cudaSuccess) return e;
  EntryParams ep{};
  ep.queries = queries;
  ep.nq = nq;
  ep.dim = dim;
  ep.nk = ix.entry_nk;
  ep.ntiles = ix.entry_tiles;
  ep.nq_dev = nq_dev;
  ep.panel = ix.entry_panel;
  ep.pnorm = ix.entry_pnorm;
  ep.keys = keys;
  ep.err = ix.err;
  e = cudaFuncSetAttribute(entry_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int tiles = (nq + kTile - 1) / kTile;
  int split = (num_sms + tiles - 1) / tiles;  // enough CTAs to cover every SM once
  split = std::max(1, std::min(split, ix.entry_tiles));
  entry_tc_kernel<<<dim3(tiles, split), kTile, smem, stream>>>(ep);
  return cudaGetLastError();
}

}  // namespace gann
