// PQ distance tables of a query batch on the 5th-generation tensor cores.
//
// The reference builds each query's table on CUDA cores (src/impl/pq.cuh:8-59):
// table[c][j] = sum over the dimensions i of chunk c of (q_i - mu_i - P[j][i])^2.
// Over a batch this is a block-diagonal GEMM. With r = q - mu,
//   table[q][c][j] = |r_qc|^2 - 2 r_qc . P_cj + |P_cj|^2,
// the cross term is r (queries x dims) times P^T restricted to chunk c.
//
// Layout: chunks are padded to p dimensions (p = next power of two >= the
// largest chunk, p <= 16), so G = 16 / p chunks share one K = 16 slice of the
// query operand A (128 queries x 16, BF16). For chunk c the operand B is a
// 256 x 16 tile that holds P_cj in the p columns of chunk c's slot and zeros
// elsewhere, so D = A . B^T (M = 128, N = 256, K = 16, FP32 accumulate in
// TMEM) is exactly r_qc . P_cj for the 256 centroids j of chunk c. The B tiles
// of every chunk are laid out once at index open (gann_api.cu) in the UMMA
// K-major no-swizzle canonical layout and copied per chunk with a bulk
// (1-D TMA) copy. With split3 the operands are split into BF16 hi + lo parts
// and D = A_hi B_hi + A_hi B_lo + A_lo B_hi (three MMAs into the same TMEM
// columns), which keeps the cross term close to FP32.
//
// One CTA of 128 threads handles 128 queries; thread t owns query row t (TMEM
// lane t). One elected thread issues tcgen05.mma; completion is tracked by
// tcgen05.commit on an mbarrier; the epilogue reads TMEM with tcgen05.ld,
// adds the norms, rounds to BF16 and stores the rows. The chunks of a CTA run
// as a two-stage pipeline: two B tile buffers and two TMEM accumulators (512
// columns), so while the epilogue drains chunk c, the MMAs of chunk c + 1 run
// and the B tiles of chunk c + 2 are on their way. Two CTAs on one SM take
// the tensor memory in turn (tcgen05.alloc waits until the columns are free).
// Every wait is bounded: on expiry the kernel sets kErrWaitLimit, lets its
// copies and MMAs land, frees its TMEM and returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

#include "search_common.cuh"
#include "tc_common.cuh"

namespace gann {
namespace {

using namespace tc;

struct TcParams {
  const float* queries;      // nq x dim
  int nq, dim, M, p, groups;
  const int* nq_dev;         // or null: the query count, read at run time (<= nq)
  const float* centroid;     // dim
  const int32_t* chunk_off;  // M + 1
  const uint8_t* bpanel_hi;  // M x 8 KB B tiles
  const uint8_t* bpanel_lo;  // M x 8 KB (split3)
  const float* pnorm;        // M x 256: |P_cj|^2
  int split3;
  __nv_bfloat16* tables;     // nq x M x 256
  unsigned int* err;
};

__global__ void __launch_bounds__(kTile, 1) table_tc_kernel(TcParams p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  // [A_hi groups][A_lo groups][B_hi x2][B_lo x2][rn: M x 128 floats][bars][tmem slot]
  uint8_t* a_hi = smem;
  uint8_t* a_lo = a_hi + (size_t)p.groups * kATileBytes;
  uint8_t* b_hi = a_lo + (size_t)p.groups * kATileBytes;  // stage s at b_hi + s * kBTileBytes
  uint8_t* b_lo = b_hi + 2 * kBTileBytes;
  float* rn = reinterpret_cast<float*>(b_lo + 2 * kBTileBytes);
  uint64_t* bars = reinterpret_cast<uint64_t*>(rn + (size_t)p.M * kTile);  // [0,1] B copies, [2,3] MMAs done
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 4);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int q0 = blockIdx.x * kTile;
  const int qi = q0 + tid;
  if (p.nq_dev) {  // tiles past the run-time count leave before taking tensor memory
    const int n = min(p.nq, *p.nq_dev);
    if (q0 >= n) return;
    p.nq = n;
  }
  const int G = kK / p.p;
  // chunk range of this CTA: whole groups, split over gridDim.y
  const int gpb = (p.groups + gridDim.y - 1) / gridDim.y;
  const int c_begin = min(p.M, (int)blockIdx.y * gpb * G), c_end = min(p.M, ((int)blockIdx.y + 1) * gpb * G);
  const int nc = c_end - c_begin;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int b = 0; b < 4; b++) mbar_init(&bars[b], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // A operand: residual r = q - mu of this thread's query, split BF16 hi/lo,
  // in each chunk's slot of its group; squared norms per chunk in FP32.
  for (int c = c_begin; c < c_end; c++) {
    const int b = __ldg(p.chunk_off + c), e = __ldg(p.chunk_off + c + 1);
    const int g = c / G, slot = (c % G) * p.p;
    float nrm = 0.0f;
    for (int t = 0; t < p.p; t++) {
      const int i = b + t;
      float r = 0.0f;
      if (qi < p.nq && i < e) r = __fsub_rn(__ldg(p.queries + (size_t)qi * p.dim + i), __ldg(p.centroid + i));
      nrm = __fmaf_rn(r, r, nrm);
      const __nv_bfloat16 hi = __float2bfloat16_rn(r);
      const __nv_bfloat16 lo = __float2bfloat16_rn(__fsub_rn(r, __bfloat162float(hi)));
      const int off = umma_kmajor_offset(tid, slot + t);
      *reinterpret_cast<__nv_bfloat16*>(a_hi + (size_t)g * kATileBytes + off) = hi;
      *reinterpret_cast<__nv_bfloat16*>(a_lo + (size_t)g * kATileBytes + off) = lo;
    }
    rn[(size_t)c * kTile + tid] = nrm;
  }
  // slots of a group not used by any chunk (M not a multiple of G) stay zero
  for (int c = max(p.M, c_begin); c < p.groups * G && c_end == p.M && c_begin < p.M; c++) {
    const int g = c / G, slot = (c % G) * p.p;
    for (int t = 0; t < p.p; t++) {
      const int off = umma_kmajor_offset(tid, slot + t);
      *reinterpret_cast<__nv_bfloat16*>(a_hi + (size_t)g * kATileBytes + off) = __float2bfloat16_rn(0.0f);
      *reinterpret_cast<__nv_bfloat16*>(a_lo + (size_t)g * kATileBytes + off) = __float2bfloat16_rn(0.0f);
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t b_bytes = kBTileBytes * (p.split3 ? 2u : 1u);
  // Chunk i of this CTA (c_begin + i) uses B stage i & 1 and TMEM columns
  // [256 (i & 1), + 256); both barriers of a stage complete once per use, so
  // use u = i >> 1 waits on parity u & 1.
  auto issue_copy = [&](int i) {
    const int st = i & 1, c = c_begin + i;
    mbar_expect_tx(&bars[st], b_bytes);
    bulk_copy_g2s(b_hi + st * kBTileBytes, p.bpanel_hi + (size_t)c * kBTileBytes, kBTileBytes, &bars[st]);
    if (p.split3)
      bulk_copy_g2s(b_lo + st * kBTileBytes, p.bpanel_lo + (size_t)c * kBTileBytes, kBTileBytes, &bars[st]);
  };
  // tid 0 only: wait for chunk i's B tiles, then issue its MMAs
  auto issue_mma = [&](int i) -> bool {
    const int st = i & 1, c = c_begin + i;
    if (!mbar_wait(&bars[st], (uint32_t)(i >> 1) & 1u)) return false;
    tc_fence_after();
    const int g = c / G;
    const uint32_t d = tmem + (uint32_t)(st * kN);
    const uint64_t ah = umma_desc(smem_u32(a_hi + (size_t)g * kATileBytes));
    const uint64_t bh = umma_desc(smem_u32(b_hi + st * kBTileBytes));
    umma_bf16(d, ah, bh, 0u);
    if (p.split3) {
      const uint64_t al = umma_desc(smem_u32(a_lo + (size_t)g * kATileBytes));
      const uint64_t bl = umma_desc(smem_u32(b_lo + st * kBTileBytes));
      umma_bf16(d, ah, bl, 1u);
      umma_bf16(d, al, bh, 1u);
    }
    umma_commit(&bars[2 + st]);
    return true;
  };
  bool ok = true;
  if (tid == 0 && nc > 0) {
    issue_copy(0);
    if (nc > 1) issue_copy(1);
    ok = issue_mma(0);
  }
  ok = __syncthreads_and(ok);

  for (int i = 0; i < nc && ok; i++) {
    const int st = i & 1, c = c_begin + i;
    bool mine = true;
    if (tid == 0 && i + 1 < nc) mine = issue_mma(i + 1);  // runs while this chunk drains
    mine = mine && mbar_wait(&bars[2 + st], (uint32_t)(i >> 1) & 1u);
    ok = __syncthreads_and(mine);
    if (!ok) break;
    tc_fence_after();
    if (tid == 0 && i + 2 < nc) issue_copy(i + 2);  // this stage's B tiles are free: MMA i is done
    // Epilogue: row tid of D (TMEM lane tid) -> table[qi][c][0..256)
    const float rq = rn[(size_t)c * kTile + tid];
    const float* pn = p.pnorm + (size_t)c * kN;
    __nv_bfloat16* out = p.tables + ((size_t)qi * p.M + c) * kN;
    const uint32_t dcol = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(st * kN);
    for (int col = 0; col < kN; col += 16) {
      uint32_t r[16];
      tmem_ld16(dcol + (uint32_t)col, r);
      tmem_wait_ld();
      if (qi < p.nq) {
        uint32_t packed[8];
#pragma unroll
        for (int j = 0; j < 16; j += 2) {
          const float v0 = __fmaf_rn(-2.0f, __uint_as_float(r[j]), __fadd_rn(rq, __ldg(pn + col + j)));
          const float v1 = __fmaf_rn(-2.0f, __uint_as_float(r[j + 1]), __fadd_rn(rq, __ldg(pn + col + j + 1)));
          const __nv_bfloat162 h = __floats2bfloat162_rn(fmaxf(v0, 0.0f), fmaxf(v1, 0.0f));
          packed[j >> 1] = *reinterpret_cast<const uint32_t*>(&h);
        }
        uint4* o = reinterpret_cast<uint4*>(out + col);
        o[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
        o[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
      }
    }
    tc_fence_before();
    __syncthreads();  // TMEM columns of stage st are read: chunk i + 2 may overwrite them
  }
  if (!ok && tid == 0) {
    atomicOr(p.err, kErrWaitLimit);
    // let copies and MMAs still in flight land before the memory is released
    for (int b = 0; b < 4; b++) {
      mbar_wait(&bars[b], 0);
      mbar_wait(&bars[b], 1);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// One warp per query: the CUDA-core table (FP32 accumulate in the
// reference's order, src/impl/pq.cuh:8-59), stored as TabT in global memory.
template <class TabT>
__global__ void table_cc_kernel(PqView pv, const float* queries, int nq, TabT* tables) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nq) return;
  build_table(pv, tables + (size_t)warp * pv.M * kPivots, queries + (size_t)warp * pv.dim, 0, 1, lane);
}

// BF16 table entries widened to FP32.
__global__ void bf16_to_f32(const __nv_bfloat16* in, float* out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = __bfloat162float(in[i]);
}

}  // namespace

cudaError_t launch_table_cc(const DeviceIndex& ix, int dim, int M, const float* queries, int nq, int fma,
                            bool bf16, void* tables, cudaStream_t stream) {
  const PqView pv{ix.pivots_t, ix.centroid, ix.chunk_off, M, dim, fma};
  const int grid = (nq * 32 + 127) / 128;
  if (bf16)
    table_cc_kernel<__nv_bfloat16><<<grid, 128, 0, stream>>>(pv, queries, nq, (__nv_bfloat16*)tables);
  else
    table_cc_kernel<float><<<grid, 128, 0, stream>>>(pv, queries, nq, (float*)tables);
  return cudaGetLastError();
}

cudaError_t widen_bf16(const __nv_bfloat16* in, float* out, size_t n, cudaStream_t stream) {
  bf16_to_f32<<<1024, 256, 0, stream>>>(in, out, n);
  return cudaGetLastError();
}

size_t table_tc_smem(int M, int groups) {
  return (size_t)groups * kATileBytes * 2 + (size_t)kBTileBytes * 4 + (size_t)M * kTile * 4 + 32 + 16;
}

// Host-side layout of the B operand tiles (one per chunk) and the centroid norms.
// pivots: 256 x dim row-major FP32. Returns false when a chunk is wider than 16.
bool make_tc_panels(const std::vector<float>& pivots, const std::vector<int32_t>& chunk_off, int dim,
                    std::vector<uint8_t>& hi, std::vector<uint8_t>& lo, std::vector<float>& pnorm, int& p_out,
                    int& groups_out) {
  const int M = (int)chunk_off.size() - 1;
  int smax = 0;
  for (int c = 0; c < M; c++) smax = std::max(smax, chunk_off[c + 1] - chunk_off[c]);
  int p = 1;
  while (p < smax) p <<= 1;
  if (p > kK) return false;
  const int G = kK / p;
  p_out = p;
  groups_out = (M + G - 1) / G;
  hi.assign((size_t)M * kBTileBytes, 0);
  lo.assign((size_t)M * kBTileBytes, 0);
  pnorm.assign((size_t)M * kN, 0.0f);
  for (int c = 0; c < M; c++) {
    const int b = chunk_off[c], e = chunk_off[c + 1], slot = (c % G) * p;
    for (int j = 0; j < kN; j++) {
      double nrm = 0.0;
      for (int i = b; i < e; i++) {
        const float v = pivots[(size_t)j * dim + i];
        nrm += (double)v * v;
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
        const int off = umma_kmajor_offset(j, slot + (i - b));
        *reinterpret_cast<__nv_bfloat16*>(&hi[(size_t)c * kBTileBytes + off]) = h;
        *reinterpret_cast<__nv_bfloat16*>(&lo[(size_t)c * kBTileBytes + off]) = l;
      }
      pnorm[(size_t)c * kN + j] = (float)nrm;
    }
  }
  return true;
}

cudaError_t launch_table_tc(const DeviceIndex& ix, int dim, int M, const float* queries, int nq, int split3,
                            __nv_bfloat16* tables, cudaStream_t stream, int num_sms, const int* nq_dev) {
  if (!ix.tc_bpanel_hi) return cudaErrorNotSupported;
  TcParams tp{};
  tp.queries = queries;
  tp.nq = nq;
  tp.nq_dev = nq_dev;
  tp.dim = dim;
  tp.M = M;
  tp.p = ix.tc_p;
  tp.groups = ix.tc_groups;
  tp.centroid = ix.centroid;
  tp.chunk_off = ix.chunk_off;
  tp.bpanel_hi = ix.tc_bpanel_hi;
  tp.bpanel_lo = ix.tc_bpanel_lo;
  tp.pnorm = ix.tc_pnorm;
  tp.split3 = split3;
  tp.tables = tables;
  tp.err = ix.err;
  const size_t smem = table_tc_smem(M, ix.tc_groups);
  if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  cudaError_t e = cudaFuncSetAttribute(table_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int tiles = (nq + kTile - 1) / kTile;
  int split = (num_sms + tiles - 1) / tiles;  // enough CTAs to cover every SM once
  split = std::max(1, std::min(split, ix.tc_groups));
  table_tc_kernel<<<dim3(tiles, split), kTile, smem, stream>>>(tp);
  return cudaGetLastError();
}

}  // namespace gann
