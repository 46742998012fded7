/*
 * gann_oracle.c -- CPU restatement of GustANN's all-in-GPU (`search_mem -G`)
 * search path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker for the CUDA product
 * (gustann_b200/libgann.so) and the timed CPU baseline. The product never
 * links, loads or calls it; only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline / reference legs do.
 *
 * Parity pinning: the outputs of this file are compared, on a B200, with the
 * reference's own kernels compiled from its sources (oracle/build_ref.sh), and
 * the resulting golden vectors are committed under tests/golden/.
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the GustANN project root). The search arithmetic is FP32 in the reference's
 * order. Two sites may be contracted into FMA by nvcc in the reference build
 * (src/impl/pq.cuh:40 and src/impl/util.cuh:37); each has a switch here.
 * Build with -ffp-contract=off so that the switch is the only source of FMA.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

#define ORC_MASK 0x7fffffffu
#define ORC_BIT 0x80000000u
#define ORC_PAGE 4096
#define ORC_PIVOTS 256

/* per-query flags reported by orc_search / orc_walk */
#define ORC_F_REF_UNDEFINED 1  /* list exhausted while shorter than L: reference reads stale memory */
#define ORC_F_KEY_COLLISION 2  /* duplicate neighbour ids in one record: reference merge collides */
#define ORC_F_BAD_ID 4         /* neighbour / entry id out of range */
#define ORC_F_BAD_DEG 8        /* degree word > max_m0 */
#define ORC_F_HOP_CAP 16       /* hop cap reached (runaway walk) */
#define ORC_F_NAV_CAP 32       /* nav iteration cap reached */

static __thread char g_err[512];
const char* orc_last_error(void) { return g_err; }
static int fail(const char* msg, const char* arg) {
  snprintf(g_err, sizeof g_err, "%s%s%s", msg, arg ? ": " : "", arg ? arg : "");
  return -1;
}

typedef struct {
  int dtype; /* 0 = uint8, 1 = float (src/common.hpp:22-25) */
  int elt;
  int64_t n, dim, medoid, node_len, npp, max_m0, data_len, num_pages;
  uint8_t* pages; /* num_pages x 4096, the file after its first sector */
  int pq_n, pq_m, pq_dim;
  uint8_t* codes;    /* pq_n x pq_m */
  float* pivots_t;   /* dim x 256 */
  float* centroid;   /* dim */
  int* chunk_id;     /* dim */
  int has_nav;
  int nav_n, nav_dim, nav_max_m, nav_start;
  uint8_t* nav_data; /* nav_n x nav_dim x elt */
  int* nav_graph;    /* nav_n x nav_max_m, padded with -1 */
  int* nav_map;      /* nav_n */
} orc_index;

/* ---------------------------------------------------------------- readers */

/* Layout::parse_diskann_metadata, src/layout.cpp:11-69 */
static int read_layout(orc_index* ix, const char* path) {
  FILE* f = fopen(path, "rb");
  if (!f) return fail("cannot open index file", path);
  uint32_t nr = 0, nc = 0;
  uint64_t v[8];
  if (fread(&nr, 4, 1, f) != 1 || fread(&nc, 4, 1, f) != 1 || fread(v, 8, 8, f) != 8) {
    fclose(f);
    return fail("short index header", path);
  }
  ix->n = (int64_t)v[0];
  ix->dim = (int64_t)v[1];
  ix->medoid = (int64_t)v[2];
  ix->node_len = (int64_t)v[3];
  ix->npp = (int64_t)v[4];
  ix->data_len = ix->dim * ix->elt;
  ix->max_m0 = (ix->node_len - ix->data_len) / 4 - 1; /* layout.cpp:46 */
  if (ix->npp <= 0 || ix->n <= 0 || ix->dim <= 0 || ix->max_m0 < 0) {
    fclose(f);
    return fail("invalid index header", path);
  }
  ix->num_pages = (ix->n + ix->npp - 1) / ix->npp;
  size_t bytes = (size_t)ix->num_pages * ORC_PAGE;
  ix->pages = (uint8_t*)malloc(bytes);
  /* PureMemExecutor::read_to_mem, src/pure_mem.cu:45-55: pages after the first sector */
  if (!ix->pages || fseek(f, ORC_PAGE, SEEK_SET) != 0 || fread(ix->pages, 1, bytes, f) != bytes) {
    fclose(f);
    return fail("short index body", path);
  }
  fclose(f);
  return 0;
}

/* read_bin, src/pq_search.cu:187-201: int npts, int ndim, then npts*ndim items */
static void* read_bin(const char* path, size_t off, size_t elt, int* npts, int* ndim) {
  FILE* f = fopen(path, "rb");
  if (!f) return NULL;
  void* data = NULL;
  if (fseek(f, (long)off, SEEK_SET) == 0 && fread(npts, 4, 1, f) == 1 && fread(ndim, 4, 1, f) == 1 &&
      *npts >= 0 && *ndim >= 0) {
    size_t len = (size_t)*npts * (size_t)*ndim;
    data = malloc(len * elt + 1);
    if (data && fread(data, elt, len, f) != len) {
      free(data);
      data = NULL;
    }
  }
  fclose(f);
  return data;
}

/* PQSearch::read_data, src/pq_search.cu:56-121 */
static int read_pq(orc_index* ix, const char* pq_prefix) {
  char piv[4096], cmp[4096];
  snprintf(piv, sizeof piv, "%s_pivots.bin", pq_prefix); /* src/ssd_search.cu:61-63 */
  snprintf(cmp, sizeof cmp, "%s_compressed.bin", pq_prefix);
  int nr, nc;
  ix->codes = (uint8_t*)read_bin(cmp, 0, 1, &ix->pq_n, &ix->pq_m);
  if (!ix->codes) return fail("cannot read PQ codes", cmp);
  uint64_t* offs = (uint64_t*)read_bin(piv, 0, 8, &nr, &nc);
  if (!offs) return fail("cannot read PQ pivots", piv);
  if (!((nr == 4 || nr == 5) && nc == 1)) { /* pq_search.cu:77-79 */
    free(offs);
    return fail("PQ offsets table must be 4 or 5 x 1", piv);
  }
  int legacy = nr == 5;
  float* pivots = (float*)read_bin(piv, offs[0], 4, &nr, &ix->pq_dim);
  if (!pivots || nr != ORC_PIVOTS) {
    free(offs);
    free(pivots);
    return fail("PQ pivots must be 256 x dim", piv);
  }
  ix->pivots_t = (float*)malloc(sizeof(float) * ORC_PIVOTS * ix->pq_dim);
  for (int i = 0; i < ORC_PIVOTS; i++) /* transpose, pq_search.cu:86-91 */
    for (int j = 0; j < ix->pq_dim; j++) ix->pivots_t[(size_t)j * ORC_PIVOTS + i] = pivots[(size_t)i * ix->pq_dim + j];
  free(pivots);
  ix->centroid = (float*)read_bin(piv, offs[1], 4, &nr, &nc);
  if (!ix->centroid || nr != ix->pq_dim || nc != 1) {
    free(offs);
    return fail("PQ centroid must be dim x 1", piv);
  }
  int* chunk_offsets = (int*)read_bin(piv, offs[legacy ? 3 : 2], 4, &nr, &nc);
  free(offs);
  if (!chunk_offsets || nr != ix->pq_m + 1 || nc != 1) {
    free(chunk_offsets);
    return fail("PQ chunk offsets must be (M+1) x 1", piv);
  }
  ix->chunk_id = (int*)malloc(sizeof(int) * ix->pq_dim);
  for (int i = 0; i < ix->pq_dim; i++) ix->chunk_id[i] = -1; /* pq_search.cu:110 */
  for (int c = 0; c < ix->pq_m; c++)
    for (int j = chunk_offsets[c]; j < chunk_offsets[c + 1]; j++)
      if (j >= 0 && j < ix->pq_dim) ix->chunk_id[j] = c;
  free(chunk_offsets);
  for (int i = 0; i < ix->pq_dim; i++)
    if (ix->chunk_id[i] < 0) return fail("PQ chunk offsets leave a dimension unassigned", piv);
  return 0;
}

/* NavGraph::init, src/nav_graph.cu:41-100 */
static int read_nav(orc_index* ix, const char* dir) {
  char pidx[4096], pdat[4096], pmap[4096];
  snprintf(pidx, sizeof pidx, "%s/nav_index", dir); /* src/ssd_search.cu:72-75 */
  snprintf(pdat, sizeof pdat, "%s/nav_index.data", dir);
  snprintf(pmap, sizeof pmap, "%s/map.txt", dir);
  FILE* f = fopen(pdat, "rb");
  if (!f) return fail("cannot open nav data", pdat);
  if (fread(&ix->nav_n, 4, 1, f) != 1 || fread(&ix->nav_dim, 4, 1, f) != 1 || ix->nav_n <= 0) {
    fclose(f);
    return fail("short nav data header", pdat);
  }
  size_t bytes = (size_t)ix->nav_n * ix->nav_dim * ix->elt;
  ix->nav_data = (uint8_t*)malloc(bytes);
  if (fread(ix->nav_data, 1, bytes, f) != bytes) {
    fclose(f);
    return fail("short nav data", pdat);
  }
  fclose(f);
  f = fopen(pmap, "r");
  if (!f) return fail("cannot open nav map", pmap);
  ix->nav_map = (int*)malloc(sizeof(int) * ix->nav_n);
  for (int i = 0; i < ix->nav_n; i++)
    if (fscanf(f, "%d", &ix->nav_map[i]) != 1) {
      fclose(f);
      return fail("short nav map", pmap);
    }
  fclose(f);
  f = fopen(pidx, "rb");
  if (!f) return fail("cannot open nav index", pidx);
  int hdr[6];
  if (fread(hdr, 4, 6, f) != 6) {
    fclose(f);
    return fail("short nav index header", pidx);
  }
  ix->nav_max_m = hdr[2]; /* nav_graph.cu:79-80 */
  ix->nav_start = hdr[3];
  if (!(ix->nav_max_m > 0 && ix->nav_max_m <= 32)) {
    fclose(f);
    return fail("nav max degree must be in 1..32", pidx);
  }
  ix->nav_graph = (int*)malloc(sizeof(int) * (size_t)ix->nav_n * ix->nav_max_m);
  for (int i = 0; i < ix->nav_n; i++) {
    int d;
    int* row = ix->nav_graph + (size_t)i * ix->nav_max_m;
    if (fread(&d, 4, 1, f) != 1 || d <= 0 || d > ix->nav_max_m || fread(row, 4, (size_t)d, f) != (size_t)d) {
      fclose(f);
      return fail("bad nav adjacency record", pidx);
    }
    for (int j = d; j < ix->nav_max_m; j++) row[j] = -1; /* nav_graph.cu:91 */
  }
  fclose(f);
  ix->has_nav = 1;
  return 0;
}

void orc_close(orc_index* ix) {
  if (!ix) return;
  free(ix->pages);
  free(ix->codes);
  free(ix->pivots_t);
  free(ix->centroid);
  free(ix->chunk_id);
  free(ix->nav_data);
  free(ix->nav_graph);
  free(ix->nav_map);
  free(ix);
}

/* GustANN::init_gustann_internal + PureMemExecutor ctor, src/ssd_search.cu:55-79,108-112 */
int orc_open(const char* index_file, const char* pq_prefix, const char* nav_dir, int dtype, orc_index** out) {
  *out = NULL;
  if (dtype != 0 && dtype != 1) return fail("dtype must be 0 (uint8) or 1 (float)", NULL);
  orc_index* ix = (orc_index*)calloc(1, sizeof(orc_index));
  ix->dtype = dtype;
  ix->elt = dtype == 0 ? 1 : 4;
  if (read_layout(ix, index_file) || read_pq(ix, pq_prefix) ||
      (nav_dir && nav_dir[0] && read_nav(ix, nav_dir))) {
    orc_close(ix);
    return -1;
  }
  if (ix->pq_dim != ix->dim || ix->pq_n != ix->n) { /* PQSearch::init_device asserts, pq_search.cu:124-125 */
    orc_close(ix);
    return fail("PQ data does not match the index (dim or point count)", NULL);
  }
  if (ix->has_nav && ix->nav_dim != ix->dim) {
    orc_close(ix);
    return fail("nav data dimension does not match the index", NULL);
  }
  *out = ix;
  return 0;
}

/* n, dim, medoid, node_len, npp, max_m0, num_pages, pq_m, has_nav, nav_n, nav_max_m, nav_start */
void orc_info(const orc_index* ix, int64_t* o) {
  o[0] = ix->n; o[1] = ix->dim; o[2] = ix->medoid; o[3] = ix->node_len; o[4] = ix->npp;
  o[5] = ix->max_m0; o[6] = ix->num_pages; o[7] = ix->pq_m; o[8] = ix->has_nav;
  o[9] = ix->nav_n; o[10] = ix->nav_max_m; o[11] = ix->nav_start;
}

/* ------------------------------------------------------------- arithmetic */

static inline float elem(const void* v, int dtype, int64_t i) {
  return dtype == 0 ? (float)((const uint8_t*)v)[i] : ((const float*)v)[i];
}

/* square_sum_32, src/impl/util.cuh:26-46: lane-strided partial sums, then a
 * __shfl_down_sync tree with offsets 16,8,4,2,1; the result is lane 0's. */
float orc_exact_dist(const float* a, const void* b, int dtype, int dim, int fma) {
  float lane[32];
  for (int l = 0; l < 32; l++) {
    float v = 0.0f;
    for (int i = l; i < dim; i += 32) {
      float d = a[i] - elem(b, dtype, i);
      v = fma ? fmaf(d, d, v) : v + d * d; /* util.cuh:36-38 */
    }
    lane[l] = v;
  }
  for (int off = 16; off > 0; off >>= 1) /* util.cuh:41-44 */
    for (int l = 0; l + off < 32; l++) lane[l] = lane[l] + lane[l + off];
  return lane[0];
}

/* PQSearchData::init_query, src/impl/pq.cuh:8-59. The table is accumulated in
 * dimension order; q is shifted by the centroid in place and restored after,
 * and the restored value (which may differ from q by an ulp) is what the
 * exact distance later uses (src/impl/pure_mem.cuh:421). */
void orc_pq_table(const orc_index* ix, const float* q, int fma, float* table, float* q_restored) {
  const int dim = (int)ix->dim, M = ix->pq_m;
  memset(table, 0, sizeof(float) * (size_t)M * ORC_PIVOTS); /* pq.cuh:12-14 */
  float* qc = (float*)malloc(sizeof(float) * dim);
  for (int i = 0; i < dim; i++) qc[i] = q[i] - ix->centroid[i]; /* pq.cuh:22-24 */
  for (int i = 0; i < dim; i++) {                                 /* pq.cuh:35-43 */
    float* row = table + (size_t)ix->chunk_id[i] * ORC_PIVOTS;
    const float* pt = ix->pivots_t + (size_t)i * ORC_PIVOTS;
    for (int j = 0; j < ORC_PIVOTS; j++) {
      float d = qc[i] - pt[j];
      row[j] = fma ? fmaf(d, d, row[j]) : row[j] + d * d;
    }
  }
  for (int i = 0; i < dim; i++) q_restored[i] = qc[i] + ix->centroid[i]; /* pq.cuh:54-56 */
  free(qc);
}

/* ADC over one code, src/impl/pure_mem.cuh:302-309: sequential FP32 adds. */
static inline float adc(const float* table, const uint8_t* code, int M) {
  float d = 0.0f;
  for (int j = 0; j < M; j++) d += table[j * ORC_PIVOTS + code[j]];
  return d;
}

/* lower_bound on the key (dist, id & 0x7fffffff), src/impl/util.cuh:166-178 */
static inline int lower_bound_key(const float* dist, const uint32_t* id, int l, int r, float d, uint32_t x) {
  x &= ORC_MASK;
  while (l < r) {
    int mid = (l + r) / 2;
    if (dist[mid] < d || (dist[mid] == d && (id[mid] & ORC_MASK) < x))
      l = mid + 1;
    else
      r = mid;
  }
  return l;
}

/* retset_push_32, src/impl/util.cuh:116-163, restated by its result: the value
 * goes after every entry whose distance is <= value; entries past max_size
 * fall off; size grows by one up to max_size. */
static void topk_push(float* dist, int32_t* idx, int* size, int max_size, float value, int value_idx) {
  int p = 0;
  while (p < *size && dist[p] <= value) p++;
  if (p < max_size) {
    int last = *size < max_size ? *size : max_size - 1;
    for (int i = last; i > p; i--) {
      dist[i] = dist[i - 1];
      idx[i] = idx[i - 1];
    }
    dist[p] = value;
    idx[p] = value_idx;
  }
  if (*size + 1 <= max_size) (*size)++;
}

/* get_entry_kernel_inner, src/impl/nav.cuh:13-135: greedy walk on the pivot
 * graph with a 32-slot list per query (4 kept + 28 neighbour slots). Slots past
 * the current node's degree keep stale entries. Four selection rounds each
 * take a warp argmin (a __shfl_down_sync tree with strict <) and swap only
 * when the distances differ. Duplicates of the previous round's pick are
 * dropped and their expanded bit is OR-ed into it (several lanes store to that
 * slot at once in the reference; the OR of all of them is used here). Returns
 * the local id (before map.txt translation), or -1 with *flags set. */
int orc_nav_entry(const orc_index* ix, const float* q, int fma, int* flags) {
  enum { NL = 4, NR = 28 };
  uint32_t id[32];
  float ds[32];
  const int dim = (int)ix->dim;
  const size_t vec_bytes = (size_t)dim * ix->elt;
  const int64_t graph_len = (int64_t)ix->nav_n * ix->nav_max_m;
  id[0] = (uint32_t)ix->nav_start; /* nav.cuh:50-57 */
  ds[0] = orc_exact_dist(q, ix->nav_data + vec_bytes * ix->nav_start, ix->dtype, dim, fma);
  for (int t = 1; t < 32; t++) {
    id[t] = 0xffffffffu;
    ds[t] = INFINITY;
  }
  int idx = 0, iters = 0;
  while (idx != -1) {
    if (++iters > 1000000) {
      *flags |= ORC_F_NAV_CAP;
      return -1;
    }
    uint32_t u = id[idx]; /* nav.cuh:62-68 */
    id[idx] |= ORC_BIT;
    for (int i = 0; i < NR; i++) { /* nav.cuh:69-81 */
      /* The row is read as 28 consecutive slots of the flat array, so rows
       * narrower than 28 run into the next row; past the last row the
       * reference reads beyond its allocation, taken here as -1. */
      int64_t e = (int64_t)ix->nav_max_m * u + i;
      int v = e < graph_len ? ix->nav_graph[e] : -1;
      if (v == -1) break;
      if (v < 0 || v >= ix->nav_n) {
        *flags |= ORC_F_BAD_ID;
        return -1;
      }
      id[i + NL] = (uint32_t)v;
      ds[i + NL] = orc_exact_dist(q, ix->nav_data + vec_bytes * v, ix->dtype, dim, fma);
    }
    for (int i = 0; i < NL; i++) { /* nav.cuh:84-119 */
      float dist[32];
      int pos[32];
      uint32_t prev = i ? id[i - 1] : 0, orv = 0;
      int any = 0;
      for (int t = 0; t < 32; t++) {
        dist[t] = ds[t];
        pos[t] = t;
        if (t < i)
          dist[t] = INFINITY;
        else if (i != 0 && ((id[t] ^ prev) & ORC_MASK) == 0) {
          orv |= id[t];
          any = 1;
          dist[t] = ds[t] = INFINITY;
        }
      }
      if (any) id[i - 1] = prev | orv;
      for (int off = 16; off > 0; off >>= 1)
        for (int t = 0; t + off < 32; t++)
          if (dist[t + off] < dist[t]) {
            dist[t] = dist[t + off];
            pos[t] = pos[t + off];
          }
      int p = pos[0];
      if (i != p && ds[i] != ds[p]) {
        float td = ds[i];
        ds[i] = ds[p];
        ds[p] = td;
        uint32_t ti = id[i];
        id[i] = id[p];
        id[p] = ti;
      }
    }
    int x = 32; /* nav.cuh:120-129: first lane whose id has the expanded bit clear */
    for (int t = 0; t < 32; t++)
      if (!(id[t] & ORC_BIT)) {
        x = t;
        break;
      }
    idx = x < NL ? x : -1;
  }
  return (int)(id[0] & ORC_MASK); /* nav.cuh:133 */
}

typedef struct {
  int cap;
  int* mv_pos;
  uint32_t *mv_id, *tmp_id;
  float *mv_dist, *tmp_dist;
  float* table;
  float* qr;
} orc_scratch;

static void scratch_init(orc_scratch* s, const orc_index* ix, int L) {
  s->cap = L + (int)ix->max_m0 + 64;
  s->mv_pos = (int*)calloc(s->cap, sizeof(int));
  s->mv_id = (uint32_t*)calloc(s->cap, sizeof(uint32_t));
  s->tmp_id = (uint32_t*)calloc(s->cap, sizeof(uint32_t));
  s->mv_dist = (float*)calloc(s->cap, sizeof(float));
  s->tmp_dist = (float*)calloc(s->cap, sizeof(float));
  s->table = (float*)malloc(sizeof(float) * (size_t)ix->pq_m * ORC_PIVOTS);
  s->qr = (float*)malloc(sizeof(float) * ix->dim);
}
static void scratch_free(orc_scratch* s) {
  free(s->mv_pos); free(s->mv_id); free(s->tmp_id); free(s->mv_dist); free(s->tmp_dist);
  free(s->table); free(s->qr);
}

/* One query of search_graph_kernel_gpumem, src/impl/pure_mem.cuh:277-428,
 * with the table and restored query already built. The mv_ and tmp_ arrays play
 * the role of the kernel's shared-memory pool (pure_mem.cuh:267-272); the
 * block-parallel steps are executed as "compute every position, then scatter",
 * exactly as the reference's __syncthreads phases order them. */
static int walk_one(const orc_index* ix, orc_scratch* s, int64_t entry, int L, int k, int fma,
                    int32_t* out_id, float* out_d, int32_t* out_found, int32_t* trace, int trace_cap,
                    int* n_hops, int* flags) {
  const int max_m = (int)ix->max_m0, M = ix->pq_m, dim = (int)ix->dim;
  int* mv_pos = s->mv_pos;
  uint32_t *mv_id = s->mv_id, *tmp_id = s->tmp_id;
  float *mv_dist = s->mv_dist, *tmp_dist = s->tmp_dist;
  const float* table = s->table;
  int ctx_size = 0, found = 0, hops = 0;
  for (int i = 0; i < k; i++) { /* thrust device_vector zero-init, pure_mem.cu:85-87 */
    out_id[i] = 0;
    out_d[i] = 0.0f;
  }
  int64_t u = entry;
  while (u != -1) {
    if (u < 0 || u >= ix->n) {
      *flags |= ORC_F_BAD_ID;
      break;
    }
    if (hops >= 10000000) {
      *flags |= ORC_F_HOP_CAP;
      break;
    }
    /* get_node_ptr, pure_mem.cuh:261-265,288-292 */
    const uint8_t* node = ix->pages + (u / ix->npp) * ORC_PAGE + (u % ix->npp) * ix->node_len;
    uint32_t meta0;
    memcpy(&meta0, node + ix->data_len, 4);
    int deg = (int)meta0;
    const uint8_t* edge = node + ix->data_len + 4;
    if (deg < 0 || deg > max_m) {
      *flags |= ORC_F_BAD_DEG;
      break;
    }
    int sz = ctx_size;
    /* ADC of every neighbour; sentinels past the degree, pure_mem.cuh:294-310 */
    for (int t = 0; t < max_m; t++) {
      if (t >= deg) {
        tmp_id[sz + t] = 0xffffffffu - (uint32_t)t;
        tmp_dist[sz + t] = INFINITY;
      } else {
        int32_t v;
        memcpy(&v, edge + 4 * (size_t)t, 4);
        if (v < 0 || v >= ix->n) {
          *flags |= ORC_F_BAD_ID;
          return -1;
        }
        tmp_id[sz + t] = (uint32_t)v;
        tmp_dist[sz + t] = adc(table, ix->codes + (size_t)v * M, M);
      }
    }
    /* local merge sort of the deg new entries, pure_mem.cuh:314-348 */
    for (int len = 2; len < 2 * deg; len *= 2) {
      for (int t = 0; t < deg; t++) {
        int start = (t / len) * len;
        int mid = start + len / 2 < deg ? start + len / 2 : deg;
        int end = start + len < deg ? start + len : deg;
        if (t < mid)
          mv_pos[t] = lower_bound_key(tmp_dist + sz + mid, tmp_id + sz + mid, 0, end - mid, tmp_dist[sz + t],
                                      tmp_id[sz + t]) + t;
        else if (t < end)
          mv_pos[t] = lower_bound_key(tmp_dist + sz, tmp_id + sz, start, mid, tmp_dist[sz + t], tmp_id[sz + t]) +
                      t - mid;
      }
      for (int t = 0; t < deg; t++)
        for (int w = t + 1; w < deg; w++)
          if (mv_pos[w] == mv_pos[t]) *flags |= ORC_F_KEY_COLLISION;
      for (int t = 0; t < deg; t++) {
        mv_id[mv_pos[t]] = tmp_id[sz + t];
        mv_dist[mv_pos[t]] = tmp_dist[sz + t];
      }
      for (int t = 0; t < deg; t++) {
        tmp_id[sz + t] = mv_id[t];
        tmp_dist[sz + t] = mv_dist[t];
      }
    }
    /* merge with the sorted list; a new entry equal to an old one goes after
     * it, pure_mem.cuh:351-376 */
    for (int t = 0; t < deg; t++) {
      int id = lower_bound_key(tmp_dist, tmp_id, 0, sz, tmp_dist[sz + t], tmp_id[sz + t]);
      if (id != sz && ((tmp_id[id] ^ tmp_id[sz + t]) & ORC_MASK) == 0) id++;
      mv_pos[sz + t] = id + t;
    }
    for (int i = 0; i < sz; i++)
      mv_pos[i] = lower_bound_key(tmp_dist + sz, tmp_id + sz, 0, deg, tmp_dist[i], tmp_id[i]) + i;
    for (int i = 0; i < sz + deg; i++) {
      mv_id[mv_pos[i]] = tmp_id[i];
      mv_dist[mv_pos[i]] = tmp_dist[i];
    }
    ctx_size = sz + deg < 2 * L ? sz + deg : 2 * L; /* pure_mem.cuh:377 */
    /* warp 0: drop adjacent duplicate ids, find the first entry without the
     * expanded bit, pure_mem.cuh:380-419 */
    int sz2 = ctx_size, count = 0, best = sz2 + 1;
    for (int i = 0; i < sz2; i++) {
      int dup = i != 0 && ((mv_id[i] ^ mv_id[i - 1]) & ORC_MASK) == 0;
      if (dup) {
        count++;
        continue;
      }
      int p = i - count;
      tmp_id[p] = mv_id[i];
      tmp_dist[p] = mv_dist[i];
      if (!(mv_id[i] & ORC_BIT) && best > p) best = p;
    }
    int64_t next;
    if (best > sz2 - count && sz2 - count < L) {
      /* No unexpanded entry and a list shorter than L: the reference then
       * selects tmp_id[sz+1] or reads list slots past the end (stale shared
       * memory). That is undefined; the walk stops here. */
      *flags |= ORC_F_REF_UNDEFINED;
      next = -1;
    } else if (best >= L) {
      next = -1;
    } else {
      next = (int64_t)tmp_id[best];
      ctx_size = sz2 - count < L ? sz2 - count : L;
      tmp_id[best] |= ORC_BIT;
    }
    /* warp 1: exact distance of this node and top-k insertion, pure_mem.cuh:420-424 */
    float d = orc_exact_dist(s->qr, node, ix->dtype, dim, fma);
    topk_push(out_d, out_id, &found, k, d, (int)u);
    if (trace && hops < trace_cap) trace[hops] = (int32_t)u;
    hops++;
    u = next;
  }
  *out_found = found;
  *n_hops = hops;
  return 0;
}

/* One query end to end: entry selection (nav.cuh or the medoid, pure_mem.cu:106-124),
 * table build, walk. fma_table: pq.cuh:40; fma_exact: util.cuh:37. */
static int search_one(const orc_index* ix, orc_scratch* s, const float* q, int k, int L, int fma_table,
                      int fma_exact, int32_t* ids, float* dists, int32_t* found, int32_t* trace, int trace_cap,
                      int* hops, int* flags, int* entry_out) {
  int64_t entry;
  if (ix->has_nav) {
    int local = orc_nav_entry(ix, q, fma_exact, flags);
    if (local < 0 || local >= ix->nav_n) {
      *flags |= ORC_F_BAD_ID;
      *hops = 0;
      *found = 0;
      return -1;
    }
    entry = ix->nav_map[local]; /* NavGraph::translate, nav_graph.cu:104-109 */
  } else {
    entry = ix->medoid;
  }
  if (entry_out) *entry_out = (int)entry;
  orc_pq_table(ix, q, fma_table, s->table, s->qr);
  return walk_one(ix, s, entry, L, k, fma_exact, ids, dists, found, trace, trace_cap, hops, flags);
}

/* Single query with a hop trace (debugging and tests). */
int orc_search_one(const orc_index* ix, const float* q, int k, int L, int fma_table, int fma_exact, int32_t* ids,
                   float* dists, int32_t* found, int32_t* trace, int trace_cap, int32_t* hops, int32_t* flags,
                   int32_t* entry) {
  orc_scratch s;
  scratch_init(&s, ix, L);
  int h = 0, f = 0, e = -1;
  int rc = search_one(ix, &s, q, k, L, fma_table, fma_exact, ids, dists, found, trace, trace_cap, &h, &f, &e);
  scratch_free(&s);
  *hops = h;
  *flags = f;
  *entry = e;
  return rc;
}

/* PureMemExecutor::search, src/pure_mem.cu:71-199: nq queries, spread over
 * nthreads host threads (<= 0: every online core) that take queries from a
 * shared counter. hops/flags/entries may be NULL. */
typedef struct {
  const orc_index* ix;
  const float* q;
  int nq, k, L, fma_table, fma_exact;
  int32_t *ids, *found, *hops, *flags, *entries;
  float* dists;
  int next; /* next query to take (atomic) */
  int rc;
} orc_job;

static void* search_worker(void* arg) {
  orc_job* j = (orc_job*)arg;
  orc_scratch s;
  scratch_init(&s, j->ix, j->L);
  for (;;) {
    int i = __atomic_fetch_add(&j->next, 1, __ATOMIC_RELAXED);
    if (i >= j->nq) break;
    int h = 0, f = 0, e = -1;
    int rc = search_one(j->ix, &s, j->q + (size_t)i * j->ix->dim, j->k, j->L, j->fma_table, j->fma_exact,
                        j->ids + (size_t)i * j->k, j->dists + (size_t)i * j->k, j->found + i, NULL, 0, &h, &f, &e);
    if (j->hops) j->hops[i] = h;
    if (j->flags) j->flags[i] = f;
    if (j->entries) j->entries[i] = e;
    if (rc) __atomic_store_n(&j->rc, -1, __ATOMIC_RELAXED);
  }
  scratch_free(&s);
  return NULL;
}

int orc_max_threads(void) {
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (int)n : 1;
}

int orc_search(const orc_index* ix, const float* q, int nq, int k, int L, int fma_table, int fma_exact, int nthreads,
               int32_t* ids, float* dists, int32_t* found, int32_t* hops, int32_t* flags, int32_t* entries) {
  if (k <= 0 || L <= 0 || nq < 0) return fail("k and L must be positive", NULL);
  if (nthreads <= 0) nthreads = orc_max_threads();
  if (nthreads > nq) nthreads = nq > 0 ? nq : 1;
  orc_job j = {ix, q, nq, k, L, fma_table, fma_exact, ids, found, hops, flags, entries, dists, 0, 0};
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nthreads);
  int started = 0;
  for (int t = 1; t < nthreads; t++)
    if (pthread_create(&th[t], NULL, search_worker, &j) == 0) started = t;
    else break;
  search_worker(&j);
  for (int t = 1; t <= started; t++) pthread_join(th[t], NULL);
  free(th);
  return j.rc;
}
