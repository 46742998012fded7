/*
 * gann.h -- C ABI of the B200-native GustANN all-in-GPU search path.
 *
 * Drop-in for the reference's `search_mem -G` entry points. Each declaration
 * cites the reference interface it replaces (paths relative to the GustANN
 * project root). All calls return a status (GANN_OK = 0); on failure
 * gann_last_error() describes the cause (the reference aborts, exits or throws
 * instead, src/common.hpp:17, src/common_cuda.cuh:10-17).
 *
 * Threading: a handle may be used from several host threads; calls on one
 * handle are serialised internally. Each handle lives on the CUDA device that
 * was current when it was opened and issues its work on its own stream.
 */
#ifndef GANN_H_
#define GANN_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gann_index gann_t;

/* status codes */
enum {
  GANN_OK = 0,
  GANN_EINVAL = 1,   /* bad argument (null pointer, k/L out of range, dtype) */
  GANN_EIO = 2,      /* a file could not be opened or is short */
  GANN_EFORMAT = 3,  /* a file is malformed or inconsistent with the others */
  GANN_ECUDA = 4,    /* a CUDA runtime call failed */
  GANN_ENOMEM = 5,   /* device or host allocation failed */
  GANN_EKERNEL = 6,  /* a kernel reported an error (bad id/degree, wait limit) */
  GANN_ERANGE = 7,   /* a size is beyond what this entry point supports */
  GANN_EBUSY = 8     /* a server's request budget is full: submit again later */
};

/* element type of the base vectors; gustann::DataType, src/common.hpp:22-25 */
enum { GANN_UINT8 = 0, GANN_FLOAT = 1 };

/* gann_open flags */
enum {
  GANN_OPEN_NO_VALIDATE = 1, /* skip the load-time check of degrees and neighbour ids */
  /* keep the records (vector + degree + neighbour ids) in pinned, mapped host
   * memory and read them from the kernels over PCIe/C2C; PQ codes, pivots and
   * the pivot graph stay in HBM. This is init_pure_mem(config, use_gpu_mem = false)
   * (src/pure_mem.cu:51-66, kernel search_graph_kernel_dram src/impl/pure_mem.cuh:50-241).
   * Results are identical to the HBM-resident mode. */
  GANN_OPEN_HOST_PAGES = 2
};

/* table precision for gann_search_batch */
enum {
  GANN_PREC_FP32 = 0,    /* FP32 tables, built per query on CUDA cores (the reference's arithmetic) */
  GANN_PREC_BF16 = 1,    /* BF16 tables built for the batch on the tensor cores, FP32 accumulate */
  GANN_PREC_BF16X3 = 2,  /* as BF16, with a three-term split-BF16 product (near-FP32 table values) */
  GANN_PREC_BF16_CC = 3  /* BF16 tables built per query on CUDA cores (FP32 then rounded) */
};

/* entry node of the batched form's walk */
enum {
  GANN_ENTRY_NAV_WALK = 0,      /* the reference's greedy walk over the pivot graph, a beam of 4
                                   (src/impl/nav.cuh:13-135), or the medoid without a pivot graph */
  GANN_ENTRY_NEAREST_PIVOT = 1  /* the nearest point of the pivot file (nav_index.data) by squared L2,
                                   found for the whole batch as one tensor-core product of the queries
                                   by the pivots (exact for uint8 vectors and integral queries; float
                                   operands rounded to BF16). Needs a pivot graph and dim <= 176. */
};

/* options of gann_search_batch; zero-initialised = defaults, except that a
 * zero precision is GANN_PREC_FP32. Passing opts = NULL selects
 * GANN_PREC_BF16X3: the split-BF16 tensor-core tables, whose error against
 * FP64 stays within BF16 storage rounding (single-pass GANN_PREC_BF16 loses
 * up to 2^-5 of a chunk's range to cancellation in |r|^2 - 2 r.P + |P|^2). */
typedef struct {
  int32_t precision;   /* GANN_PREC_*; opts = NULL means GANN_PREC_BF16X3 */
  int32_t beam_width;  /* warps (nodes expanded per step) per query: 1, 2, 4, 8 or 16; 0 = 4 (or autotuned) */
  int32_t hash_bits;   /* visited cache of 2^hash_bits ids per query; 0 = sized from L */
  int32_t entry;       /* GANN_ENTRY_*; 0 (and opts = NULL) = GANN_ENTRY_NAV_WALK */
  int32_t reserved[4];
} gann_batch_opts_t;

typedef struct {
  int64_t num_points;      /* Layout::num_data   src/layout.hpp:16 */
  int64_t dim;             /* Layout::num_dims   src/layout.hpp:8  */
  int64_t max_degree;      /* Layout::max_m0     src/layout.hpp:9  */
  int64_t medoid;          /* Layout::enter_point src/layout.hpp:10 */
  int64_t node_len;        /* Layout::node_size  src/layout.hpp:13 */
  int64_t nodes_per_page;  /* Layout::nodes_per_page src/layout.hpp:18 */
  int64_t num_pages;       /* Layout::num_pages  src/layout.hpp:15 */
  int32_t pq_chunks;       /* PQSearchData::num_chunks src/pq_search.hpp:14 */
  int32_t dtype;           /* GANN_UINT8 / GANN_FLOAT */
  int32_t has_nav;         /* pivot graph loaded */
  int32_t nav_points;      /* NavGraph::num_node src/nav_graph.hpp:12 */
  int32_t nav_max_degree;  /* NavGraph::max_m src/nav_graph.hpp:14 */
  int32_t device;          /* CUDA device the handle lives on */
  int64_t device_bytes;    /* HBM held by the index */
  int32_t host_pages;      /* records live in pinned host memory (GANN_OPEN_HOST_PAGES) */
  int32_t reserved0;
  int64_t host_bytes;      /* pinned host memory held by the index */
} gann_info_t;

/*
 * Open an index and make it resident in HBM (with GANN_OPEN_HOST_PAGES: the
 * records in pinned host memory, the rest in HBM).
 * Replaces gustann::GustANN::GustANN(DataType) + GustANN::init_pure_mem(config,
 * use_gpu_mem): src/ssd_search.hpp:70,76, src/ssd_search.cu:55-79,108-112,
 * src/pure_mem.cu:27-69. Files: index_file is DiskANN's `_disk.index`
 * (src/layout.cpp:11-69); `<pq_prefix>_pivots.bin` and `<pq_prefix>_compressed.bin`
 * (src/ssd_search.cu:61-63, src/pq_search.cu:56-121); `<nav_dir>/nav_index`,
 * `nav_index.data`, `map.txt` (src/ssd_search.cu:72-75, src/nav_graph.cu:41-100).
 * nav_dir NULL or "" means "enter at the medoid" (src/pure_mem.cu:121-123).
 */
int gann_open(const char* index_file, const char* pq_prefix, const char* nav_dir, int dtype,
              int flags, gann_t** out);

/*
 * For a handle opened with GANN_OPEN_HOST_PAGES: copy the records most often
 * expanded by a sample batch (nq device queries searched at ef_search) into
 * HBM, up to max_bytes (records padded to 16 B), and read those from HBM from
 * then on; the others stay in host memory. Results do not change (the same
 * bytes are read). A later call replaces the cache; max_bytes 0 drops it.
 * *cached_records (may be NULL) receives the number cached. The reference's
 * host-memory mode reads every record over the bus (src/pure_mem.cu:51-66,
 * src/impl/pure_mem.cuh:50-241); no counterpart.
 */
int gann_cache_hot_records(gann_t* h, const float* d_queries, int nq, int ef_search, int64_t max_bytes,
                           int64_t* cached_records);

/* Release the handle and its device memory. Replaces gustann::GustANN::~GustANN,
 * src/ssd_search.cu:29-53. NULL is accepted. */
int gann_close(gann_t* h);

/* Describe an open index. The reference keeps these in gustann::Layout
 * (src/layout.hpp:9-27); it has no accessor. */
int gann_get_info(const gann_t* h, gann_info_t* out);

/*
 * Plain search (the drop-in form): FP32 tables, the reference's summation
 * order and tie rules, ids identical to the reference's.
 * Replaces gustann::GustANN::search, src/ssd_search.hpp:78-80 ->
 * PureMemExecutor::search, src/pure_mem.cu:71-199. Host buffers:
 * queries nq x dim float (uint8 queries converted to float, bin/search_disk.cpp:160-165),
 * nns / distances nq x topk, found_cnt nq. Distances are squared L2. Unfilled
 * slots hold id 0 and distance 0. run_time (may be NULL) receives the device
 * time of entry selection + walk in seconds, the span the reference times
 * (src/pure_mem.cu:101-187). topk and ef_search are >= 1 (the reference's
 * driver also asserts ef_search >= topk, bin/search_disk.cpp:189-192; the
 * library itself, like this one, accepts either order).
 */
int gann_search(gann_t* h, const float* queries, int nq, int topk, int ef_search, int32_t* nns,
                float* distances, int32_t* found_cnt, double* run_time);

/* Same as gann_search on device pointers, enqueued on `stream` (a cudaStream_t;
 * NULL = the handle's stream) without a host synchronisation. The reference
 * has no device-pointer form; this is PureMemExecutor::search (src/pure_mem.cu:71-199)
 * minus its host<->device copies. */
int gann_search_device(gann_t* h, const float* d_queries, int nq, int topk, int ef_search,
                       int32_t* d_nns, float* d_distances, int32_t* d_found_cnt, void* stream);

/*
 * Batched search (the optimised form): every query has its own topk and
 * ef_search (arrays of nq, or NULL to use topk_max / ef_max for all), W warps
 * expand W candidates per step, a visited cache skips already-scored
 * neighbours, and the PQ tables are BF16 built on the tensor cores (or FP32).
 * Results are not bit-identical to the reference (that is gann_search); recall
 * is reported against it. Extends PureMemExecutor::search (src/pure_mem.cu:71-199)
 * to uneven L and k; the reference asserts one L >= topk per call
 * (bin/search_disk.cpp:189-192). nns / distances are nq x topk_max (row stride
 * topk_max); slots past a query's found count hold id 0 and distance 0.
 */
int gann_search_batch(gann_t* h, const float* queries, int nq, const int32_t* topk, const int32_t* ef_search,
                      int topk_max, int ef_max, const gann_batch_opts_t* opts, int32_t* nns,
                      float* distances, int32_t* found_cnt, double* run_time);

/* gann_search_batch on device buffers (topk / ef_search device arrays or NULL),
 * enqueued on `stream` (NULL = the handle's stream) without a host
 * synchronisation; d_hops / d_bytes (nq, may be NULL) receive the per-query
 * counters of gann_search_device_ex. */
int gann_search_batch_device(gann_t* h, const float* d_queries, int nq, const int32_t* d_topk,
                             const int32_t* d_ef_search, int topk_max, int ef_max,
                             const gann_batch_opts_t* opts, int32_t* d_nns, float* d_distances,
                             int32_t* d_found_cnt, int32_t* d_hops, int64_t* d_bytes, void* stream);

/* Autotuner of the batched form: times beam widths {2, 4, 8, 16} and visited
 * caches of {1/8, 1/4, 1/2, 1, 2} x the default size on nq device queries at (topk,
 * ef_search, precision), keeps the fastest, and makes it this handle's default
 * for gann_search_batch* calls that leave beam_width / hash_bits at 0. Results
 * do not depend on the cache size; the beam width changes the walk order. The
 * reference has a fixed launch shape (src/pure_mem.cu:31,137); no counterpart. */
int gann_autotune(gann_t* h, const float* d_queries, int nq, int topk, int ef_search, int precision,
                  gann_batch_opts_t* best, double* best_seconds);

/* gann_search_device plus per-query counters (device arrays of nq, each may be
 * NULL): d_hops = nodes expanded, d_bytes = algorithmic gathered bytes (degree
 * word, neighbour ids, vector and the codes of every scored neighbour per hop,
 * plus the pivot-graph rows and vectors). No counterpart in the reference. */
int gann_search_device_ex(gann_t* h, const float* d_queries, int nq, int topk, int ef_search,
                          int32_t* d_nns, float* d_distances, int32_t* d_found_cnt, int32_t* d_hops,
                          int64_t* d_bytes, void* stream);

/*
 * The nearest point of the pivot file (nav_index.data) of each query, the
 * entry node of GANN_ENTRY_NEAREST_PIVOT: d_pivot[q] = its row in the pivot
 * file, d_node[q] = its node id (map.txt); either output may be NULL. Device
 * buffers, enqueued on `stream` (NULL = the handle's stream). Exact for uint8
 * vectors with integral queries (ties to the lowest row); float operands are
 * rounded to BF16. GANN_ERANGE without a pivot graph or above dim 176. The
 * reference's entry is the pivot-graph walk (src/impl/nav.cuh:13-135,
 * src/nav_graph.cu:104-109); this is an exact search over the same points.
 */
int gann_nearest_pivots(gann_t* h, const float* d_queries, int nq, int32_t* d_pivot, int32_t* d_node,
                        void* stream);

/*
 * gann_search_batch_device for callers that cannot allocate device memory
 * while they search: a serving loop that must not stall on cudaMalloc (which
 * can synchronise the device and takes the driver's allocation lock), or a
 * host program whose memory manager owns every device allocation after
 * start-up. No counterpart in the reference (its search allocates device
 * vectors on every call, src/pure_mem.cu:78-89).
 * Same arguments as gann_search_batch_device with one topk / ef_search for the
 * whole call; no per-query counters. The call allocates nothing: its scratch
 * (work counter, BF16 tables) is a fixed 8 MiB + 256 B array inside the
 * library, held on every GPU that loads libgann until the process exits.
 * Options left 0 (or opts NULL) take the same defaults as
 * gann_search_batch_device, the handle's gann_autotune choices included; the
 * entry is the pivot-graph walk (GANN_ENTRY_NEAREST_PIVOT returns GANN_EINVAL).
 * Limits, tensor-core tables (GANN_PREC_BF16, GANN_PREC_BF16X3) only: nq <= 512
 * per call and at most 32 PQ chunks; larger requests return GANN_ERANGE. The
 * FP32 and CUDA-core BF16 precisions use only the work counter and take any nq.
 * All calls on a device share the array: calls whose work overlaps on the GPU
 * race on it and must be serialised by the caller. Each call looks up the
 * array's device address in the current context (no allocation); the first
 * call on a device may load the library's device code, so make it before any
 * stream capture.
 */
int gann_search_batch_noalloc(gann_t* h, const float* d_queries, int nq, int topk, int ef_search,
                              const gann_batch_opts_t* opts, int32_t* d_nns, float* d_distances,
                              int32_t* d_found_cnt, void* stream);

/*
 * Batched search captured once as a CUDA graph (counter reset, tensor-core
 * table build, persistent walk) and replayed by gann_batch_graph_launch. The
 * device buffers given here are baked into the graph: d_queries (max_nq x dim),
 * optional per-query d_topk / d_ef_search (NULL = topk_max / ef_max for all),
 * the outputs as in gann_search_batch_device, and d_nq, a device int holding
 * the number of queries (rows from 0) each launch processes, read by the
 * kernels at run time and clamped to max_nq. Write the queries and the count,
 * launch, read the results. Options (precision, beam width, visited cache) and
 * the handle's tuned defaults are fixed at capture. Launches of one graph run
 * one after another; graphs of one handle may run concurrently. The reference
 * launches its kernels once per call (src/pure_mem.cu:101-184); no counterpart.
 */
typedef struct gann_batch_graph gann_batch_graph_t;
int gann_batch_graph_create(gann_t* h, int max_nq, int topk_max, int ef_max, const gann_batch_opts_t* opts,
                            const float* d_queries, const int32_t* d_topk, const int32_t* d_ef_search,
                            const int32_t* d_nq, int32_t* d_nns, float* d_distances, int32_t* d_found_cnt,
                            gann_batch_graph_t** out);
/* Enqueue one replay on `stream` (a cudaStream_t; NULL = the graph's own stream). */
int gann_batch_graph_launch(gann_batch_graph_t* g, void* stream);
/* Wait for the device (replays may be on any stream) and release the graph and
 * its scratch. NULL is accepted. */
int gann_batch_graph_destroy(gann_batch_graph_t* g);

/* PQ distance tables of nq host queries (tables: nq x M x 256 FP32, host),
 * built as the chosen precision builds them: FP32 exactly as the plain form
 * (PQSearchData::init_query, src/impl/pq.cuh:8-59); the BF16 forms widened
 * from their BF16 values. For table-error studies against an FP64 oracle. */
int gann_pq_tables(gann_t* h, const float* queries, int nq, int precision, float* tables);

/*
 * Continuous-batching server over the batched form. Requests arrive one at a
 * time; a dispatcher thread packs the waiting ones into a batch whenever one of
 * `streams` batch slots is free (or the oldest has waited max_wait_us) and
 * launches it on that slot's stream, so later arrivals start while earlier
 * batches run and several batches overlap on the device. Each slot's device
 * memory is allocated at start. Admission is by memory: every request is
 * charged the device state that its own ef_search and topk need while it is
 * held (gann_server_request_bytes: its candidate list, its visited cache, its
 * PQ table, its query and its result row), and a submit is refused with
 * GANN_EBUSY when the charge of the waiting + running + finished-but-unpolled
 * requests would pass mem_budget_kib -- so when memory runs short, requests
 * with a long list are refused while short ones still enter -- or when those
 * requests already fill the server's max_batch * (streams + 1) request
 * slots. A result depends only on its query, topk,
 * ef_search and the server options, not on the other requests in its batch.
 * The reference serves one fixed batch per call (src/pure_mem.cu:71-199);
 * no counterpart.
 */
typedef struct gann_server gann_server_t;
typedef struct {
  int32_t max_batch;    /* queries per launch; 0 = 1024 */
  int32_t streams;      /* batch slots (launches in flight); 0 = 4 */
  int32_t topk_max;     /* largest topk a request may ask; 0 = 100 */
  int32_t ef_max;       /* largest ef_search a request may ask; 0 = 512 */
  int32_t precision;    /* GANN_PREC_*; with opts given, as given */
  int32_t beam_width;   /* 0 = the handle's default */
  int32_t hash_bits;    /* 0 = sized from ef_max */
  int32_t max_wait_us;  /* a batch smaller than min_batch waits this long for company; 0 = 100 */
  int32_t min_batch;    /* 0 = launch as soon as a slot is free */
  int32_t mem_budget_kib; /* admission budget in KiB; 0 = every request slot at (topk_max, ef_max) */
  int32_t entry;        /* GANN_ENTRY_* of every batch; 0 = the pivot-graph walk */
  int32_t reserved[5];
} gann_server_opts_t;

typedef struct {
  double offered_qps, achieved_qps;
  int64_t submitted, rejected, completed;
  double p50_ms, p99_ms, p999_ms, mean_ms;  /* submit -> result available on the host */
} gann_load_stats_t;

int gann_server_start(gann_t* h, const gann_server_opts_t* opts, gann_server_t** out);
/* Bytes a request of (topk, ef_search) is charged against the admission
 * budget of this server. */
int64_t gann_server_request_bytes(const gann_server_t* s, int topk, int ef_search);
/* Copy one query (dim floats) in; GANN_EBUSY when the budget is full. */
int gann_server_submit(gann_server_t* s, const float* query, int topk, int ef_search, uint64_t tag);
/* Up to max_results finished requests: tags, nns / distances (rows of
 * topk_max), found counts, latencies in seconds; *n_out = how many. */
int gann_server_poll(gann_server_t* s, int max_results, uint64_t* tags, int32_t* nns, float* distances,
                     int32_t* found_cnt, double* latency, int* n_out);
/* Finish the running batches and release the server. */
int gann_server_stop(gann_server_t* s);
/* Open-loop load: submit the nq host queries cyclically at Poisson arrival
 * times of rate rate_qps for `seconds` (topk / ef_search per query, or NULL
 * for 10 / ef_max), then drain; reports latency percentiles and throughput. */
int gann_server_open_loop(gann_server_t* s, const float* queries, int nq, const int32_t* topk,
                          const int32_t* ef_search, double rate_qps, double seconds, uint64_t seed,
                          gann_load_stats_t* out);

/* Synchronise `stream` (NULL = the handle's stream) and report, as
 * GANN_EKERNEL, any error word left by kernels enqueued with
 * gann_search_device; the word is cleared. The reference has no counterpart
 * (its kernels report through device assert, src/impl/pure_mem.cuh:373). */
int gann_check(gann_t* h, void* stream);

/* FMA behaviour of the plain form at the reference's two contraction sites:
 * the table accumulate (src/impl/pq.cuh:40) and the exact-distance accumulate
 * (src/impl/util.cuh:37). Default 1/1 (fused), which tests/golden pins against
 * the reference's own build. No counterpart in the reference (a compiler flag there). */
int gann_set_fma(gann_t* h, int fma_table, int fma_exact);

/* Pivot-graph sample (index preparation): the ids 0..num_data-1 shuffled with
 * std::shuffle and std::mt19937(seed), the first num_samp kept and sorted.
 * Replaces bin/gen_small_file.cpp:12-25 (seed 114514 there). */
int gann_sample_pivots(int64_t num_data, int64_t num_samp, uint32_t seed, int32_t* out);

/* RobustPrune for the index builder (index preparation, device buffers): for
 * each of n_rows points (d_rows[r], or r when d_rows is NULL) keep at most R of
 * its K candidate ids (d_cand, n_rows x K, -1 = none; the point itself,
 * repeats and ids outside [0, n) are ignored) in order of squared L2 distance,
 * dropping every candidate c that a kept neighbour j occludes:
 * alpha * d(j, c) < d(p, c). d_x is n x dim uint8 or float32 (dtype); d_out
 * is n_rows x R, -1 padded. Enqueued on `stream`. Replaces the pruning step of
 * DiskANN's Vamana build, which the reference calls through
 * scripts/build_diskann_index.sh:7 (DiskANN is an empty submodule there). */
int gann_build_prune(const void* d_x, int dtype, int64_t n, int dim, const int32_t* d_rows,
                     const int32_t* d_cand, int64_t n_rows, int K, int R, float alpha, int32_t* d_out,
                     void* stream);

/* Message for the last failing call on this thread. */
const char* gann_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* GANN_H_ */
