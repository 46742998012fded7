// Continuous-batching search server over the batched form.
//
// The reference answers one fixed batch per call (PureMemExecutor::search,
// src/pure_mem.cu:71-199). Here requests arrive one by one; a dispatcher thread
// packs the ones that have arrived into a batch whenever a batch slot is free
// and launches it on that slot's stream, so requests that arrive while others
// run on the GPU start as soon as a slot frees up, and up to `streams` batches
// overlap on the device. Each slot owns its device buffers (queries, per-query
// k and L, the batch size, results) and a CUDA graph of the batched search
// captured over them at start (gann_batch_graph_create: counter reset, table
// build, persistent walk reading the batch size from device memory), so a
// batch is its input copies, one graph launch and its output copies. Admission
// is by memory: each request is charged the device state its own L and k need
// (candidate list, visited cache, table, query, result row; request_bytes),
// and a submit is refused (GANN_EBUSY) when the requests held by the server --
// waiting, on the GPU, or finished and not yet polled -- would exceed the byte
// budget, or would take more request slots than the server has. Per-query
// state lives on the device for the life of its batch. A request's result
// depends only on the query, its k and L, and the server's options, not on
// the other requests in its batch.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "gann_internal.h"

int gann_internal_set_error(int code, const char* msg);

namespace {

using Clock = std::chrono::steady_clock;

double now_s() { return std::chrono::duration<double>(Clock::now().time_since_epoch()).count(); }

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  float* h_q = nullptr;
  int32_t *h_k = nullptr, *h_l = nullptr, *h_nns = nullptr, *h_f = nullptr;
  float* h_d = nullptr;
  float* d_q = nullptr;
  int32_t *d_k = nullptr, *d_l = nullptr, *d_nns = nullptr, *d_f = nullptr;
  float* d_d = nullptr;
  int32_t* h_nq = nullptr;  // batch size (pinned) and its device copy read by the graph
  int32_t* d_nq = nullptr;
  gann_batch_graph_t* graph = nullptr;
  std::vector<uint64_t> tags;
  std::vector<double> t_submit;
  std::vector<int64_t> cost;
  int count = 0;
  bool busy = false;
};

}  // namespace

struct gann_server {
  gann_t* h = nullptr;
  gann_server_opts_t o{};
  int dim = 0, M = 0;
  std::vector<Slot> slots;
  // request ring (host): queries, k, L, tag, submit time
  int cap = 0, head = 0, tail = 0, size = 0;
  std::vector<float> rq;
  std::vector<int32_t> rk, rl;
  std::vector<uint64_t> rtag;
  std::vector<double> rt;
  std::vector<int64_t> rcost;
  int in_flight = 0;  // requests inside busy slots
  int64_t budget = 0;      // admission budget in bytes
  int64_t bytes_held = 0;  // charge of the waiting + running + unpolled requests
  // completions (ring of the same capacity; counted against the budget until polled)
  int dhead = 0, dsize = 0;
  std::vector<uint64_t> dtag;
  std::vector<int32_t> dfound, dids;
  std::vector<float> ddist;
  std::vector<double> dlat;
  std::vector<int64_t> dcost;
  std::mutex mu;
  std::thread th;
  std::atomic<bool> stop{false};
  std::atomic<int> error{0};
  std::string error_msg;
};

namespace {

void free_slot(Slot& s) {
  if (s.graph) gann_batch_graph_destroy(s.graph);
  for (void* p : {(void*)s.h_q, (void*)s.h_k, (void*)s.h_l, (void*)s.h_nns, (void*)s.h_f, (void*)s.h_d,
                  (void*)s.h_nq})
    if (p) cudaFreeHost(p);
  for (void* p : {(void*)s.d_q, (void*)s.d_k, (void*)s.d_l, (void*)s.d_nns, (void*)s.d_f, (void*)s.d_d,
                  (void*)s.d_nq})
    if (p) cudaFree(p);
  if (s.done) cudaEventDestroy(s.done);
  if (s.stream) cudaStreamDestroy(s.stream);
  s = Slot{};
}

cudaError_t alloc_slot(Slot& s, int B, int dim, int kmax) {
  cudaError_t e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMallocHost(&s.h_q, sizeof(float) * (size_t)B * dim);
  if (e == cudaSuccess) e = cudaMallocHost(&s.h_k, sizeof(int32_t) * B);
  if (e == cudaSuccess) e = cudaMallocHost(&s.h_l, sizeof(int32_t) * B);
  if (e == cudaSuccess) e = cudaMallocHost(&s.h_nns, sizeof(int32_t) * (size_t)B * kmax);
  if (e == cudaSuccess) e = cudaMallocHost(&s.h_d, sizeof(float) * (size_t)B * kmax);
  if (e == cudaSuccess) e = cudaMallocHost(&s.h_f, sizeof(int32_t) * B);
  if (e == cudaSuccess) e = cudaMalloc(&s.d_q, sizeof(float) * (size_t)B * dim);
  if (e == cudaSuccess) e = cudaMalloc(&s.d_k, sizeof(int32_t) * B);
  if (e == cudaSuccess) e = cudaMalloc(&s.d_l, sizeof(int32_t) * B);
  if (e == cudaSuccess) e = cudaMalloc(&s.d_nns, sizeof(int32_t) * (size_t)B * kmax);
  if (e == cudaSuccess) e = cudaMalloc(&s.d_d, sizeof(float) * (size_t)B * kmax);
  if (e == cudaSuccess) e = cudaMalloc(&s.d_f, sizeof(int32_t) * B);
  if (e == cudaSuccess) e = cudaMallocHost(&s.h_nq, sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc(&s.d_nq, sizeof(int32_t));
  s.tags.resize(B);
  s.t_submit.resize(B);
  s.cost.resize(B);
  return e;
}

// Device state a request of (k, L) holds while the server has it: the sorted
// candidate list (id + distance per entry), the visited cache (one id per
// slot, sized from L as the batched form sizes it), the PQ table (BF16 or
// FP32 per precision), the query and the result row (id + distance per k,
// plus the found count), and the entry key with the nearest-pivot entry.
int64_t request_bytes(const gann_server* sv, int k, int L) {
  const int tab = sv->o.precision == GANN_PREC_FP32 ? 4 : 2;
  const int hb = sv->o.hash_bits ? sv->o.hash_bits : gann::batch_hash_bits(L);
  return 8ll * L + 4ll * (1ll << hb) + (int64_t)tab * sv->M * gann::kPivots + 4ll * sv->dim + 8ll * k + 4 +
         (sv->o.entry == GANN_ENTRY_NEAREST_PIVOT ? 8 : 0);
}

// Publish a finished batch into the completion ring. Dispatcher thread only.
// The ring range [dhead + dsize, + count) is free (the admission budget keeps
// waiting + in flight + completed <= cap), so it is filled without the lock
// and made visible to gann_server_poll by one locked update of dsize.
void complete(gann_server* sv, Slot& s, cudaError_t q) {
  const int kmax = sv->o.topk_max;
  const double t = now_s();
  int base;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    base = sv->dhead + sv->dsize;
  }
  for (int i = 0; i < s.count; i++) {
    const int r = (base + i) % sv->cap;
    sv->dtag[r] = s.tags[i];
    sv->dcost[r] = s.cost[i];
    sv->dfound[r] = s.h_f[i];
    sv->dlat[r] = t - s.t_submit[i];
    std::memcpy(&sv->dids[(size_t)r * kmax], s.h_nns + (size_t)i * kmax, sizeof(int32_t) * kmax);
    std::memcpy(&sv->ddist[(size_t)r * kmax], s.h_d + (size_t)i * kmax, sizeof(float) * kmax);
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  if (q != cudaSuccess && !sv->error) {
    sv->error_msg = std::string("server batch: ") + cudaGetErrorString(q);
    sv->error = GANN_ECUDA;
  }
  sv->dsize += s.count;
  sv->in_flight -= s.count;
  s.busy = false;
  s.count = 0;
}

// Launch the waiting requests on a free slot, if the batching rule allows.
// Dispatcher thread only. The ring entries [head, head + n) stay counted in
// `size` while they are copied out without the lock, so no submit can reuse
// them; head and size move in one locked update afterwards.
bool launch(gann_server* sv) {
  Slot* s = nullptr;
  for (Slot& x : sv->slots)
    if (!x.busy) {
      s = &x;
      break;
    }
  if (!s) return false;
  const int B = sv->o.max_batch, dim = sv->dim;
  int n, h0;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->size == 0) return false;
    const bool old_enough = now_s() - sv->rt[sv->head] >= sv->o.max_wait_us * 1e-6;
    if (sv->size < std::min(B, std::max(1, sv->o.min_batch)) && !old_enough) return false;
    n = std::min(B, sv->size);
    h0 = sv->head;
  }
  for (int i = 0; i < n; i++) {
    const int r = (h0 + i) % sv->cap;
    std::memcpy(s->h_q + (size_t)i * dim, sv->rq.data() + (size_t)r * dim, sizeof(float) * dim);
    s->h_k[i] = sv->rk[r];
    s->h_l[i] = sv->rl[r];
    s->tags[i] = sv->rtag[r];
    s->t_submit[i] = sv->rt[r];
    s->cost[i] = sv->rcost[r];
  }
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->head = (h0 + n) % sv->cap;
    sv->size -= n;
    sv->in_flight += n;
  }
  s->count = n;
  s->busy = true;
  const int kmax = sv->o.topk_max;
  cudaStream_t st = s->stream;
  *s->h_nq = n;
  cudaError_t e = cudaMemcpyAsync(s->d_q, s->h_q, sizeof(float) * (size_t)n * dim, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_k, s->h_k, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_l, s->h_l, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_nq, s->h_nq, sizeof(int32_t), cudaMemcpyHostToDevice, st);
  int rc = GANN_OK;
  if (e == cudaSuccess) rc = gann_batch_graph_launch(s->graph, st);
  if (e == cudaSuccess && rc == GANN_OK)
    e = cudaMemcpyAsync(s->h_nns, s->d_nns, sizeof(int32_t) * (size_t)n * kmax, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && rc == GANN_OK)
    e = cudaMemcpyAsync(s->h_d, s->d_d, sizeof(float) * (size_t)n * kmax, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && rc == GANN_OK)
    e = cudaMemcpyAsync(s->h_f, s->d_f, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaEventRecord(s->done, st);
  if (e != cudaSuccess || rc != GANN_OK) {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (!sv->error) {
      sv->error_msg = rc != GANN_OK ? "server launch failed" : std::string("server: ") + cudaGetErrorString(e);
      sv->error = rc != GANN_OK ? rc : GANN_ECUDA;
    }
  }
  return true;
}

void dispatcher(gann_server* sv) {
  cudaSetDevice(sv->h->device);
  while (!sv->stop.load(std::memory_order_relaxed)) {
    bool work = false;
    for (Slot& s : sv->slots) {
      if (!s.busy) continue;
      const cudaError_t q = cudaEventQuery(s.done);
      if (q == cudaErrorNotReady) continue;
      complete(sv, s, q);
      work = true;
    }
    work = launch(sv) || work;
    if (work) continue;
    bool idle;
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      idle = sv->size == 0 && sv->in_flight == 0;
    }
    if (idle)
      std::this_thread::sleep_for(std::chrono::microseconds(20));
    else
      std::this_thread::yield();
  }
  for (Slot& s : sv->slots)
    if (s.busy) complete(sv, s, cudaEventSynchronize(s.done));
}

// Queue one request that arrived at time t. Caller holds mu.
int submit_locked(gann_server* sv, const float* query, int topk, int ef_search, uint64_t tag, double t) {
  if (sv->error) return gann_internal_set_error(sv->error, sv->error_msg.c_str());
  // admission: waiting + on the GPU + finished but not yet polled, against
  // the byte budget and the request slots
  const int64_t cost = request_bytes(sv, topk, ef_search);
  if (sv->size + sv->in_flight + sv->dsize >= sv->cap || sv->bytes_held + cost > sv->budget) return GANN_EBUSY;
  const int r = sv->tail;
  sv->rcost[r] = cost;
  sv->bytes_held += cost;
  std::memcpy(sv->rq.data() + (size_t)r * sv->dim, query, sizeof(float) * sv->dim);
  sv->rk[r] = topk;
  sv->rl[r] = ef_search;
  sv->rtag[r] = tag;
  sv->rt[r] = t;
  sv->tail = (sv->tail + 1) % sv->cap;
  sv->size++;
  return GANN_OK;
}

}  // namespace

extern "C" {

int gann_server_start(gann_t* h, const gann_server_opts_t* opts, gann_server_t** out) {
  if (!h || !out) return gann_internal_set_error(GANN_EINVAL, "null argument");
  *out = nullptr;
  gann_server_opts_t o{};
  if (opts) o = *opts;
  if (!o.max_batch) o.max_batch = 1024;
  if (!o.streams) o.streams = 4;
  if (!o.topk_max) o.topk_max = 100;
  if (!o.ef_max) o.ef_max = 512;
  if (!o.max_wait_us) o.max_wait_us = 100;
  if (!opts) o.precision = GANN_PREC_BF16X3;
  if (o.max_batch < 1 || o.streams < 1 || o.streams > 64 || o.topk_max < 1 || o.ef_max < 1 || o.topk_max > 4096 ||
      o.ef_max > 4096 || o.max_wait_us < 0 || o.mem_budget_kib < 0)
    return gann_internal_set_error(GANN_EINVAL, "bad server options");
  auto* sv = new gann_server();
  sv->h = h;
  sv->o = o;
  sv->dim = (int)h->hx.dim;
  sv->M = h->hx.pq_m;
  sv->cap = o.max_batch * (o.streams + 1);
  sv->rq.resize((size_t)sv->cap * sv->dim);
  sv->rk.resize(sv->cap);
  sv->rl.resize(sv->cap);
  sv->rtag.resize(sv->cap);
  sv->rt.resize(sv->cap);
  sv->rcost.resize(sv->cap);
  sv->dcost.resize(sv->cap);
  sv->budget = o.mem_budget_kib > 0 ? (int64_t)o.mem_budget_kib * 1024
                                    : (int64_t)sv->cap * request_bytes(sv, o.topk_max, o.ef_max);
  sv->dtag.resize(sv->cap);
  sv->dfound.resize(sv->cap);
  sv->dlat.resize(sv->cap);
  sv->dids.resize((size_t)sv->cap * o.topk_max);
  sv->ddist.resize((size_t)sv->cap * o.topk_max);
  sv->slots.resize(o.streams);
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(h->device);
  cudaError_t e = cudaSuccess;
  int rc = GANN_OK;
  gann_batch_opts_t bo{};
  bo.precision = o.precision;
  bo.beam_width = o.beam_width;
  bo.hash_bits = o.hash_bits;
  bo.entry = o.entry;
  for (Slot& s : sv->slots) {
    e = alloc_slot(s, o.max_batch, sv->dim, o.topk_max);
    if (e != cudaSuccess) break;
    // The slot's batched search, captured over its buffers; the batch size is read from d_nq.
    rc = gann_batch_graph_create(h, o.max_batch, o.topk_max, o.ef_max, &bo, s.d_q, s.d_k, s.d_l, s.d_nq, s.d_nns,
                                 s.d_d, s.d_f, &s.graph);
    if (rc != GANN_OK) break;
  }
  if (prev >= 0) cudaSetDevice(prev);
  if (e != cudaSuccess || rc != GANN_OK) {
    const std::string msg = e != cudaSuccess ? std::string("server buffers: ") + cudaGetErrorString(e)
                                             : std::string("server batch graph: ") + gann_last_error();
    for (Slot& s : sv->slots) free_slot(s);
    delete sv;
    return gann_internal_set_error(e != cudaSuccess ? GANN_ENOMEM : rc, msg.c_str());
  }
  sv->th = std::thread(dispatcher, sv);
  *out = sv;
  return GANN_OK;
}

int64_t gann_server_request_bytes(const gann_server_t* sv, int topk, int ef_search) {
  if (!sv || topk < 1 || ef_search < 1) return -1;
  return request_bytes(sv, topk, ef_search);
}

int gann_server_submit(gann_server_t* sv, const float* query, int topk, int ef_search, uint64_t tag) {
  if (!sv || !query) return gann_internal_set_error(GANN_EINVAL, "null argument");
  if (topk < 1 || topk > sv->o.topk_max || ef_search < 1 || ef_search > sv->o.ef_max)
    return gann_internal_set_error(GANN_EINVAL, "topk / ef_search outside the server's limits");
  std::lock_guard<std::mutex> lk(sv->mu);
  return submit_locked(sv, query, topk, ef_search, tag, now_s());
}

int gann_server_poll(gann_server_t* sv, int max_results, uint64_t* tags, int32_t* nns, float* distances,
                     int32_t* found_cnt, double* latency, int* n_out) {
  if (!sv || !n_out) return gann_internal_set_error(GANN_EINVAL, "null argument");
  *n_out = 0;
  std::lock_guard<std::mutex> lk(sv->mu);
  const int n = std::min(max_results, sv->dsize);
  const int kmax = sv->o.topk_max;
  for (int i = 0; i < n; i++) {
    const int r = (sv->dhead + i) % sv->cap;
    if (tags) tags[i] = sv->dtag[r];
    if (nns) std::memcpy(nns + (size_t)i * kmax, &sv->dids[(size_t)r * kmax], sizeof(int32_t) * kmax);
    if (distances) std::memcpy(distances + (size_t)i * kmax, &sv->ddist[(size_t)r * kmax], sizeof(float) * kmax);
    if (found_cnt) found_cnt[i] = sv->dfound[r];
    if (latency) latency[i] = sv->dlat[r];
    sv->bytes_held -= sv->dcost[r];
  }
  sv->dhead = (sv->dhead + n) % sv->cap;
  sv->dsize -= n;
  *n_out = n;
  if (sv->error) return gann_internal_set_error(sv->error, sv->error_msg.c_str());
  return GANN_OK;
}

int gann_server_stop(gann_server_t* sv) {
  if (!sv) return GANN_OK;
  sv->stop = true;
  if (sv->th.joinable()) sv->th.join();
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(sv->h->device);
  for (Slot& s : sv->slots) free_slot(s);
  if (prev >= 0) cudaSetDevice(prev);
  delete sv;
  return GANN_OK;
}

int gann_server_open_loop(gann_server_t* sv, const float* queries, int nq, const int32_t* topk,
                          const int32_t* ef_search, double rate_qps, double seconds, uint64_t seed,
                          gann_load_stats_t* out) {
  if (!sv || !queries || nq < 1 || rate_qps <= 0 || seconds <= 0 || !out)
    return gann_internal_set_error(GANN_EINVAL, "bad open-loop arguments");
  std::mt19937_64 rng(seed);
  std::exponential_distribution<double> gap(rate_qps);
  std::vector<double> lat;
  lat.reserve((size_t)(rate_qps * seconds * 1.1) + 16);
  const int poll_max = 4096;
  std::vector<double> lbuf(poll_max);
  int64_t submitted = 0, rejected = 0;
  auto drain = [&]() {
    int n = 0;
    gann_server_poll(sv, poll_max, nullptr, nullptr, nullptr, nullptr, lbuf.data(), &n);
    lat.insert(lat.end(), lbuf.begin(), lbuf.begin() + n);
  };
  // Arrivals follow a Poisson process fixed in advance; each request's latency
  // is measured from its scheduled arrival, so a generator that falls behind
  // shows up as latency, not as a lower offered rate.
  const double t0 = now_s();
  double next = t0 + gap(rng), last_drain = t0;
  int64_t i = 0;
  while (true) {
    const double t = now_s();
    if (t - t0 >= seconds) break;
    if (t >= next) {
      std::lock_guard<std::mutex> lk(sv->mu);
      for (int b = 0; b < 256 && next <= t && next - t0 < seconds; b++, next += gap(rng), i++) {
        const int q = (int)(i % nq);
        const int rc = submit_locked(sv, queries + (size_t)q * sv->dim,
                                     topk ? topk[q] : std::min(10, sv->o.topk_max),
                                     ef_search ? ef_search[q] : sv->o.ef_max, (uint64_t)i, next);
        if (rc == GANN_OK)
          submitted++;
        else if (rc == GANN_EBUSY)
          rejected++;
        else
          return rc;
      }
    }
    if (t - last_drain > 50e-6) {
      drain();
      last_drain = t;
    }
  }
  const double t_end = now_s();
  double t_last = t_end;
  while ((int64_t)lat.size() < submitted && now_s() - t_end < 30.0) {
    const size_t before = lat.size();
    drain();
    if (lat.size() > before) t_last = now_s();
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  std::sort(lat.begin(), lat.end());
  auto pct = [&](double p) { return lat.empty() ? 0.0 : lat[std::min(lat.size() - 1, (size_t)(p * lat.size()))]; };
  double mean = 0.0;
  for (double x : lat) mean += x;
  out->offered_qps = rate_qps;
  out->submitted = submitted;
  out->rejected = rejected;
  out->completed = (int64_t)lat.size();
  out->achieved_qps = (double)lat.size() / std::max(seconds, t_last - t0);
  out->p50_ms = pct(0.50) * 1e3;
  out->p99_ms = pct(0.99) * 1e3;
  out->p999_ms = pct(0.999) * 1e3;
  out->mean_ms = lat.empty() ? 0.0 : mean / lat.size() * 1e3;
  return GANN_OK;
}

}  // extern "C"
