// clue_server.cu -- continuous-batching request loop (clue_server_* in clue_b200.h).
//
// One dispatcher thread per server.  Callers queue single events (clue_server_submit); the
// dispatcher packs the pending events, first come first served, into the next free slot while
// they fit its reserved points / tiles / events, copies them to the slot's device pool and
// enqueues the batched pipeline on the slot's stream.  Slots run concurrently, so events that
// arrive while a batch is on the GPU start as soon as any slot frees up.  Completion is found
// by polling each busy slot's CUDA event; results are copied from the slot's pinned buffers to
// the callers' arrays, with nearest_higher made event-local.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "clue_internal.h"

namespace clue_b200 {
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t ticket = 0;
  int32_t n = 0;
  int32_t tiles = 0;
  const float* coords = nullptr;
  int64_t stride = 0;
  const float* weight = nullptr;
  clue_outputs out{};
  int32_t offset = 0;  // first point inside its batch
  bool done = false;
  clue_request_info info{};
};

struct Slot {
  clue_context ctx = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  float* h_in = nullptr;     // pinned, (ndim + 1) rows of the batch's points
  int32_t* h_out = nullptr;  // pinned, 5 rows of the batch's points + per-event cluster counts
  float* d_in = nullptr;
  int32_t* d_out = nullptr;
  std::vector<int32_t> off;
  std::vector<Request*> reqs;
  int32_t points = 0;
  bool busy = false;
  clue_status launch_status = CLUE_OK;
};

// Tiles a slot reserves for `points` points in up to `events` events.  An event's reference
// grid has ceil(ne / ppbin) tiles rounded up to a power of N, which is below ne + 64 for most
// shapes; batches are formed against the exact per-event counts, so a slot of many tiny
// high-dimensional events simply carries fewer of them.  A tile costs about 16 bytes.
int64_t slot_tiles(int64_t points, int64_t events) { return points + 64 * events + 64; }

int64_t slot_io_bytes(int ndim, int64_t points, int64_t events) {
  return ((int64_t)(ndim + 1) * points + 5 * points + events) * 4;
}

}  // namespace
}  // namespace clue_b200

using namespace clue_b200;

struct clue_server_s {
  clue_server_config cfg{};
  clue_params params{};
  clue_kernel kernel{};
  clue_metric metric{};
  int64_t cap_points = 0, cap_tiles = 0;
  int32_t cap_events = 0;
  std::vector<Slot> slots;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> pending;
  std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;
  int64_t next_ticket = 0;
  bool stop = false;
  std::thread worker;
  Clock::time_point t0 = Clock::now();
  clue_server_stats stats{};
  int32_t in_flight = 0;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace clue_b200 {
namespace {

void free_slot(Slot& s) {
  if (s.stream) cudaStreamSynchronize(s.stream);
  if (s.ctx) clue_context_destroy(s.ctx);
  if (s.done) cudaEventDestroy(s.done);
  if (s.stream) cudaStreamDestroy(s.stream);
  if (s.h_in) cudaFreeHost(s.h_in);
  if (s.h_out) cudaFreeHost(s.h_out);
  if (s.d_in) cudaFree(s.d_in);
  if (s.d_out) cudaFree(s.d_out);
  s = Slot{};
}

clue_status alloc_slot(clue_server_s* S, Slot& s) {
  const int nd = S->cfg.ndim;
  clue_status st = clue_context_create(S->cfg.device, &s.ctx);
  if (st != CLUE_OK) return st;
  st = clue_context_reserve_batch(s.ctx, nd, S->cap_points, S->cap_tiles, S->cap_events);
  if (st != CLUE_OK) return st;
  CLUE_CUDA_TRY(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
  CLUE_CUDA_TRY(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
  const size_t in_words = (size_t)(nd + 1) * S->cap_points;
  const size_t out_words = 5 * (size_t)S->cap_points + S->cap_events;
  CLUE_CUDA_TRY(cudaMallocHost((void**)&s.h_in, in_words * 4));
  CLUE_CUDA_TRY(cudaMallocHost((void**)&s.h_out, out_words * 4));
  CLUE_CUDA_TRY(cudaMalloc((void**)&s.d_in, in_words * 4));
  CLUE_CUDA_TRY(cudaMalloc((void**)&s.d_out, out_words * 4));
  s.off.reserve(S->cap_events + 1);
  s.reqs.reserve(S->cap_events);
  return CLUE_OK;
}

// Packs the slot's requests and enqueues copy-in, pipeline, copy-out and the completion event.
clue_status launch(clue_server_s* S, Slot& s) {
  const int nd = S->cfg.ndim;
  const int64_t P = s.points;
  const int32_t E = (int32_t)s.reqs.size();
  s.off.assign(1, 0);
  for (Request* r : s.reqs) {
    for (int d = 0; d < nd; ++d)
      std::memcpy(s.h_in + (size_t)d * P + r->offset, r->coords + (size_t)d * r->stride, (size_t)r->n * 4);
    std::memcpy(s.h_in + (size_t)nd * P + r->offset, r->weight, (size_t)r->n * 4);
    s.off.push_back(r->offset + r->n);
  }
  CLUE_CUDA_TRY(cudaMemcpyAsync(s.d_in, s.h_in, (size_t)(nd + 1) * P * 4, cudaMemcpyHostToDevice, s.stream));
  clue_outputs o{};
  o.cluster_index = s.d_out;
  o.is_seed = s.d_out + P;
  o.nearest_higher = s.d_out + 2 * P;
  o.rho = reinterpret_cast<float*>(s.d_out + 3 * P);
  o.delta = reinterpret_cast<float*>(s.d_out + 4 * P);
  clue_status st = clue_batch_make_clusters_async(s.ctx, &S->params, &S->kernel, &S->metric, nd, E, s.off.data(),
                                                  s.d_in, s.d_in + (size_t)nd * P, &o, s.d_out + 5 * P, s.stream);
  if (st != CLUE_OK) return st;
  CLUE_CUDA_TRY(cudaMemcpyAsync(s.h_out, s.d_out, (size_t)(5 * P + E) * 4, cudaMemcpyDeviceToHost, s.stream));
  CLUE_CUDA_TRY(cudaEventRecord(s.done, s.stream));
  return CLUE_OK;
}

// Copies a finished slot's results to its requests (called without the server lock).
void deliver(clue_server_s* S, Slot& s, clue_status st) {
  const int64_t P = s.points;
  if (st == CLUE_OK) {
    clue_run_info ri;
    st = clue_context_read_info(s.ctx, s.stream, &ri);  // bounded-wait timeouts, non-finite input
  }
  for (size_t e = 0; e < s.reqs.size(); ++e) {
    Request* r = s.reqs[e];
    r->info.status = st;
    if (st != CLUE_OK) continue;
    r->info.n_clusters = s.h_out[5 * P + e];
    if (!r->out.cluster_index) continue;  // replay without outputs: results stay in the slot
    const size_t b = (size_t)r->n * 4;
    std::memcpy(r->out.cluster_index, s.h_out + r->offset, b);
    if (r->out.is_seed) std::memcpy(r->out.is_seed, s.h_out + P + r->offset, b);
    if (r->out.nearest_higher) {
      const int32_t* nh = s.h_out + 2 * P + r->offset;
      for (int32_t i = 0; i < r->n; ++i) r->out.nearest_higher[i] = nh[i] >= 0 ? nh[i] - r->offset : -1;
    }
    if (r->out.rho) std::memcpy(r->out.rho, s.h_out + 3 * P + r->offset, b);
    if (r->out.delta) std::memcpy(r->out.delta, s.h_out + 4 * P + r->offset, b);
  }
}

void dispatcher(clue_server_s* S) {
  cudaSetDevice(S->cfg.device);
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    bool any_busy = false;
    // completions
    for (size_t k = 0; k < S->slots.size(); ++k) {
      Slot& s = S->slots[k];
      if (!s.busy) continue;
      clue_status st = s.launch_status;
      if (st == CLUE_OK) {
        const cudaError_t q = cudaEventQuery(s.done);
        if (q == cudaErrorNotReady) {
          any_busy = true;
          continue;
        }
        if (q != cudaSuccess) {
          set_error(std::string("server batch failed: ") + cudaGetErrorString(q));
          st = CLUE_ERR_CUDA;
        }
      }
      lk.unlock();
      deliver(S, s, st);
      lk.lock();
      const double t = S->now();
      for (Request* r : s.reqs) {
        r->info.done_s = t;
        r->done = true;
        if (r->info.status == CLUE_OK)
          ++S->stats.completed;
        else
          ++S->stats.failed;
      }
      s.reqs.clear();
      s.busy = false;
      --S->in_flight;
      S->cv_done.notify_all();
    }
    if (S->stop) {
      if (any_busy) {
        S->cv_work.wait_for(lk, std::chrono::microseconds(50));
        continue;
      }
      break;
    }
    // admissions
    for (size_t k = 0; k < S->slots.size() && !S->pending.empty(); ++k) {
      Slot& s = S->slots[k];
      if (s.busy) continue;
      int64_t points = 0, tiles = 0;
      while (!S->pending.empty() && (int32_t)s.reqs.size() < S->cap_events) {
        Request* r = S->pending.front();
        if (points + r->n > S->cap_points || tiles + r->tiles > S->cap_tiles) break;
        S->pending.pop_front();
        r->offset = (int32_t)points;
        points += r->n;
        tiles += r->tiles;
        s.reqs.push_back(r);
      }
      if (s.reqs.empty()) break;  // head of the queue waits for an empty slot
      s.points = (int32_t)points;
      s.busy = true;
      ++S->in_flight;
      S->stats.max_in_flight = std::max(S->stats.max_in_flight, S->in_flight);
      ++S->stats.batches;
      S->stats.batched_points += points;
      S->stats.max_batch_seen = std::max(S->stats.max_batch_seen, (int32_t)s.reqs.size());
      const double t = S->now();
      for (Request* r : s.reqs) {
        r->info.start_s = t;
        r->info.slot = (int32_t)k;
        r->info.batch_events = (int32_t)s.reqs.size();
      }
      lk.unlock();
      s.launch_status = launch(S, s);
      if (s.launch_status != CLUE_OK) cudaStreamSynchronize(s.stream);  // nothing may still read h_in
      lk.lock();
      any_busy = true;
    }
    if (any_busy)
      S->cv_work.wait_for(lk, std::chrono::microseconds(20));
    else if (S->pending.empty() && !S->stop)
      S->cv_work.wait(lk);
  }
  // fail whatever is still queued
  for (Request* r : S->pending) {
    r->info.status = CLUE_ERR_INVALID_ARG;
    r->done = true;
    ++S->stats.failed;
  }
  S->pending.clear();
  S->cv_done.notify_all();
}

}  // namespace
}  // namespace clue_b200

extern "C" {

clue_status clue_server_create(const clue_server_config* config, const clue_params* params,
                               const clue_kernel* kernel, const clue_metric* metric, clue_server* server) {
  if (!config || !params || !kernel || !metric || !server) {
    set_error("clue_server_create: null argument");
    return CLUE_ERR_INVALID_ARG;
  }
  const clue_server_config& c = *config;
  if (c.ndim < 1 || c.ndim > CLUE_MAX_DIM || c.n_slots < 1 || c.n_slots > 16 || c.max_batch_events < 1 ||
      c.max_event_points < 1 || c.max_pending < 1 || c.device_budget_bytes <= 0) {
    set_error("clue_server_create: invalid configuration");
    return CLUE_ERR_INVALID_ARG;
  }
  clue_status st;
  if ((st = clue_check_params(params)) != CLUE_OK) return st;
  if ((st = clue_check_kernel(kernel)) != CLUE_OK) return st;
  if ((st = clue_check_metric(metric, c.ndim)) != CLUE_OK) return st;
  // Largest slot (points) whose pools fit the budget, by bisection on the arena layout.
  const int64_t E = c.max_batch_events;
  auto slot_bytes = [&](int64_t p) -> int64_t {
    const int64_t t = slot_tiles(p, E);
    return (int64_t)workspace_bytes_for(c.ndim, (size_t)p, (size_t)t, (size_t)E) + slot_io_bytes(c.ndim, p, E);
  };
  const int64_t per_slot = c.device_budget_bytes / c.n_slots;
  int64_t lo = 0, hi = 1;
  while (hi < 2000000000ll && slot_bytes(hi) <= per_slot) hi *= 2;
  while (hi - lo > 1) {
    const int64_t mid = lo + (hi - lo) / 2;
    (slot_bytes(mid) <= per_slot ? lo : hi) = mid;
  }
  int32_t npd = 0, nt_max = 0;
  grid_shape(c.max_event_points, params->points_per_tile, c.ndim, &npd, &nt_max);
  if (lo < c.max_event_points || slot_tiles(lo, E) < nt_max) {
    set_error("clue_server_create: device budget of " + std::to_string(c.device_budget_bytes) + " bytes over " +
              std::to_string(c.n_slots) + " slots cannot hold an event of " + std::to_string(c.max_event_points) +
              " points");
    return CLUE_ERR_CAPACITY;
  }
  auto* S = new (std::nothrow) clue_server_s;
  if (!S) return CLUE_ERR_OUT_OF_MEMORY;
  S->cfg = c;
  S->params = *params;
  S->kernel = *kernel;
  S->metric = *metric;
  S->cap_points = std::min<int64_t>(lo, 2147483000ll);
  S->cap_tiles = slot_tiles(S->cap_points, E);
  S->cap_events = (int32_t)E;
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(c.device) != cudaSuccess) {
    cudaGetLastError();
    delete S;
    set_error("clue_server_create: no CUDA device " + std::to_string(c.device));
    return CLUE_ERR_CUDA;
  }
  S->slots.resize(c.n_slots);
  for (auto& s : S->slots) {
    st = alloc_slot(S, s);
    if (st != CLUE_OK) {
      for (auto& q : S->slots) free_slot(q);
      delete S;
      cudaSetDevice(prev);
      return st;
    }
  }
  cudaSetDevice(prev);
  S->stats.slot_points = S->cap_points;
  S->stats.slot_events = S->cap_events;
  S->stats.device_bytes = (int64_t)c.n_slots * slot_bytes(S->cap_points);
  S->t0 = Clock::now();
  S->worker = std::thread(dispatcher, S);
  *server = S;
  return CLUE_OK;
}

clue_status clue_server_destroy(clue_server S) {
  if (!S) return CLUE_OK;
  {
    std::lock_guard<std::mutex> g(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->worker.joinable()) S->worker.join();
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(S->cfg.device);
  for (auto& s : S->slots) free_slot(s);
  cudaSetDevice(prev);
  delete S;
  return CLUE_OK;
}

}  // extern "C"

namespace clue_b200 {
namespace {

// Queues one event; out == nullptr leaves the results in the slot (load replay).
clue_status submit_impl(clue_server S, int32_t n, const float* coords, int64_t coord_stride, const float* weight,
                        const clue_outputs* out, int64_t* ticket) {
  if (!S || !coords || !weight || !ticket || n <= 0 || coord_stride < n) {
    set_error("clue_server_submit: null argument, n <= 0 or coord_stride < n");
    return CLUE_ERR_INVALID_ARG;
  }
  if (n > S->cfg.max_event_points) {
    set_error("clue_server_submit: event of " + std::to_string(n) + " points exceeds max_event_points");
    std::lock_guard<std::mutex> g(S->mu);
    ++S->stats.rejected;
    return CLUE_ERR_CAPACITY;
  }
  for (int d = 0; d < S->cfg.ndim; ++d)
    for (int32_t i = 0; i < n; ++i)
      if (!std::isfinite(coords[(size_t)d * coord_stride + i])) {
        set_error("clue_server_submit: non-finite coordinate");
        return CLUE_ERR_NONFINITE;
      }
  for (int32_t i = 0; i < n; ++i)
    if (!std::isfinite(weight[i])) {
      set_error("clue_server_submit: non-finite weight");
      return CLUE_ERR_NONFINITE;
    }
  int32_t npd = 0, nt = 0;
  grid_shape(n, S->params.points_per_tile, S->cfg.ndim, &npd, &nt);
  auto r = std::make_unique<Request>();
  r->n = n;
  r->tiles = nt;
  r->coords = coords;
  r->stride = coord_stride;
  r->weight = weight;
  if (out) r->out = *out;
  {
    std::lock_guard<std::mutex> g(S->mu);
    if (S->stop) {
      set_error("clue_server_submit: server is shutting down");
      return CLUE_ERR_INVALID_ARG;
    }
    if ((int64_t)S->pending.size() >= S->cfg.max_pending) {
      ++S->stats.rejected;
      set_error("clue_server_submit: queue full");
      return CLUE_ERR_CAPACITY;
    }
    r->ticket = S->next_ticket++;
    r->info.submit_s = S->now();
    *ticket = r->ticket;
    S->pending.push_back(r.get());
    S->reqs.emplace(r->ticket, std::move(r));
    ++S->stats.submitted;
  }
  S->cv_work.notify_one();
  return CLUE_OK;
}

}  // namespace
}  // namespace clue_b200

extern "C" {

clue_status clue_server_submit(clue_server S, int32_t n, const float* coords, int64_t coord_stride,
                               const float* weight, const clue_outputs* out, int64_t* ticket) {
  if (!out || !out->cluster_index) {
    set_error("clue_server_submit: out->cluster_index must be non-null");
    return CLUE_ERR_INVALID_ARG;
  }
  return submit_impl(S, n, coords, coord_stride, weight, out, ticket);
}

clue_status clue_server_wait(clue_server S, int64_t ticket, int32_t timeout_ms, clue_request_info* info) {
  if (!S) return CLUE_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) {
    set_error("clue_server_wait: unknown ticket " + std::to_string(ticket));
    return CLUE_ERR_INVALID_ARG;
  }
  Request* r = it->second.get();
  auto ready = [&] { return r->done; };
  if (timeout_ms < 0)
    S->cv_done.wait(lk, ready);
  else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    set_error("clue_server_wait: request not finished");
    return CLUE_ERR_TIMEOUT;
  }
  if (info) *info = r->info;
  const clue_status st = (clue_status)r->info.status;
  S->reqs.erase(it);
  return st;
}

clue_status clue_server_stats_read(clue_server S, clue_server_stats* stats) {
  if (!S || !stats) return CLUE_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(S->mu);
  *stats = S->stats;
  return CLUE_OK;
}

clue_status clue_server_replay(clue_server S, int32_t n_events, const int32_t* event_ids, const int32_t* off,
                               const double* arrival_s, const float* coords, const float* weight,
                               const clue_outputs* out, double* latency_s, int32_t* n_rejected) {
  if (!S || n_events <= 0 || !off || !arrival_s || !coords || !weight || !latency_s || (event_ids && out) ||
      (out && !out->cluster_index)) {
    set_error("clue_server_replay: null argument, n_events <= 0, or outputs requested with event_ids");
    return CLUE_ERR_INVALID_ARG;
  }
  int32_t n_pool = event_ids ? 0 : n_events;  // events in the pool: event_offsets holds n_pool + 1 entries
  if (event_ids)
    for (int32_t e = 0; e < n_events; ++e) n_pool = std::max(n_pool, event_ids[e] + 1);
  const int64_t n_total = off[n_pool];
  std::vector<int64_t> tickets((size_t)n_events, -1);
  int32_t rejected = 0;
  clue_status result = CLUE_OK;
  const double base = S->now();
  for (int32_t e = 0; e < n_events; ++e) {
    const double target = base + arrival_s[e];
    for (double t = S->now(); t < target; t = S->now())
      if (target - t > 200e-6) std::this_thread::sleep_for(std::chrono::microseconds(50));
    const int32_t id = event_ids ? event_ids[e] : e;
    if (id < 0) {
      set_error("clue_server_replay: negative event id");
      result = CLUE_ERR_INVALID_ARG;
      continue;
    }
    const int32_t a = off[id];
    clue_outputs o{};
    if (out) {
      o.cluster_index = out->cluster_index + a;
      o.is_seed = out->is_seed ? out->is_seed + a : nullptr;
      o.rho = out->rho ? out->rho + a : nullptr;
      o.nearest_higher = out->nearest_higher ? out->nearest_higher + a : nullptr;
      o.delta = out->delta ? out->delta + a : nullptr;
    }
    const clue_status st =
        submit_impl(S, off[id + 1] - a, coords + a, n_total, weight + a, out ? &o : nullptr, &tickets[e]);
    if (st != CLUE_OK) {
      tickets[e] = -1;
      if (st == CLUE_ERR_CAPACITY)
        ++rejected;
      else
        result = st;
    }
  }
  for (int32_t e = 0; e < n_events; ++e) {
    latency_s[e] = -1.0;
    if (tickets[e] < 0) continue;
    clue_request_info info{};
    const clue_status st = clue_server_wait(S, tickets[e], -1, &info);
    if (st != CLUE_OK) {
      result = st;
      continue;
    }
    latency_s[e] = info.done_s - (base + arrival_s[e]);
  }
  if (n_rejected) *n_rejected = rejected;
  return result;
}

}  // extern "C"
