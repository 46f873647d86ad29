// clue_capi.cu -- the extern "C" entry points of libclue_b200.so (include/clue_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "clue_internal.h"

namespace clue_b200 {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

template <int N>
clue_status finish_labels(Workspace& ws, const RunArgs& a, cudaStream_t s, int first_round);

#define CLUE_DECLARE_DIM(N)                                                      \
  extern template clue_status run_pipeline<N>(Workspace&, const RunArgs&, cudaStream_t); \
  extern template clue_status finish_labels<N>(Workspace&, const RunArgs&, cudaStream_t, int);
CLUE_DECLARE_DIM(1)
CLUE_DECLARE_DIM(2)
CLUE_DECLARE_DIM(3)
CLUE_DECLARE_DIM(4)
CLUE_DECLARE_DIM(5)
CLUE_DECLARE_DIM(6)
CLUE_DECLARE_DIM(7)
CLUE_DECLARE_DIM(8)
CLUE_DECLARE_DIM(9)
CLUE_DECLARE_DIM(10)

clue_status run_pipeline_dispatch(Workspace& ws, const RunArgs& a, cudaStream_t s) {
  switch (a.ndim) {
    case 1: return run_pipeline<1>(ws, a, s);
    case 2: return run_pipeline<2>(ws, a, s);
    case 3: return run_pipeline<3>(ws, a, s);
    case 4: return run_pipeline<4>(ws, a, s);
    case 5: return run_pipeline<5>(ws, a, s);
    case 6: return run_pipeline<6>(ws, a, s);
    case 7: return run_pipeline<7>(ws, a, s);
    case 8: return run_pipeline<8>(ws, a, s);
    case 9: return run_pipeline<9>(ws, a, s);
    case 10: return run_pipeline<10>(ws, a, s);
  }
  set_error("ndim must be in [1, 10]");
  return CLUE_ERR_INVALID_ARG;
}

static clue_status finish_labels_dispatch(Workspace& ws, const RunArgs& a, cudaStream_t s, int first) {
  switch (a.ndim) {
    case 1: return finish_labels<1>(ws, a, s, first);
    case 2: return finish_labels<2>(ws, a, s, first);
    case 3: return finish_labels<3>(ws, a, s, first);
    case 4: return finish_labels<4>(ws, a, s, first);
    case 5: return finish_labels<5>(ws, a, s, first);
    case 6: return finish_labels<6>(ws, a, s, first);
    case 7: return finish_labels<7>(ws, a, s, first);
    case 8: return finish_labels<8>(ws, a, s, first);
    case 9: return finish_labels<9>(ws, a, s, first);
    case 10: return finish_labels<10>(ws, a, s, first);
  }
  return CLUE_ERR_INVALID_ARG;
}

// core/detail/SetupTiles.hpp:23-26.
void grid_shape(int32_t n, int32_t ppbin, int32_t ndim, int32_t* nperdim, int32_t* ntiles) {
  const int32_t t0 = (int32_t)std::ceil((float)n / (float)ppbin);
  // The shape depends only on (t0, ndim).  A batch computes it for every event several times
  // (validation, event tables, chunk plans), and the two pow() calls cost about 60 ns: a small
  // direct-mapped per-thread cache keeps that host work off the timed path of a batched call.
  struct Entry {
    int32_t t0 = -1, ndim = 0, npd = 0, nt = 0;
  };
  thread_local Entry cache[1024];
  Entry& c = cache[((uint32_t)t0 * 16u + (uint32_t)ndim) & 1023u];
  if (c.t0 == t0 && c.ndim == ndim) {
    *nperdim = c.npd;
    *ntiles = c.nt;
    return;
  }
  const int32_t npd = (int32_t)std::ceil(std::pow((double)t0, 1.0 / (double)ndim));
  const int32_t nt = (int32_t)std::pow((double)npd, (double)ndim);
  c.t0 = t0;
  c.ndim = ndim;
  c.npd = npd;
  c.nt = nt;
  *nperdim = npd;
  *ntiles = nt;
}

// Largest s with sqrtf(s) <= r (sqrtf is correctly rounded on host and device, so
// `s <= threshold_for(r)` decides exactly what `sqrtf(s) <= r` decides); r itself for
// metrics without a square root.
float threshold_for(float r, bool root) {
  if (!root) return r;
  float s = (float)((double)r * (double)r);
  if (!std::isfinite(s)) s = FLT_MAX;
  while (s > 0.0f && std::sqrt(s) > r) s = std::nextafter(s, 0.0f);
  while (true) {
    const float nx = std::nextafter(s, INFINITY);
    if (std::isfinite(nx) && std::sqrt(nx) <= r)
      s = nx;
    else
      break;
  }
  return s;
}

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Box lower bounds of the metrics hold when no weight is negative (or NaN).
int lower_bounds_ok(const clue_metric* m, int ndim) {
  if (m->type == CLUE_METRIC_WEIGHTED_EUCLIDEAN || m->type == CLUE_METRIC_WEIGHTED_CHEBYSHEV)
    for (int d = 0; d < ndim; ++d)
      if (!(m->par[d] >= 0.0f)) return 0;
  return 1;
}

namespace {

struct ArenaItem {
  void** ptr;
  size_t bytes;
};

// The buffers of the workspace arena for n points, ntiles tiles, n_events events and w record
// words; `nw` receives the carved pointers once an arena is placed (arena_place).
std::vector<ArenaItem> arena_items(Workspace& nw, void** evtab, size_t n, size_t ntiles, size_t n_events, size_t w) {
  const size_t nb = (size_t)sort_blocks((int)n);
  const size_t hist_len = hist_words(nb);
  const size_t scan_words = scan_scratch_words(std::max(std::max(hist_len, n), ntiles)) + 1;
  return {
      {evtab, event_table_bytes(n_events)},
      {(void**)&nw.status, sizeof(DevStatus)},
      {(void**)&nw.keys[0], n * 4},
      {(void**)&nw.keys[1], n * 4},
      {(void**)&nw.vals[0], n * 4},
      {(void**)&nw.vals[1], n * 4},
      {(void**)&nw.hist, hist_len * 4},
      {(void**)&nw.scan_scratch, scan_words * 4},
      {(void**)&nw.offsets, (ntiles + 1) * 4},
      {(void**)&nw.rec_w, n * w * 16},
      {(void**)&nw.rec_r, n * w * 16},
      {(void**)&nw.delta_s, n * 4},
      {(void**)&nw.nh_s, n * 4},
      {(void**)&nw.par, n * 4},
      {(void**)&nw.is_seed_s, n * 4},
      {(void**)&nw.seed_flag, n * 4},
      {(void**)&nw.seed_total, 16},
      {(void**)&nw.blk, (n / 32 + 1) * 6 * 16},
      {(void**)&nw.mq_alt, n * 4},
      {(void**)&nw.mkeys_alt, n * 4},
      {(void**)&nw.rec_m, n * w * 16},
      {(void**)&nw.sblk, (n / 1024 + 1) * 6 * 16},
      {(void**)&nw.ord_rho, n * 4},
      {(void**)&nw.chunk_count, (ntiles + 1) * 4},
      {(void**)&nw.chunk_tile, (n / kChunkPoints + ntiles + 1) * 4},
      {(void**)&nw.chunk_total, 16},
      {(void**)&nw.tblk, std::min(n, n / 32 + ntiles + 1) * 2 * w * 16},
      {(void**)&nw.tblk_off, (ntiles + 1) * 4},
      {(void**)&nw.rho_fix, n * 8},
      {(void**)&nw.ev_chunk, ((n >> 10) + 1) * 4},
  };
}

size_t arena_total(const std::vector<ArenaItem>& items) {
  size_t total = 0;
  for (auto& it : items) total = align_up(total, 256) + align_up(it.bytes, 256);
  return total;
}

}  // namespace

size_t workspace_bytes_for(int ndim, size_t n, size_t ntiles, size_t n_events) {
  Workspace nw;
  void* evtab = nullptr;
  return arena_total(arena_items(nw, &evtab, n, ntiles, n_events, (size_t)((ndim + 1 + 3) / 4)));
}

clue_status workspace_reserve(Workspace& ws, int ndim, size_t n, size_t ntiles, size_t n_events) {
  const size_t words = (size_t)((ndim + 1 + 3) / 4);
  if (n <= ws.cap_n && ntiles <= ws.cap_tiles && words <= ws.cap_words && n_events <= ws.cap_events && ws.arena)
    return CLUE_OK;
  n = std::max(n, ws.cap_n);
  ntiles = std::max(ntiles, ws.cap_tiles);
  n_events = std::max(n_events, ws.cap_events);
  const size_t w = std::max(words, ws.cap_words);
  Workspace nw = ws;
  void* evtab = nullptr;
  const std::vector<ArenaItem> items = arena_items(nw, &evtab, n, ntiles, n_events, w);
  const size_t total = arena_total(items);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ws.device);
  if (ws.arena) {
    cudaDeviceSynchronize();
    cudaFree(ws.arena);
    ws.arena = nullptr;
  }
  void* arena = nullptr;
  cudaError_t e = cudaMalloc(&arena, total);
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaSetDevice(prev);
    ws.cap_n = ws.cap_tiles = ws.cap_words = ws.cap_events = 0;
    set_error(std::string("workspace allocation of ") + std::to_string(total) + " bytes failed: " +
              cudaGetErrorString(e));
    return CLUE_ERR_OUT_OF_MEMORY;
  }
  size_t offset = 0;
  for (auto& it : items) {
    offset = align_up(offset, 256);
    *it.ptr = static_cast<char*>(arena) + offset;
    offset += align_up(it.bytes, 256);
  }
  event_table_carve(evtab, n_events, &nw.ev, &nw.ev_pt, &nw.ev_tile);
  nw.arena = arena;
  nw.arena_bytes = total;
  nw.cap_n = n;
  nw.cap_tiles = ntiles;
  nw.cap_words = w;
  nw.cap_events = n_events;
  if (nw.pinned_bytes < event_table_bytes(n_events)) {
    if (nw.pinned) cudaFreeHost(nw.pinned);
    nw.pinned = nullptr;
    nw.pinned_bytes = 0;
    e = cudaMallocHost(&nw.pinned, event_table_bytes(n_events));
    if (e != cudaSuccess) {
      cudaGetLastError();
      cudaSetDevice(prev);
      set_error("pinned event-table allocation failed");
      return CLUE_ERR_OUT_OF_MEMORY;
    }
    nw.pinned_bytes = event_table_bytes(n_events);
  }
  if (!nw.status_host) {
    e = cudaMallocHost((void**)&nw.status_host, sizeof(DevStatus) + 64);
    if (e != cudaSuccess) {
      cudaGetLastError();
      cudaSetDevice(prev);
      set_error("pinned status allocation failed");
      return CLUE_ERR_OUT_OF_MEMORY;
    }
  }
  ws = nw;
  cudaSetDevice(prev);
  return CLUE_OK;
}

static clue_status reserve_stage(Workspace& ws, size_t bytes) {
  if (bytes <= ws.dstage_bytes) return CLUE_OK;
  if (ws.dstage) {
    cudaDeviceSynchronize();
    cudaFree(ws.dstage);
    ws.dstage = nullptr;
    ws.dstage_bytes = 0;
  }
  CLUE_CUDA_TRY(cudaMalloc(&ws.dstage, bytes));
  ws.dstage_bytes = bytes;
  return CLUE_OK;
}

void workspace_release(Workspace& ws) {
  for (auto& e : ws.tev)
    if (e) cudaEventDestroy(e);
  for (auto& e : ws.pipe_ev)
    if (e) cudaEventDestroy(e);
  if (ws.pipe_h2d) cudaStreamDestroy(ws.pipe_h2d);
  if (ws.pipe_d2h) cudaStreamDestroy(ws.pipe_d2h);
  if (ws.pipe_status_host) cudaFreeHost(ws.pipe_status_host);
  if (ws.pipe_pinned) cudaFreeHost(ws.pipe_pinned);
  if (ws.arena) cudaFree(ws.arena);
  if (ws.dstage) cudaFree(ws.dstage);
  if (ws.status_host) cudaFreeHost(ws.status_host);
  if (ws.pinned) cudaFreeHost(ws.pinned);
  ws = Workspace{};
}

static clue_status check_finite(float v, const char* what) {
  if (!std::isfinite(v)) {
    set_error(std::string(what) + " must be finite");
    return CLUE_ERR_INVALID_ARG;
  }
  return CLUE_OK;
}

template <int N>
float metric_eval_n(int32_t type, const float* a, const float* b, const float* par) {
  switch (type) {
    case CLUE_METRIC_EUCLIDEAN: {
      using M = Metric<N, CLUE_METRIC_EUCLIDEAN>;
      return M::finish(M::partial(a, b, par));
    }
    case CLUE_METRIC_WEIGHTED_EUCLIDEAN: {
      using M = Metric<N, CLUE_METRIC_WEIGHTED_EUCLIDEAN>;
      return M::finish(M::partial(a, b, par));
    }
    case CLUE_METRIC_PERIODIC_EUCLIDEAN: {
      using M = Metric<N, CLUE_METRIC_PERIODIC_EUCLIDEAN>;
      return M::finish(M::partial(a, b, par));
    }
    case CLUE_METRIC_MANHATTAN: {
      using M = Metric<N, CLUE_METRIC_MANHATTAN>;
      return M::finish(M::partial(a, b, par));
    }
    case CLUE_METRIC_CHEBYSHEV: {
      using M = Metric<N, CLUE_METRIC_CHEBYSHEV>;
      return M::finish(M::partial(a, b, par));
    }
    default: {
      using M = Metric<N, CLUE_METRIC_WEIGHTED_CHEBYSHEV>;
      return M::finish(M::partial(a, b, par));
    }
  }
}

}  // namespace clue_b200

namespace clue_b200 {

// keys[i] = cluster_index[i] + 1 (0 for outliers); labels outside [-1, n) raise *bad and count
// as outliers so that every key stays inside the offsets table.
__global__ void k_label_keys(const int32_t* __restrict__ label, int n, uint32_t* __restrict__ keys,
                             int32_t* __restrict__ bad) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int l = label[i];
    const bool ok = l >= -1 && l < n;
    if (!ok) atomicOr(bad, 1);
    keys[i] = ok ? (uint32_t)(l + 1) : 0u;
  }
}

// off[k] = first sorted position of key k (k = 0..n+1); key 0 holds the outliers, so cluster c
// owns sorted positions [off[c + 1], off[c + 2]).  Writes offsets[0..n] and the clustered points.
__global__ void k_cluster_csr(const int32_t* __restrict__ off, const int32_t* __restrict__ vals, int n,
                              int32_t* __restrict__ offsets, int32_t* __restrict__ points) {
  const int first = off[1];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
    offsets[i] = off[i + 1] - first;
    if (i < n - first) points[i] = vals[first + i];
  }
}

}  // namespace clue_b200

using namespace clue_b200;

struct clue_context_s {
  Workspace ws;
  // A second workspace and stream for the odd chunks of an overlapped host-memory batch, so that
  // consecutive chunks' pipelines run concurrently (created on the first such batch).
  Workspace* alt = nullptr;
  cudaStream_t alt_stream = nullptr;
  // The overlapped host batch's even chunks run on chunk_stream (a stream of the context, so a
  // caller's legacy default stream never has to be captured), and every chunk's pipeline is
  // captured into a graph whose executable is kept here and updated in place on the next call.
  cudaGraphExec_t chunk_exec[Workspace::kPipeMaxChunks] = {};
  cudaStream_t chunk_stream = nullptr;
  // the same for the pipeline of a blocking call (run_pipeline_graph)
  cudaGraphExec_t plain_exec = nullptr;
  cudaEvent_t plain_ev[2] = {};
};

// Captures the pipeline enqueued by run_pipeline_dispatch on `g` into a graph and launches it
// there, keeping the executable in *exec (updated in place when the captured graph has the same
// shape, else instantiated again).
static clue_status capture_and_launch(Workspace& w, const RunArgs& a, cudaStream_t g, cudaGraphExec_t* exec) {
  const bool timing = w.timing;
  w.timing = false;
  cudaGraph_t cg = nullptr;
  clue_status st = CLUE_OK;
  cudaError_t ce = cudaStreamBeginCapture(g, cudaStreamCaptureModeThreadLocal);
  if (ce == cudaSuccess) {
    st = run_pipeline_dispatch(w, a, g);
    ce = cudaStreamEndCapture(g, &cg);
  }
  w.timing = timing;
  if (ce == cudaSuccess && st == CLUE_OK) {
    cudaGraphExecUpdateResultInfo ui;
    if (!*exec || cudaGraphExecUpdate(*exec, cg, &ui) != cudaSuccess) {
      cudaGetLastError();
      if (*exec) cudaGraphExecDestroy(*exec);
      *exec = nullptr;
      ce = cudaGraphInstantiate(exec, cg, 0);
    }
    if (ce == cudaSuccess) ce = cudaGraphLaunch(*exec, g);
  }
  if (cg) cudaGraphDestroy(cg);
  if (st == CLUE_OK && ce != cudaSuccess) {
    set_error(std::string("pipeline graph: ") + cudaGetErrorString(ce));
    st = CLUE_ERR_CUDA;
  }
  return st;
}

// One pipeline of a blocking host-memory call as a graph launch on the context's chunk stream,
// ordered after the work already on the caller's stream s and before its next: enqueued kernel
// by kernel, the launch gaps cost several microseconds per kernel.  (A stream of the context,
// since a caller's legacy default stream cannot be captured.)
static clue_status run_pipeline_graph(clue_context ctx, const RunArgs& a, cudaStream_t s) {
  Workspace& ws = ctx->ws;
  if (ws.timing) return run_pipeline_dispatch(ws, a, s);  // stage timing records events per stage
  if (!ctx->chunk_stream) CLUE_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->chunk_stream, cudaStreamNonBlocking));
  for (auto& e : ctx->plain_ev)
    if (!e) CLUE_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaStream_t g = ctx->chunk_stream;
  CLUE_CUDA_TRY(cudaEventRecord(ctx->plain_ev[0], s));
  CLUE_CUDA_TRY(cudaStreamWaitEvent(g, ctx->plain_ev[0], 0));
  const clue_status st = capture_and_launch(ws, a, g, &ctx->plain_exec);
  CLUE_CUDA_TRY(cudaEventRecord(ctx->plain_ev[1], g));
  CLUE_CUDA_TRY(cudaStreamWaitEvent(s, ctx->plain_ev[1], 0));
  return st;
}

extern "C" {

int32_t clue_abi_version(void) { return CLUE_ABI_VERSION; }

const char* clue_last_error(void) { return g_last_error.c_str(); }

const char* clue_status_string(clue_status s) {
  switch (s) {
    case CLUE_OK: return "ok";
    case CLUE_ERR_INVALID_ARG: return "invalid argument";
    case CLUE_ERR_OUT_OF_MEMORY: return "out of memory";
    case CLUE_ERR_CAPACITY: return "capacity exceeded";
    case CLUE_ERR_TIMEOUT: return "timeout";
    case CLUE_ERR_CUDA: return "cuda error";
    case CLUE_ERR_NOT_SUPPORTED: return "not supported";
    case CLUE_ERR_NONFINITE: return "non-finite input";
    case CLUE_ERR_OUT_OF_RANGE: return "out of range";
  }
  return "unknown";
}

clue_status clue_check_params(const clue_params* p) {
  if (!p) {
    set_error("params is null");
    return CLUE_ERR_INVALID_ARG;
  }
  for (float v : {p->dc, p->rhoc, p->dm, p->seed_dc})
    if (check_finite(v, "clustering parameters") != CLUE_OK) return CLUE_ERR_INVALID_ARG;
  if (p->dc <= 0.f || p->rhoc < 0.f || p->dm <= 0.f || p->seed_dc <= 0.f || p->points_per_tile <= 0) {
    set_error("Invalid clustering parameters. The parameters must be positive.");
    return CLUE_ERR_INVALID_ARG;
  }
  if (p->tiebreak != CLUE_TIE_REFERENCE && p->tiebreak != CLUE_TIE_RHO_INDEX) {
    set_error("unknown tiebreak");
    return CLUE_ERR_INVALID_ARG;
  }
  return CLUE_OK;
}

clue_status clue_check_kernel(const clue_kernel* k) {
  if (!k) {
    set_error("kernel is null");
    return CLUE_ERR_INVALID_ARG;
  }
  switch (k->type) {
    case CLUE_KERNEL_FLAT:
      if (!(k->par[0] > 0.f) || !std::isfinite(k->par[0])) {
        set_error("Flat kernel parameter must be positive.");
        return CLUE_ERR_INVALID_ARG;
      }
      return CLUE_OK;
    case CLUE_KERNEL_EXPONENTIAL:
      if (!(k->par[0] > 0.f) || !(k->par[1] > 0.f) || !std::isfinite(k->par[0]) || !std::isfinite(k->par[1])) {
        set_error("Exponential kernel parameters must be positive.");
        return CLUE_ERR_INVALID_ARG;
      }
      return CLUE_OK;
    case CLUE_KERNEL_GAUSSIAN:
      if (!(k->par[0] >= 0.f) || !(k->par[1] > 0.f) || !(k->par[2] > 0.f) || !std::isfinite(k->par[0]) ||
          !std::isfinite(k->par[1]) || !std::isfinite(k->par[2])) {
        set_error("Gaussian kernel parameters must be positive (mean may be 0).");
        return CLUE_ERR_INVALID_ARG;
      }
      return CLUE_OK;
  }
  set_error("unknown kernel type");
  return CLUE_ERR_INVALID_ARG;
}

clue_status clue_check_metric(const clue_metric* m, int32_t ndim) {
  if (!m) {
    set_error("metric is null");
    return CLUE_ERR_INVALID_ARG;
  }
  if (m->type < CLUE_METRIC_EUCLIDEAN || m->type > CLUE_METRIC_WEIGHTED_CHEBYSHEV) {
    set_error("unknown metric type");
    return CLUE_ERR_INVALID_ARG;
  }
  if (ndim < 1 || ndim > CLUE_MAX_DIM) {
    set_error("ndim must be in [1, 10]");
    return CLUE_ERR_INVALID_ARG;
  }
  for (int d = 0; d < ndim; ++d)
    if (!std::isfinite(m->par[d])) {
      set_error("metric parameters must be finite");
      return CLUE_ERR_INVALID_ARG;
    }
  return CLUE_OK;
}

clue_status clue_grid_shape(int32_t n, int32_t ppbin, int32_t ndim, int32_t* n_per_dim, int32_t* n_tiles) {
  if (n <= 0 || ppbin <= 0 || ndim < 1 || ndim > CLUE_MAX_DIM || !n_per_dim || !n_tiles) {
    set_error("invalid grid request");
    return CLUE_ERR_INVALID_ARG;
  }
  grid_shape(n, ppbin, ndim, n_per_dim, n_tiles);
  return CLUE_OK;
}

float clue_metric_eval(const clue_metric* m, int32_t ndim, const float* a, const float* b) {
  if (!m || !a || !b) return NAN;
  switch (ndim) {
    case 1: return metric_eval_n<1>(m->type, a, b, m->par);
    case 2: return metric_eval_n<2>(m->type, a, b, m->par);
    case 3: return metric_eval_n<3>(m->type, a, b, m->par);
    case 4: return metric_eval_n<4>(m->type, a, b, m->par);
    case 5: return metric_eval_n<5>(m->type, a, b, m->par);
    case 6: return metric_eval_n<6>(m->type, a, b, m->par);
    case 7: return metric_eval_n<7>(m->type, a, b, m->par);
    case 8: return metric_eval_n<8>(m->type, a, b, m->par);
    case 9: return metric_eval_n<9>(m->type, a, b, m->par);
    case 10: return metric_eval_n<10>(m->type, a, b, m->par);
  }
  return NAN;
}

float clue_kernel_eval(const clue_kernel* k, float dist, int32_t i, int32_t j) {
  if (!k) return NAN;
  if (i == j) return 1.0f;
  return kernel_value(k->type, k->par, dist);
}

clue_status clue_device_count(int32_t* count) {
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *count = 0;
    set_error(std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
    return CLUE_ERR_CUDA;
  }
  *count = c;
  return CLUE_OK;
}

clue_status clue_device_alloc(int32_t device, size_t bytes, void** ptr) {
  if (!ptr) return CLUE_ERR_INVALID_ARG;
  int prev = 0;
  CLUE_CUDA_TRY(cudaGetDevice(&prev));
  CLUE_CUDA_TRY(cudaSetDevice(device));
  cudaError_t e = cudaMalloc(ptr, bytes ? bytes : 1);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? CLUE_ERR_OUT_OF_MEMORY : CLUE_ERR_CUDA;
  }
  return CLUE_OK;
}

clue_status clue_device_free(void* ptr) {
  CLUE_CUDA_TRY(cudaFree(ptr));
  return CLUE_OK;
}

clue_status clue_host_alloc_pinned(size_t bytes, void** ptr) {
  if (!ptr) return CLUE_ERR_INVALID_ARG;
  CLUE_CUDA_TRY(cudaMallocHost(ptr, bytes ? bytes : 1));
  return CLUE_OK;
}

clue_status clue_host_free_pinned(void* ptr) {
  CLUE_CUDA_TRY(cudaFreeHost(ptr));
  return CLUE_OK;
}

clue_status clue_memcpy_htod(void* dst, const void* src, size_t bytes, void* stream) {
  CLUE_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream));
  return CLUE_OK;
}
clue_status clue_memcpy_dtoh(void* dst, const void* src, size_t bytes, void* stream) {
  CLUE_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  return CLUE_OK;
}
clue_status clue_memcpy_dtod(void* dst, const void* src, size_t bytes, void* stream) {
  CLUE_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return CLUE_OK;
}
clue_status clue_stream_create(int32_t device, void** stream) {
  int prev = 0;
  CLUE_CUDA_TRY(cudaGetDevice(&prev));
  CLUE_CUDA_TRY(cudaSetDevice(device));
  cudaStream_t s;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    set_error(cudaGetErrorString(e));
    return CLUE_ERR_CUDA;
  }
  *stream = (void*)s;
  return CLUE_OK;
}
clue_status clue_stream_destroy(void* stream) {
  CLUE_CUDA_TRY(cudaStreamDestroy((cudaStream_t)stream));
  return CLUE_OK;
}
clue_status clue_stream_synchronize(void* stream) {
  CLUE_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  return CLUE_OK;
}

clue_status clue_context_create(int32_t device, clue_context* ctx) {
  if (!ctx) return CLUE_ERR_INVALID_ARG;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    set_error("no CUDA device with id " + std::to_string(device));
    return CLUE_ERR_CUDA;
  }
  auto* c = new (std::nothrow) clue_context_s;
  if (!c) return CLUE_ERR_OUT_OF_MEMORY;
  c->ws.device = device;
  *ctx = c;
  return CLUE_OK;
}

clue_status clue_context_destroy(clue_context ctx) {
  if (!ctx) return CLUE_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ctx->ws.device);
  workspace_release(ctx->ws);
  if (ctx->alt) {
    workspace_release(*ctx->alt);
    delete ctx->alt;
  }
  if (ctx->alt_stream) cudaStreamDestroy(ctx->alt_stream);
  if (ctx->chunk_stream) cudaStreamDestroy(ctx->chunk_stream);
  for (auto& ge : ctx->chunk_exec)
    if (ge) cudaGraphExecDestroy(ge);
  if (ctx->plain_exec) cudaGraphExecDestroy(ctx->plain_exec);
  for (auto& e : ctx->plain_ev)
    if (e) cudaEventDestroy(e);
  cudaSetDevice(prev);
  delete ctx;
  return CLUE_OK;
}

clue_status clue_context_reserve(clue_context ctx, int32_t ndim, int32_t n, int32_t ppbin) {
  if (!ctx || n <= 0 || ppbin <= 0 || ndim < 1 || ndim > CLUE_MAX_DIM) {
    set_error("invalid reserve request");
    return CLUE_ERR_INVALID_ARG;
  }
  int32_t npd, nt;
  grid_shape(n, ppbin, ndim, &npd, &nt);
  return workspace_reserve(ctx->ws, ndim, (size_t)n, (size_t)nt);
}

clue_status clue_context_reserve_batch(clue_context ctx, int32_t ndim, int64_t n_points, int64_t n_tiles,
                                       int32_t n_events) {
  if (!ctx || n_points <= 0 || n_tiles <= 0 || n_events <= 0 || ndim < 1 || ndim > CLUE_MAX_DIM ||
      n_points > 2147483000ll || n_tiles > 2147483000ll) {
    set_error("invalid batch reserve request");
    return CLUE_ERR_INVALID_ARG;
  }
  return workspace_reserve(ctx->ws, ndim, (size_t)n_points, (size_t)n_tiles, (size_t)n_events);
}

size_t clue_context_workspace_bytes(clue_context ctx) { return ctx ? ctx->ws.arena_bytes + ctx->ws.dstage_bytes : 0; }

}  // extern "C"

namespace clue_b200 {

static clue_status prepare(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                           const clue_metric* metric, int32_t ndim, int32_t n, const float* coords,
                           const float* weight, const clue_outputs* out, RunArgs& a) {
  if (!ctx) {
    set_error("context is null");
    return CLUE_ERR_INVALID_ARG;
  }
  clue_status st;
  if ((st = clue_check_params(params)) != CLUE_OK) return st;
  if ((st = clue_check_kernel(kernel)) != CLUE_OK) return st;
  if ((st = clue_check_metric(metric, ndim)) != CLUE_OK) return st;
  if (n <= 0) {
    set_error("Number of points must be positive.");
    return CLUE_ERR_INVALID_ARG;
  }
  if (!coords || !weight || !out || !out->cluster_index) {
    set_error("coords, weight and out->cluster_index must be non-null");
    return CLUE_ERR_INVALID_ARG;
  }
  int32_t npd, nt;
  grid_shape(n, params->points_per_tile, ndim, &npd, &nt);
  if (npd <= 0 || nt <= 0 || (double)nt > 2147483000.0) {
    set_error("tile grid too large");
    return CLUE_ERR_CAPACITY;
  }
  KParams& kp = a.kp;
  std::memset(&kp, 0, sizeof(kp));
  const bool root = metric->type == CLUE_METRIC_EUCLIDEAN || metric->type == CLUE_METRIC_WEIGHTED_EUCLIDEAN ||
                    metric->type == CLUE_METRIC_PERIODIC_EUCLIDEAN;
  kp.dc = params->dc;
  kp.dm = params->dm;
  kp.seed_dc = params->seed_dc;
  kp.rhoc = params->rhoc;
  kp.t_dc = threshold_for(params->dc, root);
  kp.t_dm = threshold_for(params->dm, root);
  kp.lb_ok = lower_bounds_ok(metric, ndim);
  kp.flags = params->flags;
  kp.ginv = kernel->type == CLUE_KERNEL_GAUSSIAN ? 1.0f / (2.0f * kernel->par[1] * kernel->par[1]) : 0.0f;
  kp.kernel_type = kernel->type;
  for (int k = 0; k < 3; ++k) kp.kpar[k] = kernel->par[k];
  for (int d = 0; d < ndim; ++d) kp.mpar[d] = metric->par[d];
  kp.nperdim0 = npd;
  kp.ntiles = nt;
  kp.n_events = 1;
  int64_t s = 1;
  for (int d = ndim - 1; d >= 0; --d) {
    kp.stride0[d] = (int32_t)s;
    s *= npd;
  }
  for (int d = 0; d < ndim; ++d) kp.wrapped[d] = params->wrapped[d] ? 1 : 0;
  kp.tiebreak = params->tiebreak;
  kp.seed_capacity = params->seed_capacity;
  kp.n = n;
  a.ndim = ndim;
  a.n = n;
  a.metric = metric->type;
  for (int d = 0; d < ndim; ++d) a.coords[d] = coords + (size_t)d * n;
  a.weight = weight;
  a.out = *out;
  a.ev_n_seeds = nullptr;
  a.ev_n_clusters = nullptr;
  ctx->ws.last_kp = kp;
  return workspace_reserve(ctx->ws, ndim, (size_t)n, (size_t)nt);
}

static clue_status read_info(Workspace& ws, const KParams& kp, cudaStream_t s, clue_run_info* info,
                             bool& unresolved) {
  DevStatus* h = ws.status_host;
  uint32_t* total = reinterpret_cast<uint32_t*>(h + 1);
  CLUE_CUDA_TRY(cudaMemcpyAsync(h, ws.status, sizeof(DevStatus), cudaMemcpyDeviceToHost, s));
  CLUE_CUDA_TRY(cudaMemcpyAsync(total, ws.seed_total, 4, cudaMemcpyDeviceToHost, s));
  CLUE_CUDA_TRY(cudaStreamSynchronize(s));
  unresolved = h->unresolved[3] != 0;
  if (h->check_site) {
    set_error(std::string("device bounds check failed in ") + check_site_name(h->check_site) + ": index " +
              std::to_string(h->check_index));
    return CLUE_ERR_CUDA;
  }
  if (h->stage_timeout) {
    set_error("a bulk-copy wait in the density / nearest-higher sweep timed out");
    return CLUE_ERR_TIMEOUT;
  }
  if (h->nonfinite) {
    set_error("coordinates or weights contain NaN or Inf");
    return CLUE_ERR_NONFINITE;
  }
  if (info) {
    const int64_t nseeds = *total;
    const int64_t cap = kp.seed_capacity < 0 ? -1
                                             : std::max<int64_t>(kp.seed_capacity, (int64_t)h->seed_candidates);
    info->n_seeds = nseeds;
    info->n_clusters = h->n_clusters;
    info->dropped_seeds = nseeds - info->n_clusters;
    info->seed_capacity_used = kp.n_events == 1 ? cap : (kp.seed_capacity < 0 ? -1 : -2);
    info->n_tiles = kp.ntiles;
    info->n_per_dim = kp.n_events == 1 ? kp.nperdim0 : 0;
    info->label_rounds = h->label_rounds;
  }
  return CLUE_OK;
}

}  // namespace clue_b200

extern "C" {

clue_status clue_make_clusters(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                               const clue_metric* metric, int32_t ndim, int32_t n, const float* coords,
                               const float* weight, const clue_outputs* out, int32_t memory, void* stream,
                               clue_run_info* info) {
  RunArgs a;
  clue_status st = prepare(ctx, params, kernel, metric, ndim, n, coords, weight, out, a);
  if (st != CLUE_OK) return st;
  Workspace& ws = ctx->ws;
  int prev = 0;
  CLUE_CUDA_TRY(cudaGetDevice(&prev));
  CLUE_CUDA_TRY(cudaSetDevice(ws.device));
  cudaStream_t s = (cudaStream_t)stream;
  const size_t nn = (size_t)n;
  clue_outputs dev_out = *out;
  if (memory == CLUE_MEM_HOST) {
    // device staging: coords, weight, then the five outputs
    st = reserve_stage(ws, (nn * (size_t)(ndim + 1) + 5 * nn) * 4);
    if (st != CLUE_OK) {
      cudaSetDevice(prev);
      return st;
    }
    float* dcoords = static_cast<float*>(ws.dstage);
    float* dweight = dcoords + nn * ndim;
    int32_t* o = reinterpret_cast<int32_t*>(dweight + nn);
    CLUE_CUDA_TRY(cudaMemcpyAsync(dcoords, coords, nn * ndim * 4, cudaMemcpyHostToDevice, s));
    CLUE_CUDA_TRY(cudaMemcpyAsync(dweight, weight, nn * 4, cudaMemcpyHostToDevice, s));
    for (int d = 0; d < ndim; ++d) a.coords[d] = dcoords + (size_t)d * nn;
    a.weight = dweight;
    dev_out.cluster_index = o;
    dev_out.is_seed = out->is_seed ? o + nn : nullptr;
    dev_out.rho = out->rho ? reinterpret_cast<float*>(o + 2 * nn) : nullptr;
    dev_out.nearest_higher = out->nearest_higher ? o + 3 * nn : nullptr;
    dev_out.delta = out->delta ? reinterpret_cast<float*>(o + 4 * nn) : nullptr;
    a.out = dev_out;
  }
  st = run_pipeline_graph(ctx, a, s);
  bool unresolved = false;
  if (st == CLUE_OK) st = read_info(ws, a.kp, s, info, unresolved);
  if (st == CLUE_OK && unresolved) {
    st = finish_labels_dispatch(ws, a, s, 4);
    if (st == CLUE_OK) st = read_info(ws, a.kp, s, info, unresolved);
  }
  if (st == CLUE_OK && memory == CLUE_MEM_HOST) {
    auto back = [&](void* dst, const void* src) -> cudaError_t {
      return dst ? cudaMemcpyAsync(dst, src, nn * 4, cudaMemcpyDeviceToHost, s) : cudaSuccess;
    };
    cudaError_t e = back(out->cluster_index, dev_out.cluster_index);
    if (e == cudaSuccess) e = back(out->is_seed, dev_out.is_seed);
    if (e == cudaSuccess) e = back(out->rho, dev_out.rho);
    if (e == cudaSuccess) e = back(out->nearest_higher, dev_out.nearest_higher);
    if (e == cudaSuccess) e = back(out->delta, dev_out.delta);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      set_error(std::string("copy back: ") + cudaGetErrorString(e));
      st = CLUE_ERR_CUDA;
    }
  }
  cudaSetDevice(prev);
  return st;
}

clue_status clue_make_clusters_async(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                                     const clue_metric* metric, int32_t ndim, int32_t n, const float* coords,
                                     const float* weight, const clue_outputs* out, void* stream) {
  RunArgs a;
  clue_status st = prepare(ctx, params, kernel, metric, ndim, n, coords, weight, out, a);
  if (st != CLUE_OK) return st;
  return run_pipeline_dispatch(ctx->ws, a, (cudaStream_t)stream);
}

clue_status clue_context_read_info(clue_context ctx, void* stream, clue_run_info* info) {
  if (!ctx || !ctx->ws.arena) {
    set_error("context has no completed run");
    return CLUE_ERR_INVALID_ARG;
  }
  bool unresolved = false;
  clue_status st = read_info(ctx->ws, ctx->ws.last_kp, (cudaStream_t)stream, info, unresolved);
  if (st == CLUE_OK && unresolved) {
    set_error("nearest-higher chains deeper than the enqueued label rounds; use clue_make_clusters");
    return CLUE_ERR_TIMEOUT;
  }
  return st;
}

clue_status clue_context_read_near_counts(clue_context ctx, void* stream, clue_near_counts* counts) {
  if (!ctx || !ctx->ws.arena || !counts) {
    set_error("context has no completed run");
    return CLUE_ERR_INVALID_ARG;
  }
  Workspace& ws = ctx->ws;
  const bool ties = (ws.last_kp.flags & CLUE_FLAG_NEAR_TIES) != 0;
  if (ws.near_from_host) {
    counts->rho_near_rhoc = ws.near_sum[0];
    counts->delta_near_seed_dc = ws.near_sum[1];
    counts->delta_near_dm = ws.near_sum[2];
    counts->nh_near_ties = ties ? ws.near_sum[3] : -1;
    return CLUE_OK;
  }
  int prev = 0;
  CLUE_CUDA_TRY(cudaGetDevice(&prev));
  CLUE_CUDA_TRY(cudaSetDevice(ws.device));
  cudaStream_t s = (cudaStream_t)stream;
  DevStatus* h = ws.status_host;
  cudaError_t e = cudaMemcpyAsync(h, ws.status, sizeof(DevStatus), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    set_error(std::string("read near counts: ") + cudaGetErrorString(e));
    return CLUE_ERR_CUDA;
  }
  counts->rho_near_rhoc = h->near_rhoc;
  counts->delta_near_seed_dc = h->near_seed_dc;
  counts->delta_near_dm = h->near_dm;
  counts->nh_near_ties = ties ? (int64_t)h->nh_near_ties : -1;
  return CLUE_OK;
}

clue_status clue_context_set_timing(clue_context ctx, int32_t enable) {
  if (!ctx) return CLUE_ERR_INVALID_ARG;
  int prev = 0;
  CLUE_CUDA_TRY(cudaGetDevice(&prev));
  CLUE_CUDA_TRY(cudaSetDevice(ctx->ws.device));
  for (auto& e : ctx->ws.tev)
    if (!e) {
      cudaError_t err = cudaEventCreate(&e);
      if (err != cudaSuccess) {
        cudaSetDevice(prev);
        set_error(cudaGetErrorString(err));
        return CLUE_ERR_CUDA;
      }
    }
  ctx->ws.timing = enable != 0;
  cudaSetDevice(prev);
  return CLUE_OK;
}

clue_status clue_context_stage_times(clue_context ctx, float* ms, int32_t n_stages) {
  if (!ctx || !ms || !ctx->ws.tev[CLUE_N_STAGES]) {
    set_error("timing not enabled");
    return CLUE_ERR_INVALID_ARG;
  }
  CLUE_CUDA_TRY(cudaEventSynchronize(ctx->ws.tev[CLUE_N_STAGES]));
  for (int k = 0; k < n_stages && k < CLUE_N_STAGES; ++k)
    CLUE_CUDA_TRY(cudaEventElapsedTime(&ms[k], ctx->ws.tev[k], ctx->ws.tev[k + 1]));
  return CLUE_OK;
}

uint64_t clue_context_kernel_launches(clue_context ctx) { return ctx ? ctx->ws.launches : 0; }

clue_status clue_get_clusters(clue_context ctx, int32_t n, const int32_t* cluster_index, int32_t* offsets,
                              int32_t* points, int32_t* n_clusters_out, int32_t* n_clustered_out, void* stream) {
  if (!ctx || n <= 0 || !cluster_index || !offsets || !points) {
    set_error("clue_get_clusters: null argument or n <= 0");
    return CLUE_ERR_INVALID_ARG;
  }
  Workspace& ws = ctx->ws;
  // keys = label + 1 in [0, n]; offsets_from_sorted needs n + 2 entries, one more word holds
  // the invalid-label flag.
  clue_status st = workspace_reserve(ws, 1, (size_t)n, (size_t)n + 2, 1);
  if (st != CLUE_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ws.device);
  int32_t* bad = ws.offsets + (n + 2);
  CLUE_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int32_t), s));
  const int threads = 256;
  const int blocks = std::min((n + threads - 1) / threads, 148 * 16);
  k_label_keys<<<blocks, threads, 0, s>>>(cluster_index, n, ws.keys[0], bad);
  const int cur = radix_sort_pairs(ws.keys, ws.vals, true, n, bits_for((uint32_t)n), ws.hist, ws.scan_scratch, s);
  offsets_from_sorted(ws.keys[cur], n, n + 1, ws.offsets, s);
  k_cluster_csr<<<blocks, threads, 0, s>>>(ws.offsets, ws.vals[cur], n, offsets, points);
  ws.launches += 3 + radix_sort_launches(bits_for((uint32_t)n));
  int32_t h[2] = {0, 0};
  uint32_t last = 0;
  CLUE_CUDA_TRY(cudaMemcpyAsync(h, ws.offsets + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  CLUE_CUDA_TRY(cudaMemcpyAsync(h + 1, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  CLUE_CUDA_TRY(cudaMemcpyAsync(&last, ws.keys[cur] + (n - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CLUE_CUDA_TRY(cudaStreamSynchronize(s));
  cudaSetDevice(prev);
  if (h[1]) {
    set_error("clue_get_clusters: cluster index outside [-1, n)");
    return CLUE_ERR_OUT_OF_RANGE;
  }
  if (n_clusters_out) *n_clusters_out = (int32_t)last;  // max label + 1 (0 when all are -1)
  if (n_clustered_out) *n_clustered_out = n - h[0];
  return CLUE_OK;
}

}  // extern "C"

namespace clue_b200 {

// Validates a batched request, computes every event's reference grid on the host
// (SetupTiles.hpp:23-26, same arithmetic as a plain call), reserves the workspace and fills the
// pinned event table.  Device pointers in `a` are left for the caller to set.
static clue_status prepare_batch(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                                 const clue_metric* metric, int32_t ndim, int32_t n_events,
                                 const int32_t* ev_off, const clue_outputs* out, RunArgs& a) {
  if (!ctx) {
    set_error("context is null");
    return CLUE_ERR_INVALID_ARG;
  }
  clue_status st;
  if ((st = clue_check_params(params)) != CLUE_OK) return st;
  if ((st = clue_check_kernel(kernel)) != CLUE_OK) return st;
  if ((st = clue_check_metric(metric, ndim)) != CLUE_OK) return st;
  if (n_events <= 0 || !ev_off || !out || !out->cluster_index) {
    set_error("n_events must be positive; event_offsets and out->cluster_index must be non-null");
    return CLUE_ERR_INVALID_ARG;
  }
  if (ev_off[0] != 0) {
    set_error("event_offsets[0] must be 0");
    return CLUE_ERR_INVALID_ARG;
  }
  int64_t tiles = 0;
  for (int e = 0; e < n_events; ++e) {
    const int64_t ne = (int64_t)ev_off[e + 1] - ev_off[e];
    if (ne <= 0) {
      set_error("every event needs at least one point (event " + std::to_string(e) + ")");
      return CLUE_ERR_INVALID_ARG;
    }
    int32_t npd, nt;
    grid_shape((int32_t)ne, params->points_per_tile, ndim, &npd, &nt);
    if (nt <= 0) {
      set_error("tile grid too large");
      return CLUE_ERR_CAPACITY;
    }
    tiles += nt;
  }
  const int64_t n = ev_off[n_events];
  if (tiles > 2147483000ll || n > 2147483000ll) {
    set_error("batch too large (points or tiles exceed 2^31)");
    return CLUE_ERR_CAPACITY;
  }
  Workspace& ws = ctx->ws;
  if ((st = workspace_reserve(ws, ndim, (size_t)n, (size_t)tiles, (size_t)n_events)) != CLUE_OK) return st;
  EvGrid* heg;
  int32_t *hpt, *htile;
  event_table_carve(ws.pinned, ws.cap_events, &heg, &hpt, &htile);
  int32_t tb = 0;
  for (int e = 0; e < n_events; ++e) {
    const int32_t ne = ev_off[e + 1] - ev_off[e];
    int32_t npd, nt;
    grid_shape(ne, params->points_per_tile, ndim, &npd, &nt);
    EvGrid g;
    std::memset(&g, 0, sizeof(g));
    int64_t sd = 1;
    for (int d = ndim - 1; d >= 0; --d) {
      g.stride[d] = (int32_t)sd;
      sd *= npd;
    }
    g.nperdim = npd;
    g.ntiles = nt;
    g.tile_base = tb;
    g.pt_base = ev_off[e];
    g.pt_count = ne;
    heg[e] = g;
    hpt[e] = ev_off[e];
    htile[e] = tb;
    tb += nt;
  }
  hpt[n_events] = (int32_t)n;
  htile[n_events] = tb;

  KParams& kp = a.kp;
  std::memset(&kp, 0, sizeof(kp));
  const bool root = metric->type == CLUE_METRIC_EUCLIDEAN || metric->type == CLUE_METRIC_WEIGHTED_EUCLIDEAN ||
                    metric->type == CLUE_METRIC_PERIODIC_EUCLIDEAN;
  kp.dc = params->dc;
  kp.dm = params->dm;
  kp.seed_dc = params->seed_dc;
  kp.rhoc = params->rhoc;
  kp.t_dc = threshold_for(params->dc, root);
  kp.t_dm = threshold_for(params->dm, root);
  kp.lb_ok = lower_bounds_ok(metric, ndim);
  kp.flags = params->flags;
  kp.ginv = kernel->type == CLUE_KERNEL_GAUSSIAN ? 1.0f / (2.0f * kernel->par[1] * kernel->par[1]) : 0.0f;
  kp.kernel_type = kernel->type;
  for (int k = 0; k < 3; ++k) kp.kpar[k] = kernel->par[k];
  for (int d = 0; d < ndim; ++d) kp.mpar[d] = metric->par[d];
  for (int d = 0; d < ndim; ++d) kp.wrapped[d] = params->wrapped[d] ? 1 : 0;
  kp.tiebreak = params->tiebreak;
  kp.seed_capacity = params->seed_capacity;
  kp.n = (int32_t)n;
  kp.n_events = n_events;
  kp.ntiles = (int32_t)tiles;
  kp.nperdim0 = heg[0].nperdim;
  for (int d = 0; d < kMaxDim; ++d) kp.stride0[d] = heg[0].stride[d];
  a.ndim = ndim;
  a.n = (int32_t)n;
  a.metric = metric->type;
  a.out = *out;
  a.ev_n_seeds = nullptr;
  a.ev_n_clusters = nullptr;
  ws.last_kp = kp;
  return CLUE_OK;
}

// Copies the event table of an E-event batch from the pinned staging to the device.
static clue_status upload_events(Workspace& ws, int E, cudaStream_t s) {
  if (E <= 1) return CLUE_OK;  // a single event's table is written by the first kernel
  EvGrid* heg;
  int32_t *hpt, *htile;
  event_table_carve(ws.pinned, ws.cap_events, &heg, &hpt, &htile);
  CLUE_CUDA_TRY(cudaMemcpyAsync(ws.ev, heg, (size_t)E * sizeof(EvGrid), cudaMemcpyHostToDevice, s));
  CLUE_CUDA_TRY(cudaMemcpyAsync(ws.ev_pt, hpt, (size_t)(E + 1) * 4, cudaMemcpyHostToDevice, s));
  CLUE_CUDA_TRY(cudaMemcpyAsync(ws.ev_tile, htile, (size_t)(E + 1) * 4, cudaMemcpyHostToDevice, s));
  return CLUE_OK;
}

// One pass over the whole batch: inputs copied in (host memory), pipeline, outputs copied out.
static clue_status batch_plain(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                               const clue_metric* metric, int32_t ndim, int32_t n_events,
                               const int32_t* event_offsets, const float* coords, const float* weight,
                               const clue_outputs* out, int32_t* ev_n_clusters, int32_t memory, void* stream,
                               clue_run_info* info) {
  RunArgs a;
  clue_status st = prepare_batch(ctx, params, kernel, metric, ndim, n_events, event_offsets, out, a);
  if (st != CLUE_OK) return st;
  if (!coords || !weight) {
    set_error("coords and weight must be non-null");
    return CLUE_ERR_INVALID_ARG;
  }
  Workspace& ws = ctx->ws;
  int prev = 0;
  CLUE_CUDA_TRY(cudaGetDevice(&prev));
  CLUE_CUDA_TRY(cudaSetDevice(ws.device));
  cudaStream_t s = (cudaStream_t)stream;
  const size_t nn = (size_t)a.n;
  clue_outputs dev_out = *out;
  int32_t* dev_ncl = ev_n_clusters;
  if (memory == CLUE_MEM_HOST) {
    st = reserve_stage(ws, (nn * (size_t)(ndim + 1) + 5 * nn + (size_t)n_events) * 4);
    if (st != CLUE_OK) {
      cudaSetDevice(prev);
      return st;
    }
    float* dcoords = static_cast<float*>(ws.dstage);
    float* dweight = dcoords + nn * ndim;
    int32_t* o = reinterpret_cast<int32_t*>(dweight + nn);
    CLUE_CUDA_TRY(cudaMemcpyAsync(dcoords, coords, nn * ndim * 4, cudaMemcpyHostToDevice, s));
    CLUE_CUDA_TRY(cudaMemcpyAsync(dweight, weight, nn * 4, cudaMemcpyHostToDevice, s));
    for (int d = 0; d < ndim; ++d) a.coords[d] = dcoords + (size_t)d * nn;
    a.weight = dweight;
    dev_out.cluster_index = o;
    dev_out.is_seed = out->is_seed ? o + nn : nullptr;
    dev_out.rho = out->rho ? reinterpret_cast<float*>(o + 2 * nn) : nullptr;
    dev_out.nearest_higher = out->nearest_higher ? o + 3 * nn : nullptr;
    dev_out.delta = out->delta ? reinterpret_cast<float*>(o + 4 * nn) : nullptr;
    dev_ncl = ev_n_clusters ? o + 5 * nn : nullptr;
  } else {
    for (int d = 0; d < ndim; ++d) a.coords[d] = coords + (size_t)d * nn;
    a.weight = weight;
  }
  a.out = dev_out;
  a.ev_n_clusters = dev_ncl;
  st = upload_events(ws, n_events, s);
  if (st == CLUE_OK) st = run_pipeline_graph(ctx, a, s);
  bool unresolved = false;
  if (st == CLUE_OK) st = read_info(ws, a.kp, s, info, unresolved);
  if (st == CLUE_OK && unresolved) {
    st = finish_labels_dispatch(ws, a, s, 4);
    if (st == CLUE_OK) st = read_info(ws, a.kp, s, info, unresolved);
  }
  if (st == CLUE_OK && memory == CLUE_MEM_HOST) {
    auto back = [&](void* dst, const void* src, size_t cnt) -> cudaError_t {
      return dst ? cudaMemcpyAsync(dst, src, cnt * 4, cudaMemcpyDeviceToHost, s) : cudaSuccess;
    };
    cudaError_t e = back(out->cluster_index, dev_out.cluster_index, nn);
    if (e == cudaSuccess) e = back(out->is_seed, dev_out.is_seed, nn);
    if (e == cudaSuccess) e = back(out->rho, dev_out.rho, nn);
    if (e == cudaSuccess) e = back(out->nearest_higher, dev_out.nearest_higher, nn);
    if (e == cudaSuccess) e = back(out->delta, dev_out.delta, nn);
    if (e == cudaSuccess) e = back(ev_n_clusters, dev_ncl, (size_t)n_events);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      set_error(std::string("copy back: ") + cudaGetErrorString(e));
      st = CLUE_ERR_CUDA;
    }
  }
  if (st == CLUE_OK && info) info->n_per_dim = 0;
  cudaSetDevice(prev);
  return st;
}

__global__ void k_shift_indices(int32_t* __restrict__ v, int n, int32_t by) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    if (v[i] >= 0) v[i] += by;
}

__global__ void k_save_status(const DevStatus* __restrict__ st, const uint32_t* __restrict__ total,
                              DevStatus* __restrict__ dst, uint32_t* __restrict__ dst_total) {
  const uint32_t* a = reinterpret_cast<const uint32_t*>(st);
  uint32_t* b = reinterpret_cast<uint32_t*>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(DevStatus) / 4); i += blockDim.x) b[i] = a[i];
  if (threadIdx.x == 0) *dst_total = *total;
}

// Host-memory batches of at least this many points overlap their copies with the pipeline.
constexpr int64_t kPipeMinPoints = 4000000;

// Whether a host-memory batch takes the overlapped path: large, several events, valid (an
// invalid request goes to the plain path, which reports it).
static bool batch_overlap_ok(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                             const clue_metric* metric, int32_t ndim, int32_t n_events, const int32_t* ev_off,
                             const float* coords, const float* weight, const clue_outputs* out) {
  if (!ctx || !params || !kernel || !metric || !ev_off || !coords || !weight || !out || !out->cluster_index)
    return false;
  if (ctx->ws.tune_overlap_chunk_points <= 0) return false;
  if (n_events < 2 || ev_off[0] != 0 || ev_off[n_events] < kPipeMinPoints) return false;
  if (clue_check_params(params) != CLUE_OK || clue_check_kernel(kernel) != CLUE_OK ||
      clue_check_metric(metric, ndim) != CLUE_OK)
    return false;
  for (int e = 0; e < n_events; ++e) {
    if (ev_off[e + 1] <= ev_off[e]) return false;
    int32_t npd, nt;
    grid_shape(ev_off[e + 1] - ev_off[e], params->points_per_tile, ndim, &npd, &nt);
    if (nt <= 0) return false;
  }
  return true;
}

// A large host-memory batch in K chunks of whole events, so the copies overlap the pipeline:
// every chunk's event table and inputs go up on a copy stream (all enqueued at once, each chunk
// with its own pinned and device event table, since a copy engine runs its queue in order and
// a small copy on the compute stream would wait behind all the inputs), chunk c runs as one
// graph launch on a stream of the context once its copies are in, and its outputs come down on
// a second copy stream while chunk c + 1 runs; the caller's stream waits for all of it.  Events are independent and a chunk's results do not depend on the
// other events in it, so the outputs are those of one pass over the whole batch (nearest-higher
// indices are shifted to the batch).  The rare chunk whose label chains outlast the fixed
// pointer-jumping rounds is run again alone.
static clue_status batch_host_overlapped(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                                         const clue_metric* metric, int32_t ndim, int32_t n_events,
                                         const int32_t* ev_off, const float* coords, const float* weight,
                                         const clue_outputs* out, int32_t* ev_n_clusters, void* stream,
                                         clue_run_info* info) {
  constexpr int KM = Workspace::kPipeMaxChunks;
  Workspace& ws = ctx->ws;
  const int64_t n = ev_off[n_events];
  const size_t nn = (size_t)n;
  // points per chunk (clue_tuning.overlap_chunk_points): 2..kPipeMaxChunks chunks
  int K = (int)std::min<int64_t>(KM, std::max<int64_t>(2, n / ws.tune_overlap_chunk_points));
  K = std::min(K, (int)n_events);
  // chunk sizes in the ratio 1 : 2 : ... : 2 : 1 -- only the first chunk's copy-in and the last
  // chunk's copy-out are not hidden behind a pipeline run
  std::vector<int> cut(1, 0);  // first event of every chunk, then n_events
  const int64_t parts = 2 * (int64_t)K - 2;
  for (int e = 1; e < n_events && (int)cut.size() < K; ++e) {
    const int64_t c = (int64_t)cut.size();  // chunk that would start at e
    const int64_t before = 2 * c - 1;       // parts in chunks 0 .. c - 1
    if ((int64_t)ev_off[e] * parts >= before * n) cut.push_back(e);
  }
  cut.push_back(n_events);
  K = (int)cut.size() - 1;
  size_t max_n = 0, max_tiles = 0, max_ev = 0;
  std::vector<int64_t> chunk_tiles(K, 0);
  for (int c = 0; c < K; ++c) {
    for (int e = cut[c]; e < cut[c + 1]; ++e) {
      int32_t npd, nt;
      grid_shape(ev_off[e + 1] - ev_off[e], params->points_per_tile, ndim, &npd, &nt);
      chunk_tiles[c] += nt;
    }
    max_n = std::max(max_n, (size_t)(ev_off[cut[c + 1]] - ev_off[cut[c]]));
    max_tiles = std::max(max_tiles, (size_t)chunk_tiles[c]);
    max_ev = std::max(max_ev, (size_t)(cut[c + 1] - cut[c]));
  }
  clue_status st = workspace_reserve(ws, ndim, max_n, max_tiles, max_ev);
  if (st != CLUE_OK) return st;
  int prev = 0;
  CLUE_CUDA_TRY(cudaGetDevice(&prev));
  CLUE_CUDA_TRY(cudaSetDevice(ws.device));
  Workspace* alt = nullptr;  // without room for a second workspace the chunks run one after another
  if (K >= 2) {
    if (!ctx->alt) {
      ctx->alt = new Workspace();
      ctx->alt->device = ws.device;
      CLUE_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->alt_stream, cudaStreamNonBlocking));
    }
    alt = ctx->alt;
    alt->tune_symmetric = ws.tune_symmetric;
    alt->tune_nh_split = ws.tune_nh_split;
    alt->tune_density_gate = ws.tune_density_gate;
    alt->tune_density_exp2 = ws.tune_density_exp2;
    alt->tune_labels_bfs = ws.tune_labels_bfs;
    if (workspace_reserve(*alt, ndim, max_n, max_tiles, max_ev) != CLUE_OK) alt = nullptr;
  }
  if (!ctx->chunk_stream) CLUE_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->chunk_stream, cudaStreamNonBlocking));
  cudaStream_t s1 = ctx->chunk_stream;
  cudaStream_t s2 = alt ? ctx->alt_stream : nullptr;
  const uint64_t alt_launches0 = alt ? alt->launches : 0;
  struct DeviceGuard {
    int prev;
    ~DeviceGuard() { cudaSetDevice(prev); }
  } guard{prev};
  const size_t io_bytes = align_up((nn * (size_t)(ndim + 1) + 5 * nn + (size_t)n_events) * 4, 256);
  const size_t status_bytes = align_up(KM * (sizeof(DevStatus) + 4), 256);
  std::vector<size_t> dev_tab(K + 1, 0);  // every chunk's device event table, after the statuses
  for (int c = 0; c < K; ++c) dev_tab[c + 1] = dev_tab[c] + align_up(event_table_bytes(cut[c + 1] - cut[c]), 256);
  if ((st = reserve_stage(ws, io_bytes + status_bytes + dev_tab[K])) != CLUE_OK) return st;
  if (!ws.pipe_h2d) {
    CLUE_CUDA_TRY(cudaStreamCreateWithFlags(&ws.pipe_h2d, cudaStreamNonBlocking));
    CLUE_CUDA_TRY(cudaStreamCreateWithFlags(&ws.pipe_d2h, cudaStreamNonBlocking));
    for (auto& e : ws.pipe_ev) CLUE_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CLUE_CUDA_TRY(cudaMallocHost((void**)&ws.pipe_status_host, KM * (sizeof(DevStatus) + 4)));
  }
  const size_t host_tab = event_table_bytes(ws.cap_events);  // one pinned table per chunk
  if (ws.pipe_pinned_bytes < (size_t)K * host_tab) {
    if (ws.pipe_pinned) cudaFreeHost(ws.pipe_pinned);
    ws.pipe_pinned = nullptr;
    ws.pipe_pinned_bytes = 0;
    CLUE_CUDA_TRY(cudaMallocHost(&ws.pipe_pinned, (size_t)KM * host_tab));
    ws.pipe_pinned_bytes = (size_t)KM * host_tab;
  }
  cudaStream_t s = (cudaStream_t)stream, h2d = ws.pipe_h2d, d2h = ws.pipe_d2h;
  float* dcoords = static_cast<float*>(ws.dstage);
  float* dweight = dcoords + nn * ndim;
  int32_t* o = reinterpret_cast<int32_t*>(dweight + nn);
  clue_outputs dev_out{};
  dev_out.cluster_index = o;
  dev_out.is_seed = out->is_seed ? o + nn : nullptr;
  dev_out.rho = out->rho ? reinterpret_cast<float*>(o + 2 * nn) : nullptr;
  dev_out.nearest_higher = out->nearest_higher ? o + 3 * nn : nullptr;
  dev_out.delta = out->delta ? reinterpret_cast<float*>(o + 4 * nn) : nullptr;
  int32_t* dev_ncl = ev_n_clusters ? o + 5 * nn : nullptr;
  DevStatus* dslot = reinterpret_cast<DevStatus*>(static_cast<char*>(ws.dstage) + io_bytes);
  uint32_t* dtotal = reinterpret_cast<uint32_t*>(dslot + KM);
  char* dtab = static_cast<char*>(ws.dstage) + io_bytes + status_bytes;
  cudaEvent_t ev_start = ws.pipe_ev[0];
  auto ev_in = [&](int c) { return ws.pipe_ev[1 + 3 * c]; };
  auto ev_done = [&](int c) { return ws.pipe_ev[3 + 3 * c]; };

  auto drain = [&]() {
    cudaStreamSynchronize(h2d);
    cudaStreamSynchronize(s1);
    cudaStreamSynchronize(s);
    if (s2) cudaStreamSynchronize(s2);
    cudaStreamSynchronize(d2h);
  };

  // 1. copy-in stream, chunk by chunk: the chunk's inputs (they need no preparation, so the copy
  //    engine starts at once), then the host computes the chunk's grids and parameters into its
  //    own pinned event table while those inputs are in flight, then the table goes up; a chunk
  //    can start as soon as its own copies are done, and the host never waits for the GPU before
  //    all chunks are enqueued
  CLUE_CUDA_TRY(cudaEventRecord(ev_start, s));
  CLUE_CUDA_TRY(cudaStreamWaitEvent(h2d, ev_start, 0));
  CLUE_CUDA_TRY(cudaStreamWaitEvent(d2h, ev_start, 0));
  CLUE_CUDA_TRY(cudaStreamWaitEvent(s1, ev_start, 0));
  if (s2) CLUE_CUDA_TRY(cudaStreamWaitEvent(s2, ev_start, 0));
  std::vector<RunArgs> args(K);
  std::vector<int32_t> rel;
  void* pinned_main = ws.pinned;
  for (int c = 0; c < K && st == CLUE_OK; ++c) {
    const int e0 = cut[c], E = cut[c + 1] - e0;
    const size_t a0 = (size_t)ev_off[e0], cnt = (size_t)ev_off[cut[c + 1]] - a0;
    cudaError_t ce = cudaSuccess;
    for (int d = 0; d < ndim && ce == cudaSuccess; ++d)
      ce = cudaMemcpyAsync(dcoords + (size_t)d * nn + a0, coords + (size_t)d * nn + a0, cnt * 4,
                           cudaMemcpyHostToDevice, h2d);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(dweight + a0, weight + a0, cnt * 4, cudaMemcpyHostToDevice, h2d);
    if (ce != cudaSuccess) {
      set_error(std::string("overlapped batch: ") + cudaGetErrorString(ce));
      st = CLUE_ERR_CUDA;
      break;
    }
    rel.assign(ev_off + e0, ev_off + e0 + E + 1);
    for (auto& v : rel) v -= ev_off[e0];
    ws.pinned = static_cast<char*>(ws.pipe_pinned) + (size_t)c * host_tab;
    st = prepare_batch(ctx, params, kernel, metric, ndim, E, rel.data(), out, args[c]);
    ws.pinned = pinned_main;
    if (st != CLUE_OK) break;
    if (E > 1) {  // a single event's table is written by the pipeline's first kernel
      EvGrid *heg, *deg;
      int32_t *hpt, *htile, *dpt, *dtile;
      event_table_carve(static_cast<char*>(ws.pipe_pinned) + (size_t)c * host_tab, ws.cap_events, &heg, &hpt,
                        &htile);
      event_table_carve(dtab + dev_tab[c], (size_t)E, &deg, &dpt, &dtile);
      ce = cudaMemcpyAsync(deg, heg, (size_t)E * sizeof(EvGrid), cudaMemcpyHostToDevice, h2d);
      if (ce == cudaSuccess) ce = cudaMemcpyAsync(dpt, hpt, (size_t)(E + 1) * 4, cudaMemcpyHostToDevice, h2d);
      if (ce == cudaSuccess) ce = cudaMemcpyAsync(dtile, htile, (size_t)(E + 1) * 4, cudaMemcpyHostToDevice, h2d);
    }
    if (ce == cudaSuccess) ce = cudaEventRecord(ev_in(c), h2d);
    if (ce != cudaSuccess) {
      set_error(std::string("overlapped batch: ") + cudaGetErrorString(ce));
      st = CLUE_ERR_CUDA;
    }
  }
  if (st != CLUE_OK) {
    drain();
    return st;
  }
  // 2. the even chunks on the context's chunk stream and the odd ones on the second workspace's
  //    stream (each with its own device event table): consecutive chunks run concurrently, so one chunk's
  //    small-kernel phases and kernel tails overlap the next one's sweeps; results go out on the
  //    copy-out stream as each chunk finishes
  for (int c = 0; c < K && st == CLUE_OK; ++c) {
    const int e0 = cut[c], E = cut[c + 1] - e0;
    const size_t a0 = (size_t)ev_off[e0], cnt = (size_t)ev_off[cut[c + 1]] - a0;
    RunArgs& a = args[c];
    for (int d = 0; d < ndim; ++d) a.coords[d] = dcoords + (size_t)d * nn + a0;
    a.weight = dweight + a0;
    a.out.cluster_index = dev_out.cluster_index + a0;
    a.out.is_seed = dev_out.is_seed ? dev_out.is_seed + a0 : nullptr;
    a.out.rho = dev_out.rho ? dev_out.rho + a0 : nullptr;
    a.out.nearest_higher = dev_out.nearest_higher ? dev_out.nearest_higher + a0 : nullptr;
    a.out.delta = dev_out.delta ? dev_out.delta + a0 : nullptr;
    a.ev_n_clusters = dev_ncl ? dev_ncl + e0 : nullptr;
    const bool on_alt = alt && (c & 1);
    Workspace& W = on_alt ? *alt : ws;
    cudaStream_t sc = on_alt ? s2 : s1;
    cudaError_t ce = cudaStreamWaitEvent(sc, ev_in(c), 0);
    if (ce == cudaSuccess) {
      EvGrid* const w_ev = W.ev;
      int32_t* const w_pt = W.ev_pt;
      int32_t* const w_tile = W.ev_tile;
      event_table_carve(dtab + dev_tab[c], (size_t)E, &W.ev, &W.ev_pt, &W.ev_tile);
      // the chunk's pipeline as one graph launch: enqueued kernel by kernel, the launch gaps
      // of four chunk pipelines cost about 0.7 ms per calo4096 batch
      st = capture_and_launch(W, a, sc, &ctx->chunk_exec[c]);
      W.ev = w_ev;
      W.ev_pt = w_pt;
      W.ev_tile = w_tile;
    }
    if (ce == cudaSuccess && st == CLUE_OK) {
      if (a.out.nearest_higher && a0 > 0)
        k_shift_indices<<<(int)std::min<size_t>((cnt + 255) / 256, 148 * 8), 256, 0, sc>>>(a.out.nearest_higher,
                                                                                          (int)cnt, (int32_t)a0);
      k_save_status<<<1, 64, 0, sc>>>(W.status, W.seed_total, dslot + c, dtotal + c);
      ce = cudaGetLastError();
    }
    if (ce == cudaSuccess && st == CLUE_OK) ce = cudaEventRecord(ev_done(c), sc);
    if (ce == cudaSuccess && st == CLUE_OK) ce = cudaStreamWaitEvent(d2h, ev_done(c), 0);
    auto back = [&](void* dst, const void* src, size_t bytes) {
      if (ce == cudaSuccess && dst) ce = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, d2h);
    };
    if (st == CLUE_OK) {
      back(out->cluster_index + a0, dev_out.cluster_index + a0, cnt * 4);
      back(out->is_seed ? out->is_seed + a0 : nullptr, dev_out.is_seed + (out->is_seed ? a0 : 0), cnt * 4);
      back(out->rho ? out->rho + a0 : nullptr, dev_out.rho + (out->rho ? a0 : 0), cnt * 4);
      back(out->nearest_higher ? out->nearest_higher + a0 : nullptr,
           dev_out.nearest_higher + (out->nearest_higher ? a0 : 0), cnt * 4);
      back(out->delta ? out->delta + a0 : nullptr, dev_out.delta + (out->delta ? a0 : 0), cnt * 4);
      back(ev_n_clusters ? ev_n_clusters + e0 : nullptr, dev_ncl + (ev_n_clusters ? e0 : 0), (size_t)E * 4);
    }
    if (ce != cudaSuccess) {
      set_error(std::string("overlapped batch: ") + cudaGetErrorString(ce));
      st = CLUE_ERR_CUDA;
    }
  }
  if (alt) ws.launches += alt->launches - alt_launches0;  // the context counts both workspaces' kernels
  if (st == CLUE_OK) {  // the caller's stream waits for the chunk streams
    CLUE_CUDA_TRY(cudaEventRecord(ws.pipe_ev[2], s1));
    CLUE_CUDA_TRY(cudaStreamWaitEvent(s, ws.pipe_ev[2], 0));
    if (s2) {
      CLUE_CUDA_TRY(cudaEventRecord(ws.pipe_ev[5], s2));
      CLUE_CUDA_TRY(cudaStreamWaitEvent(s, ws.pipe_ev[5], 0));
    }
  }
  if (st == CLUE_OK) {
    cudaError_t ce = cudaMemcpyAsync(ws.pipe_status_host, dslot, KM * (sizeof(DevStatus) + 4),
                                     cudaMemcpyDeviceToHost, s);
    drain();
    if (ce == cudaSuccess) ce = cudaGetLastError();
    if (ce != cudaSuccess) {
      set_error(std::string("overlapped batch: ") + cudaGetErrorString(ce));
      return CLUE_ERR_CUDA;
    }
  } else {
    drain();
    return st;
  }
  const DevStatus* hs = ws.pipe_status_host;
  const uint32_t* ht = reinterpret_cast<const uint32_t*>(hs + KM);
  for (int c = 0; c < K; ++c) {
    if (hs[c].check_site) {
      set_error(std::string("device bounds check failed in ") + check_site_name(hs[c].check_site) + ": index " +
                std::to_string(hs[c].check_index));
      return CLUE_ERR_CUDA;
    }
    if (hs[c].stage_timeout) {
      set_error("a bulk-copy wait in the density / nearest-higher sweep timed out");
      return CLUE_ERR_TIMEOUT;
    }
    if (hs[c].nonfinite) {
      set_error("coordinates or weights contain NaN or Inf");
      return CLUE_ERR_NONFINITE;
    }
  }
  int64_t seeds = 0, clusters = 0, rounds = 0, tiles = 0;
  for (int c = 0; c < K; ++c) {
    int64_t cs = ht[c], cc = hs[c].n_clusters, cr = hs[c].label_rounds;
    if (hs[c].unresolved[3] != 0) {
      // label chains beyond the fixed rounds: this chunk again, alone, with the plain path
      const int e0 = cut[c], E = cut[c + 1] - e0;
      const size_t a0 = (size_t)ev_off[e0], cnt = (size_t)ev_off[cut[c + 1]] - a0;
      std::vector<float> cc_in((size_t)ndim * cnt), w_in(cnt);
      for (int d = 0; d < ndim; ++d)
        std::memcpy(cc_in.data() + (size_t)d * cnt, coords + (size_t)d * nn + a0, cnt * 4);
      std::memcpy(w_in.data(), weight + a0, cnt * 4);
      rel.assign(ev_off + e0, ev_off + e0 + E + 1);
      for (auto& v : rel) v -= (int32_t)a0;
      clue_outputs oc{};
      oc.cluster_index = out->cluster_index + a0;
      oc.is_seed = out->is_seed ? out->is_seed + a0 : nullptr;
      oc.rho = out->rho ? out->rho + a0 : nullptr;
      oc.nearest_higher = out->nearest_higher ? out->nearest_higher + a0 : nullptr;
      oc.delta = out->delta ? out->delta + a0 : nullptr;
      clue_run_info ic{};
      st = batch_plain(ctx, params, kernel, metric, ndim, E, rel.data(), cc_in.data(), w_in.data(), &oc,
                       ev_n_clusters ? ev_n_clusters + e0 : nullptr, CLUE_MEM_HOST, stream, &ic);
      if (st != CLUE_OK) return st;
      if (oc.nearest_higher)
        for (size_t i = 0; i < cnt; ++i)
          if (oc.nearest_higher[i] >= 0) oc.nearest_higher[i] += (int32_t)a0;
      cs = ic.n_seeds;
      cc = ic.n_clusters;
      cr = ic.label_rounds;
    }
    seeds += cs;
    clusters += cc;
    rounds = std::max(rounds, cr);
    tiles += chunk_tiles[c];
  }
  ws.near_from_host = true;
  for (int k = 0; k < 4; ++k) ws.near_sum[k] = 0;
  for (int c = 0; c < K; ++c) {
    ws.near_sum[0] += hs[c].near_rhoc;
    ws.near_sum[1] += hs[c].near_seed_dc;
    ws.near_sum[2] += hs[c].near_dm;
    ws.near_sum[3] += hs[c].nh_near_ties;
  }
  if (info) {
    info->n_seeds = seeds;
    info->n_clusters = clusters;
    info->dropped_seeds = seeds - clusters;
    info->seed_capacity_used = params->seed_capacity < 0 ? -1 : -2;
    info->n_tiles = tiles;
    info->n_per_dim = 0;
    info->label_rounds = rounds;
  }
  return CLUE_OK;
}
}  // namespace clue_b200

struct clue_graph_s {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = 0;
  clue_b200::Workspace* ws = nullptr;  // the captured context's workspace
};

extern "C" {

clue_status clue_batch_make_clusters(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                                     const clue_metric* metric, int32_t ndim, int32_t n_events,
                                     const int32_t* event_offsets, const float* coords, const float* weight,
                                     const clue_outputs* out, int32_t* ev_n_clusters, int32_t memory,
                                     void* stream, clue_run_info* info) {
  if (memory == CLUE_MEM_HOST && batch_overlap_ok(ctx, params, kernel, metric, ndim, n_events, event_offsets,
                                                  coords, weight, out))
    return batch_host_overlapped(ctx, params, kernel, metric, ndim, n_events, event_offsets, coords, weight, out,
                                 ev_n_clusters, stream, info);
  return batch_plain(ctx, params, kernel, metric, ndim, n_events, event_offsets, coords, weight, out,
                     ev_n_clusters, memory, stream, info);
}

void clue_tuning_defaults(clue_tuning* t) {
  if (!t) return;
  const Workspace d{};
  t->symmetric_density = d.tune_symmetric;
  t->nh_split_lanes = d.tune_nh_split;
  t->overlap_chunk_points = d.tune_overlap_chunk_points;
  t->density_gate = d.tune_density_gate;
  t->density_exp2 = d.tune_density_exp2;
  t->labels_bfs = d.tune_labels_bfs;
  t->reserved = 0;
}

clue_status clue_context_set_tuning(clue_context ctx, const clue_tuning* t) {
  if (!ctx) {
    set_error("context is null");
    return CLUE_ERR_INVALID_ARG;
  }
  clue_tuning d;
  clue_tuning_defaults(&d);
  if (!t) t = &d;
  if (t->symmetric_density != 0 && t->symmetric_density != 1) {
    set_error("symmetric_density must be 0 or 1");
    return CLUE_ERR_INVALID_ARG;
  }
  if (t->nh_split_lanes < 0 || t->nh_split_lanes > 16) {
    set_error("nh_split_lanes must be in [0, 16]");
    return CLUE_ERR_INVALID_ARG;
  }
  if (t->overlap_chunk_points < 0) {
    set_error("overlap_chunk_points must be >= 0");
    return CLUE_ERR_INVALID_ARG;
  }
  if ((t->density_gate != 0 && t->density_gate != 1) || (t->density_exp2 != 0 && t->density_exp2 != 1) ||
      (t->labels_bfs != 0 && t->labels_bfs != 1)) {
    set_error("density_gate, density_exp2 and labels_bfs must be 0 or 1");
    return CLUE_ERR_INVALID_ARG;
  }
  ctx->ws.tune_symmetric = t->symmetric_density;
  ctx->ws.tune_nh_split = t->nh_split_lanes;
  ctx->ws.tune_overlap_chunk_points = t->overlap_chunk_points;
  ctx->ws.tune_density_gate = t->density_gate;
  ctx->ws.tune_density_exp2 = t->density_exp2;
  ctx->ws.tune_labels_bfs = t->labels_bfs;
  return CLUE_OK;
}

clue_status clue_context_get_tuning(clue_context ctx, clue_tuning* t) {
  if (!ctx || !t) {
    set_error("context and tuning must be non-null");
    return CLUE_ERR_INVALID_ARG;
  }
  t->symmetric_density = ctx->ws.tune_symmetric;
  t->nh_split_lanes = ctx->ws.tune_nh_split;
  t->overlap_chunk_points = ctx->ws.tune_overlap_chunk_points;
  t->density_gate = ctx->ws.tune_density_gate;
  t->density_exp2 = ctx->ws.tune_density_exp2;
  t->labels_bfs = ctx->ws.tune_labels_bfs;
  t->reserved = 0;
  return CLUE_OK;
}

clue_status clue_autotune_batch(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                                const clue_metric* metric, int32_t ndim, int32_t n_events,
                                const int32_t* event_offsets, const float* coords, const float* weight,
                                void* stream, const char* cache_path, clue_tuning* chosen) {
  if (!ctx || !params || !kernel || !metric || !event_offsets || n_events <= 0 || !coords || !weight) {
    set_error("autotune: context, parameters, event offsets and inputs must be given");
    return CLUE_ERR_INVALID_ARG;
  }
  Workspace& ws = ctx->ws;
  const int64_t n = event_offsets[n_events];
  if (n <= 0) {
    set_error("autotune: empty batch");
    return CLUE_ERR_INVALID_ARG;
  }
  auto ceil_log2 = [](int64_t v) {
    int b = 0;
    while ((int64_t(1) << b) < v) ++b;
    return b;
  };
  char key[160];
  std::snprintf(key, sizeof(key), "clue-tune-v2 ndim=%d nbucket=%d ebucket=%d kernel=%d metric=%d flags=%d", ndim,
                ceil_log2(n), ceil_log2(n_events), kernel->type, metric->type, params->flags);
  int bfs_now = 0;
  auto apply = [&](int sym, int split, int gate, int exp2) {
    ws.tune_symmetric = sym;
    ws.tune_nh_split = split;
    ws.tune_density_gate = gate;
    ws.tune_density_exp2 = exp2;
    ws.tune_labels_bfs = bfs_now;
  };
  auto report = [&]() {
    if (chosen) clue_context_get_tuning(ctx, chosen);
  };
  if (cache_path) {
    if (FILE* f = std::fopen(cache_path, "r")) {
      char line[256];
      int sym = -1, split = -1, gate = -1, exp2 = -1, bfs = -1;
      const size_t kl = std::strlen(key);
      while (std::fgets(line, sizeof(line), f))
        if (std::strncmp(line, key, kl) == 0 && line[kl] == ' ')
          std::sscanf(line + kl,
                      " | symmetric_density=%d nh_split_lanes=%d density_gate=%d density_exp2=%d labels_bfs=%d", &sym,
                      &split, &gate, &exp2, &bfs);
      std::fclose(f);
      if ((sym == 0 || sym == 1) && split >= 0 && split <= 16 && (gate == 0 || gate == 1) &&
          (exp2 == 0 || exp2 == 1) && (bfs == 0 || bfs == 1)) {  // the last entry of the key wins
        bfs_now = bfs;
        apply(sym, split, gate, exp2);
        report();
        return CLUE_OK;
      }
    }
  }
  // candidates: the split threshold first (at the symmetric default), then the density form
  const bool spatial = (params->flags & CLUE_FLAG_REFERENCE_ORDER) == 0 &&
                       (kernel->type != CLUE_KERNEL_FLAT || (params->flags & CLUE_FLAG_SPATIAL_DENSITY) != 0);
  bool sym_ok = spatial && (metric->type == CLUE_METRIC_EUCLIDEAN || metric->type == CLUE_METRIC_MANHATTAN ||
                            metric->type == CLUE_METRIC_CHEBYSHEV);
  for (int d = 0; d < ndim && d < CLUE_MAX_DIM; ++d) sym_ok = sym_ok && !params->wrapped[d];
  int prev = 0;
  CLUE_CUDA_TRY(cudaGetDevice(&prev));
  CLUE_CUDA_TRY(cudaSetDevice(ws.device));
  cudaStream_t s = (cudaStream_t)stream;
  int32_t* labels = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t ce = cudaMalloc(&labels, (size_t)n * sizeof(int32_t));
  if (ce == cudaSuccess) ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
  clue_status st = ce == cudaSuccess ? CLUE_OK : CLUE_ERR_CUDA;
  if (st != CLUE_OK) set_error(std::string("autotune: ") + cudaGetErrorString(ce));
  clue_outputs out{};
  out.cluster_index = labels;
  auto measure = [&](int sym, int split, int gate, int exp2) -> float {
    apply(sym, split, gate, exp2);
    float t[3] = {0, 0, 0};
    for (int r = 0; r < 4 && st == CLUE_OK; ++r) {  // one warm-up, then three timed runs
      if (cudaEventRecord(e0, s) != cudaSuccess) st = CLUE_ERR_CUDA;
      if (st == CLUE_OK)
        st = clue_batch_make_clusters_async(ctx, params, kernel, metric, ndim, n_events, event_offsets, coords,
                                            weight, &out, nullptr, stream);
      if (st == CLUE_OK && (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess))
        st = CLUE_ERR_CUDA;
      if (st == CLUE_OK && r > 0) cudaEventElapsedTime(&t[r - 1], e0, e1);
    }
    std::sort(t, t + 3);
    return t[1];
  };
  const int sym0 = sym_ok ? 1 : ws.tune_symmetric;
  int best_sym = sym0, best_split = 8, best_gate = 0, best_exp2 = 0;
  float best = 0.0f;
  const int splits[] = {8, 0, 4, 16};  // the default first: it wins ties
  for (int split : splits) {
    const float ms = measure(sym0, split, 0, 0);
    if (st != CLUE_OK) break;
    if (split == 8 || ms < best) {
      best = ms;
      best_split = split;
    }
  }
  // the symmetric sweep's pair-step alternatives (they apply to its Euclidean unit-amplitude
  // forms; elsewhere they time the same kernel and lose ties)
  if (st == CLUE_OK && sym_ok && metric->type == CLUE_METRIC_EUCLIDEAN && ndim <= 4) {
    const int alts[3][2] = {{1, 0}, {0, 1}, {1, 1}};
    for (const auto& a : alts) {
      const float ms = measure(1, best_split, a[0], a[1]);
      if (st != CLUE_OK) break;
      if (ms < best) {
        best = ms;
        best_gate = a[0];
        best_exp2 = a[1];
      }
    }
  }
  if (st == CLUE_OK && sym_ok) {
    const float ms = measure(0, best_split, 0, 0);
    if (st == CLUE_OK && ms < best) {
      best = ms;
      best_sym = 0;
      best_gate = best_exp2 = 0;
    }
  }
  int best_bfs = 0;
  if (st == CLUE_OK) {  // the breadth-first label form on the best of the rest (the same labels)
    bfs_now = 1;
    const float ms = measure(best_sym, best_split, best_gate, best_exp2);
    bfs_now = 0;
    if (st == CLUE_OK && ms < best) {
      best = ms;
      best_bfs = 1;
    }
  }
  bfs_now = best_bfs;
  if (labels) cudaFree(labels);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaSetDevice(prev);
  if (st != CLUE_OK) return st;
  apply(best_sym, best_split, best_gate, best_exp2);
  if (cache_path) {
    FILE* f = std::fopen(cache_path, "a");
    if (!f) {
      set_error(std::string("autotune: cannot write the cache ") + cache_path);
      return CLUE_ERR_INVALID_ARG;
    }
    std::fprintf(f,
                 "%s | symmetric_density=%d nh_split_lanes=%d density_gate=%d density_exp2=%d labels_bfs=%d | %.4f ms\n",
                 key, best_sym, best_split, best_gate, best_exp2, best_bfs, best);
    std::fclose(f);
  }
  report();
  return CLUE_OK;
}

clue_status clue_batch_make_clusters_async(clue_context ctx, const clue_params* params,
                                           const clue_kernel* kernel, const clue_metric* metric, int32_t ndim,
                                           int32_t n_events, const int32_t* event_offsets, const float* coords,
                                           const float* weight, const clue_outputs* out, int32_t* ev_n_clusters,
                                           void* stream) {
  RunArgs a;
  clue_status st = prepare_batch(ctx, params, kernel, metric, ndim, n_events, event_offsets, out, a);
  if (st != CLUE_OK) return st;
  if (!coords || !weight) {
    set_error("coords and weight must be non-null");
    return CLUE_ERR_INVALID_ARG;
  }
  for (int d = 0; d < ndim; ++d) a.coords[d] = coords + (size_t)d * a.n;
  a.weight = weight;
  a.ev_n_clusters = ev_n_clusters;
  cudaStream_t s = (cudaStream_t)stream;
  st = upload_events(ctx->ws, n_events, s);
  if (st != CLUE_OK) return st;
  return run_pipeline_dispatch(ctx->ws, a, s);
}

clue_status clue_graph_capture_batch(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                                     const clue_metric* metric, int32_t ndim, int32_t n_events,
                                     const int32_t* event_offsets, const float* coords, const float* weight,
                                     const clue_outputs* out, int32_t* ev_n_clusters, void* stream,
                                     clue_graph* graph) {
  if (!graph || !stream) {
    set_error("graph capture needs an output handle and a non-default stream");
    return CLUE_ERR_INVALID_ARG;
  }
  RunArgs a;
  clue_status st = prepare_batch(ctx, params, kernel, metric, ndim, n_events, event_offsets, out, a);
  if (st != CLUE_OK) return st;
  if (!coords || !weight) {
    set_error("coords and weight must be non-null");
    return CLUE_ERR_INVALID_ARG;
  }
  for (int d = 0; d < ndim; ++d) a.coords[d] = coords + (size_t)d * a.n;
  a.weight = weight;
  a.ev_n_clusters = ev_n_clusters;
  cudaStream_t s = (cudaStream_t)stream;
  Workspace& ws = ctx->ws;
  const bool timing = ws.timing;
  ws.timing = false;
  auto* g = new (std::nothrow) clue_graph_s;
  if (!g) return CLUE_ERR_OUT_OF_MEMORY;
  g->device = ws.device;
  g->ws = &ws;
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    st = upload_events(ws, n_events, s);
    if (st == CLUE_OK) st = run_pipeline_dispatch(ws, a, s);
    e = cudaStreamEndCapture(s, &g->graph);
  }
  ws.timing = timing;
  if (e == cudaSuccess && st == CLUE_OK) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (e != cudaSuccess || st != CLUE_OK) {
    if (e != cudaSuccess) set_error(std::string("graph capture: ") + cudaGetErrorString(e));
    cudaGetLastError();
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return st != CLUE_OK ? st : CLUE_ERR_CUDA;
  }
  *graph = g;
  return CLUE_OK;
}

clue_status clue_graph_launch(clue_graph graph, void* stream) {
  if (!graph || !graph->exec) return CLUE_ERR_INVALID_ARG;
  if (graph->ws) graph->ws->near_from_host = false;  // the replay's counts land on the device
  CLUE_CUDA_TRY(cudaGraphLaunch(graph->exec, (cudaStream_t)stream));
  return CLUE_OK;
}

clue_status clue_graph_destroy(clue_graph graph) {
  if (!graph) return CLUE_OK;
  if (graph->exec) cudaGraphExecDestroy(graph->exec);
  if (graph->graph) cudaGraphDestroy(graph->graph);
  delete graph;
  return CLUE_OK;
}

}  // extern "C"

extern "C" clue_status clue_events_loop(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                                        const clue_metric* metric, int32_t ndim, int32_t n_events,
                                        const int32_t* event_offsets, const float* coords, const float* weight,
                                        const clue_outputs* out, void* stream, float* event_ms) {
  if (!ctx || n_events <= 0 || !event_offsets || !coords || !weight || !out || !out->cluster_index) {
    set_error("invalid events loop request");
    return CLUE_ERR_INVALID_ARG;
  }
  clue_status st;
  if ((st = clue_check_params(params)) != CLUE_OK) return st;
  if ((st = clue_check_kernel(kernel)) != CLUE_OK) return st;
  if ((st = clue_check_metric(metric, ndim)) != CLUE_OK) return st;
  const int64_t n_total = event_offsets[n_events];
  int32_t nmax = 0, tmax = 0;
  for (int e = 0; e < n_events; ++e) {
    const int32_t ne = event_offsets[e + 1] - event_offsets[e];
    if (ne <= 0) {
      set_error("every event needs at least one point");
      return CLUE_ERR_INVALID_ARG;
    }
    int32_t npd, nt;
    grid_shape(ne, params->points_per_tile, ndim, &npd, &nt);
    nmax = std::max(nmax, ne);
    tmax = std::max(tmax, nt);
  }
  Workspace& ws = ctx->ws;
  if ((st = workspace_reserve(ws, ndim, (size_t)nmax, (size_t)tmax, 1)) != CLUE_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<cudaEvent_t> evs;
  if (event_ms) {
    evs.resize((size_t)n_events + 1);
    for (auto& e : evs) CLUE_CUDA_TRY(cudaEventCreate(&e));
    CLUE_CUDA_TRY(cudaEventRecord(evs[0], s));
  }
  const bool root = metric->type == CLUE_METRIC_EUCLIDEAN || metric->type == CLUE_METRIC_WEIGHTED_EUCLIDEAN ||
                    metric->type == CLUE_METRIC_PERIODIC_EUCLIDEAN;
  for (int e = 0; e < n_events && st == CLUE_OK; ++e) {
    const int32_t b = event_offsets[e], ne = event_offsets[e + 1] - b;
    RunArgs a;
    std::memset(&a, 0, sizeof(a));
    KParams& kp = a.kp;
    int32_t npd, nt;
    grid_shape(ne, params->points_per_tile, ndim, &npd, &nt);
    kp.dc = params->dc;
    kp.dm = params->dm;
    kp.seed_dc = params->seed_dc;
    kp.rhoc = params->rhoc;
    kp.t_dc = threshold_for(params->dc, root);
    kp.t_dm = threshold_for(params->dm, root);
  kp.lb_ok = lower_bounds_ok(metric, ndim);
  kp.flags = params->flags;
  kp.ginv = kernel->type == CLUE_KERNEL_GAUSSIAN ? 1.0f / (2.0f * kernel->par[1] * kernel->par[1]) : 0.0f;
    kp.kernel_type = kernel->type;
    for (int k = 0; k < 3; ++k) kp.kpar[k] = kernel->par[k];
    for (int d = 0; d < ndim; ++d) kp.mpar[d] = metric->par[d];
    for (int d = 0; d < ndim; ++d) kp.wrapped[d] = params->wrapped[d] ? 1 : 0;
    kp.tiebreak = params->tiebreak;
    kp.seed_capacity = params->seed_capacity;
    kp.n = ne;
    kp.n_events = 1;
    kp.ntiles = nt;
    kp.nperdim0 = npd;
    int64_t sd = 1;
    for (int d = ndim - 1; d >= 0; --d) {
      kp.stride0[d] = (int32_t)sd;
      sd *= npd;
    }
    a.ndim = ndim;
    a.n = ne;
    a.metric = metric->type;
    for (int d = 0; d < ndim; ++d) a.coords[d] = coords + (size_t)d * n_total + b;
    a.weight = weight + b;
    a.out.cluster_index = out->cluster_index + b;
    a.out.is_seed = out->is_seed ? out->is_seed + b : nullptr;
    a.out.rho = out->rho ? out->rho + b : nullptr;
    a.out.nearest_higher = out->nearest_higher ? out->nearest_higher + b : nullptr;
    a.out.delta = out->delta ? out->delta + b : nullptr;
    st = run_pipeline_dispatch(ws, a, s);
    if (event_ms) cudaEventRecord(evs[(size_t)e + 1], s);
  }
  if (event_ms) {
    cudaError_t err = cudaEventSynchronize(evs.back());
    for (int e = 0; e < n_events && err == cudaSuccess; ++e) err = cudaEventElapsedTime(&event_ms[e], evs[e], evs[e + 1]);
    for (auto& ev : evs) cudaEventDestroy(ev);
    if (err != cudaSuccess) {
      set_error(cudaGetErrorString(err));
      return CLUE_ERR_CUDA;
    }
  }
  return st;
}
