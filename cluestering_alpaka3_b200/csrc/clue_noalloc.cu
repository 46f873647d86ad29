// clue_noalloc.cu -- clue_make_clusters_noalloc: the clustering pipeline for callers that
// cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: code that owns every byte of device memory through
// its own pool (a serving runtime or a plugin living inside another framework), and code on a
// latency-critical path where cudaMalloc's implicit device-wide synchronisation is not
// acceptable.  For them this entry point takes device inputs and outputs from the caller and
// keeps all intermediate buffers (tile CSR, sorted point records, seed and label arrays) in
// one file-scope __device__ array of fixed size, so no allocation of any kind happens.
//
// Limits: at most kNoAllocMaxPoints points and kNoAllocMaxTiles tiles of the reference grid, and
// buffers that fit the array: 32768 points in 1 to 7 dimensions at the default 128 points per
// tile, about 29,900 to 30,300 in 8 to 10 (the capacity error names the exact limit).
// Every GPU that loads the library holds the array (kNoAllocBytes) until the process exits.
// All calls on a device share the array and it keeps the last call's contents; the pipeline
// writes every entry it later reads, so no clearing between calls is needed.  Calls whose
// work overlaps on the GPU (different streams, or different host threads on one device)
// race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "clue_internal.h"

namespace clue_b200 {

template <int N>
clue_status finish_labels(Workspace& ws, const RunArgs& a, cudaStream_t s, int first_round);

namespace {

constexpr int kNoAllocMaxPoints = 32768;
constexpr int kNoAllocMaxTiles = 65536;
constexpr size_t kNoAllocBytes = 6u << 20;  // 6 MiB

// The scratch array.  Host code must not use its name as an address: on the host it names a
// host-side stand-in; the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_addr[kMaxDevices] = {};

// Looks up (once per device, with that device current) the device address of the array.
clue_status noalloc_scratch_address(int device, void** addr) {
  if (device < 0 || device >= kMaxDevices) {
    set_error("device id out of range for the no-allocation scratch table");
    return CLUE_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error(std::string("cudaGetSymbolAddress(no-allocation scratch): ") + cudaGetErrorString(e));
      return CLUE_ERR_CUDA;
    }
    g_noalloc_addr[device] = p;
  }
  *addr = g_noalloc_addr[device];
  return CLUE_OK;
}

size_t up256(size_t x) { return (x + 255) / 256 * 256; }

// Carves the scratch array into the pipeline's buffers, those of the symmetric density sweep
// included (so a call takes the same sweeps, and gives the same bits, as clue_make_clusters);
// false if they do not fit.  With base null nothing is carved: the call only checks the fit.
bool carve(Workspace& ws, void* base, int ndim, size_t n, size_t ntiles) {
  void* evtab = nullptr;
  const size_t w = (size_t)((ndim + 1 + 3) / 4);
  const size_t nb = (size_t)sort_blocks((int)n);
  const size_t hist_len = hist_words(nb);
  const size_t scan_words = scan_scratch_words(std::max(std::max(hist_len, n), ntiles)) + 1;
  struct Item {
    void** ptr;
    size_t bytes;
  } items[] = {
      {&evtab, event_table_bytes(1)},
      {(void**)&ws.status, sizeof(DevStatus)},
      {(void**)&ws.keys[0], n * 4},
      {(void**)&ws.keys[1], n * 4},
      {(void**)&ws.vals[0], n * 4},
      {(void**)&ws.vals[1], n * 4},
      {(void**)&ws.hist, hist_len * 4},
      {(void**)&ws.scan_scratch, scan_words * 4},
      {(void**)&ws.offsets, (ntiles + 1) * 4},
      {(void**)&ws.rec_w, n * w * 16},
      {(void**)&ws.rec_r, n * w * 16},
      {(void**)&ws.delta_s, n * 4},
      {(void**)&ws.nh_s, n * 4},
      {(void**)&ws.par, n * 4},
      {(void**)&ws.is_seed_s, n * 4},
      {(void**)&ws.seed_flag, n * 4},
      {(void**)&ws.seed_total, 16},
      {(void**)&ws.blk, (n / 32 + 1) * 6 * 16},
      {(void**)&ws.mq_alt, n * 4},
      {(void**)&ws.mkeys_alt, n * 4},
      {(void**)&ws.rec_m, n * w * 16},
      {(void**)&ws.sblk, (n / 1024 + 1) * 6 * 16},
      {(void**)&ws.ord_rho, n * 4},
      {(void**)&ws.chunk_count, (ntiles + 1) * 4},
      {(void**)&ws.chunk_tile, (n / kChunkPoints + ntiles + 1) * 4},
      {(void**)&ws.chunk_total, 16},
      {(void**)&ws.tblk, std::min(n, n / 32 + ntiles + 1) * 2 * w * 16},
      {(void**)&ws.tblk_off, (ntiles + 1) * 4},
      {(void**)&ws.rho_fix, n * 8},
  };
  size_t total = 0;
  for (auto& it : items) total += up256(it.bytes);
  if (total > kNoAllocBytes) return false;
  if (!base) return true;
  size_t o = 0;
  for (auto& it : items) {
    *it.ptr = static_cast<unsigned char*>(base) + o;
    o += up256(it.bytes);
  }
  event_table_carve(evtab, 1, &ws.ev, &ws.ev_pt, &ws.ev_tile);
  ws.cap_events = 1;
  ws.arena = base;
  ws.arena_bytes = total;
  ws.cap_n = n;
  ws.cap_tiles = ntiles;
  ws.cap_words = w;
  return true;
}

// Largest point count whose grid (points_per_tile ppbin) and buffers fit the scratch in ndim
// dimensions: 32768 for up to 7 dimensions at 128 points per tile, a little less for 8 to 10
// (three float4 words per record).
int max_points(int ndim, int32_t ppbin) {
  auto fits = [&](int n) {
    int32_t npd = 0, nt = 0;
    grid_shape(n, ppbin, ndim, &npd, &nt);
    Workspace probe;
    return nt > 0 && nt <= kNoAllocMaxTiles && carve(probe, nullptr, ndim, (size_t)n, (size_t)nt);
  };
  if (!fits(1)) return 0;
  int lo = 1, hi = kNoAllocMaxPoints;
  while (lo < hi) {
    const int mid = lo + (hi - lo + 1) / 2;
    if (fits(mid))
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

clue_status finish_dispatch(Workspace& ws, const RunArgs& a, cudaStream_t s, int first) {
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

}  // namespace
}  // namespace clue_b200

using namespace clue_b200;

extern "C" clue_status clue_make_clusters_noalloc(const clue_params* params, const clue_kernel* kernel,
                                                  const clue_metric* metric, int32_t ndim, int32_t n,
                                                  const float* coords, const float* weight,
                                                  const clue_outputs* out, void* stream,
                                                  clue_run_info* info) {
  clue_status st;
  if ((st = clue_check_params(params)) != CLUE_OK) return st;
  if ((st = clue_check_kernel(kernel)) != CLUE_OK) return st;
  if ((st = clue_check_metric(metric, ndim)) != CLUE_OK) return st;
  if (n <= 0) {
    set_error("Number of points must be positive.");
    return CLUE_ERR_INVALID_ARG;
  }
  if (n > kNoAllocMaxPoints) {
    set_error("clue_make_clusters_noalloc: " + std::to_string(n) + " points requested, at most " +
              std::to_string(max_points(ndim, params->points_per_tile)) + " in " + std::to_string(ndim) +
              " dimensions (fixed scratch of 6 MiB)");
    return CLUE_ERR_CAPACITY;
  }
  if (!coords || !weight || !out || !out->cluster_index) {
    set_error("coords, weight and out->cluster_index must be non-null");
    return CLUE_ERR_INVALID_ARG;
  }
  int32_t npd = 0, nt = 0;
  grid_shape(n, params->points_per_tile, ndim, &npd, &nt);
  if (nt <= 0 || nt > kNoAllocMaxTiles) {
    set_error("clue_make_clusters_noalloc: " + std::to_string(nt) + " tiles, at most 65536 (raise points_per_tile)");
    return CLUE_ERR_CAPACITY;
  }
  int device = 0;
  CLUE_CUDA_TRY(cudaGetDevice(&device));
  void* base = nullptr;
  if ((st = noalloc_scratch_address(device, &base)) != CLUE_OK) return st;

  Workspace ws;
  ws.device = device;
  if (!carve(ws, base, ndim, (size_t)n, (size_t)nt)) {
    set_error("clue_make_clusters_noalloc: " + std::to_string(n) + " points requested, at most " +
              std::to_string(max_points(ndim, params->points_per_tile)) + " in " + std::to_string(ndim) +
              " dimensions with points_per_tile " + std::to_string(params->points_per_tile) +
              " (fixed scratch of 6 MiB)");
    return CLUE_ERR_CAPACITY;
  }

  RunArgs a;
  std::memset(&a, 0, sizeof(a));
  KParams& kp = a.kp;
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
  int64_t stride = 1;
  for (int d = ndim - 1; d >= 0; --d) {
    kp.stride0[d] = (int32_t)stride;
    stride *= npd;
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

  cudaStream_t s = (cudaStream_t)stream;
  if ((st = run_pipeline_dispatch(ws, a, s)) != CLUE_OK) return st;

  DevStatus h;
  uint32_t total = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    CLUE_CUDA_TRY(cudaMemcpyAsync(&h, ws.status, sizeof(DevStatus), cudaMemcpyDeviceToHost, s));
    CLUE_CUDA_TRY(cudaMemcpyAsync(&total, ws.seed_total, 4, cudaMemcpyDeviceToHost, s));
    CLUE_CUDA_TRY(cudaStreamSynchronize(s));
    if (h.check_site) {
      set_error(std::string("device bounds check failed in ") + check_site_name(h.check_site) + ": index " +
                std::to_string(h.check_index));
      return CLUE_ERR_CUDA;
    }
    if (h.stage_timeout) {
      set_error("a bulk-copy wait in the density / nearest-higher sweep timed out");
      return CLUE_ERR_TIMEOUT;
    }
    if (h.nonfinite) {
      set_error("coordinates or weights contain NaN or Inf");
      return CLUE_ERR_NONFINITE;
    }
    if (h.unresolved[3] == 0 || attempt == 1) break;
    if ((st = finish_dispatch(ws, a, s, 4)) != CLUE_OK) return st;
  }
  if (info) {
    const int64_t nseeds = total;
    const int64_t cap = kp.seed_capacity < 0 ? -1
                                             : std::max<int64_t>(kp.seed_capacity, (int64_t)h.seed_candidates);
    info->n_seeds = nseeds;
    info->n_clusters = h.n_clusters;
    info->dropped_seeds = nseeds - info->n_clusters;
    info->seed_capacity_used = cap;
    info->n_tiles = nt;
    info->n_per_dim = npd;
    info->label_rounds = h.label_rounds;
  }
  return CLUE_OK;
}
