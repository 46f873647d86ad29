// clue_internal.h -- host-side internals shared by the translation units of libclue_b200.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstddef>
#include <cstdint>
#include <string>

#include "clue_common.cuh"

namespace clue_b200 {

// Thread-local error message behind clue_last_error().
void set_error(const std::string& msg);

#define CLUE_CUDA_TRY(expr)                                                            \
  do {                                                                                 \
    cudaError_t err_ = (expr);                                                         \
    if (err_ != cudaSuccess) {                                                         \
      ::clue_b200::set_error(std::string(#expr) + ": " + cudaGetErrorString(err_));     \
      return err_ == cudaErrorMemoryAllocation ? CLUE_ERR_OUT_OF_MEMORY : CLUE_ERR_CUDA; \
    }                                                                                  \
  } while (0)

// ---- radix sort / scan (clue_sort.cu) -----------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // keys per radix block
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kChunkPoints = 128;  // home points per CTA of the density / nearest-higher sweeps
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

inline int sort_blocks(int n) { return (n + kSortTile - 1) / kSortTile; }
// Digit-major per-block digit counts of one radix pass, then the kRadix digit totals.
inline size_t hist_words(int nblocks) { return (size_t)kRadix * nblocks + kRadix; }
inline int bits_for(uint32_t maxkey) {
  int b = 0;
  while (b < 32 && (maxkey >> b) != 0) ++b;
  return b;
}
// Scratch words needed by exclusive_scan for a length-len array.
inline size_t scan_scratch_words(size_t len) { return (len + kScanTile - 1) / kScanTile + 1; }

// Stable LSD radix sort of (key, value) pairs by the low `bits` bits of key.  Values
// start as the identity (0..n-1) when vals_in is null.  Ping-pongs between buffer 0
// and 1 of keys/vals; returns the index (0 or 1) holding the result.
int radix_sort_pairs(uint32_t* keys[2], int32_t* vals[2], bool vals_identity, int n, int bits,
                     uint32_t* hist, uint32_t* scan_scratch, cudaStream_t s);
// Kernel launches made by radix_sort_pairs / exclusive_scan for the given sizes.
inline int radix_sort_launches(int bits) { return (bits <= 0 ? 1 : (bits + kRadixBits - 1) / kRadixBits) * 3; }
constexpr int kScanLaunches = 3;

// Exclusive scan of len uint32 values (in may alias out).  Writes the total to *total
// (device pointer) when non-null.
void exclusive_scan(const uint32_t* in, uint32_t* out, size_t len, uint32_t* scratch,
                    uint32_t* total, cudaStream_t s);

// offsets[b] = first position of key b in sorted keys (b = 0..nkeys), n at the end; the key of
// an entry is its value shifted right by `shift` bits.
void offsets_from_sorted(const uint32_t* sorted_keys, int n, int nkeys, int32_t* offsets,
                         cudaStream_t s, int shift = 0);

// ---- per-dimension pipeline (clue_dim.cu, one instantiation per N) ----------
struct Workspace;

struct RunArgs {
  KParams kp;
  int32_t ndim;
  int32_t n;
  const float* coords[kMaxDim];  // device, per dimension
  const float* weight;           // device
  clue_outputs out;              // device pointers (may be null except cluster_index)
  int32_t metric;
  int32_t* ev_n_seeds;           // device [n_events] or null (batched calls)
  int32_t* ev_n_clusters;        // device [n_events] or null (batched calls)
};

template <int N>
clue_status run_pipeline(Workspace& ws, const RunArgs& a, cudaStream_t s);

// Dispatch on ndim (clue_dim.cu).
clue_status run_pipeline_dispatch(Workspace& ws, const RunArgs& a, cudaStream_t s);

// ---- workspace ----------------------------------------------------------------
struct Workspace {
  int device = 0;
  // current capacities
  size_t cap_n = 0, cap_tiles = 0, cap_words = 0;
  size_t cap_events = 0;
  void* arena = nullptr;
  size_t arena_bytes = 0;

  // event tables, one contiguous block: EvGrid[cap_events], ev_pt[cap_events + 1],
  // ev_tile[cap_events + 1] (uploaded in one copy for batched calls)
  EvGrid* ev = nullptr;
  int32_t* ev_pt = nullptr;
  int32_t* ev_tile = nullptr;
  int32_t* ev_chunk = nullptr;  // [n / 1024 + 1] event of the first point of every 1024-point chunk
  DevStatus* status = nullptr;
  uint32_t* keys[2] = {nullptr, nullptr};
  int32_t* vals[2] = {nullptr, nullptr};
  uint32_t* hist = nullptr;
  uint32_t* scan_scratch = nullptr;
  int32_t* offsets = nullptr;
  float4* rec_w = nullptr;  // coords + weight, tile-sorted
  float4* rec_r = nullptr;  // coords + rho, tile-sorted
  float* delta_s = nullptr;
  int32_t* nh_s = nullptr;
  int32_t* par = nullptr;
  int32_t* is_seed_s = nullptr;
  uint32_t* seed_flag = nullptr;  // original order, then exclusive-scanned to ranks
  uint32_t* seed_total = nullptr;
  float4* blk = nullptr;          // bounding boxes of 32-record blocks of the sorted records
  int32_t* mq_alt = nullptr;      // second value buffer of the Morton sort
  uint32_t* mkeys_alt = nullptr;  // second key buffer of the Morton sort
  int32_t* minv = nullptr;        // tile-sorted position -> Morton position (alias after the sort)
  float4* rec_m = nullptr;        // records in Morton order inside every tile
  const float4* rec_m_cur = nullptr;  // Morton-ordered records the sweeps of this run read
  float4* sblk = nullptr;         // bounding boxes of 1024-record super-blocks
  int32_t* mq = nullptr;          // Morton position -> tile-sorted position (alias after the sort)
  int32_t* ord_rho = nullptr;     // per-tile home order for the one-sided density sweeps
  uint32_t* chunk_count = nullptr;  // [ntiles] chunks per tile, then exclusive-scanned
  int32_t* chunk_tile = nullptr;  // [max chunks] tile of every chunk
  uint32_t* chunk_total = nullptr;
  float4* tblk = nullptr;         // boxes of 32-record blocks counted from every tile's start
  uint32_t* tblk_off = nullptr;   // [ntiles] such blocks per tile, then exclusive-scanned
  int64_t* rho_fix = nullptr;     // fixed-point density contributions of the symmetric sweep
  float sym_kmax = 1.0f;          // their scale's kernel bound, for a combine run later

  // pinned host copy of the event tables (same layout as the device block)
  void* pinned = nullptr;
  size_t pinned_bytes = 0;
  DevStatus* status_host = nullptr;  // pinned mirror of *status

  // device staging for host-memory inputs/outputs
  void* dstage = nullptr;
  size_t dstage_bytes = 0;

  // runtime choices (clue_context_set_tuning; clue_autotune_batch measures and picks them)
  int32_t tune_symmetric = 1;                  // symmetric density sweep where it applies
  int32_t tune_nh_split = 8;                   // nearest higher: split a block needed by <= this many lanes
  int64_t tune_overlap_chunk_points = 2200000;  // host-memory batches; 0: no overlap
  int32_t tune_density_gate = 0;               // symmetric density: vote-gated pair steps
  int32_t tune_density_exp2 = 0;               // symmetric density: 2^x on the FMA pipe
  int32_t tune_labels_bfs = 0;                 // labels by follower CSR + frontier BFS, not pointer jumping

  // overlapped host-memory batches (clue_batch_make_clusters): copy streams, per-chunk events
  // and a pinned copy of every chunk's status and seed total
  static constexpr int kPipeMaxChunks = 8;
  cudaStream_t pipe_h2d = nullptr, pipe_d2h = nullptr;
  cudaEvent_t pipe_ev[1 + 3 * kPipeMaxChunks] = {};
  DevStatus* pipe_status_host = nullptr;  // kPipeMaxChunks statuses, then as many uint32 totals
  void* pipe_pinned = nullptr;            // every chunk's pinned event table
  size_t pipe_pinned_bytes = 0;

  int32_t* perm = nullptr;  // alias of the sorted values buffer after the tile sort
  uint32_t* sorted_keys = nullptr;

  KParams last_kp{};  // parameters of the last enqueued run (for clue_context_read_info)
  // near-threshold counts summed on the host over the chunks of an overlapped host-memory
  // batch (near_from_host); every other run leaves them in the device status block
  bool near_from_host = false;
  int64_t near_sum[4] = {0, 0, 0, 0};

  // optional per-stage timing (clue_context_set_timing)
  bool timing = false;
  uint64_t launches = 0;  // kernels launched by this workspace (clue_context_kernel_launches)
  cudaEvent_t tev[CLUE_N_STAGES + 1] = {};
};

// Records stage boundary k on s when timing is enabled.
// Also closes the previous stage's NVTX range and opens the next one, so that a profiler's
// timeline (nsys) shows the host enqueue of every stage by name; NVTX calls cost a pointer test
// when no tool is attached.
inline void stage_mark(Workspace& ws, int k, cudaStream_t s) {
  static const char* const kNames[CLUE_N_STAGES] = {"clue: tiles", "clue: local density", "clue: nearest higher",
                                                    "clue: seeds and labels"};
  if (k > 0) nvtxRangePop();
  if (k < CLUE_N_STAGES) nvtxRangePushA(kNames[k]);
  if (ws.timing && ws.tev[k]) cudaEventRecord(ws.tev[k], s);
}

clue_status workspace_reserve(Workspace& ws, int ndim, size_t n, size_t ntiles, size_t n_events = 1);

// Bytes of the event-table block for `cap` events, and its three parts inside a block.
inline size_t event_table_bytes(size_t cap) { return cap * sizeof(EvGrid) + 2 * (cap + 1) * sizeof(int32_t); }
inline void event_table_carve(void* base, size_t cap, EvGrid** eg, int32_t** pt, int32_t** tile) {
  *eg = static_cast<EvGrid*>(base);
  *pt = reinterpret_cast<int32_t*>(static_cast<char*>(base) + cap * sizeof(EvGrid));
  *tile = *pt + cap + 1;
}
void workspace_release(Workspace& ws);
// Arena bytes workspace_reserve would allocate for these capacities (nothing is allocated).
size_t workspace_bytes_for(int ndim, size_t n, size_t ntiles, size_t n_events);

// Host helpers (clue_capi.cu)
float threshold_for(float r, bool root);
int lower_bounds_ok(const clue_metric* m, int ndim);
void grid_shape(int32_t n, int32_t ppbin, int32_t ndim, int32_t* nperdim, int32_t* ntiles);

}  // namespace clue_b200
