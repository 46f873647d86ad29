/*
 * clue_b200.h -- C ABI of the B200-native CLUE clustering library (libclue_b200.so).
 *
 * Plain C types only (pointers, sizes, PODs); no CUDA or torch types appear in the
 * signatures.  Streams are passed as `void*` holding a cudaStream_t (NULL = the
 * legacy default stream of the current device).
 *
 * Every entry point returns a clue_status; on failure clue_last_error() returns a
 * thread-local message.  The reference throws std::invalid_argument /
 * std::out_of_range / std::runtime_error on the host; the C++ layer in
 * include/CLUEstering/ maps the status codes back onto those exception types.
 *
 * Reference interfaces replaced (paths relative to the reference project root):
 *   clue_make_clusters  <- clue::Clusterer::make_clusters (4 overloads)
 *                          include/CLUEstering/core/Clusterer.hpp:114-169,
 *                          pipeline include/CLUEstering/core/detail/Clusterer.hpp:134-217
 *   clue_params         <- Clusterer ctor / setParameters / setWrappedCoordinates
 *                          include/CLUEstering/core/Clusterer.hpp:84-103,174-182
 *   clue_kernel         <- FlatKernel / ExponentialKernel / GaussianKernel
 *                          include/CLUEstering/core/ConvolutionalKernel.hpp:14-85
 *   clue_metric         <- the six metrics of include/CLUEstering/core/DistanceMetrics.hpp:33-230
 *   clue_context_*      <- the Clusterer's reusable tiles / seeds / followers buffers
 *                          include/CLUEstering/core/Clusterer.hpp:47-49
 *   clue_device_alloc / clue_memcpy_* / clue_stream_*
 *                       <- PointsDevice storage and copyToHost / copyToDevice
 *                          include/CLUEstering/data_structures/PointsDevice.hpp:19-107,129-194
 *   clue_get_clusters   <- clue::get_clusters (cluster -> points association map)
 *                          include/CLUEstering/utils/detail/get_clusters.hpp:21-46
 *   clue_cluster_centroids <- clue::cluster_centroids, ClusterProperties sizes
 *                          include/CLUEstering/utils/detail/cluster_centroid.hpp:39-65
 *   clue_batch_*        <- no reference counterpart: many independent events in one launch
 */
#ifndef CLUE_B200_H
#define CLUE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CLUE_MAX_DIM 10
#define CLUE_ABI_VERSION 2

typedef enum clue_status {
  CLUE_OK = 0,
  CLUE_ERR_INVALID_ARG = 1,    /* std::invalid_argument in the reference */
  CLUE_ERR_OUT_OF_MEMORY = 2,  /* device allocation failed */
  CLUE_ERR_CAPACITY = 3,       /* request larger than a fixed capacity */
  CLUE_ERR_TIMEOUT = 4,        /* a bounded device wait gave up */
  CLUE_ERR_CUDA = 5,           /* CUDA runtime error (message holds the CUDA error string) */
  CLUE_ERR_NOT_SUPPORTED = 6,  /* option not available in this build */
  CLUE_ERR_NONFINITE = 7,      /* NaN or Inf in coordinates or weights */
  CLUE_ERR_OUT_OF_RANGE = 8    /* std::out_of_range in the reference */
} clue_status;

typedef enum clue_kernel_type {
  CLUE_KERNEL_FLAT = 0,        /* par[0] = flat height */
  CLUE_KERNEL_EXPONENTIAL = 1, /* par[0] = avg, par[1] = amplitude */
  CLUE_KERNEL_GAUSSIAN = 2     /* par[0] = avg, par[1] = std, par[2] = amplitude */
} clue_kernel_type;

typedef struct clue_kernel {
  int32_t type;
  float par[3];
} clue_kernel;

typedef enum clue_metric_type {
  CLUE_METRIC_EUCLIDEAN = 0,
  CLUE_METRIC_WEIGHTED_EUCLIDEAN = 1, /* par[d] = weight of dimension d */
  CLUE_METRIC_PERIODIC_EUCLIDEAN = 2, /* par[d] = period of dimension d (0 = not periodic) */
  CLUE_METRIC_MANHATTAN = 3,
  CLUE_METRIC_CHEBYSHEV = 4,
  CLUE_METRIC_WEIGHTED_CHEBYSHEV = 5  /* par[d] = weight of dimension d */
} clue_metric_type;

typedef struct clue_metric {
  int32_t type;
  float par[CLUE_MAX_DIM];
} clue_metric;

typedef enum clue_tiebreak {
  CLUE_TIE_REFERENCE = 0, /* nearest higher keeps the first strict minimum in tile order */
  CLUE_TIE_RHO_INDEX = 1  /* equal distances resolved by higher rho, then lower index */
} clue_tiebreak;

typedef struct clue_params {
  float dc;       /* density radius, > 0 */
  float rhoc;     /* seed density threshold, >= 0 */
  float dm;       /* nearest-higher search radius, > 0 (reference default: dc) */
  float seed_dc;  /* seed distance threshold, > 0 (reference default: dc) */
  int32_t points_per_tile;        /* > 0 (reference default 128) */
  uint8_t wrapped[CLUE_MAX_DIM];  /* 1 = periodic coordinate */
  /* Seed list capacity.  < 0: every seed is kept.  >= 0: the reference's SeedArray
   * policy -- capacity = max(seed_capacity, number of points without a nearest
   * higher); seeds beyond it (in index order) are dropped and their followers get
   * label -1, as in include/CLUEstering/data_structures/internal/SeedArray.hpp:33-41. */
  int64_t seed_capacity;
  int32_t tiebreak;               /* clue_tiebreak */
  int32_t flags;                  /* CLUE_FLAG_* */
} clue_params;

/* Local-density summation order.  By default the flat kernel sums every point's terms in the
 * reference's candidate order (search-box tiles lexicographically, ascending index inside a
 * tile), which makes rho bit-identical to the reference's serial backend; the exponential and
 * Gaussian kernels, whose device expf can differ from the host's by an ulp anyway, sum in a
 * spatial order that skips far candidate blocks (rho within 1e-5 relative of FP64). */
#define CLUE_FLAG_REFERENCE_ORDER 1 /* reference order for every kernel */
#define CLUE_FLAG_SPATIAL_DENSITY 2 /* spatial order for the flat kernel too */
/* Count the points whose nearest-higher choice compares two densities within the near-threshold
 * tolerance (clue_near_counts.nh_near_ties).  Costs one extra pruned neighbour sweep. */
#define CLUE_FLAG_NEAR_TIES 4

/* Output arrays, caller-owned, n elements each, all in the memory space given by
 * `memory` in clue_make_clusters.  Only cluster_index is required. */
typedef struct clue_outputs {
  int32_t* cluster_index;  /* cluster label, -1 for outliers / unassigned */
  int32_t* is_seed;        /* 1 for seeds */
  float* rho;              /* local density */
  int32_t* nearest_higher; /* index of the nearest higher point, -1 for seeds and outliers */
  float* delta;            /* distance to the nearest higher (FLT_MAX when none was found) */
} clue_outputs;

typedef struct clue_run_info {
  int64_t n_seeds;             /* points flagged as seeds */
  int64_t n_clusters;          /* seeds kept in the seed list (= clusters labelled) */
  int64_t dropped_seeds;       /* seeds beyond the seed capacity */
  int64_t seed_capacity_used;  /* -1 when every seed is kept; -2: per event (batched call) */
  int64_t n_tiles;             /* tiles of the reference grid */
  int64_t n_per_dim;
  int64_t label_rounds;        /* pointer-jumping rounds that changed a parent */
} clue_run_info;

/* Decisions of the last run taken on values within a relative tolerance CLUE_NEAR_TOL of their
 * threshold (ClusteringKernels.hpp:129-143 nearest higher, :232-233 seeds in the reference):
 * where another summation order or another exp rounds a density differently, these are the
 * only points whose seed flag or nearest higher can change.  Counted on the device in every
 * run; nh_near_ties only with CLUE_FLAG_NEAR_TIES (else -1). */
#define CLUE_NEAR_TOL 1e-5
typedef struct clue_near_counts {
  int64_t rho_near_rhoc;      /* |rho - rhoc| <= tol * rhoc */
  int64_t delta_near_seed_dc; /* nearest higher found and |delta - seed_dc| <= tol * seed_dc */
  int64_t delta_near_dm;      /* nearest higher found and |delta - dm| <= tol * dm */
  int64_t nh_near_ties;       /* the chosen nearest higher, or a nearer candidate that is not higher,
                                 has a density within tol of the point's own; -1: not counted */
} clue_near_counts;

typedef enum clue_memory { CLUE_MEM_DEVICE = 0, CLUE_MEM_HOST = 1 } clue_memory;

typedef struct clue_context_s* clue_context;

/* ---- version / errors ---------------------------------------------------- */
int32_t clue_abi_version(void);
const char* clue_last_error(void);
const char* clue_status_string(clue_status s);

/* ---- parameter validation (host only, no GPU needed) -------------------- */
/* Clusterer ctor / setParameters rules: include/CLUEstering/core/detail/Clusterer.hpp:24-51. */
clue_status clue_check_params(const clue_params* p);
/* Kernel ctor rules: include/CLUEstering/core/detail/ConvolutionalKernel.hpp:10-53
 * (Gaussian avg >= 0 is accepted; the reference rejects avg == 0). */
clue_status clue_check_kernel(const clue_kernel* k);
clue_status clue_check_metric(const clue_metric* m, int32_t ndim);
/* Reference tile grid shape for n points (include/CLUEstering/core/detail/SetupTiles.hpp:23-26). */
clue_status clue_grid_shape(int32_t n, int32_t points_per_tile, int32_t ndim, int32_t* n_per_dim,
                            int32_t* n_tiles);
/* Metric / kernel evaluation on the host, for known-answer tests of the plugins
 * (include/CLUEstering/core/DistanceMetrics.hpp, core/detail/ConvolutionalKernel.hpp). */
float clue_metric_eval(const clue_metric* m, int32_t ndim, const float* a, const float* b);
float clue_kernel_eval(const clue_kernel* k, float dist, int32_t i, int32_t j);

/* ---- devices, memory, streams ------------------------------------------- */
clue_status clue_device_count(int32_t* count);
clue_status clue_device_alloc(int32_t device, size_t bytes, void** ptr);
clue_status clue_device_free(void* ptr);
clue_status clue_host_alloc_pinned(size_t bytes, void** ptr);
clue_status clue_host_free_pinned(void* ptr);
clue_status clue_memcpy_htod(void* dst, const void* src, size_t bytes, void* stream);
clue_status clue_memcpy_dtoh(void* dst, const void* src, size_t bytes, void* stream);
clue_status clue_memcpy_dtod(void* dst, const void* src, size_t bytes, void* stream);
clue_status clue_stream_create(int32_t device, void** stream);
clue_status clue_stream_destroy(void* stream);
clue_status clue_stream_synchronize(void* stream);

/* ---- clustering ----------------------------------------------------------- */
/* A context owns reusable device workspace (tile CSR, sorted point records, seed and
 * label buffers) on one device; buffers only grow.  Not thread-safe: one caller
 * at a time, like a reference Clusterer. */
clue_status clue_context_create(int32_t device, clue_context* ctx);
clue_status clue_context_destroy(clue_context ctx);
/* Pre-size the workspace for up to n points of ndim dimensions (optional). */
clue_status clue_context_reserve(clue_context ctx, int32_t ndim, int32_t n, int32_t points_per_tile);
/* Bytes of device workspace the context currently holds. */
/* Pre-sizes the workspace for batched calls of up to n_points points, n_tiles tiles (the sum of
 * the events' reference grids) and n_events events, so that such calls allocate nothing. */
clue_status clue_context_reserve_batch(clue_context ctx, int32_t ndim, int64_t n_points, int64_t n_tiles,
                                       int32_t n_events);
size_t clue_context_workspace_bytes(clue_context ctx);

/*
 * Run the five CLUE stages on n points of ndim (1..10) dimensions.
 * coords: SoA, coords[d * n + i];  weight: n floats.  Both in `memory` space, as are
 * the outputs.  With CLUE_MEM_HOST the library copies through pinned staging
 * buffers on `stream`.  Blocks until the results are in `out` (the reference's
 * make_clusters waits as well); `info` may be NULL.  The pipeline itself runs as one CUDA
 * graph launch on a stream of the context, ordered after the work already on `stream` and
 * before its next (the executable graph is kept in the context and updated on the next call).
 * Non-finite coordinates or weights are rejected with CLUE_ERR_NONFINITE
 * (the reference's behaviour there is undefined: static_cast<int>(NaN)).
 */
clue_status clue_make_clusters(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                               const clue_metric* metric, int32_t ndim, int32_t n,
                               const float* coords, const float* weight, const clue_outputs* out,
                               int32_t memory, void* stream, clue_run_info* info);

/*
 * Same pipeline, device memory only, without any host synchronisation: every launch is
 * enqueued on `stream` and the call returns.  Nothing is allocated if the context was
 * reserved for (ndim, n) beforehand, so the call can be captured in a CUDA graph.
 * Run information and the non-finite check land in a device-side status block that
 * clue_context_read_info() copies back (it synchronises the stream).
 */
clue_status clue_make_clusters_async(clue_context ctx, const clue_params* params,
                                     const clue_kernel* kernel, const clue_metric* metric,
                                     int32_t ndim, int32_t n, const float* coords,
                                     const float* weight, const clue_outputs* out, void* stream);
clue_status clue_context_read_info(clue_context ctx, void* stream, clue_run_info* info);
/* Near-threshold counts of the context's last run (synchronises `stream`, the stream the run
 * was enqueued on; host-memory batches report the sum over their chunks).  No counterpart in
 * the reference, which neither counts nor reports these decisions. */
clue_status clue_context_read_near_counts(clue_context ctx, void* stream, clue_near_counts* counts);

/* Per-stage device timing of the following runs (CUDA events on the run's stream):
 * stage 0 = tile build (bounding box, bins, sort, records), 1 = local density,
 * 2 = nearest higher, 3 = seeds + labels + output scatter.  Off by default. */
#define CLUE_N_STAGES 4
clue_status clue_context_set_timing(clue_context ctx, int32_t enable);
/* Milliseconds of each stage of the last timed run (synchronises on its last event). */
clue_status clue_context_stage_times(clue_context ctx, float* ms, int32_t n_stages);
/* Kernels this context has launched so far (all runs). */
uint64_t clue_context_kernel_launches(clue_context ctx);

/* ---- batched events (no reference counterpart) -------------------------------
 * Clusters n_events independent events in one pass.  Event e is the points
 * [event_offsets[e], event_offsets[e + 1]) of the concatenated SoA input
 * (coords[d * n_total + i], n_total = event_offsets[n_events]); event_offsets is a HOST array
 * of n_events + 1 entries, every event holding at least one point.  Each event gets its
 * own reference tile grid and its labels are numbered from 0 inside the event, exactly as if
 * it had been clustered alone.  ev_n_clusters (optional, n_events entries, same memory space
 * as the outputs) receives every event's cluster count; `info` holds the totals.
 * With CLUE_MEM_HOST, a batch of 4M points or more is run in chunks of whole events whose
 * copies overlap the previous chunk's pipeline (clue_tuning.overlap_chunk_points; consecutive
 * chunks run concurrently on two workspaces and two streams of the context, each chunk as one
 * graph launch); the outputs are the same as one pass, and the call returns when they are in
 * `out`.  Pinned host buffers are needed for the copies to overlap.
 */
clue_status clue_batch_make_clusters(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                                     const clue_metric* metric, int32_t ndim, int32_t n_events,
                                     const int32_t* event_offsets, const float* coords, const float* weight,
                                     const clue_outputs* out, int32_t* ev_n_clusters, int32_t memory,
                                     void* stream, clue_run_info* info);
/* Device memory only, no host synchronisation (see clue_make_clusters_async). */
clue_status clue_batch_make_clusters_async(clue_context ctx, const clue_params* params,
                                           const clue_kernel* kernel, const clue_metric* metric, int32_t ndim,
                                           int32_t n_events, const int32_t* event_offsets, const float* coords,
                                           const float* weight, const clue_outputs* out, int32_t* ev_n_clusters,
                                           void* stream);

/* The plain single-event pipeline run once per event, back to back on `stream` (device
 * memory; same inputs, outputs and per-event label numbering as the batched call, but the
 * nearest-higher chain depth is limited to what the enqueued label rounds resolve).
 * This is the per-event launch loop that the batched path replaces.  With event_ms non-NULL
 * (host, n_events floats) the call synchronises and writes every event's device time. */
clue_status clue_events_loop(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                             const clue_metric* metric, int32_t ndim, int32_t n_events,
                             const int32_t* event_offsets, const float* coords, const float* weight,
                             const clue_outputs* out, void* stream, float* event_ms);

/* The whole batched pipeline (event-table upload and every stage) captured once into an
 * executable CUDA graph; each clue_graph_launch replays it on the same buffers.  Needs a
 * non-default stream.  The context must not run other work between capture and the last
 * launch that relies on its workspace. */
typedef struct clue_graph_s* clue_graph;
clue_status clue_graph_capture_batch(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                                     const clue_metric* metric, int32_t ndim, int32_t n_events,
                                     const int32_t* event_offsets, const float* coords, const float* weight,
                                     const clue_outputs* out, int32_t* ev_n_clusters, void* stream,
                                     clue_graph* graph);
clue_status clue_graph_launch(clue_graph graph, void* stream);
clue_status clue_graph_destroy(clue_graph graph);

/* ---- runtime choices and their autotuner (no reference counterpart) -----------------------
 * The reference fixes its launch shape per backend.  Here a few choices that never change the
 * results beyond the stated tolerance are made at run time per context:
 *   symmetric_density   1 (default): where the kernel is exponential or Gaussian, the order is
 *                       spatial and the metric bounds every coordinate difference (Euclidean,
 *                       Manhattan, Chebyshev, no wrapped coordinate), every pair within dc is
 *                       evaluated once for both points; 0: one-sided sweep.  Both are within
 *                       1e-5 of FP64.
 *   nh_split_lanes      0..16 (default 8): a nearest-higher candidate block that at most this
 *                       many lanes of a warp still need is split among all 32 lanes; 0 never
 *                       splits.  Results are identical for every value.
 *   overlap_chunk_points  host-memory batches of 4M points or more overlap their copies with
 *                       the pipeline in chunks of about this many points (default 2200000);
 *                       0 turns the overlap off.  Results are identical.
 * clue_autotune_batch times the candidate values on a device-resident sample batch (CUDA
 * events on `stream`), keeps the fastest in the context and, with cache_path non-NULL, appends
 * it to a text cache keyed by (ndim, size bucket = ceil(log2 n), event-count bucket, kernel,
 * metric, flags); a later call with the same key reads the cache and times nothing.
 */
typedef struct clue_tuning {
  int32_t symmetric_density;
  int32_t nh_split_lanes;
  int64_t overlap_chunk_points;
  /* symmetric density sweep, unit-amplitude exponential / zero-mean Gaussian kernels, Euclidean
   * metric, up to four dimensions: */
  int32_t density_gate;  /* 1: skip the kernel evaluation of candidate pairs no lane holds within dc */
  int32_t density_exp2;  /* 1: evaluate 2^x on the FMA pipe (Taylor polynomial) instead of the MUFU */
  /* 1: labels from a follower CSR (counts, scan, scatter: the reference's Followers::fill) and a
   * frontier-parallel breadth-first walk from the seeds; 0: pointer jumping.  Same labels. */
  int32_t labels_bfs;
  int32_t reserved;      /* 0 */
} clue_tuning;
void clue_tuning_defaults(clue_tuning* t);
clue_status clue_context_set_tuning(clue_context ctx, const clue_tuning* t);
clue_status clue_context_get_tuning(clue_context ctx, clue_tuning* t);
clue_status clue_autotune_batch(clue_context ctx, const clue_params* params, const clue_kernel* kernel,
                                const clue_metric* metric, int32_t ndim, int32_t n_events,
                                const int32_t* event_offsets, const float* coords, const float* weight,
                                void* stream, const char* cache_path, clue_tuning* chosen);

/*
 * clue_make_clusters_noalloc -- no counterpart in the reference.
 * The same pipeline for callers that cannot allocate device memory (a runtime that owns all
 * device memory through its own pool, a plugin inside another framework, or a
 * latency-critical path that cannot afford cudaMalloc's implicit synchronisation).  Inputs
 * and outputs are the caller's device buffers; every intermediate buffer lives in one
 * fixed 6 MiB file-scope device array, so the call allocates nothing.
 * The same density sweeps as clue_make_clusters, so the outputs are bit for bit those of
 * clue_make_clusters on the same input.
 * Limits: at most 65536 tiles, and n <= 32768 points in 1 to 7 dimensions (about 29,900 to
 * 30,300 in 8 to 10 at the default 128 points per tile); larger requests return
 * CLUE_ERR_CAPACITY with the exact limit for the request's dimensionality in the message.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current: make that first call before any stream capture.  All calls on a device
 * share the array (it keeps the last call's contents); calls that overlap on the GPU race and
 * must be serialised by the caller.  Every call waits for `stream` to finish its work before
 * it returns; the results are then in `out`.  `info` may be NULL.
 */
clue_status clue_make_clusters_noalloc(const clue_params* params, const clue_kernel* kernel,
                                       const clue_metric* metric, int32_t ndim, int32_t n,
                                       const float* coords, const float* weight,
                                       const clue_outputs* out, void* stream, clue_run_info* info);

/*
 * Cluster -> points association map (CSR) from device labels, the device side of
 * clue::get_clusters (include/CLUEstering/utils/get_clusters.hpp:34-36 and
 * data_structures/internal/MakeAssociator.hpp:11-34 in the reference): keys 0..max_label,
 * offsets[c]..offsets[c + 1] are the points of cluster c, point indexes ascending inside a
 * cluster (the order of the reference's host fill); labels -1 are left out.  All device
 * pointers: `offsets` must hold n + 1 entries (entries past n_clusters repeat the total) and
 * `points` n entries.  n_clusters_out (= max label + 1) and n_clustered_out are written on the
 * host; the call synchronises `stream`.  A label outside [-1, n) gives CLUE_ERR_OUT_OF_RANGE.
 */
clue_status clue_get_clusters(clue_context ctx, int32_t n, const int32_t* cluster_index,
                              int32_t* offsets, int32_t* points, int32_t* n_clusters_out,
                              int32_t* n_clustered_out, void* stream);

/*
 * Silhouette score on the GPU (reference include/CLUEstering/utils/detail/scores.hpp:17-99,
 * computed there on the host): for a point of a cluster with at least two points,
 * s = (b - a) / max(a, b) with a the mean distance to the other points of its cluster and b the
 * smallest mean distance to another cluster's points; Euclidean distances, cluster sums in
 * ascending point order as the reference's association map gives them.  coords (SoA) and
 * cluster_index are device arrays of n points (-1 = not clustered).  per_point (device, n
 * floats, optional) receives every point's score, NaN for points not scored; *mean (host,
 * optional) the average over the scored points.  n x (clustered points) distances; allocates
 * its temporaries and synchronises `stream`.
 */
clue_status clue_silhouette(clue_context ctx, int32_t ndim, int32_t n, const float* coords,
                            const int32_t* cluster_index, float* per_point, float* mean, void* stream);

/*
 * Cluster centroids on the GPU (reference include/CLUEstering/utils/detail/cluster_centroid.hpp:
 * 39-65, computed there on the host): for every cluster c, the unweighted mean of its points'
 * coordinates, summed in ascending point order in FP32 and divided by the cluster size as a
 * float (bit for bit the reference's loop).  coords (SoA) and cluster_index are device arrays
 * of n points (-1 = not clustered).  centroids (device, capacity x ndim floats) receives
 * centroid c at [c * ndim, c * ndim + ndim); sizes (device, capacity, optional) every cluster's
 * point count (the reference's ClusterProperties::cluster sizes,
 * data_structures/ClusterProperties.hpp:19-51).  *n_clusters_out (host, optional) = max label
 * + 1; more clusters than `capacity` gives CLUE_ERR_CAPACITY with *n_clusters_out set
 * (capacity 0 with centroids NULL asks for the count alone).  Allocates its temporaries and
 * synchronises `stream`.
 */
clue_status clue_cluster_centroids(clue_context ctx, int32_t ndim, int32_t n, const float* coords,
                                   const int32_t* cluster_index, int32_t capacity, float* centroids,
                                   int32_t* sizes, int32_t* n_clusters_out, void* stream);

/* ---- serving (no reference counterpart) -------------------------------------------------
 * A request loop with continuous batching on one GPU.  Callers submit single events (host
 * memory) from any thread; a dispatcher thread owned by the server packs every pending event
 * that fits into the next free slot and runs them as one batched pipeline, while the other
 * slots' batches are still on the GPU.  Each slot is a preallocated device pool (workspace,
 * input and output buffers) plus pinned staging and a stream; together the slots stay inside
 * device_budget_bytes, and an event is admitted to a slot only while the slot's points,
 * tiles and events stay within what was reserved for it.  Results are identical to clustering
 * the event alone (same per-event grids and label numbering; nearest_higher is event-local).
 */
typedef struct clue_server_s* clue_server;

typedef struct clue_server_config {
  int32_t device;
  int32_t ndim;                 /* 1..10 */
  int32_t n_slots;              /* batches that may be on the GPU at once, 1..16 */
  int32_t max_batch_events;     /* events per batch, >= 1 */
  int32_t max_event_points;     /* larger events are refused (CLUE_ERR_CAPACITY) */
  int32_t max_pending;          /* queued events before submit refuses (CLUE_ERR_CAPACITY) */
  int64_t device_budget_bytes;  /* device memory for all slots; each slot holds >= max_event_points */
} clue_server_config;

typedef struct clue_request_info {
  int32_t status;          /* clue_status of the request */
  int32_t n_clusters;      /* clusters of the event */
  int32_t batch_events;    /* events in the batch that carried it */
  int32_t slot;            /* slot that ran it */
  double submit_s;         /* server clock (seconds since creation): accepted */
  double start_s;          /* its batch was enqueued on the GPU */
  double done_s;           /* results were in the caller's buffers */
} clue_request_info;

typedef struct clue_server_stats {
  int64_t submitted, completed, rejected, failed;
  int64_t batches, batched_points;
  int64_t slot_points;     /* points one slot holds */
  int64_t slot_events;
  int64_t device_bytes;    /* device memory held by all slots */
  int32_t max_batch_seen;  /* largest batch (events) so far */
  int32_t max_in_flight;   /* most slots on the GPU at once so far */
} clue_server_stats;

clue_status clue_server_create(const clue_server_config* config, const clue_params* params,
                               const clue_kernel* kernel, const clue_metric* metric, clue_server* server);
/* Waits for the batches on the GPU, then frees everything; pending requests fail. */
clue_status clue_server_destroy(clue_server server);
/* Queues one event: coords[d * coord_stride + i] (host), weight[i], i < n.  Inputs and the
 * host output arrays in `out` (cluster_index required) must stay valid until the request is
 * waited for.  Writes the request's ticket. */
clue_status clue_server_submit(clue_server server, int32_t n, const float* coords, int64_t coord_stride,
                               const float* weight, const clue_outputs* out, int64_t* ticket);
/* Waits up to timeout_ms (< 0: no limit) for a request, then releases it and fills `info`
 * (may be NULL).  CLUE_ERR_TIMEOUT leaves the request pending; the returned status is the
 * request's own otherwise. */
clue_status clue_server_wait(clue_server server, int64_t ticket, int32_t timeout_ms, clue_request_info* info);
clue_status clue_server_stats_read(clue_server server, clue_server_stats* stats);
/* Open-loop load replay from the calling thread.  Trace event e is pool event
 * id = event_ids ? event_ids[e] : e, i.e. points [event_offsets[id], event_offsets[id + 1]) of
 * the concatenated SoA host arrays (coords[d * n_pool_points + i], n_pool_points =
 * event_offsets[max id + 1]); it is submitted arrival_s[e] seconds after the call.  With `out`
 * given (only without event_ids) results land at the event's offsets; with out == NULL they
 * stay in the server (throughput / latency runs).  latency_s[e] = completion - scheduled
 * arrival, or -1 for an event the server refused (counted in *n_rejected).  Returns when every
 * admitted event is done. */
clue_status clue_server_replay(clue_server server, int32_t n_events, const int32_t* event_ids,
                               const int32_t* event_offsets, const double* arrival_s, const float* coords,
                               const float* weight, const clue_outputs* out, double* latency_s,
                               int32_t* n_rejected);

#ifdef __cplusplus
}
#endif
#endif /* CLUE_B200_H */
