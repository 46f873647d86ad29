/*
 * clue_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's serial CPU CLUE path
 * (clue::Clusterer::make_clusters on the alpaka CpuSerial backend), used as the
 * parity checker by tests/, by __graft_entry__.smoke() and by bench.py's
 * cpu_baseline / --impl reference leg.  Nothing in the product links or calls it.
 *
 * Arithmetic contract (FP32 mirror): every float operation is performed in the
 * order the reference's headers write it, without FMA contraction
 * (build with -ffp-contract=off).  Iteration order over candidates is the
 * reference's: search-box tiles lexicographically (dim 0 outermost, ascending
 * bins), inside a tile ascending point index (what the serial
 * KernelFillAssociator produces).
 */
#ifndef CLUE_ORACLE_H
#define CLUE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_MAX_DIM 10

enum { ORACLE_KERNEL_FLAT = 0, ORACLE_KERNEL_EXP = 1, ORACLE_KERNEL_GAUSS = 2 };
enum {
  ORACLE_METRIC_EUCLID = 0,
  ORACLE_METRIC_WEUCLID = 1,
  ORACLE_METRIC_PERIODIC = 2,
  ORACLE_METRIC_MANHATTAN = 3,
  ORACLE_METRIC_CHEBYSHEV = 4,
  ORACLE_METRIC_WCHEBYSHEV = 5
};
enum { ORACLE_TIE_REFERENCE = 0, ORACLE_TIE_RHO_INDEX = 1 };

typedef struct {
  float dc, rhoc, dm, seed_dc;
  int32_t ppbin;
  int32_t ndim;
  uint8_t wrapped[ORACLE_MAX_DIM];
  int32_t kernel_type;
  float kernel_par[3];
  int32_t metric_type;
  float metric_par[ORACLE_MAX_DIM];
  /* <0: keep every seed; >=0: the reference SeedArray policy, capacity =
   * max(seed_capacity, #points with nearest_higher == -1) */
  int64_t seed_capacity;
  int32_t tiebreak;
  int32_t nthreads; /* <=1 serial; >1 OpenMP over points for density / NH */
} oracle_params;

typedef struct {
  int32_t* cluster_index; /* [n] */
  int32_t* is_seed;       /* [n] */
  float* rho;             /* [n] */
  int32_t* nearest_higher;/* [n], after seed reset (seeds -> -1) */
  float* delta;           /* [n] or NULL: distance to nearest higher, FLT_MAX if none */
  int64_t n_seeds;        /* seeds found (is_seed == 1) */
  int64_t n_clusters;     /* seeds kept in the seed list */
  int64_t dropped_seeds;  /* seeds beyond the SeedArray capacity */
  int64_t seed_capacity_used;
  int64_t max_dfs_stack;  /* deepest follower DFS stack (reference limit: 256) */
  int64_t candidates_rho; /* candidate pairs scanned by the density loop */
  int64_t candidates_nh;  /* candidate pairs scanned by the nearest-higher loop */
  int64_t nh_distance_ties; /* qualifying candidates whose distance tied the running best */
} oracle_out;

typedef struct {
  int32_t nperdim;
  int32_t ntiles;
  float minmax[2 * ORACLE_MAX_DIM]; /* min(d) = [2d], max(d) = [2d+1] */
  float tilesize[ORACLE_MAX_DIM];
} oracle_grid;

/* Full pipeline. coords is SoA: coords[d * n + i]. Returns 0 on success. */
int oracle_run(const oracle_params* p, int32_t n, const float* coords, const float* weight,
               oracle_out* out);

/* Tile grid + tile CSR (offsets[ntiles+1], indexes[n]); offsets/indexes may be NULL to
 * query the grid only. */
/* Nearest-higher stage alone on caller-supplied densities (same grid, candidate order and
 * tie-break as oracle_run).  delta and distance_ties may be NULL. */
int oracle_nearest_higher(const oracle_params* p, int32_t n, const float* coords, const float* rho,
                          int32_t* nearest_higher, float* delta, int64_t* distance_ties);

/* Silhouette score of labelled points (per point, NAN where not scored, and the mean). */
int oracle_silhouette(int32_t ndim, int32_t n, const float* coords, const int32_t* labels, float* per_point,
                      float* mean);

int oracle_tiles(const oracle_params* p, int32_t n, const float* coords, oracle_grid* grid,
                 int32_t* offsets, int32_t* indexes);

/* Local density in FP64 over the same candidate sets (box from the FP32 grid), the
 * tolerance reference for rho.  near_dc (may be NULL) flags points with a candidate whose
 * FP64 distance lies within rel_tol * dc of dc: FP32 and FP64 may disagree on whether that
 * candidate counts, so their rho is reported apart instead of held to the tolerance. */
int oracle_rho_f64(const oracle_params* p, int32_t n, const float* coords, const float* weight,
                   double* rho64, uint8_t* near_dc, double rel_tol);

/* Distance metric on two points (ndim floats each), exposed for metric known-answer tests. */
float oracle_metric(const oracle_params* p, const float* a, const float* b);

/* Convolutional kernel value for a distance, exposed for kernel known-answer tests. */
float oracle_kernel(const oracle_params* p, float dist, int32_t i, int32_t j);


/* Batch of independent events (event e = points [offsets[e], offsets[e+1]) of SoA arrays with
 * stride ld), one event per OpenMP thread, each event clustered alone as oracle_run does.
 * out's arrays cover the whole batch; nearest highers are batch-global; stats are summed
 * (max_dfs_stack: maximum).  ev_n_clusters (may be NULL) receives each event's clusters. */
int oracle_run_events(const oracle_params* p, int32_t n_events, const int32_t* offsets, int32_t ld,
                      const float* coords, const float* weight, oracle_out* out, int64_t* ev_n_clusters);

/* Near-threshold decision points of two density vectors of the same points (see
 * clue_oracle.c).  flags[i] is an OR of the bits below. */
enum {
  ORACLE_NEAR_RHOC = 1,
  ORACLE_NEAR_FLIP = 2,
  ORACLE_NEAR_TIE = 4,
  ORACLE_NEAR_SEED_DC = 8,
  ORACLE_NEAR_DM = 16
};
int oracle_near_flags(const oracle_params* p, int32_t n, const float* coords, const float* rho_a,
                      const float* rho_b, const float* delta_a, double tol, uint8_t* flags,
                      double* max_flip_rel);

/* Per-event forms (OpenMP over events): kind ORACLE_AUX_RHO_F64 fills rho64 (and the near-dc
 * flags when flags is not NULL); ORACLE_AUX_NEAREST_HIGHER fills nearest_higher (batch-global)
 * and delta from the densities rho_a; ORACLE_AUX_NEAR_FLAGS fills flags and max_flip_rel. */
enum { ORACLE_AUX_RHO_F64 = 0, ORACLE_AUX_NEAREST_HIGHER = 1, ORACLE_AUX_NEAR_FLAGS = 2 };
int oracle_events_aux(int kind, const oracle_params* p, int32_t n_events, const int32_t* offsets, int32_t ld,
                      const float* coords, const float* weight, const float* rho_a, const float* rho_b,
                      const float* delta_a, double tol, double* rho64, uint8_t* flags, int32_t* nearest_higher,
                      float* delta, double* max_flip_rel);

#ifdef __cplusplus
}
#endif
#endif
