/*
 * clue_oracle.c -- TEST INFRASTRUCTURE ONLY (see clue_oracle.h).
 *
 * CPU restatement of the reference's serial CLUE path.  Each function names the
 * reference file:line it follows (paths relative to the reference project root,
 * headers under include/CLUEstering/).  Build with -ffp-contract=off so that no
 * multiply-add is fused: the reference's arithmetic is restated operation by
 * operation.
 */
#include "clue_oracle.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* float -> int32 truncation with x86 cvttss2si semantics: NaN and out-of-range
 * inputs give INT32_MIN.  The reference's static_cast<int>(float) compiles to
 * this instruction on the serial CPU backend (TilesView.hpp:41-43,95). */
static inline int32_t cvt_i32(float f) {
  if (!(f > -2147483904.0f && f < 2147483648.0f)) return INT32_MIN;
  return (int32_t)f;
}

typedef struct {
  int32_t ndim, nperdim, ntiles;
  float mn[ORACLE_MAX_DIM], mx[ORACLE_MAX_DIM], size[ORACLE_MAX_DIM];
  uint8_t wrapped[ORACLE_MAX_DIM];
  int64_t stride[ORACLE_MAX_DIM];
} grid_t;

/* core/detail/SetupTiles.hpp:23-26: ntiles = ceil(n / (float)ppbin),
 * nperdim = ceil(pow(ntiles, 1.0 / N)), ntiles = pow(nperdim, N). */
static void grid_shape(int32_t n, int32_t ppbin, int32_t ndim, int32_t* nperdim, int32_t* ntiles) {
  int32_t t0 = (int32_t)ceilf((float)n / (float)ppbin);
  int32_t npd = (int32_t)ceil(pow((double)t0, 1.0 / (double)ndim));
  *nperdim = npd;
  *ntiles = (int32_t)pow((double)npd, (double)ndim);
}

/* core/detail/ComputeTiles.hpp:13-27: per-dimension min/max over the host SoA and
 * tile size (max - min) / nperdim in FP32. */
static void grid_build(const oracle_params* p, int32_t n, const float* coords, grid_t* g) {
  g->ndim = p->ndim;
  grid_shape(n, p->ppbin, p->ndim, &g->nperdim, &g->ntiles);
  for (int d = 0; d < p->ndim; ++d) {
    const float* x = coords + (size_t)d * n;
    float mn = x[0], mx = x[0];
    for (int32_t i = 1; i < n; ++i) {
      if (x[i] < mn) mn = x[i];
      if (mx < x[i]) mx = x[i];
    }
    g->mn[d] = mn;
    g->mx[d] = mx;
    g->size[d] = (mx - mn) / (float)g->nperdim;
    g->wrapped[d] = p->wrapped[d];
  }
  /* TilesView.hpp:53-70: global bin = sum_d nperdim^(N-1-d) * bin_d (exact integers). */
  int64_t s = 1;
  for (int d = p->ndim - 1; d >= 0; --d) {
    g->stride[d] = s;
    s *= g->nperdim;
  }
}

/* TilesView.hpp:93-101 normalizeCoordinate. */
static inline float normalize_coord(const grid_t* g, float coord, int d) {
  const float range = g->mx[d] - g->mn[d];
  float rem = coord - (float)cvt_i32(coord / range) * range;
  if (rem >= g->mx[d])
    rem -= range;
  else if (rem < g->mn[d])
    rem += range;
  return rem;
}

/* TilesView.hpp:37-51 getBin. */
static inline int32_t get_bin(const grid_t* g, float coord, int d) {
  int32_t b;
  if (g->wrapped[d])
    b = cvt_i32((normalize_coord(g, coord, d) - g->mn[d]) / g->size[d]);
  else
    b = cvt_i32((coord - g->mn[d]) / g->size[d]);
  if (b > g->nperdim - 1) b = g->nperdim - 1;
  if (b < 0) b = 0;
  return b;
}

/* TilesView.hpp:53-61 getGlobalBin (Tiles.hpp:193-206 GetGlobalBin). */
static inline int64_t global_bin(const grid_t* g, int32_t n, const float* coords, int32_t i) {
  int64_t gb = 0;
  for (int d = 0; d < g->ndim; ++d) gb += g->stride[d] * get_bin(g, coords[(size_t)d * n + i], d);
  return gb;
}

/* TilesView.hpp:72-82 searchBox. */
static inline void search_box(const grid_t* g, const float* xi, float r, int32_t* lo, int32_t* hi) {
  for (int d = 0; d < g->ndim; ++d) {
    int32_t a = get_bin(g, xi[d] - r, d);
    int32_t b = get_bin(g, xi[d] + r, d);
    if (g->wrapped[d] && a > b) b += g->nperdim;
    lo[d] = a;
    hi[d] = b;
  }
}

/* TilesView.hpp:63-70 getGlobalBinByBin (wrapped dims reduced modulo nperdim). */
static inline int64_t global_bin_by_bin(const grid_t* g, const int32_t* v) {
  int64_t gb = 0;
  for (int d = 0; d < g->ndim; ++d) {
    int32_t b = g->wrapped[d] ? (v[d] % g->nperdim) : v[d];
    gb += g->stride[d] * b;
  }
  return gb;
}

/* core/DistanceMetrics.hpp:33-230; sums are meta::accumulate's right fold
 * t0 + (t1 + (... + (t_{N-1} + 0))) (internal/meta/accumulate.hpp:13-17), maxima are
 * meta::maximum's left-to-right std::max starting at 0 (internal/meta/maximum.hpp). */
float oracle_metric(const oracle_params* p, const float* a, const float* b) {
  const int N = p->ndim;
  const float* w = p->metric_par;
  float acc = 0.0f;
  switch (p->metric_type) {
    case ORACLE_METRIC_EUCLID:
      for (int d = N - 1; d >= 0; --d) {
        float t = (a[d] - b[d]) * (a[d] - b[d]);
        acc = t + acc;
      }
      return sqrtf(acc);
    case ORACLE_METRIC_WEUCLID:
      for (int d = N - 1; d >= 0; --d) {
        float t = w[d] * (a[d] - b[d]) * (a[d] - b[d]);
        acc = t + acc;
      }
      return sqrtf(acc);
    case ORACLE_METRIC_PERIODIC:
      for (int d = N - 1; d >= 0; --d) {
        float diff = fabsf(a[d] - b[d]);
        float alt = w[d] - diff;
        float pd = (alt < diff) ? alt : diff; /* alpaka::math::min == std::fmin for non-NaN */
        float t = pd * pd;
        acc = t + acc;
      }
      return sqrtf(acc);
    case ORACLE_METRIC_MANHATTAN:
      for (int d = N - 1; d >= 0; --d) {
        float t = fabsf(a[d] - b[d]);
        acc = t + acc;
      }
      return acc;
    case ORACLE_METRIC_CHEBYSHEV: {
      float m = 0.0f;
      for (int d = 0; d < N; ++d) {
        float t = fabsf(a[d] - b[d]);
        m = (m < t) ? t : m;
      }
      return m;
    }
    case ORACLE_METRIC_WCHEBYSHEV: {
      float m = 0.0f;
      for (int d = 0; d < N; ++d) {
        float t = w[d] * fabsf(a[d] - b[d]);
        m = (m < t) ? t : m;
      }
      return m;
    }
  }
  return NAN;
}

/* core/detail/ConvolutionalKernel.hpp:16-65. */
float oracle_kernel(const oracle_params* p, float dist, int32_t i, int32_t j) {
  if (i == j) return 1.0f;
  const float* k = p->kernel_par;
  switch (p->kernel_type) {
    case ORACLE_KERNEL_FLAT:
      return k[0];
    case ORACLE_KERNEL_EXP:
      return k[1] * expf(-k[0] * dist);
    case ORACLE_KERNEL_GAUSS: {
      float e = -(dist - k[0]) * (dist - k[0]) / (2.0f * k[1] * k[1]);
      return k[2] * expf(e);
    }
  }
  return NAN;
}

/* Host association map fill (data_structures/AssociationMap.hpp:53-74); the serial
 * KernelFillAssociator (data_structures/detail/AssociationMap.hpp:50-67) yields the
 * same index-ascending order inside each key. Keys outside [0, nkeys) are skipped. */
static void csr_fill(const int32_t* keys, int32_t n, int32_t nkeys, int32_t* offsets, int32_t* values) {
  memset(offsets, 0, sizeof(int32_t) * ((size_t)nkeys + 1));
  for (int32_t i = 0; i < n; ++i)
    if (keys[i] >= 0 && keys[i] < nkeys) offsets[keys[i] + 1]++;
  for (int32_t k = 0; k < nkeys; ++k) offsets[k + 1] += offsets[k];
  int32_t* cur = (int32_t*)malloc(sizeof(int32_t) * ((size_t)nkeys + 1));
  memcpy(cur, offsets, sizeof(int32_t) * ((size_t)nkeys + 1));
  for (int32_t i = 0; i < n; ++i)
    if (keys[i] >= 0 && keys[i] < nkeys) values[cur[keys[i]]++] = i;
  free(cur);
}

static void load_point(int N, int32_t n, const float* coords, int32_t i, float* out) {
  for (int d = 0; d < N; ++d) out[d] = coords[(size_t)d * n + i];
}

typedef struct {
  const oracle_params* p;
  const grid_t* g;
  int32_t n;
  const float* coords;
  const float* weight;
  const int32_t* off;
  const int32_t* idx;
} ctx_t;

/* Odometer over the search box, dim 0 outermost (ClusteringKernels.hpp:18-64). */
#define BOX_LOOP_BEGIN(g, lo, hi)                                  \
  {                                                                \
    int32_t v_[ORACLE_MAX_DIM];                                    \
    int empty_ = 0;                                                \
    for (int d_ = 0; d_ < (g)->ndim; ++d_) {                       \
      v_[d_] = (lo)[d_];                                           \
      if ((lo)[d_] > (hi)[d_]) empty_ = 1;                         \
    }                                                              \
    while (!empty_) {                                              \
      const int64_t tile_ = global_bin_by_bin((g), v_);

#define BOX_LOOP_END(g, lo, hi)                                    \
  int d_ = (g)->ndim - 1;                                          \
  for (; d_ >= 0; --d_) {                                          \
    if (v_[d_] < (hi)[d_]) {                                       \
      ++v_[d_];                                                    \
      break;                                                       \
    }                                                              \
    v_[d_] = (lo)[d_];                                             \
  }                                                                \
  if (d_ < 0) break;                                               \
  }                                                                \
  }

/* KernelCalculateLocalDensity (ClusteringKernels.hpp:66-107): rho_i accumulated in
 * candidate order, term = (float)(d <= dc) * k * w_j.  Terms with d > dc are +-0 and
 * leave the sum unchanged unless k * w_j is not finite, in which case the literal
 * product is added so that NaN propagates as in the reference. */
static float density_point(const ctx_t* c, int32_t i, int64_t* ncand) {
  const oracle_params* p = c->p;
  const int N = p->ndim;
  float xi[ORACLE_MAX_DIM], xj[ORACLE_MAX_DIM];
  int32_t lo[ORACLE_MAX_DIM], hi[ORACLE_MAX_DIM];
  load_point(N, c->n, c->coords, i, xi);
  search_box(c->g, xi, p->dc, lo, hi);
  float rho = 0.0f;
  int64_t cnt = 0;
  BOX_LOOP_BEGIN(c->g, lo, hi)
  for (int32_t q = c->off[tile_]; q < c->off[tile_ + 1]; ++q) {
    const int32_t j = c->idx[q];
    load_point(N, c->n, c->coords, j, xj);
    const float dist = oracle_metric(p, xi, xj);
    ++cnt;
    if (dist <= p->dc) {
      const float k = oracle_kernel(p, dist, i, j);
      rho += 1.0f * k * c->weight[j];
    } else if (!isfinite(c->weight[j]) || (isnan(dist) && p->kernel_type != ORACLE_KERNEL_FLAT)) {
      const float k = oracle_kernel(p, dist, i, j);
      rho += 0.0f * k * c->weight[j];
    }
  }
  BOX_LOOP_END(c->g, lo, hi)
  *ncand += cnt;
  return rho;
}

/* KernelCalculateNearestHigher (ClusteringKernels.hpp:109-212). */
static int32_t nh_point(const ctx_t* c, const float* rho, int32_t i, float* delta_out, int64_t* ncand,
                        int64_t* nties) {
  const oracle_params* p = c->p;
  const int N = p->ndim;
  float xi[ORACLE_MAX_DIM], xj[ORACLE_MAX_DIM];
  int32_t lo[ORACLE_MAX_DIM], hi[ORACLE_MAX_DIM];
  load_point(N, c->n, c->coords, i, xi);
  search_box(c->g, xi, p->dm, lo, hi);
  float delta = FLT_MAX;
  int32_t nh = -1;
  const float rho_i = rho[i];
  int64_t cnt = 0, ties = 0;
  BOX_LOOP_BEGIN(c->g, lo, hi)
  for (int32_t q = c->off[tile_]; q < c->off[tile_ + 1]; ++q) {
    const int32_t j = c->idx[q];
    const float rho_j = rho[j];
    int higher = (rho_j > rho_i);
    higher = higher || ((rho_j == rho_i) && (rho_j > 0.0f) && (j > i));
    load_point(N, c->n, c->coords, j, xj);
    const float dist = oracle_metric(p, xi, xj);
    ++cnt;
    if (higher && dist <= p->dm) {
      if (dist < delta) {
        delta = dist;
        nh = j;
      } else if (dist == delta) {
        ++ties;
        if (p->tiebreak == ORACLE_TIE_RHO_INDEX && nh >= 0) {
          const float rho_nh = rho[nh];
          if (rho_j > rho_nh || (rho_j == rho_nh && j < nh)) nh = j;
        }
      }
    }
  }
  BOX_LOOP_END(c->g, lo, hi)
  *ncand += cnt;
  *nties += ties;
  if (delta_out) *delta_out = delta;
  return nh;
}

static int build_tiles(const oracle_params* p, int32_t n, const float* coords, grid_t* g,
                       int32_t** off, int32_t** idx) {
  grid_build(p, n, coords, g);
  int32_t* bins = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  *off = (int32_t*)malloc(sizeof(int32_t) * ((size_t)g->ntiles + 1));
  *idx = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  if (!bins || !*off || !*idx) return -1;
  for (int32_t i = 0; i < n; ++i) bins[i] = (int32_t)global_bin(g, n, coords, i);
  csr_fill(bins, n, g->ntiles, *off, *idx);
  free(bins);
  return 0;
}

static int check_params(const oracle_params* p, int32_t n) {
  if (n <= 0 || p->ndim < 1 || p->ndim > ORACLE_MAX_DIM) return -1;
  if (p->dc <= 0.f || p->rhoc < 0.f || p->dm <= 0.f || p->seed_dc <= 0.f || p->ppbin <= 0) return -1;
  return 0;
}

int oracle_tiles(const oracle_params* p, int32_t n, const float* coords, oracle_grid* grid,
                 int32_t* offsets, int32_t* indexes) {
  if (check_params(p, n)) return -1;
  grid_t g;
  int32_t *off = NULL, *idx = NULL;
  if (build_tiles(p, n, coords, &g, &off, &idx)) return -2;
  grid->nperdim = g.nperdim;
  grid->ntiles = g.ntiles;
  for (int d = 0; d < p->ndim; ++d) {
    grid->minmax[2 * d] = g.mn[d];
    grid->minmax[2 * d + 1] = g.mx[d];
    grid->tilesize[d] = g.size[d];
  }
  if (offsets) memcpy(offsets, off, sizeof(int32_t) * ((size_t)g.ntiles + 1));
  if (indexes) memcpy(indexes, idx, sizeof(int32_t) * (size_t)n);
  free(off);
  free(idx);
  return 0;
}

/* Nearest-higher stage alone, on densities the caller supplies (KernelCalculateNearestHigher,
 * ClusteringKernels.hpp:109-212, over the tiles of setup_tiles).  Lets a test check the
 * candidate order and tie-break of an implementation whose densities differ from this
 * restatement's in the last bits. */
int oracle_nearest_higher(const oracle_params* p, int32_t n, const float* coords, const float* rho,
                          int32_t* nearest_higher, float* delta, int64_t* distance_ties) {
  if (check_params(p, n)) return -1;
  grid_t g;
  int32_t *off = NULL, *idx = NULL;
  if (build_tiles(p, n, coords, &g, &off, &idx)) return -2;
  ctx_t c = {p, &g, n, coords, NULL, off, idx};
  int64_t cand = 0, ties = 0;
  const int nt = p->nthreads > 1 ? p->nthreads : 1;
  (void)nt;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(nt) reduction(+ : cand, ties)
#endif
  for (int32_t i = 0; i < n; ++i) {
    float dl;
    nearest_higher[i] = nh_point(&c, rho, i, &dl, &cand, &ties);
    if (delta) delta[i] = dl;
  }
  if (distance_ties) *distance_ties = ties;
  free(off);
  free(idx);
  return 0;
}

int oracle_run(const oracle_params* p, int32_t n, const float* coords, const float* weight,
               oracle_out* out) {
  if (check_params(p, n)) return -1;
  const int N = p->ndim;
  grid_t g;
  int32_t *off = NULL, *idx = NULL;
  if (build_tiles(p, n, coords, &g, &off, &idx)) return -2;
  ctx_t c = {p, &g, n, coords, weight, off, idx};

  float* rho = out->rho;
  int32_t* nh = out->nearest_higher;
  int64_t cand_rho = 0, cand_nh = 0, ties = 0;
  int nt = p->nthreads > 1 ? p->nthreads : 1;
  (void)nt;

  /* stage 2: local density */
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(nt) reduction(+ : cand_rho)
#endif
  for (int32_t i = 0; i < n; ++i) rho[i] = density_point(&c, i, &cand_rho);

  /* stage 3: nearest higher + seed candidates (ClusteringKernels.hpp:306-330) */
  int64_t seed_candidates = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(nt) reduction(+ : cand_nh, ties, seed_candidates)
#endif
  for (int32_t i = 0; i < n; ++i) {
    float dl;
    nh[i] = nh_point(&c, rho, i, &dl, &cand_nh, &ties);
    if (out->delta) out->delta[i] = dl;
    if (nh[i] == -1) ++seed_candidates;
  }

  /* stage 4: seeds (KernelFindClusters, ClusteringKernels.hpp:214-244; SeedArray push_back
   * SeedArray.hpp:33-41; capacity from setup_seeds SetupSeeds.hpp:10-20).  The serial
   * backend visits points in index order, so the seed list is index-ascending. */
  int64_t cap = p->seed_capacity < 0 ? (int64_t)n
                                     : (p->seed_capacity > seed_candidates ? p->seed_capacity
                                                                           : seed_candidates);
  int32_t* seeds = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  int64_t nseeds_list = 0, nseeds = 0, dropped = 0;
  float sentinel[ORACLE_MAX_DIM];
  for (int d = 0; d < N; ++d) sentinel[d] = FLT_MAX; /* PointsCommon.hpp:75-81 operator[](-1) */
  for (int32_t i = 0; i < n; ++i) {
    out->cluster_index[i] = -1;
    float xi[ORACLE_MAX_DIM], xn[ORACLE_MAX_DIM];
    load_point(N, n, coords, i, xi);
    if (nh[i] >= 0)
      load_point(N, n, coords, nh[i], xn);
    else
      memcpy(xn, sentinel, sizeof(float) * N);
    const float dist = oracle_metric(p, xi, xn);
    const int is_seed = (dist > p->seed_dc) && (rho[i] >= p->rhoc);
    if (is_seed) {
      out->is_seed[i] = 1;
      nh[i] = -1;
      ++nseeds;
      if (nseeds_list < cap)
        seeds[nseeds_list++] = i;
      else
        ++dropped;
    } else {
      out->is_seed[i] = 0;
    }
  }

  /* stage 5: followers CSR keyed by nearest_higher (Followers.hpp:27-30) and the
   * per-seed DFS (KernelAssignClusters, ClusteringKernels.hpp:246-281). */
  int32_t* foff = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
  int32_t* fidx = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  csr_fill(nh, n, n, foff, fidx);
  int32_t* stack = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
  int64_t max_stack = 0;
  for (int64_t c_ = 0; c_ < nseeds_list; ++c_) {
    int64_t sp = 0;
    const int32_t s = seeds[c_];
    out->cluster_index[s] = (int32_t)c_;
    stack[sp++] = s;
    if (sp > max_stack) max_stack = sp;
    while (sp > 0) {
      const int32_t e = stack[--sp];
      const int32_t lab = out->cluster_index[e];
      for (int32_t q = foff[e]; q < foff[e + 1]; ++q) {
        const int32_t f = fidx[q];
        out->cluster_index[f] = lab;
        stack[sp++] = f;
        if (sp > max_stack) max_stack = sp;
      }
    }
  }

  out->n_seeds = nseeds;
  out->n_clusters = nseeds_list;
  out->dropped_seeds = dropped;
  out->seed_capacity_used = p->seed_capacity < 0 ? -1 : cap;
  out->max_dfs_stack = max_stack;
  out->candidates_rho = cand_rho;
  out->candidates_nh = cand_nh;
  out->nh_distance_ties = ties;
  free(seeds);
  free(foff);
  free(fidx);
  free(stack);
  free(off);
  free(idx);
  return 0;
}

/* FP64 metric on float inputs, same operation order as oracle_metric. */
static double metric_f64(const oracle_params* p, const float* a, const float* b) {
  const int N = p->ndim;
  const float* w = p->metric_par;
  double acc = 0.0;
  switch (p->metric_type) {
    case ORACLE_METRIC_EUCLID:
      for (int d = N - 1; d >= 0; --d) acc = ((double)a[d] - b[d]) * ((double)a[d] - b[d]) + acc;
      return sqrt(acc);
    case ORACLE_METRIC_WEUCLID:
      for (int d = N - 1; d >= 0; --d) acc = (double)w[d] * ((double)a[d] - b[d]) * ((double)a[d] - b[d]) + acc;
      return sqrt(acc);
    case ORACLE_METRIC_PERIODIC:
      for (int d = N - 1; d >= 0; --d) {
        double diff = fabs((double)a[d] - b[d]);
        double alt = (double)w[d] - diff;
        double pd = alt < diff ? alt : diff;
        acc = pd * pd + acc;
      }
      return sqrt(acc);
    case ORACLE_METRIC_MANHATTAN:
      for (int d = N - 1; d >= 0; --d) acc = fabs((double)a[d] - b[d]) + acc;
      return acc;
    case ORACLE_METRIC_CHEBYSHEV:
      for (int d = 0; d < N; ++d) {
        double t = fabs((double)a[d] - b[d]);
        acc = acc < t ? t : acc;
      }
      return acc;
    case ORACLE_METRIC_WCHEBYSHEV:
      for (int d = 0; d < N; ++d) {
        double t = (double)w[d] * fabs((double)a[d] - b[d]);
        acc = acc < t ? t : acc;
      }
      return acc;
  }
  return NAN;
}

static double kernel_f64(const oracle_params* p, double dist, int32_t i, int32_t j) {
  if (i == j) return 1.0;
  const float* k = p->kernel_par;
  switch (p->kernel_type) {
    case ORACLE_KERNEL_FLAT:
      return k[0];
    case ORACLE_KERNEL_EXP:
      return (double)k[1] * exp(-(double)k[0] * dist);
    case ORACLE_KERNEL_GAUSS:
      return (double)k[2] * exp(-(dist - k[0]) * (dist - k[0]) / (2.0 * k[1] * k[1]));
  }
  return NAN;
}

int oracle_rho_f64(const oracle_params* p, int32_t n, const float* coords, const float* weight,
                   double* rho64, uint8_t* near_dc, double rel_tol) {
  if (check_params(p, n)) return -1;
  grid_t g;
  int32_t *off = NULL, *idx = NULL;
  if (build_tiles(p, n, coords, &g, &off, &idx)) return -2;
  const int N = p->ndim;
  int nt = p->nthreads > 1 ? p->nthreads : 1;
  (void)nt;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(nt)
#endif
  for (int32_t i = 0; i < n; ++i) {
    float xi[ORACLE_MAX_DIM], xj[ORACLE_MAX_DIM];
    int32_t lo[ORACLE_MAX_DIM], hi[ORACLE_MAX_DIM];
    load_point(N, n, coords, i, xi);
    search_box(&g, xi, p->dc, lo, hi);
    double rho = 0.0;
    int near = 0;
    const double dc = (double)p->dc;
    BOX_LOOP_BEGIN(&g, lo, hi)
    for (int32_t q = off[tile_]; q < off[tile_ + 1]; ++q) {
      const int32_t j = idx[q];
      load_point(N, n, coords, j, xj);
      const double dist = metric_f64(p, xi, xj);
      if (dist <= dc) rho += kernel_f64(p, dist, i, j) * (double)weight[j];
      if (fabs(dist - dc) <= rel_tol * dc) near = 1;
    }
    BOX_LOOP_END(&g, lo, hi)
    rho64[i] = rho;
    if (near_dc) near_dc[i] = (uint8_t)near;
  }
  free(off);
  free(idx);
  return 0;
}

/* Silhouette score (include/CLUEstering/utils/detail/scores.hpp:17-99): per point of a cluster
 * with at least two points, a = sum of distances to the other points of its cluster / (size-1),
 * b = min over the other clusters (ascending label) of sum of distances / size, both sums over
 * the cluster's points in ascending index order; s = (b - a) / max(a, b).  Distances:
 * d = 0; d += (l - r) * (l - r) per dimension in order; sqrt(d), separately rounded.  per_point
 * gets NAN for points not scored; *mean the FP32 sum of the scores in index order / count. */
int oracle_silhouette(int32_t ndim, int32_t n, const float* coords, const int32_t* labels, float* per_point,
                      float* mean) {
  if (n <= 0 || ndim < 1 || ndim > ORACLE_MAX_DIM) return -1;
  int32_t k = 0;
  for (int32_t i = 0; i < n; ++i)
    if (labels[i] + 1 > k) k = labels[i] + 1;
  int32_t* off = (int32_t*)calloc((size_t)k + 1, sizeof(int32_t));
  int32_t* idx = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  int32_t* fill = (int32_t*)calloc((size_t)k + 1, sizeof(int32_t));
  if (!off || !idx || !fill) return -2;
  for (int32_t i = 0; i < n; ++i)
    if (labels[i] >= 0) ++off[labels[i] + 1];
  for (int32_t c = 0; c < k; ++c) off[c + 1] += off[c];
  for (int32_t i = 0; i < n; ++i)
    if (labels[i] >= 0) idx[off[labels[i]] + fill[labels[i]]++] = i; /* ascending index */
  float acc = 0.0f;
  int64_t cnt = 0;
  for (int32_t i = 0; i < n; ++i) {
    const int32_t own = labels[i];
    if (own < 0 || off[own + 1] - off[own] < 2) {
      per_point[i] = NAN;
      continue;
    }
    float a = 0.0f, b = FLT_MAX;
    for (int32_t c = 0; c < k; ++c) {
      float sum = 0.0f;
      for (int32_t q = off[c]; q < off[c + 1]; ++q) {
        const int32_t j = idx[q];
        if (c == own && j == i) continue;
        float d = 0.0f;
        for (int dd = 0; dd < ndim; ++dd) {
          const float t = coords[(size_t)dd * n + i] - coords[(size_t)dd * n + j];
          d = d + t * t;
        }
        sum = sum + sqrtf(d);
      }
      const int32_t sz = off[c + 1] - off[c];
      if (c == own) {
        a = sum / (float)(sz - 1);
      } else if (sz > 0) {
        const float m = sum / (float)sz;
        b = m < b ? m : b;
      }
    }
    const float sc = (b - a) / (a < b ? b : a); /* std::max(a, b) */
    per_point[i] = sc;
    acc += sc;
    ++cnt;
  }
  if (mean) *mean = acc / (float)cnt;
  free(off);
  free(idx);
  free(fill);
  return 0;
}

/* ---- per-event runs (a batch of independent events, OpenMP over events) ----------------
 * The reference clusters one event per make_clusters call; a caller with many events loops
 * over them.  These helpers run that loop with one event per thread (each event serial, as
 * the serial backend computes it), which is the fastest use of the host cores for a batch of
 * small events.  Event e owns points [offsets[e], offsets[e+1]) of the SoA arrays (stride ld). */

static float* gather_event(const float* coords, int32_t ld, int N, int32_t b, int32_t ne) {
  float* c = (float*)malloc(sizeof(float) * (size_t)N * (size_t)(ne > 0 ? ne : 1));
  if (!c) return NULL;
  for (int d = 0; d < N; ++d) memcpy(c + (size_t)d * ne, coords + (size_t)d * ld + b, sizeof(float) * (size_t)ne);
  return c;
}

int oracle_run_events(const oracle_params* p, int32_t n_events, const int32_t* offsets, int32_t ld,
                      const float* coords, const float* weight, oracle_out* out, int64_t* ev_n_clusters) {
  const int nt = p->nthreads > 1 ? p->nthreads : 1;
  (void)nt;
  int64_t n_seeds = 0, n_clusters = 0, dropped = 0, cand_rho = 0, cand_nh = 0, ties = 0, max_stack = 0;
  int err = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt) \
    reduction(+ : n_seeds, n_clusters, dropped, cand_rho, cand_nh, ties) reduction(max : max_stack) reduction(| : err)
#endif
  for (int32_t e = 0; e < n_events; ++e) {
    const int32_t b = offsets[e], ne = offsets[e + 1] - offsets[e];
    if (ne <= 0) continue;
    oracle_params pe = *p;
    pe.nthreads = 1;
    float* c = gather_event(coords, ld, p->ndim, b, ne);
    if (!c) {
      err |= 1;
      continue;
    }
    oracle_out oe;
    memset(&oe, 0, sizeof(oe));
    oe.cluster_index = out->cluster_index + b;
    oe.is_seed = out->is_seed + b;
    oe.rho = out->rho + b;
    oe.nearest_higher = out->nearest_higher + b;
    oe.delta = out->delta ? out->delta + b : NULL;
    if (oracle_run(&pe, ne, c, weight + b, &oe) != 0) err |= 1;
    free(c);
    for (int32_t i = 0; i < ne; ++i)
      if (oe.nearest_higher[i] >= 0) oe.nearest_higher[i] += b; /* batch-global index */
    n_seeds += oe.n_seeds;
    n_clusters += oe.n_clusters;
    dropped += oe.dropped_seeds;
    cand_rho += oe.candidates_rho;
    cand_nh += oe.candidates_nh;
    ties += oe.nh_distance_ties;
    if (oe.max_dfs_stack > max_stack) max_stack = oe.max_dfs_stack;
    if (ev_n_clusters) ev_n_clusters[e] = oe.n_clusters;
  }
  out->n_seeds = n_seeds;
  out->n_clusters = n_clusters;
  out->dropped_seeds = dropped;
  out->seed_capacity_used = -1;
  out->max_dfs_stack = max_stack;
  out->candidates_rho = cand_rho;
  out->candidates_nh = cand_nh;
  out->nh_distance_ties = ties;
  return err ? -2 : 0;
}

/* ---- near-threshold classification ------------------------------------------------------
 * Two density vectors of the same points -- rho_a from this restatement, rho_b from another
 * implementation that sums the same terms in another order or with another exp -- agree to a
 * few ulp.  The nearest-higher and seed stages (ClusteringKernels.hpp:129-143, 232-233) turn
 * them into discrete decisions, and a decision can differ only where it compares values that
 * are that close.  oracle_near_flags marks those decision points per point:
 *   ORACLE_NEAR_RHOC     rho_a and rho_b lie on different sides of rhoc, or |rho_a - rhoc| <= tol*rhoc
 *   ORACLE_NEAR_FLIP     some candidate j of i's dm search box with d(i, j) <= dm is higher than i
 *                        under one vector and not under the other (the rule of
 *                        ClusteringKernels.hpp:129-131)
 *   ORACLE_NEAR_TIE      some such candidate has |rho_a[j] - rho_a[i]| <= tol * max(|rho_a[i]|, |rho_a[j]|)
 *   ORACLE_NEAR_SEED_DC  |delta_a - seed_dc| <= tol * seed_dc
 *   ORACLE_NEAR_DM       |delta_a - dm| <= tol * dm
 * max_flip_rel (may be NULL) receives the largest |rho_a[j] - rho_a[i]| / max(|rho_a[i]|, |rho_a[j]|)
 * over the flipped pairs: small when every flip is a genuine near-tie. */

static inline int is_higher(float rho_i, float rho_j, int32_t i, int32_t j) {
  return (rho_j > rho_i) || ((rho_j == rho_i) && (rho_j > 0.0f) && (j > i));
}

int oracle_near_flags(const oracle_params* p, int32_t n, const float* coords, const float* rho_a,
                      const float* rho_b, const float* delta_a, double tol, uint8_t* flags,
                      double* max_flip_rel) {
  if (check_params(p, n)) return -1;
  grid_t g;
  int32_t *off = NULL, *idx = NULL;
  if (build_tiles(p, n, coords, &g, &off, &idx)) return -2;
  const int N = p->ndim;
  const int nt = p->nthreads > 1 ? p->nthreads : 1;
  (void)nt;
  double worst = 0.0;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 256) num_threads(nt) reduction(max : worst)
#endif
  for (int32_t i = 0; i < n; ++i) {
    float xi[ORACLE_MAX_DIM], xj[ORACLE_MAX_DIM];
    int32_t lo[ORACLE_MAX_DIM], hi[ORACLE_MAX_DIM];
    uint8_t f = 0;
    const float ra = rho_a[i], rb = rho_b[i];
    if ((ra >= p->rhoc) != (rb >= p->rhoc) || fabs((double)ra - p->rhoc) <= tol * p->rhoc) f |= ORACLE_NEAR_RHOC;
    if (delta_a) {
      if (fabs((double)delta_a[i] - p->seed_dc) <= tol * p->seed_dc) f |= ORACLE_NEAR_SEED_DC;
      if (fabs((double)delta_a[i] - p->dm) <= tol * p->dm) f |= ORACLE_NEAR_DM;
    }
    load_point(N, n, coords, i, xi);
    search_box(&g, xi, p->dm, lo, hi);
    BOX_LOOP_BEGIN(&g, lo, hi)
    for (int32_t q = off[tile_]; q < off[tile_ + 1]; ++q) {
      const int32_t j = idx[q];
      if (j == i) continue;
      load_point(N, n, coords, j, xj);
      if (!(oracle_metric(p, xi, xj) <= p->dm)) continue;
      const double m = fmax(fabs((double)ra), fabs((double)rho_a[j]));
      const double gap = fabs((double)rho_a[j] - (double)ra);
      if (gap <= tol * m) f |= ORACLE_NEAR_TIE;
      if (is_higher(ra, rho_a[j], i, j) != is_higher(rb, rho_b[j], i, j)) {
        f |= ORACLE_NEAR_FLIP;
        const double rel = m > 0.0 ? gap / m : 0.0;
        if (rel > worst) worst = rel;
      }
    }
    BOX_LOOP_END(&g, lo, hi)
    flags[i] = f;
  }
  if (max_flip_rel) *max_flip_rel = worst;
  free(off);
  free(idx);
  return 0;
}

/* Per-event forms of the FP64 density, the nearest-higher stage on given densities and the
 * near-threshold flags (nearest highers returned batch-global). */
int oracle_events_aux(int kind, const oracle_params* p, int32_t n_events, const int32_t* offsets, int32_t ld,
                      const float* coords, const float* weight, const float* rho_a, const float* rho_b,
                      const float* delta_a, double tol, double* rho64, uint8_t* flags, int32_t* nearest_higher,
                      float* delta, double* max_flip_rel) {
  const int nt = p->nthreads > 1 ? p->nthreads : 1;
  (void)nt;
  int err = 0;
  double worst = 0.0;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt) reduction(| : err) reduction(max : worst)
#endif
  for (int32_t e = 0; e < n_events; ++e) {
    const int32_t b = offsets[e], ne = offsets[e + 1] - offsets[e];
    if (ne <= 0) continue;
    oracle_params pe = *p;
    pe.nthreads = 1;
    float* c = gather_event(coords, ld, p->ndim, b, ne);
    if (!c) {
      err |= 1;
      continue;
    }
    int rc = 0;
    if (kind == ORACLE_AUX_RHO_F64) {
      rc = oracle_rho_f64(&pe, ne, c, weight + b, rho64 + b, flags ? flags + b : NULL, tol);
    } else if (kind == ORACLE_AUX_NEAREST_HIGHER) {
      int64_t t = 0;
      rc = oracle_nearest_higher(&pe, ne, c, rho_a + b, nearest_higher + b, delta ? delta + b : NULL, &t);
      for (int32_t i = 0; i < ne && rc == 0; ++i)
        if (nearest_higher[b + i] >= 0) nearest_higher[b + i] += b;
    } else {
      double w = 0.0;
      rc = oracle_near_flags(&pe, ne, c, rho_a + b, rho_b + b, delta_a ? delta_a + b : NULL, tol, flags + b, &w);
      if (w > worst) worst = w;
    }
    if (rc != 0) err |= 1;
    free(c);
  }
  if (max_flip_rel) *max_flip_rel = worst;
  return err ? -2 : 0;
}
