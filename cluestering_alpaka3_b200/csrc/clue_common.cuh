// clue_common.cuh -- definitions shared by host and device code of libclue_b200.
//
// The binning, metric and kernel arithmetic restates the reference bit for bit:
// every float operation is a separately rounded IEEE op (explicit __f*_rn
// intrinsics on the device, -ffp-contract=off on the host), in the order the
// reference's headers write it.  References are to the reference project's
// include/CLUEstering/ tree.
#pragma once

#include <cstdint>
#include <cfloat>
#include <cmath>

#include "../../include/clue_b200.h"

#if defined(__CUDACC__)
#define CLUE_HD __host__ __device__ __forceinline__
#else
#define CLUE_HD inline
#endif

namespace clue_b200 {

constexpr int kMaxDim = CLUE_MAX_DIM;

// Number of float4 words of one tile-sorted point record: N coordinates followed by
// one payload float (the weight in the density record, rho in the nearest-higher
// record), payload in the last float of the last word.
template <int N>
struct Rec {
  static constexpr int kWords = (N + 1 + 3) / 4;
  static constexpr int kPayload = 4 * kWords - 1;
};

// Host-computed launch parameters, passed by value to every kernel.
struct KParams {
  float dc, dm, seed_dc, rhoc;
  float t_dc, t_dm;  // thresholds on the metric's pre-root value (see threshold_for)
  int32_t kernel_type;
  float kpar[3];
  float mpar[kMaxDim];
  uint8_t wrapped[kMaxDim];
  int32_t tiebreak;
  int64_t seed_capacity;
  int32_t n;          // points over all events
  int32_t n_events;   // events (1 for a plain make_clusters call)
  int32_t ntiles;     // tiles over all events
  // grid of the single event of a plain call (written to the event table by k_init)
  int32_t nperdim0;
  int32_t stride0[kMaxDim];
  int32_t lb_ok;  // metric parameters allow box lower bounds (no negative weights)
  int32_t flags;  // clue_params.flags
  float ginv;     // 1 / (2 std^2) of the Gaussian kernel (spatial-order density)
};

// Bounding box of 32 consecutive tile-sorted records: lo[N], hi[N], max payload.
template <int N>
struct Blk {
  static constexpr int kWords = (2 * N + 1 + 3) / 4;
};

// Tile grid of one event.  The host fills nperdim, ntiles, strides and the point / tile
// bases (the reference computes the grid shape on the host, SetupTiles.hpp:23-26); the
// device fills the bounding box and tile sizes.
struct EvGrid {
  uint32_t enc_min[kMaxDim];
  uint32_t enc_max[kMaxDim];
  float mn[kMaxDim];
  float mx[kMaxDim];
  float size[kMaxDim];
  int32_t stride[kMaxDim];
  int32_t nperdim;
  int32_t ntiles;
  int32_t tile_base;        // first global tile of the event
  int32_t pt_base;          // first point of the event
  int32_t pt_count;
  uint32_t seed_candidates; // points of the event without nearest higher
  uint32_t wmax_bits;       // largest |weight| of the event (float bits; non-negative floats order as integers)
};

// Levels of the breadth-first label form (clue_tuning.labels_bfs) enqueued without host
// synchronisation; deeper forests continue by pointer jumping from the host.
constexpr int kBfsLevels = 64;

// Device-side status block (counters and flags), read back once per call.
struct DevStatus {
  uint32_t nonfinite;
  uint32_t seed_candidates;  // points with no nearest higher (before the seed reset)
  uint32_t n_seeds;
  uint32_t unresolved[64];   // label rounds that left an unresolved parent chain
  uint32_t label_rounds;
  uint32_t stage_timeout;  // a bulk-copy wait in a staged sweep gave up
  uint32_t n_clusters;     // seeds kept in the seed lists, summed over events
  // near-threshold decisions (relative tolerance kNearTol, counted by k_seeds and k_near_ties)
  uint32_t near_rhoc;      // |rho - rhoc| <= tol * rhoc
  uint32_t near_seed_dc;   // nearest higher found and |delta - seed_dc| <= tol * seed_dc
  uint32_t near_dm;        // nearest higher found and |delta - dm| <= tol * dm
  uint32_t nh_near_ties;   // nearest-higher choice compares densities within tol (CLUE_FLAG_NEAR_TIES)
  uint32_t bfs_count[kBfsLevels + 1];  // frontier sizes of the breadth-first label form
  uint32_t check_site;   // device bounds checks (CLUE_DEVICE_CHECKS builds): first failing site
  int32_t check_index;   // and the index it rejected
};

// Relative tolerance of the near-threshold counts: the tolerance rho is held to against FP64.
constexpr float kNearTol = 1e-5f;

// ---- device bounds checks -----------------------------------------------------
// A build with -DCLUE_DEVICE_CHECKS=1 tests every index that the pipeline reads from its own
// data (permutations, parents, nearest highers, tile numbers) before it addresses memory with
// it.  A bad index records the first failing site and the index in the status block, and the
// access is skipped: the kernel neither traps nor reads or writes out of bounds, and the host
// turns the record into an error after the run.  Without the flag the test compiles away.
#ifndef CLUE_DEVICE_CHECKS
#define CLUE_DEVICE_CHECKS 0
#endif
enum : uint32_t {
  kChkGatherPerm = 1,    // k_gather: the tile sort's permutation
  kChkSeedsPerm = 2,     // k_seeds: the permutation
  kChkJumpParent = 3,    // k_jump: a parent pointer
  kChkFinalizeRoot = 4,  // k_finalize: a label root and its original index
  kChkFinalizeNh = 5,    // k_finalize: a nearest higher
  kChkDensityTile = 6,   // k_density_sym: a tile of the search box
  kChkDensityMirror = 7, // k_density_sym: the mirrored term's point
};
inline const char* check_site_name(uint32_t site) {
  switch (site) {
    case kChkGatherPerm: return "record gather (tile-sort permutation)";
    case kChkSeedsPerm: return "seed flags (permutation)";
    case kChkJumpParent: return "pointer jumping (parent)";
    case kChkFinalizeRoot: return "labels (root)";
    case kChkFinalizeNh: return "outputs (nearest higher)";
    case kChkDensityTile: return "symmetric density (search-box tile)";
    case kChkDensityMirror: return "symmetric density (mirrored point)";
  }
  return "unknown";
}
#if defined(__CUDACC__)
__device__ __forceinline__ bool dcheck_bad(DevStatus* st, long long idx, long long n, uint32_t site) {
#if CLUE_DEVICE_CHECKS
  if (idx >= 0 && idx < n) return false;
  if (atomicCAS(&st->check_site, 0u, site) == 0u) st->check_index = (int32_t)idx;
  return true;
#else
  (void)st, (void)idx, (void)n, (void)site;
  return false;
#endif
}
#endif

// float -> int32 truncation with x86 cvttss2si semantics (NaN and out-of-range give
// INT32_MIN), which is what the reference's static_cast<int>(float) does on its
// serial CPU backend (data_structures/internal/TilesView.hpp:41-43,95).
CLUE_HD int32_t cvt_i32(float f) {
  if (!(f > -2147483904.0f && f < 2147483648.0f)) return INT32_MIN;
  return (int32_t)f;
}

// Monotone float <-> uint32 encoding for atomic min/max.
CLUE_HD uint32_t enc_float(float f) {
#if defined(__CUDA_ARCH__)
  uint32_t u = __float_as_uint(f);
#else
  uint32_t u;
  __builtin_memcpy(&u, &f, 4);
#endif
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
CLUE_HD float dec_float(uint32_t e) {
  uint32_t u = (e & 0x80000000u) ? (e & 0x7fffffffu) : ~e;
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  __builtin_memcpy(&f, &u, 4);
  return f;
#endif
}

// Separately rounded float ops (never contracted into FMA).
#if defined(__CUDA_ARCH__)
CLUE_HD float fadd(float a, float b) { return __fadd_rn(a, b); }
CLUE_HD float fsub(float a, float b) { return __fsub_rn(a, b); }
CLUE_HD float fmul(float a, float b) { return __fmul_rn(a, b); }
CLUE_HD float fdiv(float a, float b) { return __fdiv_rn(a, b); }
CLUE_HD float fsqrt(float a) { return __fsqrt_rn(a); }
#else
CLUE_HD float fadd(float a, float b) { return a + b; }
CLUE_HD float fsub(float a, float b) { return a - b; }
CLUE_HD float fmul(float a, float b) { return a * b; }
CLUE_HD float fdiv(float a, float b) { return a / b; }
CLUE_HD float fsqrt(float a) { return sqrtf(a); }
#endif

// ---- tile grid (data_structures/internal/TilesView.hpp) ---------------------

// normalizeCoordinate, TilesView.hpp:93-101.
CLUE_HD float normalize_coord(float coord, float mn, float mx) {
  const float range = fsub(mx, mn);
  float rem = fsub(coord, fmul((float)cvt_i32(fdiv(coord, range)), range));
  if (rem >= mx)
    rem = fsub(rem, range);
  else if (rem < mn)
    rem = fadd(rem, range);
  return rem;
}

// getBin, TilesView.hpp:37-51.
CLUE_HD int32_t get_bin(float coord, float mn, float mx, float size, bool wrapped, int32_t nperdim) {
  int32_t b;
  if (wrapped)
    b = cvt_i32(fdiv(fsub(normalize_coord(coord, mn, mx), mn), size));
  else
    b = cvt_i32(fdiv(fsub(coord, mn), size));
  b = b < nperdim - 1 ? b : nperdim - 1;
  b = b > 0 ? b : 0;
  return b;
}

// ---- distance metrics (core/DistanceMetrics.hpp:33-230) ---------------------
// partial() returns the value before the final square root, summed as
// meta::accumulate's right fold t0 + (t1 + (... + (t_{N-1} + 0))) or, for the
// Chebyshev family, meta::maximum's left-to-right std::max starting from 0.
// finish() applies the square root where the reference takes one.

template <int N, int MT>
struct Metric;

template <int N>
struct Metric<N, CLUE_METRIC_EUCLIDEAN> {
  static constexpr bool kRoot = true;
  // Right fold t_0 + (t_1 + (... + (t_{N-1} + 0))).  A square is never -0, so t_{N-1} + 0 is
  // t_{N-1} itself and the fold starts there.
  CLUE_HD static float partial(const float* a, const float* b, const float*) {
    float acc = fmul(fsub(a[N - 1], b[N - 1]), fsub(a[N - 1], b[N - 1]));
#pragma unroll
    for (int d = N - 2; d >= 0; --d) {
      const float t = fmul(fsub(a[d], b[d]), fsub(a[d], b[d]));
      acc = fadd(t, acc);
    }
    return acc;
  }
  // Lower bound of partial(x, c) over every c in the box [lo, hi], with the same monotone
  // rounded operations, so lower() > t implies partial(x, c) > t for every c in the box.
  CLUE_HD static float lower(const float* x, const float* lo, const float* hi, const float*) {
    float acc = 0.0f;
#pragma unroll
    for (int d = N - 1; d >= 0; --d) {
      const float gap = x[d] < lo[d] ? fsub(lo[d], x[d]) : (x[d] > hi[d] ? fsub(x[d], hi[d]) : 0.0f);
      acc = fadd(fmul(gap, gap), acc);
    }
    return acc;
  }
  CLUE_HD static float finish(float s) { return fsqrt(s); }
};

template <int N>
struct Metric<N, CLUE_METRIC_WEIGHTED_EUCLIDEAN> {
  static constexpr bool kRoot = true;
  CLUE_HD static float partial(const float* a, const float* b, const float* w) {
    float acc = 0.0f;
#pragma unroll
    for (int d = N - 1; d >= 0; --d) {
      const float t = fmul(fmul(w[d], fsub(a[d], b[d])), fsub(a[d], b[d]));
      acc = fadd(t, acc);
    }
    return acc;
  }
  CLUE_HD static float lower(const float* x, const float* lo, const float* hi, const float* w) {
    float acc = 0.0f;
#pragma unroll
    for (int d = N - 1; d >= 0; --d) {
      const float gap = x[d] < lo[d] ? fsub(lo[d], x[d]) : (x[d] > hi[d] ? fsub(x[d], hi[d]) : 0.0f);
      acc = fadd(fmul(fmul(w[d], gap), gap), acc);
    }
    return acc;
  }
  CLUE_HD static float finish(float s) { return fsqrt(s); }
};

template <int N>
struct Metric<N, CLUE_METRIC_PERIODIC_EUCLIDEAN> {
  static constexpr bool kRoot = true;
  CLUE_HD static float term(float a, float b, float period) {
    const float diff = fabsf(fsub(a, b));
    const float alt = fsub(period, diff);
    const float pd = alt < diff ? alt : diff;
    return fmul(pd, pd);
  }
  // Right fold as for the Euclidean metric; a square is never -0, so the fold starts at the
  // last term.
  CLUE_HD static float partial(const float* a, const float* b, const float* period) {
    float acc = term(a[N - 1], b[N - 1], period[N - 1]);
#pragma unroll
    for (int d = N - 2; d >= 0; --d) acc = fadd(term(a[d], b[d], period[d]), acc);
    return acc;
  }
  // Periodic dimensions contribute no bound; the others bound like the Euclidean metric.
  CLUE_HD static float lower(const float* x, const float* lo, const float* hi, const float* period) {
    float acc = 0.0f;
#pragma unroll
    for (int d = N - 1; d >= 0; --d) {
      const float gap = x[d] < lo[d] ? fsub(lo[d], x[d]) : (x[d] > hi[d] ? fsub(x[d], hi[d]) : 0.0f);
      acc = fadd(period[d] == 0.0f ? fmul(gap, gap) : 0.0f, acc);
    }
    return acc;
  }
  CLUE_HD static float finish(float s) { return fsqrt(s); }
};

template <int N>
struct Metric<N, CLUE_METRIC_MANHATTAN> {
  static constexpr bool kRoot = false;
  // Right fold of |a_d - b_d|; an absolute value is never -0, so the fold starts at the last term.
  CLUE_HD static float partial(const float* a, const float* b, const float*) {
    float acc = fabsf(fsub(a[N - 1], b[N - 1]));
#pragma unroll
    for (int d = N - 2; d >= 0; --d) acc = fadd(fabsf(fsub(a[d], b[d])), acc);
    return acc;
  }
  CLUE_HD static float lower(const float* x, const float* lo, const float* hi, const float*) {
    float acc = 0.0f;
#pragma unroll
    for (int d = N - 1; d >= 0; --d) {
      const float gap = x[d] < lo[d] ? fsub(lo[d], x[d]) : (x[d] > hi[d] ? fsub(x[d], hi[d]) : 0.0f);
      acc = fadd(gap, acc);
    }
    return acc;
  }
  CLUE_HD static float finish(float s) { return s; }
};

template <int N>
struct Metric<N, CLUE_METRIC_CHEBYSHEV> {
  static constexpr bool kRoot = false;
  CLUE_HD static float partial(const float* a, const float* b, const float*) {
    float m = 0.0f;
#pragma unroll
    for (int d = 0; d < N; ++d) {
      const float t = fabsf(fsub(a[d], b[d]));
      m = (m < t) ? t : m;
    }
    return m;
  }
  CLUE_HD static float lower(const float* x, const float* lo, const float* hi, const float*) {
    float m = 0.0f;
#pragma unroll
    for (int d = 0; d < N; ++d) {
      const float gap = x[d] < lo[d] ? fsub(lo[d], x[d]) : (x[d] > hi[d] ? fsub(x[d], hi[d]) : 0.0f);
      m = (m < gap) ? gap : m;
    }
    return m;
  }
  CLUE_HD static float finish(float s) { return s; }
};

template <int N>
struct Metric<N, CLUE_METRIC_WEIGHTED_CHEBYSHEV> {
  static constexpr bool kRoot = false;
  CLUE_HD static float partial(const float* a, const float* b, const float* w) {
    float m = 0.0f;
#pragma unroll
    for (int d = 0; d < N; ++d) {
      const float t = fmul(w[d], fabsf(fsub(a[d], b[d])));
      m = (m < t) ? t : m;
    }
    return m;
  }
  CLUE_HD static float lower(const float* x, const float* lo, const float* hi, const float* w) {
    float m = 0.0f;
#pragma unroll
    for (int d = 0; d < N; ++d) {
      const float gap = x[d] < lo[d] ? fsub(lo[d], x[d]) : (x[d] > hi[d] ? fsub(x[d], hi[d]) : 0.0f);
      const float t = fmul(w[d], gap);
      m = (m < t) ? t : m;
    }
    return m;
  }
  CLUE_HD static float finish(float s) { return s; }
};

#if defined(__CUDACC__)
// Paired single-precision arithmetic (sm_100 f32x2 instructions: two IEEE round-to-nearest
// operations in one issue slot, each rounded exactly like its scalar form).
__device__ __forceinline__ unsigned long long pk2(float2 v) {
  unsigned long long u;
  asm("mov.b64 %0, {%1, %2};" : "=l"(u) : "f"(v.x), "f"(v.y));
  return u;
}
__device__ __forceinline__ float2 upk2(unsigned long long u) {
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(u));
  return v;
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
  return upk2(r);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
  return upk2(r);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
  return upk2(r);
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)), "l"(pk2(c)));
  return upk2(r);
}

// Metric values of one point against two others, bit-identical to two Metric::partial calls;
// the Euclidean metric takes paired differences and squares.  The sums stay scalar: ptxas
// (CUDA 12.9) contracts a paired multiply feeding a paired add into a fused multiply-add even
// under --fmad=false, which would change the rounding.
template <int N, int MT>
__device__ __forceinline__ float2 partial_pair(const float* x, const float* a, const float* b, const float* mpar) {
  if constexpr (MT == CLUE_METRIC_EUCLIDEAN) {
    float2 df = sub2(make_float2(x[N - 1], x[N - 1]), make_float2(a[N - 1], b[N - 1]));
    float2 acc = mul2(df, df);
#pragma unroll
    for (int d = N - 2; d >= 0; --d) {
      df = sub2(make_float2(x[d], x[d]), make_float2(a[d], b[d]));
      const float2 t = mul2(df, df);
      acc = make_float2(fadd(t.x, acc.x), fadd(t.y, acc.y));
    }
    return acc;
  } else {
    return make_float2(Metric<N, MT>::partial(x, a, mpar), Metric<N, MT>::partial(x, b, mpar));
  }
}
#endif

// ---- convolutional kernels (core/detail/ConvolutionalKernel.hpp:16-65) -------
#if defined(__CUDACC__)
// Hardware approximations used by the spatial-order density (whose sums are not bit-exact):
// sqrt.approx (about 1 ulp) and 2^x of x * log2(e) (ex2.approx, a few ulp); the relative error
// of a term stays below 1e-6, well inside the 1e-5 tolerance on rho.
__device__ __forceinline__ float sqrt_approx(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// 2^e of two values on the FMA pipe instead of the MUFU (XU) pipe, for e <= 0: e is split as
// n + f with n the nearest integer (adding and subtracting 1.5 * 2^23 rounds to an integer) and
// |f| <= 1/2; 2^f = exp(f ln 2) is the Taylor series of exp truncated after degree 6 (Horner
// form, paired fused multiply-adds), and 2^n is added to the exponent field.  Truncation error
// (ln2 / 2)^7 / 7! * exp(ln2 / 2) < 1.7e-7 relative to 2^f >= 0.7, plus a few ulp of rounding:
// below 5e-7 relative.  e below -126 is clamped (the result stays a normal number); e = 0 gives
// exactly 1.
__device__ __forceinline__ float2 exp2_poly2(float2 e) {
  constexpr double kLn2 = 0.69314718055994530942;
  constexpr float c1 = (float)kLn2, c2 = (float)(kLn2 * kLn2 / 2.0), c3 = (float)(kLn2 * kLn2 * kLn2 / 6.0),
                  c4 = (float)(kLn2 * kLn2 * kLn2 * kLn2 / 24.0),
                  c5 = (float)(kLn2 * kLn2 * kLn2 * kLn2 * kLn2 / 120.0),
                  c6 = (float)(kLn2 * kLn2 * kLn2 * kLn2 * kLn2 * kLn2 / 720.0);
  const float2 magic = make_float2(12582912.0f, 12582912.0f);
  e = make_float2(fmaxf(e.x, -126.0f), fmaxf(e.y, -126.0f));
  const float2 t = add2(e, magic);
  const float2 f = sub2(e, sub2(t, magic));
  float2 p = fma2(make_float2(c6, c6), f, make_float2(c5, c5));
  p = fma2(p, f, make_float2(c4, c4));
  p = fma2(p, f, make_float2(c3, c3));
  p = fma2(p, f, make_float2(c2, c2));
  p = fma2(p, f, make_float2(c1, c1));
  p = fma2(p, f, make_float2(1.0f, 1.0f));
  const int nx = __float_as_int(t.x) - 0x4B400000, ny = __float_as_int(t.y) - 0x4B400000;
  return make_float2(__int_as_float(__float_as_int(p.x) + (nx << 23)),
                     __int_as_float(__float_as_int(p.y) + (ny << 23)));
}
__device__ __forceinline__ float exp_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x * 1.4426950408889634f));
  return y;
}
// Kernel value of the spatial-order density (distance from the pre-root metric value s).
// ginv = 1 / (2 std^2) precomputed on the host.
__device__ __forceinline__ float kernel_value_fast(int32_t type, const float* k, float ginv, float dist) {
  if (type == CLUE_KERNEL_FLAT) return k[0];
  if (type == CLUE_KERNEL_EXPONENTIAL) return k[1] * exp_approx(-k[0] * dist);
  const float u = dist - k[0];
  return k[2] * exp_approx(-u * u * ginv);
}
#endif
// Value for a pair of distinct points; the self pair (i == j) is 1.
CLUE_HD float kernel_value(int32_t type, const float* k, float dist) {
  if (type == CLUE_KERNEL_FLAT) return k[0];
  if (type == CLUE_KERNEL_EXPONENTIAL) return fmul(k[1], expf(fmul(-k[0], dist)));
  // Gaussian: amp * exp(-(d - avg) * (d - avg) / (2 * std * std))
  const float u = fsub(dist, k[0]);
  const float e = fdiv(fmul(-u, u), fmul(fmul(2.0f, k[1]), k[1]));
  return fmul(k[2], expf(e));
}

}  // namespace clue_b200
