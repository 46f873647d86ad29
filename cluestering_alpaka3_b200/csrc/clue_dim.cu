// clue_dim.cu -- the five CLUE stages for points of CLUE_NDIM dimensions.
//
// Compiled once per dimensionality (-DCLUE_NDIM=1..10) so the templates of one
// dimension build in parallel.  Stage map against the reference's serial path
// (include/CLUEstering/core/detail/Clusterer.hpp:134-171):
//   k_bbox / k_grid      compute_tile_size        core/detail/ComputeTiles.hpp:13-27
//   k_bin + radix sort   Tiles::fill              data_structures/internal/Tiles.hpp:92-96
//   k_density            KernelCalculateLocalDensity  core/detail/ClusteringKernels.hpp:66-107
//   k_nearest_higher     KernelCalculateNearestHigher core/detail/ClusteringKernels.hpp:109-212
//   k_seeds              KernelFindClusters       core/detail/ClusteringKernels.hpp:214-244
//   k_jump + k_finalize  Followers::fill + KernelAssignClusters
//                        data_structures/internal/Followers.hpp:27-30,
//                        core/detail/ClusteringKernels.hpp:246-281
//
// Layout in HBM: points are reordered by tile (stable: ascending index inside a tile)
// into float4 records {coords..., payload}; one warp lane owns one home point and the
// whole warp walks the same candidate sequence, so every candidate record is one
// broadcast 16-byte load per warp.
#include "clue_internal.h"

#ifndef CLUE_NDIM
#error "CLUE_NDIM must be defined"
#endif

namespace clue_b200 {
namespace {

constexpr int kTileThreads = 128;
constexpr int kTileWarps = kTileThreads / 32;
constexpr int kCap = 2048;  // home points signature-sorted per pass

struct InPtrs {
  const float* c[kMaxDim];
  const float* w;
};

__device__ __forceinline__ int warp_min_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ int warp_max_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ uint32_t warp_min_u(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ uint32_t warp_max_u(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <int N>
__device__ __forceinline__ void load_rec(const float4* __restrict__ rec, int pos, float* x, float& payload) {
  constexpr int W = Rec<N>::kWords;
  float buf[4 * W];
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const float4 v = __ldg(rec + (size_t)pos * W + k);
    buf[4 * k + 0] = v.x;
    buf[4 * k + 1] = v.y;
    buf[4 * k + 2] = v.z;
    buf[4 * k + 3] = v.w;
  }
#pragma unroll
  for (int d = 0; d < N; ++d) x[d] = buf[d];
  payload = buf[Rec<N>::kPayload];
}

template <int N>
__device__ __forceinline__ void store_rec(float4* __restrict__ rec, int pos, const float* x, float payload) {
  constexpr int W = Rec<N>::kWords;
  float buf[4 * W];
#pragma unroll
  for (int k = 0; k < 4 * W; ++k) buf[k] = 0.0f;
#pragma unroll
  for (int d = 0; d < N; ++d) buf[d] = x[d];
  buf[Rec<N>::kPayload] = payload;
#pragma unroll
  for (int k = 0; k < W; ++k)
    rec[(size_t)pos * W + k] = make_float4(buf[4 * k], buf[4 * k + 1], buf[4 * k + 2], buf[4 * k + 3]);
}

// Search box of one point in "virtual" bins: the reference's [getBin(x - r), getBin(x + r)]
// (TilesView.hpp:72-82, wrapped boxes extended by nperdim), shifted down by nperdim when a
// wrapped box starts above the home bin, so that every lane of a warp expresses its box
// in the same frame around the home tile.  The tile of virtual bin v is v mod nperdim.
template <int N>
__device__ __forceinline__ void lane_box(const KParams& kp, const DevGrid* __restrict__ g, const float* x,
                                         float r, const int* hb, int* lo, int* hi) {
#pragma unroll
  for (int d = 0; d < N; ++d) {
    const bool wr = kp.wrapped[d] != 0;
    int a = get_bin(fsub(x[d], r), g->mn[d], g->mx[d], g->size[d], wr, kp.nperdim);
    int b = get_bin(fadd(x[d], r), g->mn[d], g->mx[d], g->size[d], wr, kp.nperdim);
    if (wr && a > b) b += kp.nperdim;
    if (wr && a > hb[d]) {
      a -= kp.nperdim;
      b -= kp.nperdim;
    }
    lo[d] = a;
    hi[d] = b;
  }
}

template <int N>
__device__ __forceinline__ void home_bins(const KParams& kp, int t, int* hb) {
#pragma unroll
  for (int d = 0; d < N; ++d) hb[d] = (t / kp.stride[d]) % kp.nperdim;
}

__device__ __forceinline__ int wrap_bin(int v, int npd) {
  int b = v % npd;
  return b < 0 ? b + npd : b;
}

// Orders the home points [cb, cb + cnt) of a tile by which neighbour tiles their search
// box reaches (2 bits per dimension), so that the 32 lanes of a warp share one box.
template <int N>
__device__ void signature_sort(const KParams& kp, const DevGrid* __restrict__ g, const float4* __restrict__ rec,
                               int cb, int cnt, float r, const int* hb, int32_t* s_order, uint8_t* s_key,
                               int32_t* s_hist) {
  if constexpr (N <= 4) {
    constexpr int K = 1 << (2 * N);
    for (int e = threadIdx.x; e < K; e += blockDim.x) s_hist[e] = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
      float x[N], pl;
      load_rec<N>(rec, cb + k, x, pl);
      int lo[N], hi[N];
      lane_box<N>(kp, g, x, r, hb, lo, hi);
      int key = 0;
#pragma unroll
      for (int d = 0; d < N; ++d) key |= ((lo[d] < hb[d] ? 1 : 0) | (hi[d] > hb[d] ? 2 : 0)) << (2 * d);
      s_key[k] = (uint8_t)key;
      atomicAdd(&s_hist[key], 1);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      int carry = 0;
      for (int base = 0; base < K; base += 32) {
        const int e = base + (int)threadIdx.x;
        const int v = e < K ? s_hist[e] : 0;
        int inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t = __shfl_up_sync(0xffffffffu, inc, o);
          if ((int)threadIdx.x >= o) inc += t;
        }
        if (e < K) s_hist[e] = carry + inc - v;
        carry += __shfl_sync(0xffffffffu, inc, 31);
      }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) s_order[atomicAdd(&s_hist[s_key[k]], 1)] = k;
    __syncthreads();
  } else {
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) s_order[k] = k;
    __syncthreads();
  }
}

// ---- stage 1: bounding box, grid, bins --------------------------------------

template <int N>
__global__ void k_init(DevGrid* g, DevStatus* st) {
  const int t = threadIdx.x;
  if (t < kMaxDim) {
    g->enc_min[t] = 0xffffffffu;
    g->enc_max[t] = 0u;
  }
  uint32_t* s = reinterpret_cast<uint32_t*>(st);
  for (int k = t; k < (int)(sizeof(DevStatus) / 4); k += blockDim.x) s[k] = 0u;
}

template <int N>
__global__ void __launch_bounds__(256) k_bbox(InPtrs in, int n, DevGrid* g, DevStatus* st) {
  uint32_t emn[N], emx[N];
#pragma unroll
  for (int d = 0; d < N; ++d) {
    emn[d] = 0xffffffffu;
    emx[d] = 0u;
  }
  bool bad = false;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
#pragma unroll
    for (int d = 0; d < N; ++d) {
      const float x = in.c[d][i];
      bad |= !isfinite(x);
      const uint32_t e = enc_float(x);
      emn[d] = min(emn[d], e);
      emx[d] = max(emx[d], e);
    }
    bad |= !isfinite(in.w[i]);
  }
#pragma unroll
  for (int d = 0; d < N; ++d) {
    emn[d] = warp_min_u(emn[d]);
    emx[d] = warp_max_u(emx[d]);
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int d = 0; d < N; ++d) {
      atomicMin(&g->enc_min[d], emn[d]);
      atomicMax(&g->enc_max[d], emx[d]);
    }
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&st->nonfinite, 1u);
}

// Tile size (max - min) / nperdim in FP32 (ComputeTiles.hpp:20-23).
template <int N>
__global__ void k_grid(const KParams kp, DevGrid* g) {
  const int d = threadIdx.x;
  if (d < N) {
    const float mn = dec_float(g->enc_min[d]);
    const float mx = dec_float(g->enc_max[d]);
    g->mn[d] = mn;
    g->mx[d] = mx;
    g->size[d] = fdiv(fsub(mx, mn), (float)kp.nperdim);
  }
}

// Global bin of every point (TilesView.hpp:53-61, exact integer arithmetic).
template <int N>
__global__ void __launch_bounds__(256) k_bin(const KParams kp, InPtrs in, int n, const DevGrid* __restrict__ g,
                                             uint32_t* __restrict__ keys) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    int gb = 0;
#pragma unroll
    for (int d = 0; d < N; ++d)
      gb += kp.stride[d] *
            get_bin(in.c[d][i], g->mn[d], g->mx[d], g->size[d], kp.wrapped[d] != 0, kp.nperdim);
    keys[i] = (uint32_t)gb;
  }
}

template <int N>
__global__ void __launch_bounds__(256) k_gather(InPtrs in, int n, const int32_t* __restrict__ perm,
                                                float4* __restrict__ rec_w) {
  const int stride = gridDim.x * blockDim.x;
  for (int pos = blockIdx.x * blockDim.x + threadIdx.x; pos < n; pos += stride) {
    const int i = perm[pos];
    float x[N];
#pragma unroll
    for (int d = 0; d < N; ++d) x[d] = in.c[d][i];
    store_rec<N>(rec_w, pos, x, in.w[i]);
  }
}

// ---- stage 2: local density --------------------------------------------------
// rho_i accumulates, in the reference's candidate order (search-box tiles
// lexicographically, ascending index inside a tile), term = k(d, i, j) * w_j for every
// candidate with d <= dc; candidates beyond dc contribute +-0 and are skipped.
template <int N, int MT>
__global__ void __launch_bounds__(kTileThreads) k_density(const KParams kp, const DevGrid* __restrict__ g,
                                                          const int32_t* __restrict__ off,
                                                          const float4* __restrict__ rec_w,
                                                          float4* __restrict__ rec_r) {
  using M = Metric<N, MT>;
  __shared__ int32_t s_order[kCap];
  __shared__ uint8_t s_key[kCap];
  __shared__ int32_t s_hist[N <= 4 ? (1 << (2 * N)) : 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool flat = kp.kernel_type == CLUE_KERNEL_FLAT;
  for (int t = blockIdx.x; t < kp.ntiles; t += gridDim.x) {
    const int beg = off[t], end = off[t + 1];
    if (beg == end) continue;
    int hb[N];
    home_bins<N>(kp, t, hb);
    for (int cb = beg; cb < end; cb += kCap) {
      const int cnt = min(kCap, end - cb);
      signature_sort<N>(kp, g, rec_w, cb, cnt, kp.dc, hb, s_order, s_key, s_hist);
      for (int slice = warp; slice * 32 < cnt; slice += kTileWarps) {
        const int k = slice * 32 + lane;
        const bool valid = k < cnt;
        const int pos = cb + (valid ? s_order[k] : 0);
        float x[N], wi;
        load_rec<N>(rec_w, pos, x, wi);
        int lo[N], hi[N], ulo[N], uhi[N];
        lane_box<N>(kp, g, x, kp.dc, hb, lo, hi);
#pragma unroll
        for (int d = 0; d < N; ++d) {
          ulo[d] = warp_min_i(valid ? lo[d] : INT_MAX);
          uhi[d] = warp_max_i(valid ? hi[d] : INT_MIN);
        }
        float rho = 0.0f;
        int v[N];
#pragma unroll
        for (int d = 0; d < N; ++d) v[d] = ulo[d];
        while (true) {
          bool inbox = valid;
          int u = 0;
#pragma unroll
          for (int d = 0; d < N; ++d) {
            inbox = inbox && v[d] >= lo[d] && v[d] <= hi[d];
            u += kp.stride[d] * wrap_bin(v[d], kp.nperdim);
          }
          if (__any_sync(0xffffffffu, inbox)) {
            const int qb = off[u], qe = off[u + 1];
#pragma unroll 4
            for (int q = qb; q < qe; ++q) {
              float c[N], wj;
              load_rec<N>(rec_w, q, c, wj);
              const float s = M::partial(x, c, kp.mpar);
              if (inbox && s <= kp.t_dc) {
                float term;
                if (flat) {
                  term = (q == pos) ? wj : fmul(kp.kpar[0], wj);
                } else {
                  const float kv = (q == pos) ? 1.0f : kernel_value(kp.kernel_type, kp.kpar, M::finish(s));
                  term = fmul(kv, wj);
                }
                rho = fadd(rho, term);
              }
            }
          }
          int d = N - 1;
          for (; d >= 0; --d) {
            if (v[d] < uhi[d]) {
              ++v[d];
              break;
            }
            v[d] = ulo[d];
          }
          if (d < 0) break;
        }
        if (valid) store_rec<N>(rec_r, pos, x, rho);
      }
      __syncthreads();
    }
  }
}

// ---- stage 3: nearest higher -------------------------------------------------
// j is higher than i iff rho_j > rho_i or (rho_j == rho_i, rho_j > 0, j > i) with
// original indices; the nearest higher is the first candidate, in the reference's
// order, with the strictly smallest distance <= dm (TIE == CLUE_TIE_REFERENCE), or the
// candidate with the smallest (distance, -rho, index) (TIE == CLUE_TIE_RHO_INDEX).
template <int N, int MT, int TIE>
__global__ void __launch_bounds__(kTileThreads) k_nearest_higher(
    const KParams kp, const DevGrid* __restrict__ g, const int32_t* __restrict__ off,
    const float4* __restrict__ rec_r, const int32_t* __restrict__ perm, int32_t* __restrict__ nh_s,
    float* __restrict__ delta_s, DevStatus* st) {
  using M = Metric<N, MT>;
  __shared__ int32_t s_order[kCap];
  __shared__ uint8_t s_key[kCap];
  __shared__ int32_t s_hist[N <= 4 ? (1 << (2 * N)) : 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int t = blockIdx.x; t < kp.ntiles; t += gridDim.x) {
    const int beg = off[t], end = off[t + 1];
    if (beg == end) continue;
    int hb[N];
    home_bins<N>(kp, t, hb);
    for (int cb = beg; cb < end; cb += kCap) {
      const int cnt = min(kCap, end - cb);
      signature_sort<N>(kp, g, rec_r, cb, cnt, kp.dm, hb, s_order, s_key, s_hist);
      for (int slice = warp; slice * 32 < cnt; slice += kTileWarps) {
        const int k = slice * 32 + lane;
        const bool valid = k < cnt;
        const int pos = cb + (valid ? s_order[k] : 0);
        float x[N], rho_i;
        load_rec<N>(rec_r, pos, x, rho_i);
        const int orig_i = perm[pos];
        int lo[N], hi[N], ulo[N], uhi[N];
        lane_box<N>(kp, g, x, kp.dm, hb, lo, hi);
#pragma unroll
        for (int d = 0; d < N; ++d) {
          ulo[d] = warp_min_i(valid ? lo[d] : INT_MAX);
          uhi[d] = warp_max_i(valid ? hi[d] : INT_MIN);
        }
        float delta = FLT_MAX, s_best = INFINITY, rho_best = 0.0f;
        int nh = -1, orig_best = INT_MAX;
        int v[N];
#pragma unroll
        for (int d = 0; d < N; ++d) v[d] = ulo[d];
        while (true) {
          bool inbox = valid;
          int u = 0;
#pragma unroll
          for (int d = 0; d < N; ++d) {
            inbox = inbox && v[d] >= lo[d] && v[d] <= hi[d];
            u += kp.stride[d] * wrap_bin(v[d], kp.nperdim);
          }
          if (__any_sync(0xffffffffu, inbox)) {
            const int qb = off[u], qe = off[u + 1];
#pragma unroll 4
            for (int q = qb; q < qe; ++q) {
              float c[N], rho_j;
              load_rec<N>(rec_r, q, c, rho_j);
              const float s = M::partial(x, c, kp.mpar);
              bool cand = inbox && s <= kp.t_dm && rho_j >= rho_i;
              if (TIE == CLUE_TIE_REFERENCE) cand = cand && s < s_best;
              if (cand) {
                int orig_j = -1;
                bool higher = rho_j > rho_i;
                if (!higher && rho_j > 0.0f) {
                  orig_j = __ldg(perm + q);
                  higher = orig_j > orig_i;
                }
                if (higher) {
                  const float dist = M::finish(s);
                  if (dist < delta) {
                    delta = dist;
                    s_best = s;
                    nh = q;
                    rho_best = rho_j;
                    orig_best = orig_j;
                  } else if (TIE == CLUE_TIE_RHO_INDEX && dist == delta) {
                    if (orig_j < 0) orig_j = __ldg(perm + q);
                    if (orig_best < 0) orig_best = __ldg(perm + nh);
                    if (rho_j > rho_best || (rho_j == rho_best && orig_j < orig_best)) {
                      nh = q;
                      rho_best = rho_j;
                      orig_best = orig_j;
                    }
                  }
                }
              }
            }
          }
          int d = N - 1;
          for (; d >= 0; --d) {
            if (v[d] < uhi[d]) {
              ++v[d];
              break;
            }
            v[d] = ulo[d];
          }
          if (d < 0) break;
        }
        if (valid) {
          nh_s[pos] = nh;
          delta_s[pos] = delta;
        }
        const uint32_t none = __ballot_sync(0xffffffffu, valid && nh < 0);
        if (lane == 0 && none) atomicAdd(&st->seed_candidates, (uint32_t)__popc(none));
      }
      __syncthreads();
    }
  }
}

// ---- stage 4: seeds (KernelFindClusters) ---------------------------------------
template <int N, int MT>
__global__ void __launch_bounds__(256) k_seeds(const KParams kp, int n, const float4* __restrict__ rec_r,
                                               const int32_t* __restrict__ nh_s,
                                               const int32_t* __restrict__ perm, int32_t* __restrict__ is_seed_s,
                                               int32_t* __restrict__ par, uint32_t* __restrict__ seed_flag) {
  using M = Metric<N, MT>;
  const int stride = gridDim.x * blockDim.x;
  for (int pos = blockIdx.x * blockDim.x + threadIdx.x; pos < n; pos += stride) {
    float x[N], rho, c[N], pl;
    load_rec<N>(rec_r, pos, x, rho);
    const int nh = nh_s[pos];
    if (nh >= 0) {
      load_rec<N>(rec_r, nh, c, pl);
    } else {
#pragma unroll
      for (int d = 0; d < N; ++d) c[d] = FLT_MAX;  // PointsView::operator[](-1), PointsCommon.hpp:75-81
    }
    const float dist = M::finish(M::partial(x, c, kp.mpar));
    const bool seed = (dist > kp.seed_dc) && (rho >= kp.rhoc);
    is_seed_s[pos] = seed ? 1 : 0;
    par[pos] = seed ? -1 : nh;
    seed_flag[perm[pos]] = seed ? 1u : 0u;
  }
}

// ---- stage 5: labels ---------------------------------------------------------

// Pointer jumping on the nearest-higher forest: every parent pointer is replaced by its
// grandparent until it names a root (a seed or a point without nearest higher).  All
// writes move a pointer to an ancestor, so concurrent updates are safe.  At most
// `iters` jumps per point per launch; a launch that leaves a point unresolved records it
// in st->unresolved[round] and the next launch continues.
__global__ void __launch_bounds__(256) k_jump(int32_t* par, int n, int iters, DevStatus* st, int round) {
  if (round > 0 && st->unresolved[round - 1] == 0) return;
  bool unres = false;
  const int stride = gridDim.x * blockDim.x;
  for (int pos = blockIdx.x * blockDim.x + threadIdx.x; pos < n; pos += stride) {
    int p = par[pos];
    if (p < 0) continue;
    int it = 0;
    for (; it < iters; ++it) {
      const int pp = __ldcg(par + p);
      if (pp < 0) break;
      p = pp;
      par[pos] = p;
    }
    if (it == iters && __ldcg(par + p) >= 0) unres = true;
  }
  if (__any_sync(0xffffffffu, unres) && (threadIdx.x & 31) == 0) atomicAdd(&st->unresolved[round], 1u);
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicMax(&st->label_rounds, (uint32_t)round + 1);
}

// Labels from the roots and scatter of every output back to the caller's order.
template <int N>
__global__ void __launch_bounds__(256) k_finalize(const KParams kp, int n, const int32_t* __restrict__ par,
                                                  const int32_t* __restrict__ is_seed_s,
                                                  const uint32_t* __restrict__ seed_rank,
                                                  const int32_t* __restrict__ perm,
                                                  const int32_t* __restrict__ nh_s,
                                                  const float4* __restrict__ rec_r,
                                                  const float* __restrict__ delta_s, const DevStatus* st,
                                                  clue_outputs out) {
  const int64_t cap = kp.seed_capacity < 0
                          ? INT64_MAX
                          : (kp.seed_capacity > (int64_t)st->seed_candidates ? kp.seed_capacity
                                                                             : (int64_t)st->seed_candidates);
  const int stride = gridDim.x * blockDim.x;
  for (int pos = blockIdx.x * blockDim.x + threadIdx.x; pos < n; pos += stride) {
    const int p = par[pos];
    const int root = p >= 0 ? p : pos;
    int lab = -1;
    if (is_seed_s[root]) {
      const uint32_t rk = seed_rank[perm[root]];
      if ((int64_t)rk < cap) lab = (int)rk;
    }
    const int i = perm[pos];
    out.cluster_index[i] = lab;
    const int seed = is_seed_s[pos];
    if (out.is_seed) out.is_seed[i] = seed;
    if (out.rho) {
      float x[N], rho;
      load_rec<N>(rec_r, pos, x, rho);
      out.rho[i] = rho;
    }
    if (out.nearest_higher) {
      const int nh = seed ? -1 : nh_s[pos];
      out.nearest_higher[i] = nh >= 0 ? perm[nh] : -1;
    }
    if (out.delta) out.delta[i] = delta_s[pos];
  }
}

int grid_for(int n, int threads) {
  int b = (n + threads - 1) / threads;
  const int cap = 148 * 32;
  return b < 1 ? 1 : (b > cap ? cap : b);
}

template <int N, int MT>
void launch_density(const KParams& kp, Workspace& ws, cudaStream_t s) {
  k_density<N, MT><<<kp.ntiles, kTileThreads, 0, s>>>(kp, ws.grid, ws.offsets, ws.rec_w, ws.rec_r);
}
template <int N, int MT>
void launch_nh(const KParams& kp, Workspace& ws, cudaStream_t s) {
  if (kp.tiebreak == CLUE_TIE_RHO_INDEX)
    k_nearest_higher<N, MT, CLUE_TIE_RHO_INDEX><<<kp.ntiles, kTileThreads, 0, s>>>(
        kp, ws.grid, ws.offsets, ws.rec_r, ws.perm, ws.nh_s, ws.delta_s, ws.status);
  else
    k_nearest_higher<N, MT, CLUE_TIE_REFERENCE><<<kp.ntiles, kTileThreads, 0, s>>>(
        kp, ws.grid, ws.offsets, ws.rec_r, ws.perm, ws.nh_s, ws.delta_s, ws.status);
}
template <int N, int MT>
void launch_seeds(const KParams& kp, Workspace& ws, int n, cudaStream_t s) {
  k_seeds<N, MT><<<grid_for(n, 256), 256, 0, s>>>(kp, n, ws.rec_r, ws.nh_s, ws.perm, ws.is_seed_s, ws.par,
                                                  ws.seed_flag);
}

#define CLUE_METRIC_SWITCH(mt, FN, ...)                                           \
  switch (mt) {                                                                   \
    case CLUE_METRIC_EUCLIDEAN: FN<N, CLUE_METRIC_EUCLIDEAN>(__VA_ARGS__); break; \
    case CLUE_METRIC_WEIGHTED_EUCLIDEAN:                                          \
      FN<N, CLUE_METRIC_WEIGHTED_EUCLIDEAN>(__VA_ARGS__);                         \
      break;                                                                      \
    case CLUE_METRIC_PERIODIC_EUCLIDEAN:                                          \
      FN<N, CLUE_METRIC_PERIODIC_EUCLIDEAN>(__VA_ARGS__);                         \
      break;                                                                      \
    case CLUE_METRIC_MANHATTAN: FN<N, CLUE_METRIC_MANHATTAN>(__VA_ARGS__); break; \
    case CLUE_METRIC_CHEBYSHEV: FN<N, CLUE_METRIC_CHEBYSHEV>(__VA_ARGS__); break; \
    default: FN<N, CLUE_METRIC_WEIGHTED_CHEBYSHEV>(__VA_ARGS__); break;           \
  }

}  // namespace

// Number of pointer-jumping launches enqueued without host synchronisation.
constexpr int kJumpLaunches = 4;
constexpr int kJumpIters = 64;

template <int N>
clue_status run_pipeline(Workspace& ws, const RunArgs& a, cudaStream_t s) {
  const KParams& kp = a.kp;
  const int n = a.n;
  InPtrs in{};
  for (int d = 0; d < N; ++d) in.c[d] = a.coords[d];
  in.w = a.weight;

  stage_mark(ws, 0, s);
  k_init<N><<<1, 64, 0, s>>>(ws.grid, ws.status);
  k_bbox<N><<<grid_for(n, 256), 256, 0, s>>>(in, n, ws.grid, ws.status);
  k_grid<N><<<1, 32, 0, s>>>(kp, ws.grid);
  k_bin<N><<<grid_for(n, 256), 256, 0, s>>>(kp, in, n, ws.grid, ws.keys[0]);
  const int cur = radix_sort_pairs(ws.keys, ws.vals, true, n, bits_for((uint32_t)(kp.ntiles - 1)), ws.hist,
                                   ws.scan_scratch, s);
  ws.perm = ws.vals[cur];
  ws.sorted_keys = ws.keys[cur];
  offsets_from_sorted(ws.sorted_keys, n, kp.ntiles, ws.offsets, s);
  k_gather<N><<<grid_for(n, 256), 256, 0, s>>>(in, n, ws.perm, ws.rec_w);

  stage_mark(ws, 1, s);
  CLUE_METRIC_SWITCH(a.metric, launch_density, kp, ws, s);
  stage_mark(ws, 2, s);
  CLUE_METRIC_SWITCH(a.metric, launch_nh, kp, ws, s);
  stage_mark(ws, 3, s);
  CLUE_METRIC_SWITCH(a.metric, launch_seeds, kp, ws, n, s);
  exclusive_scan(ws.seed_flag, ws.seed_flag, (size_t)n, ws.scan_scratch, ws.seed_total, s);
  for (int r = 0; r < kJumpLaunches; ++r)
    k_jump<<<grid_for(n, 256), 256, 0, s>>>(ws.par, n, kJumpIters, ws.status, r);
  k_finalize<N><<<grid_for(n, 256), 256, 0, s>>>(kp, n, ws.par, ws.is_seed_s, ws.seed_flag, ws.perm, ws.nh_s,
                                                 ws.rec_r, ws.delta_s, ws.status, a.out);
  stage_mark(ws, 4, s);
  // init, bbox, grid, bin, sort, offsets, gather, density, nh, seeds, scan, jumps, finalize
  ws.launches += 4 + radix_sort_launches(bits_for((uint32_t)(kp.ntiles - 1))) + 2 + 3 + kScanLaunches +
                 kJumpLaunches + 1;
  CLUE_CUDA_TRY(cudaGetLastError());
  return CLUE_OK;
}

// Continue pointer jumping from the host after the enqueued launches left chains
// unresolved (only for very deep nearest-higher chains); synchronises per launch.
template <int N>
clue_status finish_labels(Workspace& ws, const RunArgs& a, cudaStream_t s, int first_round) {
  const int n = a.n;
  for (int r = first_round; r < 64; ++r) {
    k_jump<<<grid_for(n, 256), 256, 0, s>>>(ws.par, n, 1 << 12, ws.status, r);
    ++ws.launches;
    uint32_t unres = 0;
    CLUE_CUDA_TRY(cudaMemcpyAsync(&unres, &ws.status->unresolved[r], 4, cudaMemcpyDeviceToHost, s));
    CLUE_CUDA_TRY(cudaStreamSynchronize(s));
    if (unres == 0) break;
  }
  k_finalize<N><<<grid_for(n, 256), 256, 0, s>>>(a.kp, n, ws.par, ws.is_seed_s, ws.seed_flag, ws.perm, ws.nh_s,
                                                 ws.rec_r, ws.delta_s, ws.status, a.out);
  ++ws.launches;
  CLUE_CUDA_TRY(cudaGetLastError());
  return CLUE_OK;
}

template clue_status run_pipeline<CLUE_NDIM>(Workspace&, const RunArgs&, cudaStream_t);
template clue_status finish_labels<CLUE_NDIM>(Workspace&, const RunArgs&, cudaStream_t, int);

}  // namespace clue_b200
