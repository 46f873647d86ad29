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
#include "clue_tma.cuh"

#ifndef CLUE_NDIM
#error "CLUE_NDIM must be defined"
#endif

namespace clue_b200 {
namespace {

constexpr int kTileThreads = 128;
constexpr int kChunkWarps = kTileThreads / 32;
constexpr int kChunk = kChunkPoints;      // home points per CTA in the density / nearest-higher sweeps
static_assert(kChunkPoints == kTileThreads, "one home point per thread");
constexpr int kCap = 2048;                // home points signature-sorted per pass
constexpr int kStageWords = 1024;         // float4 words per staging buffer (16 KiB)
constexpr int kMaxSeg = 32;               // tile segments per staged piece

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

// ---- work orders and chunks --------------------------------------------------
// Every tile's points are ordered twice by search-box signature (radius dc for the
// density, dm for the nearest higher) and cut into chunks of kChunk home points; one CTA
// processes one chunk, so a heavy tile is spread over many CTAs.
template <int N>
__global__ void __launch_bounds__(kTileThreads) k_order(const KParams kp, const DevGrid* __restrict__ g,
                                                        const int32_t* __restrict__ off,
                                                        const float4* __restrict__ rec_w,
                                                        int32_t* __restrict__ ord_rho, int32_t* __restrict__ ord_nh,
                                                        uint32_t* __restrict__ chunk_count) {
  __shared__ int32_t s_order[kCap];
  __shared__ uint8_t s_key[kCap];
  __shared__ int32_t s_hist[N <= 4 ? (1 << (2 * N)) : 1];
  for (int t = blockIdx.x; t < kp.ntiles; t += gridDim.x) {
    const int beg = off[t], end = off[t + 1];
    if (threadIdx.x == 0) chunk_count[t] = (uint32_t)((end - beg + kChunk - 1) / kChunk);
    if (beg == end) continue;
    int hb[N];
    home_bins<N>(kp, t, hb);
    for (int cb = beg; cb < end; cb += kCap) {
      const int cnt = min(kCap, end - cb);
      signature_sort<N>(kp, g, rec_w, cb, cnt, kp.dc, hb, s_order, s_key, s_hist);
      for (int k = threadIdx.x; k < cnt; k += blockDim.x) ord_rho[cb + k] = cb + s_order[k];
      __syncthreads();
      signature_sort<N>(kp, g, rec_w, cb, cnt, kp.dm, hb, s_order, s_key, s_hist);
      for (int k = threadIdx.x; k < cnt; k += blockDim.x) ord_nh[cb + k] = cb + s_order[k];
      __syncthreads();
    }
  }
}

__global__ void k_chunk_map(int ntiles, const int32_t* __restrict__ off, const uint32_t* __restrict__ chunk_off,
                            int32_t* __restrict__ chunk_tile) {
  const int stride = gridDim.x * blockDim.x;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += stride) {
    const int nch = (off[t + 1] - off[t] + kChunk - 1) / kChunk;
    const uint32_t c0 = chunk_off[t];
    for (int c = 0; c < nch; ++c) chunk_tile[c0 + c] = t;
  }
}

// ---- staged sweep over the search-box tiles of one chunk ------------------------
// The CTA's 4 warps (128 home points of one tile) walk the union of their search boxes
// in the reference's lexicographic tile order.  Thread 0 packs consecutive tile segments
// into pieces of at most kStageWords float4 words and copies each piece into shared memory
// with bulk copies (TMA) completing on an mbarrier; two buffers alternate so the copy of
// piece p + 1 overlaps the scan of piece p.  Each warp scans only the segments of tiles in
// its own union; each lane only counts candidates of tiles inside its own box.

template <int N>
struct StageSmem {
  float4 buf[2][kStageWords];
  int32_t seg_v[2][kMaxSeg][N];
  int32_t seg_qb[2][kMaxSeg];
  int32_t seg_cnt[2][kMaxSeg];
  int32_t seg_boff[2][kMaxSeg];
  int32_t nseg[2];
  int32_t wlo[kChunkWarps][N], whi[kChunkWarps][N];
  int32_t ulo[N], uhi[N];
  int32_t any_valid;
  alignas(8) uint64_t full[2];
};

// Thread-0 iterator over the tiles of the CTA union that some warp needs.
template <int N>
struct TileIter {
  int v[N];
  bool started = false;
  int q = 0, qe = 0;

  __device__ bool needed(const StageSmem<N>& sm) const {
    for (int w = 0; w < kChunkWarps; ++w) {
      bool in = true;
#pragma unroll
      for (int d = 0; d < N; ++d) in = in && v[d] >= sm.wlo[w][d] && v[d] <= sm.whi[w][d];
      if (in) return true;
    }
    return false;
  }

  // Advances to the next needed, non-empty tile; false when the union is exhausted.
  __device__ bool next(const KParams& kp, const int32_t* __restrict__ off, const StageSmem<N>& sm) {
    while (true) {
      if (!started) {
#pragma unroll
        for (int d = 0; d < N; ++d) v[d] = sm.ulo[d];
        started = true;
      } else {
        int d = N - 1;
        for (; d >= 0; --d) {
          if (v[d] < sm.uhi[d]) {
            ++v[d];
            break;
          }
          v[d] = sm.ulo[d];
        }
        if (d < 0) return false;
      }
      if (!needed(sm)) continue;
      int u = 0;
#pragma unroll
      for (int d = 0; d < N; ++d) u += kp.stride[d] * wrap_bin(v[d], kp.nperdim);
      q = off[u];
      qe = off[u + 1];
      if (qe > q) return true;
    }
  }
};

// Builds piece b (thread 0 only) and issues its bulk copies; returns the words staged.
template <int N>
__device__ int build_piece(const KParams& kp, const int32_t* __restrict__ off, const float4* __restrict__ rec,
                           StageSmem<N>& sm, TileIter<N>& it, bool& done, int b) {
  constexpr int W = Rec<N>::kWords;
  constexpr int cap = kStageWords / W;
  int nseg = 0, fill = 0;
  while (!done && nseg < kMaxSeg && fill < cap) {
    if (it.q >= it.qe) {
      if (!it.next(kp, off, sm)) {
        done = true;
        break;
      }
    }
    const int take = min(it.qe - it.q, cap - fill);
#pragma unroll
    for (int d = 0; d < N; ++d) sm.seg_v[b][nseg][d] = it.v[d];
    sm.seg_qb[b][nseg] = it.q;
    sm.seg_cnt[b][nseg] = take;
    sm.seg_boff[b][nseg] = fill;
    ++nseg;
    fill += take;
    it.q += take;
  }
  sm.nseg[b] = nseg;
  if (fill > 0) {
    mbar_arrive_expect_tx(&sm.full[b], (uint32_t)(fill * W * 16));
    for (int s = 0; s < nseg; ++s)
      bulk_g2s(&sm.buf[b][sm.seg_boff[b][s] * W], rec + (size_t)sm.seg_qb[b][s] * W,
               (uint32_t)(sm.seg_cnt[b][s] * W * 16), &sm.full[b]);
  }
  return fill;
}

constexpr uint64_t kWaitLimitNs = 1000000000ull;  // 1 s per bulk-copy wait

// Runs the staged sweep; `vis(seg_inbox, c, payload, q)` is called for every staged
// candidate of a segment the warp needs.  Returns false if a bulk copy did not complete
// within the wait limit (the caller reports it and the CTA exits).
template <int N, class Visit>
__device__ bool staged_sweep(const KParams& kp, const int32_t* __restrict__ off, const float4* __restrict__ rec,
                             StageSmem<N>& sm, const int* lo, const int* hi, bool valid, Visit&& vis) {
  constexpr int W = Rec<N>::kWords;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int wl[N], wh[N];
  const bool warp_valid = __any_sync(0xffffffffu, valid);
#pragma unroll
  for (int d = 0; d < N; ++d) {
    wl[d] = warp_min_i(valid ? lo[d] : INT_MAX);
    wh[d] = warp_max_i(valid ? hi[d] : INT_MIN);
  }
  if (lane == 0) {
#pragma unroll
    for (int d = 0; d < N; ++d) {
      sm.wlo[warp][d] = wl[d];
      sm.whi[warp][d] = wh[d];
    }
  }
  if (threadIdx.x == 0) {
    mbar_init(&sm.full[0], 1);
    mbar_init(&sm.full[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int any = 0;
#pragma unroll
    for (int d = 0; d < N; ++d) {
      int a = INT_MAX, z = INT_MIN;
      for (int w = 0; w < kChunkWarps; ++w) {
        a = min(a, sm.wlo[w][d]);
        z = max(z, sm.whi[w][d]);
      }
      sm.ulo[d] = a;
      sm.uhi[d] = z;
    }
    for (int w = 0; w < kChunkWarps; ++w) any |= sm.wlo[w][0] != INT_MAX;
    sm.any_valid = any;
  }
  __syncthreads();
  TileIter<N> it;
  bool done = sm.any_valid == 0;
  int has_next = 0;
  if (threadIdx.x == 0) has_next = build_piece<N>(kp, off, rec, sm, it, done, 0) > 0;
  __shared__ int s_has[2];
  if (threadIdx.x == 0) s_has[0] = has_next;
  __syncthreads();
  bool ok = true;
  for (int p = 0; s_has[p & 1]; ++p) {
    const int b = p & 1;
    if (threadIdx.x == 0) s_has[b ^ 1] = build_piece<N>(kp, off, rec, sm, it, done, b ^ 1) > 0;
    if (!mbar_wait_bounded(&sm.full[b], (uint32_t)((p >> 1) & 1), kWaitLimitNs)) {
      ok = false;
      break;
    }
    const int nseg = sm.nseg[b];
    for (int s = 0; s < nseg; ++s) {
      bool wneed = warp_valid, inbox = valid;
#pragma unroll
      for (int d = 0; d < N; ++d) {
        const int vd = sm.seg_v[b][s][d];
        wneed = wneed && vd >= wl[d] && vd <= wh[d];
        inbox = inbox && vd >= lo[d] && vd <= hi[d];
      }
      if (!wneed) continue;
      const float4* sb = &sm.buf[b][sm.seg_boff[b][s] * W];
      const int qb = sm.seg_qb[b][s], cnt = sm.seg_cnt[b][s];
      vis(inbox, sb, qb, cnt);
    }
    __syncthreads();
  }
  return ok;
}

template <int N>
__device__ __forceinline__ void unpack_rec(const float4* r, float* c, float& payload) {
  constexpr int W = Rec<N>::kWords;
  float buf[4 * W];
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const float4 v = r[k];
    buf[4 * k + 0] = v.x;
    buf[4 * k + 1] = v.y;
    buf[4 * k + 2] = v.z;
    buf[4 * k + 3] = v.w;
  }
#pragma unroll
  for (int d = 0; d < N; ++d) c[d] = buf[d];
  payload = buf[Rec<N>::kPayload];
}

// ---- stage 2: local density --------------------------------------------------
// rho_i accumulates, in the reference's candidate order (search-box tiles
// lexicographically, ascending index inside a tile), term = k(d, i, j) * w_j for every
// candidate with d <= dc; candidates beyond dc contribute +-0 and are skipped.
template <int N, int MT>
__global__ void __launch_bounds__(kTileThreads) k_density(const KParams kp, const DevGrid* __restrict__ g,
                                                          const int32_t* __restrict__ off,
                                                          const int32_t* __restrict__ ord,
                                                          const int32_t* __restrict__ chunk_tile,
                                                          const uint32_t* __restrict__ chunk_off,
                                                          const uint32_t* __restrict__ chunk_total,
                                                          const float4* __restrict__ rec_w,
                                                          float4* __restrict__ rec_r, DevStatus* st) {
  using M = Metric<N, MT>;
  constexpr int W = Rec<N>::kWords;
  __shared__ StageSmem<N> sm;
  const int w = blockIdx.x;
  if (w >= (int)*chunk_total) return;
  const int t = chunk_tile[w];
  const int beg = off[t];
  const int start = (w - (int)chunk_off[t]) * kChunk;
  const int cnt = min(kChunk, off[t + 1] - beg - start);
  const int k = threadIdx.x;
  const bool valid = k < cnt;
  const int pos = ord[beg + start + (valid ? k : 0)];
  float x[N], wi;
  load_rec<N>(rec_w, pos, x, wi);
  int hb[N], lo[N], hi[N];
  home_bins<N>(kp, t, hb);
  lane_box<N>(kp, g, x, kp.dc, hb, lo, hi);
  const bool flat = kp.kernel_type == CLUE_KERNEL_FLAT;
  const float kflat = kp.kpar[0];
  const float tdc = kp.t_dc;
  float rho = 0.0f;
  const bool ok = staged_sweep<N>(kp, off, rec_w, sm, lo, hi, valid,
                                  [&](bool inbox, const float4* sb, int qb, int n_) {
    if (flat) {
#pragma unroll 4
      for (int j = 0; j < n_; ++j) {
        float c[N], wj;
        unpack_rec<N>(sb + j * W, c, wj);
        const float s = M::partial(x, c, kp.mpar);
        const float term = (qb + j == pos) ? wj : fmul(kflat, wj);
        if (inbox && s <= tdc) rho = fadd(rho, term);
      }
    } else {
      for (int j = 0; j < n_; ++j) {
        float c[N], wj;
        unpack_rec<N>(sb + j * W, c, wj);
        const float s = M::partial(x, c, kp.mpar);
        if (inbox && s <= tdc) {
          const float kv = (qb + j == pos) ? 1.0f : kernel_value(kp.kernel_type, kp.kpar, M::finish(s));
          rho = fadd(rho, fmul(kv, wj));
        }
      }
    }
  });
  if (!ok) {
    if (threadIdx.x == 0) atomicOr(&st->stage_timeout, 1u);
    return;
  }
  if (valid) store_rec<N>(rec_r, pos, x, rho);
}

// ---- stage 3: nearest higher -------------------------------------------------
// j is higher than i iff rho_j > rho_i or (rho_j == rho_i, rho_j > 0, j > i) with
// original indices; the nearest higher is the first candidate, in the reference's
// order, with the strictly smallest distance <= dm (TIE == CLUE_TIE_REFERENCE), or the
// candidate with the smallest (distance, -rho, index) (TIE == CLUE_TIE_RHO_INDEX).
template <int N, int MT, int TIE>
__global__ void __launch_bounds__(kTileThreads) k_nearest_higher(
    const KParams kp, const DevGrid* __restrict__ g, const int32_t* __restrict__ off,
    const int32_t* __restrict__ ord, const int32_t* __restrict__ chunk_tile,
    const uint32_t* __restrict__ chunk_off, const uint32_t* __restrict__ chunk_total,
    const float4* __restrict__ rec_r, const int32_t* __restrict__ perm, int32_t* __restrict__ nh_s,
    float* __restrict__ delta_s, DevStatus* st) {
  using M = Metric<N, MT>;
  constexpr int W = Rec<N>::kWords;
  __shared__ StageSmem<N> sm;
  const int w = blockIdx.x;
  if (w >= (int)*chunk_total) return;
  const int t = chunk_tile[w];
  const int beg = off[t];
  const int start = (w - (int)chunk_off[t]) * kChunk;
  const int cnt = min(kChunk, off[t + 1] - beg - start);
  const int k = threadIdx.x;
  const bool valid = k < cnt;
  const int pos = ord[beg + start + (valid ? k : 0)];
  float x[N], rho_i;
  load_rec<N>(rec_r, pos, x, rho_i);
  const int orig_i = perm[pos];
  int hb[N], lo[N], hi[N];
  home_bins<N>(kp, t, hb);
  lane_box<N>(kp, g, x, kp.dm, hb, lo, hi);
  const float tdm = kp.t_dm;
  float delta = FLT_MAX, s_best = INFINITY, rho_best = 0.0f;
  int nh = -1, orig_best = INT_MAX;
  const bool ok = staged_sweep<N>(kp, off, rec_r, sm, lo, hi, valid,
                                  [&](bool inbox, const float4* sb, int qb, int n_) {
    if (!__any_sync(0xffffffffu, inbox)) return;
#pragma unroll 4
    for (int j = 0; j < n_; ++j) {
      float c[N], rho_j;
      unpack_rec<N>(sb + j * W, c, rho_j);
      const float s = M::partial(x, c, kp.mpar);
      bool cand = inbox && s <= tdm && rho_j >= rho_i;
      if (TIE == CLUE_TIE_REFERENCE) cand = cand && s < s_best;
      if (cand) {
        const int q = qb + j;
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
  });
  if (!ok) {
    if (threadIdx.x == 0) atomicOr(&st->stage_timeout, 1u);
    return;
  }
  if (valid) {
    nh_s[pos] = nh;
    delta_s[pos] = delta;
  }
  const uint32_t none = __ballot_sync(0xffffffffu, valid && nh < 0);
  if ((threadIdx.x & 31) == 0 && none) atomicAdd(&st->seed_candidates, (uint32_t)__popc(none));
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

inline int chunk_grid(const KParams& kp) { return kp.n / kChunk + kp.ntiles + 1; }

template <int N, int MT>
void launch_density(const KParams& kp, Workspace& ws, cudaStream_t s) {
  k_density<N, MT><<<chunk_grid(kp), kTileThreads, 0, s>>>(kp, ws.grid, ws.offsets, ws.ord_rho, ws.chunk_tile,
                                                            ws.chunk_count, ws.chunk_total, ws.rec_w, ws.rec_r,
                                                            ws.status);
}
template <int N, int MT>
void launch_nh(const KParams& kp, Workspace& ws, cudaStream_t s) {
  if (kp.tiebreak == CLUE_TIE_RHO_INDEX)
    k_nearest_higher<N, MT, CLUE_TIE_RHO_INDEX><<<chunk_grid(kp), kTileThreads, 0, s>>>(
        kp, ws.grid, ws.offsets, ws.ord_nh, ws.chunk_tile, ws.chunk_count, ws.chunk_total, ws.rec_r, ws.perm,
        ws.nh_s, ws.delta_s, ws.status);
  else
    k_nearest_higher<N, MT, CLUE_TIE_REFERENCE><<<chunk_grid(kp), kTileThreads, 0, s>>>(
        kp, ws.grid, ws.offsets, ws.ord_nh, ws.chunk_tile, ws.chunk_count, ws.chunk_total, ws.rec_r, ws.perm,
        ws.nh_s, ws.delta_s, ws.status);
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
  k_order<N><<<kp.ntiles, kTileThreads, 0, s>>>(kp, ws.grid, ws.offsets, ws.rec_w, ws.ord_rho, ws.ord_nh,
                                                ws.chunk_count);
  exclusive_scan(ws.chunk_count, ws.chunk_count, (size_t)kp.ntiles, ws.scan_scratch, ws.chunk_total, s);
  k_chunk_map<<<grid_for(kp.ntiles, 256), 256, 0, s>>>(kp.ntiles, ws.offsets, ws.chunk_count, ws.chunk_tile);

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
  // init, bbox, grid, bin, sort, offsets, gather, order, scan, chunk map, density, nh, seeds, scan,
  // jumps, finalize
  ws.launches += 4 + radix_sort_launches(bits_for((uint32_t)(kp.ntiles - 1))) + 2 + 1 + kScanLaunches + 1 + 3 +
                 kScanLaunches + kJumpLaunches + 1;
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
