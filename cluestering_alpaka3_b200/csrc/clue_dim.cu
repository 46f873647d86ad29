// clue_dim.cu -- the five CLUE stages for points of CLUE_NDIM dimensions.
//
// Compiled once per dimensionality (-DCLUE_NDIM=1..10) so the templates of one
// dimension build in parallel.  Stage map against the reference's serial path
// (include/CLUEstering/core/detail/Clusterer.hpp:134-171):
//   k_bbox_* / k_grid    compute_tile_size        core/detail/ComputeTiles.hpp:13-27
//   k_bin + radix sort   Tiles::fill              data_structures/internal/Tiles.hpp:92-96
//   (k_bin_composite)    (one (tile, Morton) sort on the symmetric density path)
//   k_density            KernelCalculateLocalDensity  core/detail/ClusteringKernels.hpp:66-107
//   k_density_sym /      the same sums in spatial order (exponential / Gaussian kernels):
//   k_density_spatial    symmetric pair sweep or one-sided sweep over Morton blocks
//   k_nearest_higher     KernelCalculateNearestHigher core/detail/ClusteringKernels.hpp:109-212
//   k_seeds              KernelFindClusters       core/detail/ClusteringKernels.hpp:214-244
//   k_jump + k_finalize  Followers::fill + KernelAssignClusters
//                        data_structures/internal/Followers.hpp:27-30,
//                        core/detail/ClusteringKernels.hpp:246-281
//
// One call clusters E independent events (E = 1 for a plain make_clusters).  Event e owns
// points [pt_base, pt_base + pt_count) and global tiles [tile_base, tile_base + ntiles) of its
// own reference grid; tile keys are event-major, so one stable sort of (tile, index) pairs
// orders every event by tile while keeping events contiguous.
//
// Layout in HBM: points are reordered by tile into float4 records {coords..., payload}: by
// ascending index inside a tile for the reference-order density, by Morton code inside a tile
// for the spatial sweeps.  A CTA processes a chunk of 128 home points of one tile (four warps
// of 32).  The reference-order density stages whole candidate tiles into shared memory with
// bulk copies; the spatial sweeps stage one 32-record Morton block per warp, skip blocks whose
// bounding box is out of reach, and read every candidate as one broadcast 16-byte
// shared-memory load (nearest higher) or from its owner lane by shuffle (symmetric density).
#include "clue_internal.h"
#include "clue_tma.cuh"

#ifndef CLUE_NDIM
#error "CLUE_NDIM must be defined"
#endif

namespace clue_b200 {
namespace {

constexpr int kTileThreads = 128;
constexpr int kChunkWarps = kTileThreads / 32;
constexpr int kChunk = kChunkPoints;  // home points per CTA in the density / nearest-higher sweeps
static_assert(kChunkPoints == kTileThreads, "one home point per thread");
// float4 words per staging buffer (12 KiB).  Two 16 KiB buffers held the reference-order density
// to six CTAs per SM by shared memory; at 12 KiB it runs eight (63 registers; measured on the 1M
// 2-D points: 0.630 -> 0.587 ms, the same bits).
constexpr int kStageWords = 768;
constexpr int kMaxSeg = 32;        // tile segments per staged piece

struct InPtrs {
  const float* c[kMaxDim];
  const float* w;
};

// Event tables of one call.
struct Events {
  EvGrid* eg;               // [E]
  const int32_t* pt;        // [E + 1] point offsets
  const int32_t* tile;      // [E + 1] global tile offsets
  const int32_t* chunk_ev;  // [n / 1024 + 1] event of the first point of every 1024-point chunk
};
constexpr int kEvChunkShift = 10;

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

// Largest e in [0, E) with base[e] <= x.
__device__ __forceinline__ int find_event(const int32_t* __restrict__ base, int E, int x) {
  int lo = 0, hi = E - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(base + mid) <= x)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
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

// Search box of one point in "virtual" bins: the reference's [getBin(x - r), getBin(x + r)]
// (TilesView.hpp:72-82, wrapped boxes extended by nperdim), shifted down by nperdim when a
// wrapped box starts above the home bin, so that every lane of a warp expresses its box
// in the same frame around the home tile.  The tile of virtual bin v is v mod nperdim.
template <int N>
__device__ __forceinline__ void lane_box(const KParams& kp, const EvGrid* __restrict__ g, const float* x,
                                         float r, const int* hb, int* lo, int* hi) {
  const int npd = g->nperdim;
#pragma unroll
  for (int d = 0; d < N; ++d) {
    const bool wr = kp.wrapped[d] != 0;
    int a = get_bin(fsub(x[d], r), g->mn[d], g->mx[d], g->size[d], wr, npd);
    int b = get_bin(fadd(x[d], r), g->mn[d], g->mx[d], g->size[d], wr, npd);
    if (wr && a > b) b += npd;
    if (wr && a > hb[d]) {
      a -= npd;
      b -= npd;
    }
    lo[d] = a;
    hi[d] = b;
  }
}

template <int N>
__device__ __forceinline__ void home_bins(const EvGrid* __restrict__ g, int t, int* hb) {
  const int lt = t - g->tile_base;
#pragma unroll
  for (int d = 0; d < N; ++d) hb[d] = (lt / g->stride[d]) % g->nperdim;
}

__device__ __forceinline__ int wrap_bin(int v, int npd) {
  int b = v % npd;
  return b < 0 ? b + npd : b;
}

// Box of one warp's 32 records (lanes past the end repeat a record of the block): lo[N],
// hi[N] and the largest payload, written as block b.
template <int N>
__device__ __forceinline__ void write_block_box(float4* __restrict__ blk, int b, const float* x, float pl) {
  constexpr int BW = Blk<N>::kWords;
  const int lane = threadIdx.x & 31;
  float out[4 * BW];
#pragma unroll
  for (int k = 0; k < 4 * BW; ++k) out[k] = 0.0f;
#pragma unroll
  for (int d = 0; d < N; ++d) {
    float a = x[d], z = x[d];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a = fminf(a, __shfl_xor_sync(0xffffffffu, a, o));
      z = fmaxf(z, __shfl_xor_sync(0xffffffffu, z, o));
    }
    out[d] = a;
    out[N + d] = z;
  }
  float pm = pl;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) pm = fmaxf(pm, __shfl_xor_sync(0xffffffffu, pm, o));
  out[2 * N] = pm;
  if (lane < BW) {
    float4 v;
#pragma unroll
    for (int k = 0; k < BW; ++k)
      if (k == lane) v = make_float4(out[4 * k], out[4 * k + 1], out[4 * k + 2], out[4 * k + 3]);
    blk[(size_t)b * BW + lane] = v;
  }
}

// Bounding box (and largest payload) of every 32 consecutive tile-sorted records.
template <int N>
__global__ void __launch_bounds__(256) k_block_bbox(const float4* __restrict__ rec, int n, float4* __restrict__ blk) {
  const int lane = threadIdx.x & 31;
  const int nblk = (n + 31) >> 5;
  const int wstride = (gridDim.x * blockDim.x) >> 5;
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nblk; b += wstride) {
    const int q = (b << 5) + lane;
    float x[N], pl;
    load_rec<N>(rec, q < n ? q : b << 5, x, pl);  // lanes past the end duplicate the first record
    write_block_box<N>(blk, b, x, pl);
  }
}

// Bounding boxes of super-blocks (32 consecutive blocks = 1024 records) from the block boxes.
template <int N>
__global__ void __launch_bounds__(256) k_superblock_bbox(const float4* __restrict__ blk, int n,
                                                         float4* __restrict__ sblk) {
  constexpr int BW = Blk<N>::kWords;
  const int lane = threadIdx.x & 31;
  const int nblk = (n + 31) >> 5;
  const int nsb = (nblk + 31) >> 5;
  const int wstride = (gridDim.x * blockDim.x) >> 5;
  for (int sb = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; sb < nsb; sb += wstride) {
    const int b = min((sb << 5) + lane, nblk - 1);
    float v[4 * BW];
#pragma unroll
    for (int k = 0; k < BW; ++k) {
      const float4 t4 = __ldg(blk + (size_t)b * BW + k);
      v[4 * k] = t4.x;
      v[4 * k + 1] = t4.y;
      v[4 * k + 2] = t4.z;
      v[4 * k + 3] = t4.w;
    }
#pragma unroll
    for (int d = 0; d < N; ++d) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        v[d] = fminf(v[d], __shfl_xor_sync(0xffffffffu, v[d], o));
        v[N + d] = fmaxf(v[N + d], __shfl_xor_sync(0xffffffffu, v[N + d], o));
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[2 * N] = fmaxf(v[2 * N], __shfl_xor_sync(0xffffffffu, v[2 * N], o));
    if (lane < BW) {
      float4 out;
#pragma unroll
      for (int k = 0; k < BW; ++k)
        if (k == lane) out = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
      sblk[(size_t)sb * BW + lane] = out;
    }
  }
}

template <int N>
__device__ __forceinline__ void load_box(const float4* __restrict__ a, int i, float* bb) {
  constexpr int BW = Blk<N>::kWords;
#pragma unroll
  for (int k = 0; k < BW; ++k) {
    const float4 t4 = __ldg(a + (size_t)i * BW + k);
    bb[4 * k] = t4.x;
    bb[4 * k + 1] = t4.y;
    bb[4 * k + 2] = t4.z;
    bb[4 * k + 3] = t4.w;
  }
}

// A block of up to 32 consecutive records staged in the warp's shared-memory slot: lane k
// copies record p0 + k; smem_rec() then reads record j with broadcast loads (every lane reads
// the same address), one 16-byte load per record word.
// With sq / mq given, the records' tile-sorted positions mq[p0 + k] are staged in sq as well.
template <int N>
__device__ __forceinline__ void stage_block(float4* sm, const float4* __restrict__ rec, int p0, int cnt,
                                            int32_t* sq = nullptr, const int32_t* __restrict__ mq = nullptr) {
  constexpr int W = Rec<N>::kWords;
  const int lane = threadIdx.x & 31;
  __syncwarp();  // the previous block's readers are done
  if (lane < cnt) {
#pragma unroll
    for (int k = 0; k < W; ++k) sm[lane * W + k] = __ldg(rec + (size_t)(p0 + lane) * W + k);
    if (sq) sq[lane] = __ldg(mq + p0 + lane);
  }
  __syncwarp();
}
template <int N>
__device__ __forceinline__ void smem_rec(const float4* sm, int j, float* c, float& payload) {
  constexpr int W = Rec<N>::kWords;
  float r[4 * W];
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const float4 v = sm[j * W + k];
    r[4 * k] = v.x;
    r[4 * k + 1] = v.y;
    r[4 * k + 2] = v.z;
    r[4 * k + 3] = v.w;
  }
#pragma unroll
  for (int d = 0; d < N; ++d) c[d] = r[d];
  payload = r[Rec<N>::kPayload];
}

// Spatial sweep of one warp over the Morton-ordered records of its search-box tiles (any
// order: the own tile first, then the union of the warp's boxes lexicographically).  Super-blocks
// and blocks whose bounding box lies beyond bound() for every lane, or whose largest payload is
// below pmin for every lane, are skipped; vis(p0, p1, inbox, lexpos) gets the rest.  lexpos is
// the tile's position in this lane's reference iteration order (lexicographic over its box).
// With PREVISIT, p_home is the lane's own Morton position: the blocks around the warp's own
// positions in the home tile are visited first (the nearest candidates are there, which tightens
// bound() for the rest of the sweep) and skipped later.  Without it every tile's blocks are
// visited in Morton order, so order-sensitive sums do not depend on how records are aligned to
// blocks (a batch and a single event give identical results).
template <int N, class M, bool PREVISIT, class Bound, class Visit>
__device__ __forceinline__ void spatial_sweep(const KParams& kp, const EvGrid* __restrict__ g,
                                              const int32_t* __restrict__ off, const int* hb, const int* lo,
                                              const int* hi, bool valid, const float* x,
                                              const float4* __restrict__ blk, const float4* __restrict__ sblk,
                                              float pmin, int p_home, Bound&& bound, Visit&& vis) {
  constexpr int BW = Blk<N>::kWords;
  const int ph_lo = warp_min_i(valid ? p_home : INT_MAX);
  const int ph_hi = warp_max_i(valid ? p_home : INT_MIN);
  int skip_lo = 1, skip_hi = 0;  // home-tile blocks already visited
  int wl[N], wh[N];
#pragma unroll
  for (int d = 0; d < N; ++d) {
    wl[d] = warp_min_i(valid ? lo[d] : INT_MAX);
    wh[d] = warp_max_i(valid ? hi[d] : INT_MIN);
  }
  int64_t ext[N];
  {
    int64_t m = 1;
#pragma unroll
    for (int d = N - 1; d >= 0; --d) {
      ext[d] = m;
      m *= (int64_t)(hi[d] - lo[d] + 1);
    }
  }
  // one tile of the search boxes: its super-blocks and blocks that some lane may need
  auto visit_tile = [&](const int* v, bool is_home_tile) {
    bool inbox = valid;
    int u = g->tile_base;
    int64_t lexpos = 0;
#pragma unroll
    for (int d = 0; d < N; ++d) {
      inbox = inbox && v[d] >= lo[d] && v[d] <= hi[d];
      u += g->stride[d] * wrap_bin(v[d], g->nperdim);
      lexpos += (int64_t)(v[d] - lo[d]) * ext[d];
    }
    if (!__any_sync(0xffffffffu, inbox)) return;
    const int pb = off[u], pe = off[u + 1];
    if (pb >= pe) return;
    const bool home_tile = PREVISIT && is_home_tile;
    if (home_tile && ph_lo <= ph_hi) {
      skip_lo = max(pb >> 5, (ph_lo >> 5) - 1);
      skip_hi = min((pe - 1) >> 5, (ph_hi >> 5) + 1);
      for (int b = skip_lo; b <= skip_hi; ++b) {
        const int q0 = max(pb, b << 5), q1 = min(pe, (b + 1) << 5);
        bool need = inbox;
        if (kp.lb_ok) {
          float bb[4 * BW];
          load_box<N>(blk, b, bb);
          need = need && M::lower(x, bb, bb + N, kp.mpar) <= bound() && bb[2 * N] >= pmin;
        }
        if (__any_sync(0xffffffffu, need)) vis(q0, q1, need, lexpos);
      }
    }
    for (int sbk = pb >> 10; sbk <= (pe - 1) >> 10; ++sbk) {
      if (kp.lb_ok) {
        float bb[4 * BW];
        load_box<N>(sblk, sbk, bb);
        const bool need = inbox && M::lower(x, bb, bb + N, kp.mpar) <= bound() && bb[2 * N] >= pmin;
        if (!__any_sync(0xffffffffu, need)) continue;
      }
      const int sp0 = max(pb, sbk << 10), sp1 = min(pe, (sbk + 1) << 10);
      for (int b = sp0 >> 5; b <= (sp1 - 1) >> 5; ++b) {
        if (home_tile && b >= skip_lo && b <= skip_hi) continue;
        bool need = inbox;
        if (kp.lb_ok) {
          float bb[4 * BW];
          load_box<N>(blk, b, bb);
          need = need && M::lower(x, bb, bb + N, kp.mpar) <= bound() && bb[2 * N] >= pmin;
        }
        if (!__any_sync(0xffffffffu, need)) continue;
        vis(max(sp0, b << 5), min(sp1, (b + 1) << 5), need, lexpos);
      }
    }
  };
  visit_tile(hb, true);
  int v[N];
  if (PREVISIT && N <= 3) {
    // the other tiles ring by ring around the home tile (nearest first, so the bound shrinks
    // early and far blocks are skipped), lexicographic inside a ring
    int R = 0;
#pragma unroll
    for (int d = 0; d < N; ++d) R = max(R, max(hb[d] - wl[d], wh[d] - hb[d]));
    for (int r = 1; r <= R; ++r) {
#pragma unroll
      for (int d = 0; d < N; ++d) v[d] = wl[d];
      while (true) {
        int ring = 0;
#pragma unroll
        for (int d = 0; d < N; ++d) ring = max(ring, abs(v[d] - hb[d]));
        if (ring == r) visit_tile(v, false);
        int d = N - 1;
        for (; d >= 0; --d) {
          if (v[d] < wh[d]) {
            ++v[d];
            break;
          }
          v[d] = wl[d];
        }
        if (d < 0) break;
      }
    }
  } else {
    // the other tiles of the union box lexicographically
#pragma unroll
    for (int d = 0; d < N; ++d) v[d] = wl[d];
    while (true) {
      bool is_home = true;
#pragma unroll
      for (int d = 0; d < N; ++d) is_home = is_home && v[d] == hb[d];
      if (!is_home) visit_tile(v, false);
      int d = N - 1;
      for (; d >= 0; --d) {
        if (v[d] < wh[d]) {
          ++v[d];
          break;
        }
        v[d] = wl[d];
      }
      if (d < 0) break;
    }
  }
}

// Walks the staged segment [qb, qb + n) block by block (blocks are 32 aligned records) and
// calls inner(j0, j1) for the parts whose block some lane of the warp may need: the lane's
// box holds the tile, the block's box lower bound is within `bound` (strictly below it when
// `strict`) and the block's largest payload reaches `pmin`.
template <int N, class M, class Inner>
__device__ __forceinline__ void scan_blocks(const KParams& kp, const float4* __restrict__ blk, const float* x,
                                            bool inbox, float bound, bool strict, float pmin, int qb, int n,
                                            Inner&& inner) {
  constexpr int BW = Blk<N>::kWords;
  int j = 0;
  while (j < n) {
    const int b = (qb + j) >> 5;
    const int je = min(n, ((b + 1) << 5) - qb);
    bool need = inbox;
    if (kp.lb_ok) {
      float buf[4 * BW];
#pragma unroll
      for (int k = 0; k < BW; ++k) {
        const float4 v = __ldg(blk + (size_t)b * BW + k);
        buf[4 * k] = v.x;
        buf[4 * k + 1] = v.y;
        buf[4 * k + 2] = v.z;
        buf[4 * k + 3] = v.w;
      }
      const float lb = M::lower(x, buf, buf + N, kp.mpar);
      need = need && (strict ? lb < bound : lb <= bound) && buf[2 * N] >= pmin;
    }
    if (__any_sync(0xffffffffu, need)) inner(j, je);
    j = je;
  }
}

// ---- stage 1: bounding box, grid, bins --------------------------------------

// Resets the per-call state; for a plain call also writes the event table of its one event.
template <int N>
__global__ void k_init(const KParams kp, Events ev, int32_t* ev_pt, int32_t* ev_tile, DevStatus* st) {
  if (blockIdx.x == 0) {
    uint32_t* s = reinterpret_cast<uint32_t*>(st);
    for (int k = threadIdx.x; k < (int)(sizeof(DevStatus) / 4); k += blockDim.x) s[k] = 0u;
  }
  const int stride = gridDim.x * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < kp.n_events; e += stride) {
    EvGrid& g = ev.eg[e];
    for (int d = 0; d < kMaxDim; ++d) {
      g.enc_min[d] = 0xffffffffu;
      g.enc_max[d] = 0u;
    }
    g.seed_candidates = 0;
    g.wmax_bits = 0u;
    if (kp.n_events == 1) {
      g.nperdim = kp.nperdim0;
      g.ntiles = kp.ntiles;
      g.tile_base = 0;
      g.pt_base = 0;
      g.pt_count = kp.n;
      for (int d = 0; d < kMaxDim; ++d) g.stride[d] = kp.stride0[d];
      ev_pt[0] = 0;
      ev_pt[1] = kp.n;
      ev_tile[0] = 0;
      ev_tile[1] = kp.ntiles;
    }
  }
}

// Bounding box and largest |weight| of a single event: per-thread, warp and block reductions,
// then one set of atomics per CTA.
template <int N>
__global__ void __launch_bounds__(256) k_bbox_single(InPtrs in, int n, EvGrid* g, DevStatus* st) {
  uint32_t emn[N], emx[N];
#pragma unroll
  for (int d = 0; d < N; ++d) {
    emn[d] = 0xffffffffu;
    emx[d] = 0u;
  }
  bool bad = false;
  uint32_t wmax = 0u;
  auto take = [&](const float* x, float w) {
#pragma unroll
    for (int d = 0; d < N; ++d) {
      bad |= !isfinite(x[d]);
      const uint32_t e = enc_float(x[d]);
      emn[d] = min(emn[d], e);
      emx[d] = max(emx[d], e);
    }
    bad |= !isfinite(w);
    wmax = max(wmax, __float_as_uint(fabsf(w)));
  };
  const int stride = gridDim.x * blockDim.x;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  // four points per thread and step, their loads in flight together
  for (; i + 3 * stride < n; i += 4 * stride) {
    float x[4][N], w[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
#pragma unroll
      for (int d = 0; d < N; ++d) x[k][d] = in.c[d][i + k * stride];
      w[k] = in.w[i + k * stride];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) take(x[k], w[k]);
  }
  for (; i < n; i += stride) {
    float x[N];
#pragma unroll
    for (int d = 0; d < N; ++d) x[d] = in.c[d][i];
    take(x, in.w[i]);
  }
  // warp, then block reduction: one set of atomics per CTA (same-address atomics from every
  // warp of a large grid serialise at the L2)
  __shared__ uint32_t s_red[8][2 * N + 2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < N; ++d) {
    emn[d] = warp_min_u(emn[d]);
    emx[d] = warp_max_u(emx[d]);
  }
  wmax = warp_max_u(wmax);
  const bool wbad = __any_sync(0xffffffffu, bad);
  if (lane == 0) {
#pragma unroll
    for (int d = 0; d < N; ++d) {
      s_red[warp][d] = emn[d];
      s_red[warp][N + d] = emx[d];
    }
    s_red[warp][2 * N] = wmax;
    s_red[warp][2 * N + 1] = wbad ? 1u : 0u;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    for (int w = 1; w < nw; ++w) {
#pragma unroll
      for (int d = 0; d < N; ++d) {
        s_red[0][d] = min(s_red[0][d], s_red[w][d]);
        s_red[0][N + d] = max(s_red[0][N + d], s_red[w][N + d]);
      }
      s_red[0][2 * N] = max(s_red[0][2 * N], s_red[w][2 * N]);
      s_red[0][2 * N + 1] |= s_red[w][2 * N + 1];
    }
#pragma unroll
    for (int d = 0; d < N; ++d) {
      atomicMin(&g->enc_min[d], s_red[0][d]);
      atomicMax(&g->enc_max[d], s_red[0][N + d]);
    }
    atomicMax(&g->wmax_bits, s_red[0][2 * N]);
    if (s_red[0][2 * N + 1]) atomicOr(&st->nonfinite, 1u);
  }
}

// Event of point i.  Events are contiguous, ascending point ranges: chunk_ev holds the event of
// the first point of i's 1024-point chunk, and the events that start later inside the chunk are
// stepped over (a few steps at most for events of 100 points and more), which replaces a binary
// search of about log2(E) dependent loads.  Without the table (one event, or a workspace
// without it) the binary search.
__device__ __forceinline__ int event_of(const int32_t* __restrict__ ev_pt, const int32_t* __restrict__ chunk_ev,
                                        int E, int i) {
  if (E == 1) return 0;
  if (!chunk_ev) return find_event(ev_pt, E, i);
  int e = __ldg(chunk_ev + (i >> kEvChunkShift));
  while (__ldg(ev_pt + e + 1) <= i) ++e;
  return e;
}

// Event of point i, looked up once per warp when the warp's points share one event (the usual
// case: events are contiguous ranges of points) and per lane otherwise.
__device__ __forceinline__ int warp_event(const int32_t* __restrict__ ev_pt, const int32_t* __restrict__ chunk_ev,
                                          int E, int i, bool active, bool& uniform) {
  const unsigned am = __activemask();
  const int first = __shfl_sync(am, i, __ffs(am) - 1);
  const int last = __shfl_sync(am, i, 31 - __clz(am));
  const int e0 = event_of(ev_pt, chunk_ev, E, first);
  uniform = last < ev_pt[e0 + 1];
  return uniform ? e0 : (active ? event_of(ev_pt, chunk_ev, E, i) : e0);
}

// The chunk table of event_of: chunk c (points [1024 c, 1024 c + 1024)) gets the event that
// holds its first point; every non-empty event writes the chunks whose first point it holds.
__global__ void __launch_bounds__(256) k_event_chunks(int E, const int32_t* __restrict__ ev_pt,
                                                      int32_t* __restrict__ chunk_ev) {
  const int stride = gridDim.x * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += stride) {
    const int a = ev_pt[e], b = ev_pt[e + 1];
    if (a >= b) continue;
    for (int c = (a + (1 << kEvChunkShift) - 1) >> kEvChunkShift; c <= (b - 1) >> kEvChunkShift; ++c) chunk_ev[c] = e;
  }
}

// Bounding box and largest |weight| of many events.  Every warp takes spans of `span`
// consecutive points (a multiple of 32) and keeps a running box while its 32-point groups stay
// inside one event, so a span inside an event costs one warp reduction and 2N + 1 atomics; a
// group that straddles events falls back to per-lane atomics.
template <int N>
__global__ void __launch_bounds__(256) k_bbox_events(InPtrs in, int n, int E, const int32_t* __restrict__ ev_pt,
                                                     const int32_t* __restrict__ chunk_ev, EvGrid* eg, DevStatus* st,
                                                     int span) {
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  bool bad = false;
  for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * span; base < n; base += nwarps * span) {
    const int end = min(n, base + span);
    {
      // the usual case, a span inside one event: four 32-point groups per step with their loads
      // in flight together, one warp reduction and 2N + 1 atomics
      const int e0 = event_of(ev_pt, chunk_ev, E, base);
      if (ev_pt[e0 + 1] >= end) {
        uint32_t bmn[N], bmx[N], bw = 0;
#pragma unroll
        for (int d = 0; d < N; ++d) {
          bmn[d] = 0xffffffffu;
          bmx[d] = 0;
        }
        for (int i0 = base; i0 < end; i0 += 128) {
          float xs[4][N], wv[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int i = min(i0 + 32 * k + lane, end - 1);  // lanes past the end repeat the last point
#pragma unroll
            for (int d = 0; d < N; ++d) xs[k][d] = in.c[d][i];
            wv[k] = in.w[i];
          }
#pragma unroll
          for (int k = 0; k < 4; ++k) {
#pragma unroll
            for (int d = 0; d < N; ++d) {
              bad |= !isfinite(xs[k][d]);
              const uint32_t u = enc_float(xs[k][d]);
              bmn[d] = min(bmn[d], u);
              bmx[d] = max(bmx[d], u);
            }
            bad |= !isfinite(wv[k]);
            bw = max(bw, __float_as_uint(fabsf(wv[k])));
          }
        }
#pragma unroll
        for (int d = 0; d < N; ++d) {
          bmn[d] = warp_min_u(bmn[d]);
          bmx[d] = warp_max_u(bmx[d]);
        }
        bw = warp_max_u(bw);
        if (lane == 0) {
#pragma unroll
          for (int d = 0; d < N; ++d) {
            atomicMin(&eg[e0].enc_min[d], bmn[d]);
            atomicMax(&eg[e0].enc_max[d], bmx[d]);
          }
          atomicMax(&eg[e0].wmax_bits, bw);
        }
        continue;
      }
    }
    int cur = -1;  // event of the running box (warp-uniform), -1: none
    uint32_t amn[N], amx[N], aw = 0;
#pragma unroll
    for (int d = 0; d < N; ++d) amn[d] = amx[d] = 0;
    auto flush = [&]() {
#pragma unroll
      for (int d = 0; d < N; ++d) {
        amn[d] = warp_min_u(amn[d]);
        amx[d] = warp_max_u(amx[d]);
      }
      aw = warp_max_u(aw);
      if (lane == 0) {
#pragma unroll
        for (int d = 0; d < N; ++d) {
          atomicMin(&eg[cur].enc_min[d], amn[d]);
          atomicMax(&eg[cur].enc_max[d], amx[d]);
        }
        atomicMax(&eg[cur].wmax_bits, aw);
      }
    };
    for (int i0 = base; i0 < end; i0 += 32) {
      const int i = min(i0 + lane, end - 1);  // lanes past the end repeat the last point
      bool uniform;
      const int e = warp_event(ev_pt, chunk_ev, E, i, true, uniform);
      uint32_t emn[N];
#pragma unroll
      for (int d = 0; d < N; ++d) {
        const float x = in.c[d][i];
        bad |= !isfinite(x);
        emn[d] = enc_float(x);
      }
      const float w = in.w[i];
      bad |= !isfinite(w);
      const uint32_t wm = __float_as_uint(fabsf(w));
      if (uniform && e == cur) {
#pragma unroll
        for (int d = 0; d < N; ++d) {
          amn[d] = min(amn[d], emn[d]);
          amx[d] = max(amx[d], emn[d]);
        }
        aw = max(aw, wm);
        continue;
      }
      if (cur >= 0) flush();
      if (uniform) {
        cur = e;
#pragma unroll
        for (int d = 0; d < N; ++d) amn[d] = amx[d] = emn[d];
        aw = wm;
      } else {
        cur = -1;
#pragma unroll
        for (int d = 0; d < N; ++d) {
          atomicMin(&eg[e].enc_min[d], emn[d]);
          atomicMax(&eg[e].enc_max[d], emn[d]);
        }
        atomicMax(&eg[e].wmax_bits, wm);
      }
    }
    if (cur >= 0) flush();
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&st->nonfinite, 1u);
}

// Tile size (max - min) / nperdim in FP32 (ComputeTiles.hpp:20-23), per event.
template <int N>
__global__ void k_grid(int E, EvGrid* eg) {
  const int stride = gridDim.x * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += stride) {
    EvGrid& g = eg[e];
#pragma unroll
    for (int d = 0; d < N; ++d) {
      const float mn = dec_float(g.enc_min[d]);
      const float mx = dec_float(g.enc_max[d]);
      g.mn[d] = mn;
      g.mx[d] = mx;
      g.size[d] = fdiv(fsub(mx, mn), (float)g.nperdim);
    }
  }
}

// Event-major global tile key of every point (TilesView.hpp:53-61, exact integers).
template <int N>
__global__ void __launch_bounds__(256) k_bin(const KParams kp, InPtrs in, Events ev,
                                             uint32_t* __restrict__ keys) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kp.n; i += stride) {
    bool uniform;
    const EvGrid* g = ev.eg + warp_event(ev.pt, ev.chunk_ev, kp.n_events, i, true, uniform);
    int gb = g->tile_base;
#pragma unroll
    for (int d = 0; d < N; ++d)
      gb += g->stride[d] * get_bin(in.c[d][i], g->mn[d], g->mx[d], g->size[d], kp.wrapped[d] != 0, g->nperdim);
    keys[i] = (uint32_t)gb;
  }
}

template <int N>
__global__ void __launch_bounds__(256) k_gather(InPtrs in, int n, const int32_t* __restrict__ perm,
                                                float4* __restrict__ rec_w, DevStatus* st,
                                                int32_t* __restrict__ ida, int32_t* __restrict__ idb) {
  const int stride = gridDim.x * blockDim.x;
  for (int pos = blockIdx.x * blockDim.x + threadIdx.x; pos < n; pos += stride) {
    if (ida) ida[pos] = idb[pos] = pos;  // identity orders, when asked for
    const int i = perm[pos];
    if (dcheck_bad(st, i, n, kChkGatherPerm)) continue;
    float x[N];
#pragma unroll
    for (int d = 0; d < N; ++d) x[d] = in.c[d][i];
    store_rec<N>(rec_w, pos, x, in.w[i]);
  }
}

// Morton bits per dimension of the fine order inside a tile (16 bits per key in total, so the
// order -- and the spatial-order sums -- depend only on the tile's own points).
template <int N>
struct MortonBits {
  static constexpr int kPerDim = N == 1 ? 16 : (16 / N > 0 ? 16 / N : 1);
  static constexpr int kBits = kPerDim * N;
};

// Morton bits the tile-internal order sorts on: the top bits of the interleaved code, a fixed
// count per dimension, so an event's record order (and with it the bits of its densities) never
// depends on the batch around it or on which of the two sort paths built it.  Two dimensions keep
// 15 of 16 bits, so a (tile, Morton) composite key fits 32 bits up to 2^17 tiles.
template <int N>
struct MortonSortBits {
  static constexpr int kBits = N == 2 ? 15 : MortonBits<N>::kBits;
};

// The bits of c (below 2^kPerDim) moved to positions 0, N, 2N, ... of a Morton code.
template <int N>
__device__ __forceinline__ uint32_t spread_bits(uint32_t c) {
  if constexpr (N == 1) {
    return c;
  } else if constexpr (N == 2) {  // 8 bits
    c = (c | (c << 4)) & 0x0f0fu;
    c = (c | (c << 2)) & 0x3333u;
    return (c | (c << 1)) & 0x5555u;
  } else {
    uint32_t m = 0;
#pragma unroll
    for (int bit = 0; bit < MortonBits<N>::kPerDim; ++bit) m |= ((c >> bit) & 1u) << (bit * N);
    return m;
  }
}

// Morton key of every tile-sorted record inside its tile (tile keys are read from tile_keys).
template <int N>
__global__ void __launch_bounds__(256) k_morton_keys(const KParams kp, Events ev, const float4* __restrict__ rec,
                                                     const uint32_t* __restrict__ tile_keys,
                                                     uint32_t* __restrict__ keys) {
  constexpr int bpd = MortonBits<N>::kPerDim;
  const float scale = (float)(1u << bpd);
  const int stride = gridDim.x * blockDim.x;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < kp.n; q += stride) {
    const uint32_t t = tile_keys[q];
    bool uniform;  // tile-sorted positions are event-major: event e holds [ev.pt[e], ev.pt[e + 1])
    const EvGrid* g = ev.eg + warp_event(ev.pt, ev.chunk_ev, kp.n_events, q, true, uniform);
    int hb[N];
    home_bins<N>(g, (int)t, hb);
    float x[N], pl;
    load_rec<N>(rec, q, x, pl);
    uint32_t m = 0;
#pragma unroll
    for (int d = 0; d < N; ++d) {
      // position inside the tile from getBin's quotient, as in k_bin_composite
      const float xd = kp.wrapped[d] ? normalize_coord(x[d], g->mn[d], g->mx[d]) : x[d];
      const float qd = fdiv(fsub(xd, g->mn[d]), g->size[d]);
      int c = g->size[d] > 0.0f ? (int)((qd - (float)hb[d]) * scale) : 0;
      c = c < 0 ? 0 : (c > (1 << bpd) - 1 ? (1 << bpd) - 1 : c);
      m |= spread_bits<N>((uint32_t)c) << d;
    }
    keys[q] = m >> (MortonBits<N>::kBits - MortonSortBits<N>::kBits);
  }
}

// Tile key of every record in the Morton-sorted order (second, stable sort by tile).
__global__ void __launch_bounds__(256) k_tile_of(const uint32_t* __restrict__ tile_keys,
                                                 const int32_t* __restrict__ mq, int n, uint32_t* __restrict__ out) {
  const int stride = gridDim.x * blockDim.x;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) out[p] = tile_keys[mq[p]];
}

// Composite key (tile << mbits | Morton code of the point inside its tile, top mbits bits) of
// every point, for the single sort that yields the (tile, Morton) order directly.  Every thread
// takes four points per step, their coordinates loaded together before the keys are computed.
template <int N>
__global__ void __launch_bounds__(256) k_bin_composite(const KParams kp, InPtrs in, Events ev, int mbits,
                                                       uint32_t* __restrict__ keys) {
  constexpr int bpd = MortonBits<N>::kPerDim;
  constexpr int kPer = 4;
  const float scale = (float)(1u << bpd);
  for (int base = blockIdx.x * (256 * kPer); base < kp.n; base += gridDim.x * 256 * kPer) {
    float xs[kPer][N];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int i = min(base + k * 256 + (int)threadIdx.x, kp.n - 1);
#pragma unroll
      for (int d = 0; d < N; ++d) xs[k][d] = in.c[d][i];
    }
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int i = base + k * 256 + (int)threadIdx.x;
      if (i >= kp.n) break;
      bool uniform;
      const EvGrid* g = ev.eg + warp_event(ev.pt, ev.chunk_ev, kp.n_events, i, true, uniform);
      int gb = g->tile_base;
      uint32_t m = 0;
#pragma unroll
      for (int d = 0; d < N; ++d) {
        // getBin without wrapped coordinates (the composite sort is only taken without them):
        // the quotient also places the point inside its tile for the Morton code
        const float q = fdiv(fsub(xs[k][d], g->mn[d]), g->size[d]);
        int b = cvt_i32(q);
        b = b < g->nperdim - 1 ? b : g->nperdim - 1;
        b = b > 0 ? b : 0;
        gb += g->stride[d] * b;
        int c = g->size[d] > 0.0f ? (int)((q - (float)b) * scale) : 0;
        c = c < 0 ? 0 : (c > (1 << bpd) - 1 ? (1 << bpd) - 1 : c);
        m |= spread_bits<N>((uint32_t)c) << d;
      }
      keys[i] = ((uint32_t)gb << mbits) | (m >> (MortonBits<N>::kBits - mbits));
    }
  }
}

// Inverse permutation: minv[mq[p]] = p.
__global__ void __launch_bounds__(256) k_invert(const int32_t* __restrict__ mq, int n, int32_t* __restrict__ minv) {
  const int stride = gridDim.x * blockDim.x;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) minv[mq[p]] = p;
}

template <int N>
__global__ void __launch_bounds__(256) k_gather_morton(const float4* __restrict__ rec_r, int n,
                                                       const int32_t* __restrict__ mq, float4* __restrict__ rec_m) {
  constexpr int W = Rec<N>::kWords;
  const int stride = gridDim.x * blockDim.x;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
    const int q = mq[p];
#pragma unroll
    for (int k = 0; k < W; ++k) rec_m[(size_t)p * W + k] = __ldg(rec_r + (size_t)q * W + k);
  }
}

// ---- work orders and chunks --------------------------------------------------
// Home points of every tile are taken in the fine Morton order of the tile (so 32 consecutive
// points are close together at the data's own density scale).  For the one-sided density
// sweeps they are also stably partitioned by search-box signature -- which neighbour tiles the
// box of radius dc reaches, 2 bits per dimension -- so the 32 lanes of a warp share one box.
// (The nearest-higher sweep and the symmetric density sweep take the Morton order as it is.)
// The orders are cut into chunks of kChunk home points; one CTA processes one chunk, so a heavy
// tile is spread over many CTAs.  One CTA per tile; warp w partitions the w-th quarter of the
// tile and the quarters are concatenated per key, which keeps the partition stable.
template <int N>
__global__ void __launch_bounds__(kTileThreads) k_order(const KParams kp, Events ev,
                                                        const int32_t* __restrict__ off,
                                                        const float4* __restrict__ rec_w,
                                                        const int32_t* __restrict__ mq,
                                                        int32_t* __restrict__ ord_rho,
                                                        uint32_t* __restrict__ chunk_count) {
  constexpr int K = N <= 4 ? (1 << (2 * N)) : 1;
  __shared__ uint32_t s_cnt[kChunkWarps][K];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  for (int t = blockIdx.x; t < kp.ntiles; t += gridDim.x) {
    const int beg = off[t], end = off[t + 1];
    if (threadIdx.x == 0) chunk_count[t] = (uint32_t)((end - beg + kChunk - 1) / kChunk);
    if (beg == end) continue;
    const EvGrid* g = ev.eg + find_event(ev.tile, kp.n_events, t);
    int hb[N];
    home_bins<N>(g, t, hb);
    const int quarter = ((end - beg + kChunkWarps - 1) / kChunkWarps + 31) & ~31;
    const int wb = min(end, beg + warp * quarter), we = min(end, wb + quarter);
    for (int e = threadIdx.x; e < kChunkWarps * K; e += blockDim.x) (&s_cnt[0][0])[e] = 0;
    __syncthreads();
    for (int pass = 0; pass < 2; ++pass) {
      for (int base = wb; base < we; base += 32) {
        const int p = base + lane;
        const bool valid = p < we;
        const int q = valid ? mq[p] : mq[beg];
        int key = 0;
        if (K > 1) {
          float x[N], pl;
          load_rec<N>(rec_w, q, x, pl);
          int lo[N], hi[N];
          lane_box<N>(kp, g, x, kp.dc, hb, lo, hi);
#pragma unroll
          for (int d = 0; d < N; ++d) key |= ((lo[d] < hb[d] ? 1 : 0) | (hi[d] > hb[d] ? 2 : 0)) << (2 * d);
        }
        const uint32_t peers = __match_any_sync(0xffffffffu, valid ? key : -1);
        const bool leader = valid && (peers & lt) == 0;
        if (pass == 1 && valid) ord_rho[beg + s_cnt[warp][key] + __popc(peers & lt)] = q;
        __syncwarp();
        if (leader) s_cnt[warp][key] += __popc(peers);
        __syncwarp();
      }
      if (pass == 0) {
        __syncthreads();
        // first slot of (warp, key): keys in order, warps in order inside a key
        if (threadIdx.x == 0) {
          uint32_t run = 0;
          for (int k = 0; k < K; ++k)
            for (int w = 0; w < kChunkWarps; ++w) {
              const uint32_t c = s_cnt[w][k];
              s_cnt[w][k] = run;
              run += c;
            }
        }
        __syncthreads();
      }
    }
    __syncthreads();
  }
}

// Chunks of kChunk and blocks of 32 points of every tile (when no density home order is built).
__global__ void k_tile_counts(int ntiles, const int32_t* __restrict__ off, uint32_t* __restrict__ chunk_count,
                              uint32_t* __restrict__ blk_count) {
  const int stride = gridDim.x * blockDim.x;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += stride) {
    const int cnt = off[t + 1] - off[t];
    chunk_count[t] = (uint32_t)((cnt + kChunk - 1) / kChunk);
    blk_count[t] = (uint32_t)((cnt + 31) / 32);
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
  int32_t has[2];
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
  __device__ bool next(const EvGrid* __restrict__ g, const int32_t* __restrict__ off, const StageSmem<N>& sm) {
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
      int u = g->tile_base;
#pragma unroll
      for (int d = 0; d < N; ++d) u += g->stride[d] * wrap_bin(v[d], g->nperdim);
      q = off[u];
      qe = off[u + 1];
      if (qe > q) return true;
    }
  }
};

// Builds piece b (thread 0 only) and issues its bulk copies; returns the words staged.
template <int N>
__device__ int build_piece(const EvGrid* __restrict__ g, const int32_t* __restrict__ off,
                           const float4* __restrict__ rec, StageSmem<N>& sm, TileIter<N>& it, bool& done,
                           int b) {
  constexpr int W = Rec<N>::kWords;
  constexpr int cap = kStageWords / W;
  int nseg = 0, fill = 0;
  while (!done && nseg < kMaxSeg && fill < cap) {
    if (it.q >= it.qe) {
      if (!it.next(g, off, sm)) {
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

// Runs the staged sweep; `vis(inbox, staged_records, first_position, count)` is called for
// every staged segment of a tile the warp needs.  Returns false if a bulk copy did not
// complete within the wait limit (the caller reports it and the CTA exits).
//
// The give-up decision is made for the whole CTA: every thread waits on the piece's mbarrier
// with its own time limit, a warp whose lanes did not all see the copy complete skips the
// piece as a whole (no lane leaves the warp's shuffles and votes), and the barrier that ends
// the piece is __syncthreads_or of the warps' give-ups, so every thread leaves the loop at the
// same point and no thread passes a barrier that its siblings do not reach.  Before the CTA
// returns, the copies it has issued (the timed-out piece and the one issued ahead of it) are
// waited for once more, again with a time limit: a bulk copy cannot be cancelled, and shared
// memory must not be released to the next CTA while one may still write into it.
template <int N, class Visit>
__device__ bool staged_sweep(const EvGrid* __restrict__ g, const int32_t* __restrict__ off,
                             const float4* __restrict__ rec, StageSmem<N>& sm, const int* lo, const int* hi,
                             bool valid, Visit&& vis) {
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
  if (threadIdx.x == 0) sm.has[0] = build_piece<N>(g, off, rec, sm, it, done, 0) > 0;
  __syncthreads();
  for (int p = 0; sm.has[p & 1]; ++p) {
    const int b = p & 1;
    if (threadIdx.x == 0) sm.has[b ^ 1] = build_piece<N>(g, off, rec, sm, it, done, b ^ 1) > 0;
    const bool arrived = mbar_wait_bounded(&sm.full[b], (uint32_t)((p >> 1) & 1), kWaitLimitNs);
    // warp-uniform: a warp visits the piece only if all of its lanes saw the copy complete
    const bool warp_gave_up = __any_sync(0xffffffffu, !arrived);
    if (!warp_gave_up) {
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
        vis(inbox, &sm.buf[b][sm.seg_boff[b][s] * W], sm.seg_qb[b][s], sm.seg_cnt[b][s]);
      }
    }
    // CTA-uniform: every thread takes the same branch after this barrier
    if (__syncthreads_or(warp_gave_up ? 1 : 0)) {
      // drain what this CTA has issued: piece p (timed out) and piece p + 1 (issued above)
      if (threadIdx.x == 0) {
        mbar_wait_bounded(&sm.full[b], (uint32_t)((p >> 1) & 1), kWaitLimitNs);
        if (sm.has[b ^ 1]) mbar_wait_bounded(&sm.full[b ^ 1], (uint32_t)(((p + 1) >> 1) & 1), kWaitLimitNs);
      }
      __syncthreads();
      return false;
    }
  }
  return true;
}

// Chunk of the CTA: tile, event grid and home position of this thread.
struct ChunkHome {
  int t;
  const EvGrid* g;
  int pos;
  bool valid;
};

__device__ __forceinline__ bool chunk_home(const KParams& kp, Events ev, const int32_t* __restrict__ off,
                                           const int32_t* __restrict__ ord, const int32_t* __restrict__ chunk_tile,
                                           const uint32_t* __restrict__ chunk_off,
                                           const uint32_t* __restrict__ chunk_total, ChunkHome& h) {
  const int w = blockIdx.x;
  if (w >= (int)*chunk_total) return false;
  h.t = chunk_tile[w];
  h.g = ev.eg + find_event(ev.tile, kp.n_events, h.t);
  const int beg = off[h.t];
  const int start = (w - (int)chunk_off[h.t]) * kChunk;
  const int cnt = min(kChunk, off[h.t + 1] - beg - start);
  h.valid = (int)threadIdx.x < cnt;
  h.pos = ord[beg + start + (h.valid ? (int)threadIdx.x : 0)];
  return true;
}

// ---- stage 2: local density --------------------------------------------------
// rho_i accumulates, in the reference's candidate order (search-box tiles
// lexicographically, ascending index inside a tile), term = k(d, i, j) * w_j for every
// candidate with d <= dc; candidates beyond dc contribute +-0 and are skipped.
template <int N, int MT>
__global__ void __launch_bounds__(kTileThreads) k_density(const KParams kp, Events ev,
                                                          const int32_t* __restrict__ off,
                                                          const int32_t* __restrict__ ord,
                                                          const int32_t* __restrict__ chunk_tile,
                                                          const uint32_t* __restrict__ chunk_off,
                                                          const uint32_t* __restrict__ chunk_total,
                                                          const float4* __restrict__ rec_w,
                                                          const float4* __restrict__ blk,
                                                          float4* __restrict__ rec_r, DevStatus* st) {
  using M = Metric<N, MT>;
  constexpr int W = Rec<N>::kWords;
  __shared__ StageSmem<N> sm;
  ChunkHome h;
  if (!chunk_home(kp, ev, off, ord, chunk_tile, chunk_off, chunk_total, h)) return;
  const int pos = h.pos;
  const bool valid = h.valid;
  float x[N], wi;
  load_rec<N>(rec_w, pos, x, wi);
  int hb[N], lo[N], hi[N];
  home_bins<N>(h.g, h.t, hb);
  lane_box<N>(kp, h.g, x, kp.dc, hb, lo, hi);
  const bool flat = kp.kernel_type == CLUE_KERNEL_FLAT;
  const float kflat = kp.kpar[0];
  const float tdc = kp.t_dc;
  float rho = 0.0f;
  const bool ok = staged_sweep<N>(h.g, off, rec_w, sm, lo, hi, valid, [&](bool inbox, const float4* sb, int qb, int n_) {
    scan_blocks<N, M>(kp, blk, x, inbox, tdc, false, -INFINITY, qb, n_, [&](int j0, int j1) {
      if (flat) {
#pragma unroll 4
        for (int j = j0; j < j1; ++j) {
          float c[N], wj;
          unpack_rec<N>(sb + j * W, c, wj);
          const float s = M::partial(x, c, kp.mpar);
          const float term = (qb + j == pos) ? wj : fmul(kflat, wj);
          if (inbox && s <= tdc) rho = fadd(rho, term);
        }
      } else {
        for (int j = j0; j < j1; ++j) {
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
  });
  if (!ok) {
    if (threadIdx.x == 0) atomicOr(&st->stage_timeout, 1u);
    return;
  }
  if (valid) store_rec<N>(rec_r, pos, x, rho);
}

// ---- stage 3: nearest higher -------------------------------------------------
// j is higher than i iff rho_j > rho_i or (rho_j == rho_i, rho_j > 0, j > i) with original
// indices.  The reference keeps the first candidate of its iteration order (search-box tiles
// lexicographically, ascending index inside a tile) with the strictly smallest distance <= dm,
// i.e. the minimum of (distance, iteration rank); that minimum does not depend on the order in
// which candidates are visited, so the search here is spatial: every tile's records are also
// kept in Morton order of a fine grid inside the tile, the own tile is searched first, and a
// 32-record block is skipped when its bounding box is farther than every lane's current best
// (or than dm) or holds no density reaching the lane's.  TIE == CLUE_TIE_RHO_INDEX resolves equal
// distances by higher rho, then lower index.

template <int N, int MT, int TIE>
__global__ void __launch_bounds__(kTileThreads, (N <= 4 ? 8 : 4) * 128 / kTileThreads) k_nearest_higher(
    const KParams kp, Events ev, const int32_t* __restrict__ off, const int32_t* __restrict__ ord,
    const int32_t* __restrict__ chunk_tile, const uint32_t* __restrict__ chunk_off,
    const uint32_t* __restrict__ chunk_total, const float4* __restrict__ rec_r, const float4* __restrict__ rec_m,
    const int32_t* __restrict__ mq, const float4* __restrict__ blk, const float4* __restrict__ sblk,
    const int32_t* __restrict__ minv, const int32_t* __restrict__ perm, int32_t* __restrict__ nh_s,
    float* __restrict__ delta_s, DevStatus* st, int split_lanes) {
  using M = Metric<N, MT>;
  ChunkHome h;
  if (!chunk_home(kp, ev, off, ord, chunk_tile, chunk_off, chunk_total, h)) return;
  const int pos = h.pos;
  const bool valid = h.valid;
  float x[N], rho_i;
  load_rec<N>(rec_r, pos, x, rho_i);
  const int orig_i = perm[pos];
  int hb[N], lo[N], hi[N];
  home_bins<N>(h.g, h.t, hb);
  lane_box<N>(kp, h.g, x, kp.dm, hb, lo, hi);
  if (!__any_sync(0xffffffffu, valid)) return;
  const float tdm = kp.t_dm;
  __shared__ float4 s_rec[kTileThreads / 32][32 * Rec<N>::kWords];
  __shared__ int32_t s_q[kTileThreads / 32][32];
  float4* sm = s_rec[threadIdx.x >> 5];
  int32_t* sq = s_q[threadIdx.x >> 5];
  const float slack = M::kRoot ? 1.0f + 1.0f / 524288.0f : 1.0f;  // s range of one rounded distance
  float s_best = INFINITY, rho_best = 0.0f;  // metric value of the nearest higher so far
  // Candidates beyond bnd cannot be nearer than the best so far (nor within dm): its distance
  // would round above delta.
  float bnd = tdm;
  int nh = -1, orig_best = -1;
  int lex_best = 0;  // search-box position of the best one's tile (below the tile count)
  spatial_sweep<N, M, true>(kp, h.g, off, hb, lo, hi, valid, x, blk, sblk, rho_i, minv[pos],
                      [&]() { return bnd; },
                      [&](int p0, int p1, bool need, int64_t lexpos) {
    const int cnt = p1 - p0;
    stage_block<N>(sm, rec_m, p0, cnt, sq, mq);
    // Update of the lane's best by candidate j (called by the whole warp).  The common case, a
    // strictly denser candidate whose distance rounds strictly below the best one's, is a
    // predicated update; equal densities (index rule) and distances that may round to the best
    // one's (rank rule) take the full test, entered only when some lane has such a case.
    // Update of the lane's best by candidate j, in two parts.  consider_fast() takes the common
    // case, a strictly denser candidate whose distance rounds strictly below the best one's, with
    // selects, and returns whether the candidate needs the full test (equal densities: index
    // rule; distances that may round to the best one's: rank rule).  consider_full() is that
    // test; it may run after other candidates' updates, since the best is an exact minimum.
    auto consider_fast = [&](int j, float s, float rho_j, bool in_block) -> bool {
      // selects rather than a branch: the candidate's position is a shared-memory broadcast
      const int qj = sq[j];
      // The home point itself (equal density, never higher) is left out here: the full test
      // would reject it only after a global load of its original index, and every pair of
      // candidates holding some lane's own point would take that path (measured: nearest
      // higher on calo4096 4.04 -> 3.79 ms, on the 4M 3-D points 2.40 -> 2.17 ms).
      const bool c = need && in_block && s <= bnd && rho_j >= rho_i && qj != pos;
      const bool fast = c && rho_j > rho_i && s * slack < s_best;
      const float bj = fminf(tdm, s * slack);
      s_best = fast ? s : s_best;
      bnd = fast ? bj : bnd;
      nh = fast ? qj : nh;
      lex_best = fast ? (int)lexpos : lex_best;
      if (TIE != CLUE_TIE_REFERENCE) {
        rho_best = fast ? rho_j : rho_best;
        orig_best = fast ? -1 : orig_best;  // -1: read from perm when a tie needs it
      }
      return c && !fast;
    };
    auto consider_full = [&](int j, float s, float rho_j) {
      const int q = sq[j];
      int orig_j = -1;
      bool higher = rho_j > rho_i;
      if (!higher && rho_j > 0.0f) {
        orig_j = __ldg(perm + q);
        higher = orig_j > orig_i;
      }
      if (!higher) return;
      bool better;
      if (s * slack < s_best) {
        better = true;  // its distance rounds strictly below the best one's
      } else {
        // the two distances may round to the same value: decide on the rounded distances,
        // then on the iteration rank (search-box position of the tile, then the original
        // index, which orders the points of one tile in the reference's iteration)
        const float dist = M::finish(s), dbest = M::finish(s_best);
        if (dist != dbest || nh < 0) {
          better = dist < dbest;
        } else if (TIE == CLUE_TIE_REFERENCE && (int)lexpos != lex_best) {
          better = (int)lexpos < lex_best;
        } else {
          if (orig_j < 0) orig_j = __ldg(perm + q);
          const int ob = TIE == CLUE_TIE_REFERENCE || orig_best < 0 ? __ldg(perm + nh) : orig_best;
          better = TIE == CLUE_TIE_REFERENCE ? orig_j < ob
                                             : rho_j > rho_best || (rho_j == rho_best && orig_j < ob);
        }
      }
      if (better) {
        s_best = s;
        bnd = fminf(tdm, s * slack);
        nh = q;
        lex_best = (int)lexpos;
        if (TIE != CLUE_TIE_REFERENCE) {
          rho_best = rho_j;
          orig_best = orig_j;
        }
      }
    };
    // both parts for one candidate (called by the whole warp)
    auto consider = [&](int j, float s, float rho_j, bool in_block) {
      const bool slow = consider_fast(j, s, rho_j, in_block);
      if (__any_sync(0xffffffffu, slow) && slow) consider_full(j, s, rho_j);
    };
    // Few lanes need this block: its candidates are split among all 32 lanes, G lanes per
    // needing home (G = 32 / P, P >= the number of such homes, a power of two); each group finds
    // its home's best candidate of the block, and the home lane takes it through consider().
    // Inside one block every candidate has the same search-box position, so the best is the
    // least (rounded distance, then [density, for TIE_RHO_INDEX] then original index), a strict
    // total order that the group reduces exactly.
    const unsigned nm = __ballot_sync(0xffffffffu, need);
    const int k = __popc(nm);
    if (k <= split_lanes) {
      const int lg = k <= 1 ? 5 : (k <= 2 ? 4 : (k <= 4 ? 3 : (k <= 8 ? 2 : 1)));  // log2 G
      const int lane = threadIdx.x & 31;
      const int hs = lane >> lg;  // home slot of this lane's group
      unsigned m = nm;
      for (int i = 0; i < hs && m; ++i) m &= m - 1;
      const bool gv = hs < k;
      const int hl = gv ? __ffs(m) - 1 : 0;  // lane of the group's home
      float xh[N];
#pragma unroll
      for (int d = 0; d < N; ++d) xh[d] = __shfl_sync(0xffffffffu, x[d], hl);
      const float rho_h = __shfl_sync(0xffffffffu, rho_i, hl);
      const float bnd_h = __shfl_sync(0xffffffffu, bnd, hl);
      const int orig_h = __shfl_sync(0xffffffffu, orig_i, hl);
      const int pos_h = __shfl_sync(0xffffffffu, pos, hl);
      // a before b (both higher than the home, same tile)
      auto less = [&](float sa, float ra, int ja, float sb, float rb, int jb) -> bool {
        if (sa * slack < sb) return true;
        if (sb * slack < sa) return false;
        const float da = M::finish(sa), db = M::finish(sb);
        if (da != db) return da < db;
        if (TIE != CLUE_TIE_REFERENCE && ra != rb) return ra > rb;
        return __ldg(perm + sq[ja]) < __ldg(perm + sq[jb]);
      };
      float s_loc = INFINITY, r_loc = 0.0f;
      int j_loc = -1;
      const int G = 1 << lg;
      for (int j = lane & (G - 1); j < cnt; j += G) {
        float c[N], rj;
        smem_rec<N>(sm, j, c, rj);
        const float sj = M::partial(xh, c, kp.mpar);
        if (gv && sj <= bnd_h && rj >= rho_h) {
          bool higher = rj > rho_h;
          if (!higher && rj > 0.0f) {  // (the home point itself needs no load: never higher)
            const int qj = sq[j];
            higher = qj != pos_h && __ldg(perm + qj) > orig_h;
          }
          if (higher && (j_loc < 0 || less(sj, rj, j, s_loc, r_loc, j_loc))) {
            s_loc = sj;
            r_loc = rj;
            j_loc = j;
          }
        }
      }
      for (int o = G >> 1; o > 0; o >>= 1) {
        const float s_o = __shfl_xor_sync(0xffffffffu, s_loc, o);
        const float r_o = __shfl_xor_sync(0xffffffffu, r_loc, o);
        const int j_o = __shfl_xor_sync(0xffffffffu, j_loc, o);
        if (j_o >= 0 && (j_loc < 0 || less(s_o, r_o, j_o, s_loc, r_loc, j_loc))) {
          s_loc = s_o;
          r_loc = r_o;
          j_loc = j_o;
        }
      }
      const int src = need ? __popc(nm & ((1u << lane) - 1u)) << lg : 0;
      const float s_g = __shfl_sync(0xffffffffu, s_loc, src);
      const float r_g = __shfl_sync(0xffffffffu, r_loc, src);
      const int j_g = __shfl_sync(0xffffffffu, j_loc, src);
      consider(j_g >= 0 ? j_g : 0, s_g, r_g, j_g >= 0);
      return;
    }
    // two candidates at a time: their metric values and densities first, then the update,
    // entered only when some lane holds a candidate that passes the bound (the bound only
    // shrinks between the two, and consider() checks it again)
    for (int j = 0; j < cnt; j += 2) {
      float ca[N], cb[N], ra, rb;
      smem_rec<N>(sm, j, ca, ra);
      smem_rec<N>(sm, j + 1, cb, rb);
      // paired differences and squares pay from three dimensions on (measured)
      const float2 s2 = N >= 3 ? partial_pair<N, MT>(x, ca, cb, kp.mpar)
                               : make_float2(M::partial(x, ca, kp.mpar), M::partial(x, cb, kp.mpar));
      const bool any = (s2.x <= bnd && ra >= rho_i) || (j + 1 < cnt && s2.y <= bnd && rb >= rho_i);
      if (__any_sync(0xffffffffu, need && any)) {
        const bool slow_a = consider_fast(j, s2.x, ra, true);
        const bool slow_b = consider_fast(j + 1, s2.y, rb, j + 1 < cnt);
        if (__any_sync(0xffffffffu, slow_a || slow_b)) {  // one vote for both full tests
          if (slow_a) consider_full(j, s2.x, ra);
          if (slow_b) consider_full(j + 1, s2.y, rb);
        }
      }
    }
  });
  if (valid) {
    nh_s[pos] = nh;
    delta_s[pos] = nh >= 0 ? M::finish(s_best) : FLT_MAX;
  }
  const uint32_t none = __ballot_sync(0xffffffffu, valid && nh < 0);
  if ((threadIdx.x & 31) == 0 && none) {
    atomicAdd(&st->seed_candidates, (uint32_t)__popc(none));
    atomicAdd(const_cast<uint32_t*>(&h.g->seed_candidates), (uint32_t)__popc(none));
  }
}

// Forms of the spatial-order density.  With unit amplitude the exponential kernel is
// exp2(kexp * d) and the zero-mean Gaussian exp2(kexp * d^2), kexp folding -avg or -1/(2 std^2)
// with log2(e); their value at d = 0 is exp2(0) = 1, the reference's self term, so no per-pair
// self test is needed.  Every other kernel takes the generic form.
enum { kDensGeneric = 0, kDensExpUnit = 1, kDensGauss0Unit = 2 };

// Local density over the Morton-ordered records (any order, kernels other than flat): the
// same candidate set as the reference (search-box tiles, d <= dc, self term 1), summed in
// spatial order.  Blocks farther than dc from every lane are skipped; inside a block, candidates
// that no lane of the warp holds within dc skip the kernel evaluation.
template <int N, int MT, int FORM>
__global__ void __launch_bounds__(kTileThreads, (N <= 4 ? 8 : 4) * 128 / kTileThreads) k_density_spatial(
    const KParams kp, Events ev, const int32_t* __restrict__ off, const int32_t* __restrict__ ord,
    const int32_t* __restrict__ chunk_tile, const uint32_t* __restrict__ chunk_off,
    const uint32_t* __restrict__ chunk_total, const float4* __restrict__ rec_w, const float4* __restrict__ rec_m,
    const int32_t* __restrict__ mq, const float4* __restrict__ blk, const float4* __restrict__ sblk,
    float4* __restrict__ rec_r, const int32_t* __restrict__ minv, float kexp) {
  using M = Metric<N, MT>;
  __shared__ float4 s_rec[kTileThreads / 32][32 * Rec<N>::kWords];
  ChunkHome h;
  if (!chunk_home(kp, ev, off, ord, chunk_tile, chunk_off, chunk_total, h)) return;
  const int pos = h.pos;
  const bool valid = h.valid;
  float x[N], wi;
  load_rec<N>(rec_w, pos, x, wi);
  const int p_home = minv[pos];
  int hb[N], lo[N], hi[N];
  home_bins<N>(h.g, h.t, hb);
  lane_box<N>(kp, h.g, x, kp.dc, hb, lo, hi);
  if (!__any_sync(0xffffffffu, valid)) return;
  const float tdc = kp.t_dc;
  float4* sm = s_rec[threadIdx.x >> 5];
  float rho = 0.0f;
  spatial_sweep<N, M, false>(kp, h.g, off, hb, lo, hi, valid, x, blk, sblk, -INFINITY, p_home, [&]() { return tdc; },
                      [&](int p0, int p1, bool need, int64_t) {
    const int cnt = p1 - p0;
    stage_block<N>(sm, rec_m, p0, cnt);
    const int jself = p_home - p0;
    auto pair = [&](int j, bool in_block) {
      float c[N], wj;
      smem_rec<N>(sm, j, c, wj);
      const float s = M::partial(x, c, kp.mpar);
      const bool in = need && in_block && s <= tdc;
      if (__any_sync(0xffffffffu, in)) {
        float kv;
        if (FORM == kDensExpUnit) {
          kv = ex2_approx(kexp * (M::kRoot ? sqrt_approx(s) : s));
        } else if (FORM == kDensGauss0Unit) {
          kv = ex2_approx(kexp * (M::kRoot ? s : s * s));
        } else {
          const float dist = M::kRoot ? sqrt_approx(s) : s;
          kv = (j == jself) ? 1.0f : kernel_value_fast(kp.kernel_type, kp.kpar, kp.ginv, dist);
        }
        const float t = kv * wj;
        if (in) rho = fadd(rho, t);
      }
    };
    int j0 = 0;
    for (; j0 + 8 <= cnt; j0 += 8) {
#pragma unroll
      for (int u = 0; u < 8; ++u) pair(j0 + u, true);
    }
    if (j0 < cnt) {
#pragma unroll
      for (int u = 0; u < 8; ++u) pair(j0 + u, j0 + u < cnt);
    }
  });
  if (valid) store_rec<N>(rec_r, pos, x, rho);
}

// ---- symmetric spatial density -------------------------------------------------
// For metrics whose value bounds every coordinate difference (Euclidean, Manhattan, Chebyshev)
// and no wrapped coordinate, d(i, j) <= dc already places j's tile inside i's search box, so the
// candidate set is {j : d(i, j) <= dc} and every pair can be evaluated once for both points.
// Blocks are 32 consecutive Morton-ordered records counted from their tile's start (so the
// result does not depend on where a tile lies in a batch): block slot 4 c + w is warp w of
// chunk c.  The warp of block A evaluates A against itself one-sidedly and every block B of its
// tile after A and of the later tiles of its search-box union both ways: the candidate records
// rotate through the lanes, each lane adding K(d) w_j to its own sum and K(d) w_i to the
// travelling candidate's sum, which is then added in fixed point (exact integer adds, so the
// order of arrival does not matter) to the candidate's accumulator.

// Block boxes in compact order: block b of tile u is entry bo[u] + b (bo = exclusive scan of
// the tiles' block counts).  One thread per (chunk, warp) slot; slots past a tile's end write
// nothing.
template <int N>
__global__ void __launch_bounds__(256) k_tblock_bbox(int max_slots, const uint32_t* __restrict__ chunk_total,
                                                    const int32_t* __restrict__ off,
                                                    const int32_t* __restrict__ chunk_tile,
                                                    const uint32_t* __restrict__ chunk_off,
                                                    const uint32_t* __restrict__ bo,
                                                    const float4* __restrict__ rec_m, float4* __restrict__ tblk) {
  constexpr int BW = Blk<N>::kWords;
  const int nslots = min(max_slots, kChunkWarps * (int)*chunk_total);
  const int stride = gridDim.x * blockDim.x;
  for (int sl = blockIdx.x * blockDim.x + threadIdx.x; sl < nslots; sl += stride) {
    const int c = sl / kChunkWarps;
    const int t = chunk_tile[c];
    const int b = (c - (int)chunk_off[t]) * kChunkWarps + sl % kChunkWarps;
    const int first = off[t] + (b << 5);
    const int cnt = min(32, off[t + 1] - first);
    if (cnt <= 0) continue;
    float bb[4 * BW];
#pragma unroll
    for (int d = 0; d < N; ++d) {
      bb[d] = INFINITY;
      bb[N + d] = -INFINITY;
    }
#pragma unroll
    for (int k = 2 * N; k < 4 * BW; ++k) bb[k] = 0.0f;
    for (int r = 0; r < cnt; ++r) {
      float x[N], pl;
      load_rec<N>(rec_m, first + r, x, pl);
#pragma unroll
      for (int d = 0; d < N; ++d) {
        bb[d] = fminf(bb[d], x[d]);
        bb[N + d] = fmaxf(bb[N + d], x[d]);
      }
    }
    const size_t id = (size_t)bo[t] + b;
#pragma unroll
    for (int k = 0; k < BW; ++k)
      tblk[id * BW + k] = make_float4(bb[4 * k], bb[4 * k + 1], bb[4 * k + 2], bb[4 * k + 3]);
  }
}

// Fixed-point exponent of an event: contributions times 2^F stay below 2^61 in total
// (|sum| <= count * max|w| * max kernel value).
__device__ __forceinline__ int fix_exponent(const EvGrid* g, float kmax) {
  const float bound = __uint_as_float(g->wmax_bits) * (float)g->pt_count * kmax;
  int e = 0;
  frexpf(bound, &e);  // bound < 2^e
  return max(-126, min(126, 61 - e));
}

// VAR selects measured alternatives of the pair step (clue_tuning.density_gate / density_exp2):
// bit 0: a warp vote per pair of steps skips the kernel evaluation and the mirrored shuffles when
// no lane of the warp has a candidate within dc (the same bits: the skipped terms are zeros);
// bit 1: the unit-amplitude forms evaluate 2^x with exp2_poly2 on the FMA pipe instead of
// ex2.approx on the MUFU pipe (within 5e-7 relative per term).
template <int N, int MT, int FORM, int VAR>
__global__ void __launch_bounds__(kTileThreads, (N <= 4 ? 8 : 4) * 128 / kTileThreads) k_density_sym(
    const KParams kp, Events ev, const int32_t* __restrict__ off, const int32_t* __restrict__ chunk_tile,
    const uint32_t* __restrict__ chunk_off, const uint32_t* __restrict__ chunk_total,
    const float4* __restrict__ rec_m, const int32_t* __restrict__ mq, const uint32_t* __restrict__ bo,
    const float4* __restrict__ tblk, float4* __restrict__ rec_r, int64_t* __restrict__ rho_fix, float kexp,
    float kmax, DevStatus* st) {
  using M = Metric<N, MT>;
  constexpr int BW = Blk<N>::kWords;
  __shared__ float4 s_rec[kTileThreads / 32][32 * Rec<N>::kWords];
  const int c = blockIdx.x;
  if (c >= (int)*chunk_total) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int t = chunk_tile[c];
  const int a_loc = (c - (int)chunk_off[t]) * kChunkWarps + warp;  // block of the tile
  const int startA = off[t] + (a_loc << 5);
  const int cntA = min(32, off[t + 1] - startA);
  if (cntA <= 0) return;  // whole warp: this block of the chunk is past the tile's end
  const EvGrid* g = ev.eg + find_event(ev.tile, kp.n_events, t);
  const bool hv = lane < cntA;
  const int pA = startA + (hv ? lane : 0);
  float x[N], wi;
  load_rec<N>(rec_m, pA, x, wi);
  int hb[N], lo[N], hi[N];
  home_bins<N>(g, t, hb);
  lane_box<N>(kp, g, x, kp.dc, hb, lo, hi);
  int wl[N], wh[N];
#pragma unroll
  for (int d = 0; d < N; ++d) {
    wl[d] = warp_min_i(hv ? lo[d] : INT_MAX);
    wh[d] = warp_max_i(hv ? hi[d] : INT_MIN);
  }
  const float tdc = kp.t_dc;
  const float scale = ldexpf(1.0f, fix_exponent(g, kmax));
  auto kval = [&](float s, bool self) -> float {
    if (FORM == kDensExpUnit) return ex2_approx(kexp * (M::kRoot ? sqrt_approx(s) : s));
    if (FORM == kDensGauss0Unit) return ex2_approx(kexp * (M::kRoot ? s : s * s));
    const float dist = M::kRoot ? sqrt_approx(s) : s;
    return self ? 1.0f : kernel_value_fast(kp.kernel_type, kp.kpar, kp.ginv, dist);
  };
  const float2 kexp2 = make_float2(kexp, kexp);
  auto kval2 = [&](float2 s) -> float2 {
    if (FORM == kDensExpUnit) {
      const float2 d = M::kRoot ? make_float2(sqrt_approx(s.x), sqrt_approx(s.y)) : s;
      const float2 e = mul2(kexp2, d);
      if (VAR & 2) return exp2_poly2(e);
      return make_float2(ex2_approx(e.x), ex2_approx(e.y));
    }
    if (FORM == kDensGauss0Unit) {
      const float2 e = mul2(kexp2, M::kRoot ? s : mul2(s, s));
      if (VAR & 2) return exp2_poly2(e);
      return make_float2(ex2_approx(e.x), ex2_approx(e.y));
    }
    return make_float2(kval(s.x, false), kval(s.y, false));
  };
  float acc = 0.0f;
  // block A against itself, one-sided (the self pair gives the reference's self term)
  {
    float4* sm = s_rec[warp];
    stage_block<N>(sm, rec_m, startA, cntA);
    if (FORM == kDensGeneric) {  // the generic kernel needs the self test
      for (int j = 0; j < cntA; ++j) {
        float cx[N], wj;
        smem_rec<N>(sm, j, cx, wj);
        const float sd = M::partial(x, cx, kp.mpar);
        const bool in = hv && sd <= tdc;
        if (__any_sync(0xffffffffu, in)) {
          const float t2 = kval(sd, j == lane) * wj;
          if (in) acc = fadd(acc, t2);
        }
      }
    } else {
      // two candidates at a time, no branch (the own block almost always has pairs within dc);
      // a record past the block's end (stale shared memory) is masked with its weight
      float2 acc2 = make_float2(0.0f, 0.0f);
      for (int j = 0; j < cntA; j += 2) {
        float ca[N], cb[N], wa, wb;
        smem_rec<N>(sm, j, ca, wa);
        smem_rec<N>(sm, j + 1, cb, wb);
        const bool bv = j + 1 < cntA;
        const float2 sd = partial_pair<N, MT>(x, ca, cb, kp.mpar);
        float2 kv = kval2(sd);
        kv.x = hv && sd.x <= tdc ? kv.x : 0.0f;
        kv.y = hv && bv && sd.y <= tdc ? kv.y : 0.0f;
        acc2 = fma2(kv, make_float2(wa, bv ? wb : 0.0f), acc2);
      }
      acc = fadd(acc, fadd(acc2.x, acc2.y));
    }
  }
  // later blocks of the own tile, then the later tiles of the union box, both ways
  int v[N];
#pragma unroll
  for (int d = 0; d < N; ++d) v[d] = wl[d];
  while (true) {
    int u = g->tile_base;
#pragma unroll
    for (int d = 0; d < N; ++d) u += g->stride[d] * v[d];
    if (u >= t && !dcheck_bad(st, u, kp.ntiles, kChkDensityTile)) {
      const int pb = off[u], pe = off[u + 1];
      const int nb = (pe - pb + 31) >> 5;
      for (int b = (u == t ? a_loc + 1 : 0); b < nb; ++b) {
        float bb[4 * BW];
        load_box<N>(tblk, (int)bo[u] + b, bb);
        const bool need = hv && M::lower(x, bb, bb + N, kp.mpar) <= tdc;
        if (!__any_sync(0xffffffffu, need)) continue;
        const int first = pb + (b << 5);
        const int cntB = min(32, pe - first);
        const bool cv = lane < cntB;
        // lane m owns candidate m of the block; at step k lane l meets candidate l ^ k and the
        // candidate's owner collects the term from lane m ^ k = l (butterfly shuffles with
        // immediate lane masks), so no value is carried from one step to the next
        float ox[N], ow;
        load_rec<N>(rec_m, first + (cv ? lane : 0), ox, ow);
        if (!cv) {
#pragma unroll
          for (int d = 0; d < N; ++d) ox[d] = INFINITY;  // never within dc
          ow = 0.0f;
        }
        // two steps at a time, with paired arithmetic; the own terms of this block are summed
        // (fused multiply-add) in two running sums, even and odd steps, added at the block's end
        float2 acc2 = make_float2(0.0f, 0.0f), cacc2 = make_float2(0.0f, 0.0f);
        const float2 wi2 = make_float2(wi, wi);
#pragma unroll
        for (int k = 0; k < 32; k += 2) {
          float ca[N], cb[N];
#pragma unroll
          for (int d = 0; d < N; ++d) {
            ca[d] = __shfl_xor_sync(0xffffffffu, ox[d], k);
            cb[d] = __shfl_xor_sync(0xffffffffu, ox[d], k + 1);
          }
          const float2 cw = make_float2(__shfl_xor_sync(0xffffffffu, ow, k), __shfl_xor_sync(0xffffffffu, ow, k + 1));
          const float2 sd = partial_pair<N, MT>(x, ca, cb, kp.mpar);
          const bool ix = hv && sd.x <= tdc, iy = hv && sd.y <= tdc;
          if ((VAR & 1) == 0 || __any_sync(0xffffffffu, ix || iy)) {
            float2 kv = kval2(sd);
            kv.x = ix ? kv.x : 0.0f;
            kv.y = iy ? kv.y : 0.0f;
            acc2 = fma2(kv, cw, acc2);
            const float2 tc = mul2(kv, wi2);
            cacc2 = add2(cacc2, make_float2(__shfl_xor_sync(0xffffffffu, tc.x, k),
                                            __shfl_xor_sync(0xffffffffu, tc.y, k + 1)));
          }
        }
        acc = fadd(acc, fadd(acc2.x, acc2.y));
        const float cacc = fadd(cacc2.x, cacc2.y);
        if (cv && cacc != 0.0f) {
          const int mi = mq[first + lane];
          if (!dcheck_bad(st, mi, kp.n, kChkDensityMirror))
            atomicAdd(reinterpret_cast<unsigned long long*>(rho_fix + mi), (unsigned long long)__float2ll_rn(cacc * scale));
        }
      }
    }
    int d = N - 1;
    for (; d >= 0; --d) {
      if (v[d] < wh[d]) {
        ++v[d];
        break;
      }
      v[d] = wl[d];
    }
    if (d < 0) break;
  }
  if (hv) store_rec<N>(rec_r, mq[pA], x, acc);
}

// rho = own-side sum + the fixed-point sum of the contributions received as a candidate.
template <int N>
__global__ void __launch_bounds__(256) k_density_combine(const KParams kp, Events ev, int n,
                                                         const int64_t* __restrict__ rho_fix,
                                                         float4* __restrict__ rec_r, float kmax) {
  const int stride = gridDim.x * blockDim.x;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    bool uniform;
    const EvGrid* g = ev.eg + warp_event(ev.pt, ev.chunk_ev, kp.n_events, q, true, uniform);
    float x[N], acc;
    load_rec<N>(rec_r, q, x, acc);
    const float recv = (float)((double)rho_fix[q] * ldexp(1.0, -fix_exponent(g, kmax)));
    store_rec<N>(rec_r, q, x, fadd(acc, recv));
  }
}

// The symmetric density's fixed-point sums added in (as k_density_combine) and the block
// boxes with the final densities (as k_block_bbox) in one pass over the records, for the
// composite sort whose tile-ordered records are also the Morton-ordered ones.
template <int N>
__global__ void __launch_bounds__(256) k_combine_block_bbox(const KParams kp, Events ev, int n,
                                                            const int64_t* __restrict__ rho_fix,
                                                            float4* __restrict__ rec_r, float kmax,
                                                            float4* __restrict__ blk) {
  const int lane = threadIdx.x & 31;
  const int nblk = (n + 31) >> 5;
  const int wstride = (gridDim.x * blockDim.x) >> 5;
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nblk; b += wstride) {
    const int q = (b << 5) + lane;
    const bool valid = q < n;
    const int qq = valid ? q : b << 5;
    bool uniform;
    const EvGrid* g = ev.eg + warp_event(ev.pt, ev.chunk_ev, kp.n_events, qq, true, uniform);
    float x[N], acc;
    load_rec<N>(rec_r, qq, x, acc);
    const float rho = fadd(acc, (float)((double)rho_fix[qq] * ldexp(1.0, -fix_exponent(g, kmax))));
    if (valid) store_rec<N>(rec_r, q, x, rho);
    write_block_box<N>(blk, b, x, rho);
  }
}

// ---- stage 4: seeds (KernelFindClusters) ---------------------------------------
// Also counts the near-threshold decisions of this stage: densities within kNearTol of rhoc and
// nearest-higher distances within kNearTol of seed_dc or dm.
template <int N, int MT>
__global__ void __launch_bounds__(256) k_seeds(const KParams kp, int n, const float4* __restrict__ rec_r,
                                               const int32_t* __restrict__ nh_s, const float* __restrict__ delta_s,
                                               const int32_t* __restrict__ perm, int32_t* __restrict__ is_seed_s,
                                               int32_t* __restrict__ par, uint32_t* __restrict__ seed_flag,
                                               DevStatus* st) {
  const int stride = gridDim.x * blockDim.x;
  uint32_t c_rhoc = 0, c_seed_dc = 0, c_dm = 0;
  for (int pos = blockIdx.x * blockDim.x + threadIdx.x; pos < n; pos += stride) {
    float x[N], rho;
    load_rec<N>(rec_r, pos, x, rho);
    const int nh = nh_s[pos];
    // d(i, nh) is the nearest-higher stage's delta, the same metric value bit for bit; without a
    // nearest higher the reference measures the distance to PointsView::operator[](-1), whose
    // coordinates are FLT_MAX (PointsCommon.hpp:75-81): an infinite or FLT_MAX distance, above
    // any finite seed_dc, which +inf decides the same way
    const float dist = nh >= 0 ? delta_s[pos] : INFINITY;
    const bool seed = (dist > kp.seed_dc) && (rho >= kp.rhoc);
    is_seed_s[pos] = seed ? 1 : 0;
    par[pos] = seed ? -1 : nh;
    const int orig = perm[pos];
    if (!dcheck_bad(st, orig, n, kChkSeedsPerm)) seed_flag[orig] = seed ? 1u : 0u;
    c_rhoc += fabsf(rho - kp.rhoc) <= kNearTol * kp.rhoc ? 1u : 0u;
    c_seed_dc += nh >= 0 && fabsf(dist - kp.seed_dc) <= kNearTol * kp.seed_dc ? 1u : 0u;
    c_dm += nh >= 0 && fabsf(dist - kp.dm) <= kNearTol * kp.dm ? 1u : 0u;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    c_rhoc += __shfl_xor_sync(0xffffffffu, c_rhoc, o);
    c_seed_dc += __shfl_xor_sync(0xffffffffu, c_seed_dc, o);
    c_dm += __shfl_xor_sync(0xffffffffu, c_dm, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (c_rhoc) atomicAdd(&st->near_rhoc, c_rhoc);
    if (c_seed_dc) atomicAdd(&st->near_seed_dc, c_seed_dc);
    if (c_dm) atomicAdd(&st->near_dm, c_dm);
  }
}

// Near-tie count of the nearest-higher stage (CLUE_FLAG_NEAR_TIES), after k_nearest_higher:
// a point counts when its chosen nearest higher, or a candidate of its search box at most as
// far as that one (within dm when none was found) that is not its own record, has a density
// within kNearTol of the point's own.  These are the points whose nearest higher can change
// when densities move by that much (ClusteringKernels.hpp:129-143).  A pruned sweep like
// nearest higher's: blocks beyond the chosen distance, or whose densities all lie below
// rho_i - tol |rho_i|, are skipped.
template <int N, int MT>
__global__ void __launch_bounds__(kTileThreads) k_near_ties(
    const KParams kp, Events ev, const int32_t* __restrict__ off, const int32_t* __restrict__ ord,
    const int32_t* __restrict__ chunk_tile, const uint32_t* __restrict__ chunk_off,
    const uint32_t* __restrict__ chunk_total, const float4* __restrict__ rec_r, const float4* __restrict__ rec_m,
    const int32_t* __restrict__ mq, const float4* __restrict__ blk, const float4* __restrict__ sblk,
    const int32_t* __restrict__ minv, const int32_t* __restrict__ nh_s, DevStatus* st) {
  using M = Metric<N, MT>;
  ChunkHome h;
  if (!chunk_home(kp, ev, off, ord, chunk_tile, chunk_off, chunk_total, h)) return;
  const int pos = h.pos;
  const bool valid = h.valid;
  float x[N], rho_i;
  load_rec<N>(rec_r, pos, x, rho_i);
  int hb[N], lo[N], hi[N];
  home_bins<N>(h.g, h.t, hb);
  lane_box<N>(kp, h.g, x, kp.dm, hb, lo, hi);
  if (!__any_sync(0xffffffffu, valid)) return;
  __shared__ float4 s_rec[kTileThreads / 32][32 * Rec<N>::kWords];
  __shared__ int32_t s_q[kTileThreads / 32][32];
  float4* sm = s_rec[threadIdx.x >> 5];
  int32_t* sq = s_q[threadIdx.x >> 5];
  auto near = [&](float r) {
    const float m = fmaxf(fabsf(r), fabsf(rho_i));
    return m > 0.0f && fabsf(r - rho_i) <= kNearTol * m;
  };
  const int nh = nh_s[pos];
  float bnd = kp.t_dm;
  bool flag = false;
  if (nh >= 0) {
    float c[N], rho_nh;
    load_rec<N>(rec_r, nh, c, rho_nh);
    bnd = M::partial(x, c, kp.mpar);
    flag = near(rho_nh);
  }
  const float pmin = rho_i - kNearTol * fabsf(rho_i);
  spatial_sweep<N, M, false>(kp, h.g, off, hb, lo, hi, valid, x, blk, sblk, pmin, minv[pos], [&]() { return bnd; },
                             [&](int p0, int p1, bool need, int64_t) {
    const int cnt = p1 - p0;
    stage_block<N>(sm, rec_m, p0, cnt, sq, mq);
    for (int j = 0; j < cnt; ++j) {
      float c[N], rj;
      smem_rec<N>(sm, j, c, rj);
      const float s = M::partial(x, c, kp.mpar);
      flag = flag || (need && s <= bnd && sq[j] != pos && near(rj));
    }
  });
  const uint32_t cnt_w = __ballot_sync(0xffffffffu, valid && flag);
  if ((threadIdx.x & 31) == 0 && cnt_w) atomicAdd(&st->nh_near_ties, (uint32_t)__popc(cnt_w));
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
  // four chains per thread walked in lockstep: each step's four parent loads are independent,
  // so they are in flight together (the walk is bound by load latency, not bandwidth)
  constexpr int K = 4;
  for (int64_t pos0 = blockIdx.x * blockDim.x + threadIdx.x; pos0 < n; pos0 += (int64_t)K * stride) {
    int p[K];
    bool act[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int64_t pos = pos0 + (int64_t)k * stride;
      p[k] = pos < n ? par[pos] : -1;
      act[k] = p[k] >= 0;
    }
    for (int it = 0; it < iters; ++it) {
      bool any = false;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (act[k] && dcheck_bad(st, p[k], n, kChkJumpParent)) act[k] = false;
        if (act[k]) {
          const int pp = __ldcg(par + p[k]);
          if (pp < 0) {
            act[k] = false;
          } else {
            p[k] = pp;
            par[pos0 + (int64_t)k * stride] = pp;
          }
        }
        any |= act[k];
      }
      if (!any) break;
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (act[k] && __ldcg(par + p[k]) >= 0) unres = true;  // still climbing after `iters` jumps
  }
  if (__any_sync(0xffffffffu, unres) && (threadIdx.x & 31) == 0) atomicAdd(&st->unresolved[round], 1u);
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicMax(&st->label_rounds, (uint32_t)round + 1);
}

// ---- stage 5, breadth-first form (clue_tuning.labels_bfs) ----------------------
// The reference's follower association map (Followers::fill, AssociationMap.hpp:193-251: counts
// per nearest higher, a scan, a scatter) and its assignment from the seeds
// (KernelAssignClusters, ClusteringKernels.hpp:246-281, a depth-first walk per seed), here with
// the walk done level by level over all seeds at once: the frontier of level l holds the points
// l steps below a seed, and each of their followers takes the seed as its parent.  Points no
// seed reaches keep their nearest higher as parent, whose chain ends at a point that is not a
// seed, so k_finalize labels them -1 as pointer jumping does.

// counts[p] = followers of p (par[i] = p >= 0).
__global__ void __launch_bounds__(256) k_follower_count(const int32_t* __restrict__ par, int n,
                                                        uint32_t* __restrict__ counts) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int p = par[i];
    if (p >= 0) atomicAdd(counts + p, 1u);
  }
}

// Scatter of every follower into its parent's run (order inside a run is the atomic order; the
// labels do not depend on it).  cursor starts as the exclusive scan of the counts.
__global__ void __launch_bounds__(256) k_follower_fill(const int32_t* __restrict__ par, int n,
                                                       uint32_t* __restrict__ cursor, int32_t* __restrict__ followers) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int p = par[i];
    if (p >= 0) followers[atomicAdd(cursor + p, 1u)] = i;
  }
}

// Level 0: the seeds (parent -1 and the seed flag).
__global__ void __launch_bounds__(256) k_bfs_seeds(const int32_t* __restrict__ par,
                                                   const int32_t* __restrict__ is_seed_s, int n,
                                                   int32_t* __restrict__ frontier, DevStatus* st) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    if (par[i] < 0 && is_seed_s[i]) frontier[atomicAdd(&st->bfs_count[0], 1u)] = i;
}

// One level: every frontier point hands its seed to its followers, which form the next frontier.
// off[p] .. off[p] + counts[p] is p's run (off = the scanned counts before the fill advanced
// them, i.e. the cursor minus the count).
__global__ void __launch_bounds__(256) k_bfs_level(const uint32_t* __restrict__ end, const uint32_t* __restrict__ counts,
                                                   const int32_t* __restrict__ followers, int32_t* __restrict__ par,
                                                   const int32_t* __restrict__ fin, int32_t* __restrict__ fout,
                                                   DevStatus* st, int level) {
  const uint32_t nin = st->bfs_count[level];
  if (nin == 0) return;
  const int stride = gridDim.x * blockDim.x;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < (int)nin; t += stride) {
    const int u = fin[t];
    const int seed = level == 0 ? u : par[u];
    const uint32_t e = end[u], b = e - counts[u];
    for (uint32_t q = b; q < e; ++q) {
      const int c = followers[q];
      par[c] = seed;
      if (counts[c]) fout[atomicAdd(&st->bfs_count[level + 1], 1u)] = c;  // leaves end the walk
    }
  }
}

// After the last enqueued level: a frontier left over marks the run unresolved in the slot the
// host checks after the enqueued label rounds (unresolved[3]), and the host continues by
// pointer jumping (finish_labels), which completes any mix of seed and nearest-higher parents.
__global__ void k_bfs_done(DevStatus* st) {
  if (st->bfs_count[kBfsLevels] != 0) st->unresolved[3] = 1u;
}

// Seed list capacity of an event: every seed, or the reference's SeedArray capacity
// max(seed_capacity, points without nearest higher) (SetupSeeds.hpp:10-20).
__device__ __forceinline__ int64_t seed_cap(const KParams& kp, const EvGrid* g) {
  if (kp.seed_capacity < 0) return INT64_MAX;
  return kp.seed_capacity > (int64_t)g->seed_candidates ? kp.seed_capacity : (int64_t)g->seed_candidates;
}

// Labels from the roots (seed rank inside its event) and scatter of every output back to
// the caller's order.
template <int N>
__global__ void __launch_bounds__(256) k_finalize(const KParams kp, Events ev, const int32_t* __restrict__ par,
                                                  const int32_t* __restrict__ is_seed_s,
                                                  const uint32_t* __restrict__ seed_rank,
                                                  const int32_t* __restrict__ perm,
                                                  const int32_t* __restrict__ nh_s,
                                                  const float4* __restrict__ rec_r,
                                                  const float* __restrict__ delta_s, clue_outputs out,
                                                  DevStatus* st) {
  const int stride = gridDim.x * blockDim.x;
  for (int pos = blockIdx.x * blockDim.x + threadIdx.x; pos < kp.n; pos += stride) {
    bool uniform;
    const int e = warp_event(ev.pt, ev.chunk_ev, kp.n_events, pos, true, uniform);
    const int p = par[pos];
    const int root = p >= 0 ? p : pos;
    if (dcheck_bad(st, root, kp.n, kChkFinalizeRoot) || dcheck_bad(st, perm[root], kp.n, kChkFinalizeRoot)) continue;
    int lab = -1;
    if (is_seed_s[root]) {
      const uint32_t rk = seed_rank[perm[root]] - seed_rank[ev.pt[e]];
      if ((int64_t)rk < seed_cap(kp, ev.eg + e)) lab = (int)rk;
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
      out.nearest_higher[i] = nh >= 0 && !dcheck_bad(st, nh, kp.n, kChkFinalizeNh) ? perm[nh] : -1;
    }
    if (out.delta) out.delta[i] = delta_s[pos];
  }
}

// Per-event seeds and clusters: n_seeds[e], n_clusters[e] (optional outputs) and the total of
// clusters over all events in st->n_clusters.
__global__ void k_event_info(const KParams kp, const EvGrid* __restrict__ eg, const int32_t* __restrict__ ev_pt,
                             const uint32_t* __restrict__ seed_rank, const uint32_t* __restrict__ seed_total,
                             int32_t* __restrict__ n_seeds, int32_t* __restrict__ n_clusters, DevStatus* st) {
  const int stride = gridDim.x * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < kp.n_events; e += stride) {
    const uint32_t a = seed_rank[ev_pt[e]];
    const uint32_t b = e + 1 < kp.n_events ? seed_rank[ev_pt[e + 1]] : *seed_total;
    const int64_t ns = (int64_t)(b - a);
    const int64_t cap = seed_cap(kp, eg + e);
    const int64_t nc = ns < cap ? ns : cap;
    if (n_seeds) n_seeds[e] = (int32_t)ns;
    if (n_clusters) n_clusters[e] = (int32_t)nc;
    atomicAdd(&st->n_clusters, (uint32_t)nc);
  }
}

int grid_for(int n, int threads) {
  int b = (n + threads - 1) / threads;
  const int cap = 148 * 32;
  return b < 1 ? 1 : (b > cap ? cap : b);
}

inline int chunk_grid(const KParams& kp) { return kp.n / kChunk + kp.ntiles + 1; }

inline Events events_of(Workspace& ws) { return Events{ws.ev, ws.ev_pt, ws.ev_tile, ws.ev_chunk}; }

template <int N, int MT>
void launch_density(const KParams& kp, Workspace& ws, cudaStream_t s) {
  k_density<N, MT><<<chunk_grid(kp), kTileThreads, 0, s>>>(kp, events_of(ws), ws.offsets, ws.ord_rho,
                                                            ws.chunk_tile, ws.chunk_count, ws.chunk_total,
                                                            ws.rec_w, ws.blk, ws.rec_r, ws.status);
}
template <int N, int MT>
void launch_nh(const KParams& kp, Workspace& ws, cudaStream_t s) {
  // a block needed by at most this many lanes is split among all lanes (at most 16: the split
  // gives every needing lane a group of 2 lanes or more)
  const int split_lanes = std::max(0, std::min(16, (int)ws.tune_nh_split));
  if (kp.tiebreak == CLUE_TIE_RHO_INDEX)
    k_nearest_higher<N, MT, CLUE_TIE_RHO_INDEX><<<chunk_grid(kp), kTileThreads, 0, s>>>(
        kp, events_of(ws), ws.offsets, ws.mq, ws.chunk_tile, ws.chunk_count, ws.chunk_total, ws.rec_r,
        ws.rec_m_cur, ws.mq, ws.blk, ws.sblk, ws.minv, ws.perm, ws.nh_s, ws.delta_s, ws.status,
        split_lanes);
  else
    k_nearest_higher<N, MT, CLUE_TIE_REFERENCE><<<chunk_grid(kp), kTileThreads, 0, s>>>(
        kp, events_of(ws), ws.offsets, ws.mq, ws.chunk_tile, ws.chunk_count, ws.chunk_total, ws.rec_r,
        ws.rec_m_cur, ws.mq, ws.blk, ws.sblk, ws.minv, ws.perm, ws.nh_s, ws.delta_s, ws.status,
        split_lanes);
}
template <int N, int MT, int FORM>
void launch_density_spatial_form(const KParams& kp, Workspace& ws, cudaStream_t s, float kexp) {
  k_density_spatial<N, MT, FORM><<<chunk_grid(kp), kTileThreads, 0, s>>>(
      kp, events_of(ws), ws.offsets, ws.ord_rho, ws.chunk_tile, ws.chunk_count, ws.chunk_total, ws.rec_w,
      ws.rec_m_cur, ws.mq, ws.blk, ws.sblk, ws.rec_r, ws.minv, kexp);
}
template <int N, int MT>
void launch_density_spatial(const KParams& kp, Workspace& ws, cudaStream_t s) {
  const float log2e = 1.4426950408889634f;
  if (kp.kernel_type == CLUE_KERNEL_EXPONENTIAL && kp.kpar[1] == 1.0f)
    launch_density_spatial_form<N, MT, kDensExpUnit>(kp, ws, s, -kp.kpar[0] * log2e);
  else if (kp.kernel_type == CLUE_KERNEL_GAUSSIAN && kp.kpar[0] == 0.0f && kp.kpar[2] == 1.0f)
    launch_density_spatial_form<N, MT, kDensGauss0Unit>(kp, ws, s, -kp.ginv * log2e);
  else
    launch_density_spatial_form<N, MT, kDensGeneric>(kp, ws, s, 0.0f);
}
// Symmetric density: kernel form and largest kernel value (the self term is 1).
template <int N, int MT, int FORM, int VAR>
void launch_density_sym_var(const KParams& kp, Workspace& ws, cudaStream_t s, float kexp, float kmax) {
  k_density_sym<N, MT, FORM, VAR><<<chunk_grid(kp), kTileThreads, 0, s>>>(
      kp, events_of(ws), ws.offsets, ws.chunk_tile, ws.chunk_count, ws.chunk_total, ws.rec_m_cur, ws.mq, ws.tblk_off,
      ws.tblk, ws.rec_r, ws.rho_fix, kexp, kmax, ws.status);
}
template <int N, int MT, int FORM>
void launch_density_sym_form(const KParams& kp, Workspace& ws, cudaStream_t s, float kexp, float kmax) {
  // the pair-step alternatives are built for the Euclidean metric and the unit-amplitude forms
  // in up to four dimensions (the benchmark configurations); elsewhere the plain step runs
  if constexpr (MT == CLUE_METRIC_EUCLIDEAN && FORM != kDensGeneric && N <= 4) {
    const int var = (ws.tune_density_gate ? 1 : 0) | (ws.tune_density_exp2 ? 2 : 0);
    switch (var) {
      case 1: launch_density_sym_var<N, MT, FORM, 1>(kp, ws, s, kexp, kmax); return;
      case 2: launch_density_sym_var<N, MT, FORM, 2>(kp, ws, s, kexp, kmax); return;
      case 3: launch_density_sym_var<N, MT, FORM, 3>(kp, ws, s, kexp, kmax); return;
      default: break;
    }
  }
  launch_density_sym_var<N, MT, FORM, 0>(kp, ws, s, kexp, kmax);
}
template <int N, int MT>
void launch_density_sym(const KParams& kp, Workspace& ws, cudaStream_t s, bool fuse_combine) {
  const float log2e = 1.4426950408889634f;
  float kmax = 1.0f;
  if (kp.kernel_type == CLUE_KERNEL_FLAT) kmax = fmaxf(1.0f, fabsf(kp.kpar[0]));
  if (kp.kernel_type == CLUE_KERNEL_EXPONENTIAL) kmax = fmaxf(1.0f, fabsf(kp.kpar[1]));
  if (kp.kernel_type == CLUE_KERNEL_GAUSSIAN) kmax = fmaxf(1.0f, fabsf(kp.kpar[2]));
  cudaMemsetAsync(ws.rho_fix, 0, (size_t)kp.n * sizeof(int64_t), s);
  if (kp.kernel_type == CLUE_KERNEL_EXPONENTIAL && kp.kpar[1] == 1.0f)
    launch_density_sym_form<N, MT, kDensExpUnit>(kp, ws, s, -kp.kpar[0] * log2e, kmax);
  else if (kp.kernel_type == CLUE_KERNEL_GAUSSIAN && kp.kpar[0] == 0.0f && kp.kpar[2] == 1.0f)
    launch_density_sym_form<N, MT, kDensGauss0Unit>(kp, ws, s, -kp.ginv * log2e, kmax);
  else
    launch_density_sym_form<N, MT, kDensGeneric>(kp, ws, s, 0.0f, kmax);
  if (fuse_combine) {
    ws.sym_kmax = kmax;  // the combine runs with the nearest-higher block boxes
  } else {
    k_density_combine<N><<<grid_for(kp.n, 256), 256, 0, s>>>(kp, events_of(ws), kp.n, ws.rho_fix, ws.rec_r, kmax);
  }
}
// The symmetric sweep covers exactly the reference's candidates when the metric bounds every
// coordinate difference and no coordinate wraps.
inline bool symmetric_density_ok(const KParams& kp, int metric, int ndim) {
  if (metric != CLUE_METRIC_EUCLIDEAN && metric != CLUE_METRIC_MANHATTAN && metric != CLUE_METRIC_CHEBYSHEV)
    return false;
  for (int d = 0; d < ndim; ++d)
    if (kp.wrapped[d]) return false;
  return true;
}
template <int N>
void launch_density_sym_metric(int metric, const KParams& kp, Workspace& ws, cudaStream_t s, bool fuse_combine) {
  if (metric == CLUE_METRIC_MANHATTAN)
    launch_density_sym<N, CLUE_METRIC_MANHATTAN>(kp, ws, s, fuse_combine);
  else if (metric == CLUE_METRIC_CHEBYSHEV)
    launch_density_sym<N, CLUE_METRIC_CHEBYSHEV>(kp, ws, s, fuse_combine);
  else
    launch_density_sym<N, CLUE_METRIC_EUCLIDEAN>(kp, ws, s, fuse_combine);
}
template <int N, int MT>
void launch_seeds(const KParams& kp, Workspace& ws, cudaStream_t s) {
  k_seeds<N, MT><<<grid_for(kp.n, 256), 256, 0, s>>>(kp, kp.n, ws.rec_r, ws.nh_s, ws.delta_s, ws.perm, ws.is_seed_s, ws.par,
                                                     ws.seed_flag, ws.status);
}
template <int N, int MT>
void launch_near_ties(const KParams& kp, Workspace& ws, cudaStream_t s) {
  k_near_ties<N, MT><<<chunk_grid(kp), kTileThreads, 0, s>>>(
      kp, events_of(ws), ws.offsets, ws.mq, ws.chunk_tile, ws.chunk_count, ws.chunk_total, ws.rec_r, ws.rec_m_cur,
      ws.mq, ws.blk, ws.sblk, ws.minv, ws.nh_s, ws.status);
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
  const int n = kp.n;
  InPtrs in{};
  for (int d = 0; d < N; ++d) in.c[d] = a.coords[d];
  in.w = a.weight;
  const Events ev = events_of(ws);
  ws.near_from_host = false;  // this run's counts land in the device status block

  stage_mark(ws, 0, s);
  k_init<N><<<grid_for(kp.n_events, 256), 256, 0, s>>>(kp, ev, ws.ev_pt, ws.ev_tile, ws.status);
  int launches_pre = 0;
  if (kp.n_events == 1)
    k_bbox_single<N><<<std::max(1, std::min(grid_for(n, 1024), 148 * 4)), 256, 0, s>>>(in, n, ws.ev, ws.status);
  else
  {
    // spans of 32..1024 points: about four spans per resident warp (64 per SM) when there
    // are enough points, so the loads of many spans are in flight
    const int span = std::max(32, std::min(1024, (n / (148 * 64 * 4)) & ~31));
    const int blocks = std::max(1, std::min(grid_for(n, 256), ((n + span - 1) / span + 7) / 8));
    if (ws.ev_chunk) {
      k_event_chunks<<<grid_for(kp.n_events, 256), 256, 0, s>>>(kp.n_events, ws.ev_pt, ws.ev_chunk);
      ++launches_pre;
    }
    k_bbox_events<N><<<blocks, 256, 0, s>>>(in, n, kp.n_events, ws.ev_pt, ws.ev_chunk, ws.ev, ws.status, span);
  }
  k_grid<N><<<grid_for(kp.n_events, 256), 256, 0, s>>>(kp.n_events, ws.ev);
  int launches = 4 + launches_pre;  // init, (chunk table,) bbox, grid, bin
  // density order: the reference's candidate order for the flat kernel (bit-exact sums), spatial
  // order for the exponential and Gaussian kernels (whose device expf already differs from the
  // host's by an ulp) unless the caller asks for the reference order
  const bool spatial_density = (kp.flags & CLUE_FLAG_REFERENCE_ORDER) == 0 &&
                               (kp.kernel_type != CLUE_KERNEL_FLAT || (kp.flags & CLUE_FLAG_SPATIAL_DENSITY) != 0);
  // (a workspace without the symmetric sweep's buffers, such as the fixed scratch of the
  // no-allocation entry point, keeps the one-sided sweep)
  const bool symmetric =
      spatial_density && symmetric_density_ok(kp, a.metric, N) && ws.tblk && ws.tblk_off && ws.rho_fix &&
      ws.tune_symmetric != 0;
  const int bits = bits_for((uint32_t)(kp.ntiles - 1));
  const int mbits = MortonSortBits<N>::kBits;
  // The symmetric sweep needs no tile order by point index: one sort by (tile, Morton) composite
  // keys gives its record order, and positions inside a tile are only compared through the
  // points' indices.  The other sweeps take the tile order by index and a Morton order beside it.
  const bool composite = symmetric && bits + mbits <= 32;
  if (composite) {
    k_bin_composite<N><<<grid_for(n, 1024), 256, 0, s>>>(kp, in, ev, mbits, ws.keys[0]);
    const int cur = radix_sort_pairs(ws.keys, ws.vals, true, n, bits + mbits, ws.hist, ws.scan_scratch, s);
    ws.perm = ws.vals[cur];
    ws.sorted_keys = ws.keys[cur];
    offsets_from_sorted(ws.sorted_keys, n, kp.ntiles, ws.offsets, s, mbits);
    ws.mq = ws.vals[cur ^ 1];
    ws.minv = ws.mq_alt;
    k_gather<N><<<grid_for(n, 256), 256, 0, s>>>(in, n, ws.perm, ws.rec_w, ws.status, ws.mq, ws.minv);
    ws.rec_m_cur = ws.rec_w;
    launches += radix_sort_launches(bits + mbits) + 2;
  } else {
    k_bin<N><<<grid_for(n, 256), 256, 0, s>>>(kp, in, ev, ws.keys[0]);
    const int cur = radix_sort_pairs(ws.keys, ws.vals, true, n, bits, ws.hist, ws.scan_scratch, s);
    ws.perm = ws.vals[cur];
    ws.sorted_keys = ws.keys[cur];
    offsets_from_sorted(ws.sorted_keys, n, kp.ntiles, ws.offsets, s);
    k_gather<N><<<grid_for(n, 256), 256, 0, s>>>(in, n, ws.perm, ws.rec_w, ws.status, nullptr, nullptr);
    // fine Morton order inside every tile: a stable sort by Morton key, then a stable sort by
    // tile; mq[p] = tile-sorted position of the p-th record in (tile, Morton) order
    uint32_t* mkeys[2] = {ws.keys[cur ^ 1], ws.mkeys_alt};
    int32_t* mvals[2] = {ws.vals[cur ^ 1], ws.mq_alt};
    k_morton_keys<N><<<grid_for(n, 256), 256, 0, s>>>(kp, ev, ws.rec_w, ws.sorted_keys, mkeys[0]);
    int mc = radix_sort_pairs(mkeys, mvals, true, n, MortonSortBits<N>::kBits, ws.hist, ws.scan_scratch, s);
    if (mc != 0) {
      std::swap(mkeys[0], mkeys[1]);
      std::swap(mvals[0], mvals[1]);
    }
    k_tile_of<<<grid_for(n, 256), 256, 0, s>>>(ws.sorted_keys, mvals[0], n, mkeys[0]);
    mc = radix_sort_pairs(mkeys, mvals, false, n, bits, ws.hist, ws.scan_scratch, s);
    ws.mq = mvals[mc];
    ws.minv = mvals[mc ^ 1];
    k_invert<<<grid_for(n, 256), 256, 0, s>>>(ws.mq, n, ws.minv);
    ws.rec_m_cur = ws.rec_m;
    launches += radix_sort_launches(bits) + 2 + 1 + radix_sort_launches(MortonSortBits<N>::kBits) + 1 +
                radix_sort_launches(bits) + 1;
  }
  if (symmetric)
    k_tile_counts<<<grid_for(kp.ntiles, 256), 256, 0, s>>>(kp.ntiles, ws.offsets, ws.chunk_count, ws.tblk_off);
  else
    k_order<N><<<kp.ntiles, kTileThreads, 0, s>>>(kp, ev, ws.offsets, ws.rec_w, ws.mq, ws.ord_rho, ws.chunk_count);
  exclusive_scan(ws.chunk_count, ws.chunk_count, (size_t)kp.ntiles, ws.scan_scratch, ws.chunk_total, s);
  if (symmetric) exclusive_scan(ws.tblk_off, ws.tblk_off, (size_t)kp.ntiles, ws.scan_scratch, nullptr, s);
  k_chunk_map<<<grid_for(kp.ntiles, 256), 256, 0, s>>>(kp.ntiles, ws.offsets, ws.chunk_count, ws.chunk_tile);
  launches += 1 + kScanLaunches + (symmetric ? kScanLaunches : 0) + 1;

  const int nblk_threads = ((n + 31) >> 5) * 32;
  const int nsb_threads = ((((n + 31) >> 5) + 31) >> 5) * 32;
  const int max_slots = kChunkWarps * (n / kChunk + kp.ntiles + 1);
  if (symmetric) {
    if (!composite) {
      k_gather_morton<N><<<grid_for(n, 256), 256, 0, s>>>(ws.rec_w, n, ws.mq, ws.rec_m);
      ++launches;
    }
    k_tblock_bbox<N><<<grid_for(max_slots, 256), 256, 0, s>>>(max_slots, ws.chunk_total, ws.offsets, ws.chunk_tile,
                                                               ws.chunk_count, ws.tblk_off, ws.rec_m_cur, ws.tblk);
    ++launches;
  } else if (spatial_density) {
    k_gather_morton<N><<<grid_for(n, 256), 256, 0, s>>>(ws.rec_w, n, ws.mq, ws.rec_m);
    k_block_bbox<N><<<grid_for(nblk_threads, 256), 256, 0, s>>>(ws.rec_m, n, ws.blk);
    k_superblock_bbox<N><<<grid_for(nsb_threads, 256), 256, 0, s>>>(ws.blk, n, ws.sblk);
    launches += 3;
  } else {
    k_block_bbox<N><<<grid_for(nblk_threads, 256), 256, 0, s>>>(ws.rec_w, n, ws.blk);
    ++launches;
  }

  stage_mark(ws, 1, s);
  if (symmetric) {
    launch_density_sym_metric<N>(a.metric, kp, ws, s, composite);
  } else if (spatial_density) {
    CLUE_METRIC_SWITCH(a.metric, launch_density_spatial, kp, ws, s);
  } else {
    CLUE_METRIC_SWITCH(a.metric, launch_density, kp, ws, s);
  }
  launches += symmetric && !composite ? 2 : 1;  // (a composite run combines with the block boxes)
  stage_mark(ws, 2, s);
  // Morton-ordered copy of the records with their densities (the tile-ordered records themselves
  // after a composite sort) and its block / super-block boxes with the largest rho, for the
  // nearest-higher search
  if (composite) {
    // the tile-ordered records are the Morton-ordered ones; the density's fixed-point sums are
    // added in while the block boxes are built
    ws.rec_m_cur = ws.rec_r;
    k_combine_block_bbox<N><<<grid_for(nblk_threads, 256), 256, 0, s>>>(kp, ev, n, ws.rho_fix, ws.rec_r,
                                                                         ws.sym_kmax, ws.blk);
  } else {
    k_gather_morton<N><<<grid_for(n, 256), 256, 0, s>>>(ws.rec_r, n, ws.mq, ws.rec_m);
    ws.rec_m_cur = ws.rec_m;
    ++launches;
    k_block_bbox<N><<<grid_for(nblk_threads, 256), 256, 0, s>>>(ws.rec_m_cur, n, ws.blk);
  }
  k_superblock_bbox<N><<<grid_for(nsb_threads, 256), 256, 0, s>>>(ws.blk, n, ws.sblk);
  CLUE_METRIC_SWITCH(a.metric, launch_nh, kp, ws, s);
  if (kp.flags & CLUE_FLAG_NEAR_TIES) {
    CLUE_METRIC_SWITCH(a.metric, launch_near_ties, kp, ws, s);
    ++launches;
  }
  stage_mark(ws, 3, s);
  CLUE_METRIC_SWITCH(a.metric, launch_seeds, kp, ws, s);
  exclusive_scan(ws.seed_flag, ws.seed_flag, (size_t)n, ws.scan_scratch, ws.seed_total, s);
  int label_launches = kJumpLaunches;
  if (ws.tune_labels_bfs) {
    // follower CSR in buffers that are dead by now: the sort keys and the weight records
    uint32_t* counts = ws.keys[0];
    uint32_t* run_end = ws.keys[1];
    int32_t* followers = reinterpret_cast<int32_t*>(ws.rec_w);
    int32_t* front[2] = {followers + n, followers + 2 * (size_t)n};
    cudaMemsetAsync(counts, 0, (size_t)n * sizeof(uint32_t), s);
    k_follower_count<<<grid_for(n, 256), 256, 0, s>>>(ws.par, n, counts);
    exclusive_scan(counts, run_end, (size_t)n, ws.scan_scratch, nullptr, s);
    k_follower_fill<<<grid_for(n, 256), 256, 0, s>>>(ws.par, n, run_end, followers);
    k_bfs_seeds<<<grid_for(n, 256), 256, 0, s>>>(ws.par, ws.is_seed_s, n, front[0], ws.status);
    const int lg = std::min(grid_for(n, 256), 148 * 8);
    for (int l = 0; l < kBfsLevels; ++l)
      k_bfs_level<<<lg, 256, 0, s>>>(run_end, counts, followers, ws.par, front[l & 1], front[(l + 1) & 1], ws.status,
                                     l);
    k_bfs_done<<<1, 1, 0, s>>>(ws.status);
    label_launches = kScanLaunches + kBfsLevels + 4;  // count, scan, fill, seeds, levels, done
  } else {
    for (int r = 0; r < kJumpLaunches; ++r)
      k_jump<<<grid_for(n, 256), 256, 0, s>>>(ws.par, n, kJumpIters, ws.status, r);
  }
  k_finalize<N><<<grid_for(n, 256), 256, 0, s>>>(kp, ev, ws.par, ws.is_seed_s, ws.seed_flag, ws.perm, ws.nh_s,
                                                 ws.rec_r, ws.delta_s, a.out, ws.status);
  k_event_info<<<grid_for(kp.n_events, 256), 256, 0, s>>>(kp, ws.ev, ws.ev_pt, ws.seed_flag, ws.seed_total,
                                                         a.ev_n_seeds, a.ev_n_clusters, ws.status);
  stage_mark(ws, 4, s);
  // Morton boxes, nh, seeds, scan, jumps, finalize, event info
  ws.launches += launches + 3 + 1 + kScanLaunches + label_launches + 1 + 1;
  CLUE_CUDA_TRY(cudaGetLastError());
  return CLUE_OK;
}

// Continue pointer jumping from the host after the enqueued launches left chains
// unresolved (only for very deep nearest-higher chains); synchronises per launch.
template <int N>
clue_status finish_labels(Workspace& ws, const RunArgs& a, cudaStream_t s, int first_round) {
  const int n = a.kp.n;
  for (int r = first_round; r < 64; ++r) {
    k_jump<<<grid_for(n, 256), 256, 0, s>>>(ws.par, n, 1 << 12, ws.status, r);
    ++ws.launches;
    uint32_t unres = 0;
    CLUE_CUDA_TRY(cudaMemcpyAsync(&unres, &ws.status->unresolved[r], 4, cudaMemcpyDeviceToHost, s));
    CLUE_CUDA_TRY(cudaStreamSynchronize(s));
    if (unres == 0) break;
  }
  k_finalize<N><<<grid_for(n, 256), 256, 0, s>>>(a.kp, events_of(ws), ws.par, ws.is_seed_s, ws.seed_flag, ws.perm,
                                                 ws.nh_s, ws.rec_r, ws.delta_s, a.out, ws.status);
  ++ws.launches;
  CLUE_CUDA_TRY(cudaGetLastError());
  return CLUE_OK;
}

template clue_status run_pipeline<CLUE_NDIM>(Workspace&, const RunArgs&, cudaStream_t);
template clue_status finish_labels<CLUE_NDIM>(Workspace&, const RunArgs&, cudaStream_t, int);

}  // namespace clue_b200
