// clue_sort.cu -- stable LSD radix sort, exclusive scan and CSR offsets.
//
// These replace the reference's atomic association-map fill
// (data_structures/AssociationMap.hpp:122-191 with the kernels of
// data_structures/detail/AssociationMap.hpp:13-67) and alpaka's inclusiveScan: the
// tile CSR is produced by a stable sort of (tile, point index) pairs, so the order
// inside every tile is ascending point index -- the order the reference's serial
// backend produces -- instead of the GPU atomic order.
#include "clue_internal.h"

namespace clue_b200 {

namespace {

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Per-block digit histogram; hist is digit-major: hist[d * nblocks + block].  Every warp counts
// into its own shared-memory histogram (plain shared atomics), the warps' counts are summed at
// the end; keys are read four at a time where the tile is complete.
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const uint32_t* __restrict__ keys, int n,
                                                             int shift, uint32_t* __restrict__ hist,
                                                             int nblocks) {
  constexpr int kWarps = kSortThreads / 32;
  __shared__ uint32_t h[kWarps][kRadix];
  const int warp = threadIdx.x >> 5;
  for (int e = threadIdx.x; e < kWarps * kRadix; e += blockDim.x) (&h[0][0])[e] = 0;
  __syncthreads();
  const int base = blockIdx.x * kSortTile;
  uint32_t* hw = h[warp];
  if (base + kSortTile <= n) {
    const uint4* k4 = reinterpret_cast<const uint4*>(keys + base);
#pragma unroll
    for (int r = 0; r < kSortItems / 4; ++r) {
      const uint4 v = __ldg(k4 + r * kSortThreads + threadIdx.x);
      atomicAdd(&hw[(v.x >> shift) & (kRadix - 1)], 1u);
      atomicAdd(&hw[(v.y >> shift) & (kRadix - 1)], 1u);
      atomicAdd(&hw[(v.z >> shift) & (kRadix - 1)], 1u);
      atomicAdd(&hw[(v.w >> shift) & (kRadix - 1)], 1u);
    }
  } else {
    for (int i = base + threadIdx.x; i < n; i += kSortThreads) atomicAdd(&hw[(keys[i] >> shift) & (kRadix - 1)], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += blockDim.x) {
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) c += h[w][d];
    hist[(size_t)d * nblocks + blockIdx.x] = c;
  }
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread; returns the block total via *tot.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* tot) {
  __shared__ uint32_t ws[33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t inc = warp_incl_scan(v);
  if (lane == 31) ws[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const uint32_t x = lane < nw ? ws[lane] : 0u;
    const uint32_t xi = warp_incl_scan(x);
    if (lane < nw) ws[lane] = xi - x;
    if (lane == nw - 1) ws[32] = xi;
  }
  __syncthreads();
  const uint32_t r = ws[warp] + inc - v;
  if (tot) *tot = ws[32];
  __syncthreads();
  return r;
}

// Stable scatter of one tile of kSortTile items.  Warp w ranks the w-th slice of the tile
// (kSortItems steps of 32 consecutive items) against warp-private digit counters, so inside a
// warp items keep index order without block barriers; one block-wide pass then turns the
// per-warp counts into slice bases (digits in order, warps in order inside a digit).  Items are
// placed digit-sorted in shared memory and written out in that order, so consecutive threads
// write consecutive slots of a digit's run.  The tile's count of digit d is the difference of
// consecutive entries of the digit-major scanned histogram.
// Four CTAs per SM (64 registers, a few bytes spilled): measured faster than three with 80
// registers (tile stage of calo4096 1.104 -> 1.068 ms), and again with the ballot ranking below
// against three and five CTAs (tile stage 0.855 ms against 0.950 and 0.959 ms).
__global__ void __launch_bounds__(kSortThreads, 4) k_radix_scatter(
    const uint32_t* __restrict__ kin, const int32_t* __restrict__ vin, uint32_t* __restrict__ kout,
    int32_t* __restrict__ vout, int n, int shift, const uint32_t* __restrict__ scanned,
    const uint32_t* __restrict__ tot, int nblocks) {
  static_assert(kSortThreads == kRadix, "one thread per digit");
  constexpr int kWarps = kSortThreads / 32;
  constexpr int kSlice = kSortItems * 32;  // items per warp
  __shared__ uint32_t s_key[kSortTile];
  __shared__ int32_t s_val[kSortTile];
  __shared__ uint32_t gbase[kRadix];
  __shared__ uint32_t wcnt[kWarps][kRadix];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int base = blockIdx.x * kSortTile;
  const int tile_n = min(kSortTile, n - base);
  for (int e = threadIdx.x; e < kWarps * kRadix; e += blockDim.x) (&wcnt[0][0])[e] = 0;
  uint32_t dstart;
  {
    const int d = threadIdx.x;
    const size_t idx = (size_t)d * nblocks + blockIdx.x;
    const uint32_t first = scanned[idx];  // digit d's items in earlier blocks
    const uint32_t total = tot[d];
    const uint32_t next = (int)blockIdx.x + 1 < nblocks ? scanned[idx + 1] : total;
    const uint32_t dbase = block_excl_scan(total, nullptr);  // items of smaller digits
    dstart = block_excl_scan(next - first, nullptr);          // ends with a block barrier
    gbase[d] = dbase + first - dstart;
  }
  uint32_t key[kSortItems], off[kSortItems];
  int32_t val[kSortItems];
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int k = warp * kSlice + r * 32 + lane;
    const bool valid = k < tile_n;
    key[r] = valid ? kin[base + k] : 0u;
    val[r] = valid ? (vin ? vin[base + k] : base + k) : 0;
    const uint32_t d = valid ? (key[r] >> shift) & (kRadix - 1) : (uint32_t)kRadix;
    // lanes holding the same digit: one ballot per digit bit (and one for validity), measured
    // faster than __match_any_sync (tile stage of calo4096 1.04 -> 0.92 ms)
    uint32_t peers = __ballot_sync(0xffffffffu, valid);
    peers = valid ? peers : ~peers;
#pragma unroll
    for (int b = 0; b < kRadixBits; ++b) {
      const bool bit = (d >> b) & 1u;
      const uint32_t bb = __ballot_sync(0xffffffffu, bit);
      peers &= bit ? bb : ~bb;
    }
    const uint32_t rank = __popc(peers & lt);
    off[r] = valid ? wcnt[warp][d] + rank : 0u;
    __syncwarp();
    if (valid && rank == 0) wcnt[warp][d] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {
    const int d = threadIdx.x;
    uint32_t acc = dstart;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t c = wcnt[w][d];
      wcnt[w][d] = acc;
      acc += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int k = warp * kSlice + r * 32 + lane;
    if (k < tile_n) {
      const uint32_t pos = wcnt[warp][(key[r] >> shift) & (kRadix - 1)] + off[r];
      s_key[pos] = key[r];
      s_val[pos] = val[r];
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < tile_n; k += kSortThreads) {
    const uint32_t kk = s_key[k];
    const uint32_t g = gbase[(kk >> shift) & (kRadix - 1)] + (uint32_t)k;
    kout[g] = kk;
    vout[g] = s_val[k];
  }
}

// Exclusive scan of every digit's row of the digit-major histogram, one CTA per digit (rows are
// contiguous); the row's total goes to tot[d].
__global__ void __launch_bounds__(1024) k_scan_rows(uint32_t* __restrict__ hist, int nblocks,
                                                    uint32_t* __restrict__ tot) {
  uint32_t* row = hist + (size_t)blockIdx.x * nblocks;
  const int per = (nblocks + 1023) / 1024;
  const int beg = min(nblocks, (int)threadIdx.x * per), end = min(nblocks, beg + per);
  uint32_t s = 0;
  for (int b = beg; b < end; ++b) s += row[b];
  uint32_t total;
  uint32_t run = block_excl_scan(s, &total);
  for (int b = beg; b < end; ++b) {
    const uint32_t c = row[b];
    row[b] = run;
    run += c;
  }
  if (threadIdx.x == 0) tot[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const uint32_t* __restrict__ in, size_t len,
                                                              uint32_t* __restrict__ partial) {
  const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < len) s += in[base + k];
  uint32_t tot;
  block_excl_scan(s, &tot);
  if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

// Single block: exclusive scan of the per-block partials (any count, looped).
__global__ void __launch_bounds__(1024) k_scan_partials(uint32_t* partial, int nparts, uint32_t* total) {
  uint32_t carry = 0;
  for (int base = 0; base < nparts; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const uint32_t v = i < nparts ? partial[i] : 0u;
    uint32_t tot;
    const uint32_t ex = block_excl_scan(v, &tot);
    if (i < nparts) partial[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

// `in` and `out` may alias (in-place scan): every thread reads its items before writing them.
__global__ void __launch_bounds__(kScanThreads) k_scan_down(const uint32_t* in, size_t len,
                                                            const uint32_t* __restrict__ partial,
                                                            uint32_t* out) {
  const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < len ? in[base + k] : 0u;
    s += v[k];
  }
  uint32_t run = partial[blockIdx.x] + block_excl_scan(s, nullptr);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < len) out[base + k] = run;
    run += v[k];
  }
}

__global__ void k_offsets(const uint32_t* __restrict__ keys, int n, int nkeys, int shift, int32_t* __restrict__ off) {
  const int stride = gridDim.x * blockDim.x;
  for (int pos = blockIdx.x * blockDim.x + threadIdx.x; pos <= n; pos += stride) {
    const int prev = pos > 0 ? (int)(keys[pos - 1] >> shift) : -1;
    const int cur = pos < n ? (int)(keys[pos] >> shift) : nkeys;
    for (int b = prev + 1; b <= cur; ++b) off[b] = pos;
  }
}

}  // namespace

void exclusive_scan(const uint32_t* in, uint32_t* out, size_t len, uint32_t* scratch, uint32_t* total,
                    cudaStream_t s) {
  const int nb = (int)((len + kScanTile - 1) / kScanTile);
  if (nb == 0) {
    if (total) cudaMemsetAsync(total, 0, sizeof(uint32_t), s);
    return;
  }
  k_scan_reduce<<<nb, kScanThreads, 0, s>>>(in, len, scratch);
  k_scan_partials<<<1, 1024, 0, s>>>(scratch, nb, total);
  k_scan_down<<<nb, kScanThreads, 0, s>>>(in, len, scratch, out);
}

int radix_sort_pairs(uint32_t* keys[2], int32_t* vals[2], bool vals_identity, int n, int bits,
                     uint32_t* hist, uint32_t* scan_scratch, cudaStream_t s) {
  const int nb = sort_blocks(n);
  int cur = 0;
  const int passes = bits <= 0 ? 1 : (bits + kRadixBits - 1) / kRadixBits;
  for (int p = 0; p < passes; ++p) {
    const int shift = p * kRadixBits;
    uint32_t* tot = hist + (size_t)kRadix * nb;
    k_radix_hist<<<nb, kSortThreads, 0, s>>>(keys[cur], n, shift, hist, nb);
    k_scan_rows<<<kRadix, 1024, 0, s>>>(hist, nb, tot);
    const int32_t* vin = (p == 0 && vals_identity) ? nullptr : vals[cur];
    k_radix_scatter<<<nb, kSortThreads, 0, s>>>(keys[cur], vin, keys[cur ^ 1], vals[cur ^ 1], n, shift,
                                                hist, tot, nb);
    cur ^= 1;
  }
  return cur;
}

void offsets_from_sorted(const uint32_t* sorted_keys, int n, int nkeys, int32_t* offsets, cudaStream_t s,
                         int shift) {
  const int threads = 256;
  int blocks = (n + 1 + threads - 1) / threads;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_offsets<<<blocks, threads, 0, s>>>(sorted_keys, n, nkeys, shift, offsets);
}

}  // namespace clue_b200
