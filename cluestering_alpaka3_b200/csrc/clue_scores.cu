// clue_scores.cu -- post-processing of clustered points on the GPU: silhouette score
// (clue_silhouette) and cluster centroids (clue_cluster_centroids).
//
// The reference computes it on the host (include/CLUEstering/utils/detail/scores.hpp:17-99):
// for a point i of a cluster with at least two points, a = mean distance to the other points of
// its cluster, b = the smallest mean distance to the points of another cluster, and
// s_i = (b - a) / max(a, b); silhouette(points) averages s_i over those points.  Cluster sums
// run over the cluster's points in ascending index order (the association map's order), and a
// distance is sqrt(sum over dimensions of (l - r)^2) accumulated from 0 in dimension order.
//
// Here every point is one thread that streams all clustered points in (cluster, index) order
// (the CSR of clue_get_clusters), staged through shared memory by its block; a cluster's sum
// runs in exactly the reference's order and is turned into a mean when the stream moves to the
// next cluster, so per-point scores are bit-identical to a sequential evaluation without
// contracted multiply-adds.  The work is n x (clustered points) distances.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <string>
#include <vector>

#include "clue_internal.h"

namespace clue_b200 {
namespace {

constexpr int kSilThreads = 128;
constexpr int kSilTile = 512;  // clustered points staged per block step

// sorted coordinates (SoA over the clustered points) and cluster ids in (cluster, index) order
__global__ void k_sil_gather(int ndim, int n, int n_clustered, const float* __restrict__ coords,
                             const int32_t* __restrict__ cluster_index, const int32_t* __restrict__ points,
                             float* __restrict__ sc, int32_t* __restrict__ scid) {
  const int stride = gridDim.x * blockDim.x;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n_clustered; p += stride) {
    const int i = points[p];
    for (int d = 0; d < ndim; ++d) sc[(size_t)d * n_clustered + p] = coords[(size_t)d * n + i];
    scid[p] = cluster_index[i];
  }
}

template <int N>
__global__ void __launch_bounds__(kSilThreads) k_silhouette(int n, int n_clustered, const float* __restrict__ coords,
                                                           const int32_t* __restrict__ cluster_index,
                                                           const int32_t* __restrict__ offsets,
                                                           const float* __restrict__ sc,
                                                           const int32_t* __restrict__ scid,
                                                           float* __restrict__ score) {
  __shared__ float s_c[N][kSilTile];
  __shared__ int32_t s_id[kSilTile];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool inr = i < n;
  float x[N];
  int own = -1;
  if (inr) {
#pragma unroll
    for (int d = 0; d < N; ++d) x[d] = coords[(size_t)d * n + i];
    own = cluster_index[i];
  } else {
#pragma unroll
    for (int d = 0; d < N; ++d) x[d] = 0.0f;
  }
  float a = 0.0f, b = FLT_MAX, sum = 0.0f;
  int cur = -1;
  auto close_cluster = [&]() {
    if (cur < 0) return;
    const int cnt = offsets[cur + 1] - offsets[cur];
    if (cur == own) {
      a = __fdiv_rn(sum, (float)(cnt - 1));
    } else {
      const float m = __fdiv_rn(sum, (float)cnt);
      b = m < b ? m : b;  // std::min(acc, val)
    }
  };
  for (int base = 0; base < n_clustered; base += kSilTile) {
    const int cnt = min(kSilTile, n_clustered - base);
    __syncthreads();
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
#pragma unroll
      for (int d = 0; d < N; ++d) s_c[d][k] = sc[(size_t)d * n_clustered + base + k];
      s_id[k] = scid[base + k];
    }
    __syncthreads();
    for (int k = 0; k < cnt; ++k) {
      const int c = s_id[k];
      if (c != cur) {  // the same for every thread of the block
        close_cluster();
        cur = c;
        sum = 0.0f;
      }
      float dist = 0.0f;
#pragma unroll
      for (int d = 0; d < N; ++d) {
        const float t = __fsub_rn(x[d], s_c[d][k]);
        dist = __fadd_rn(dist, __fmul_rn(t, t));
      }
      dist = __fsqrt_rn(dist);
      // (the point itself adds its distance 0 to its own cluster's sum: the sums are
      // non-negative, so that leaves them as the reference's skip of the point does)
      sum = __fadd_rn(sum, dist);
    }
  }
  close_cluster();
  if (!inr) return;
  bool valid = own >= 0;
  if (valid) valid = offsets[own + 1] - offsets[own] >= 2;
  score[i] = valid ? __fdiv_rn(__fsub_rn(b, a), a < b ? b : a) : NAN;  // std::max(a, b)
}

template <int N>
void launch_silhouette(int n, int n_clustered, const float* coords, const int32_t* cluster_index,
                       const int32_t* offsets, const float* sc, const int32_t* scid, float* score, cudaStream_t s) {
  k_silhouette<N><<<(n + kSilThreads - 1) / kSilThreads, kSilThreads, 0, s>>>(n, n_clustered, coords, cluster_index,
                                                                              offsets, sc, scid, score);
}

}  // namespace
}  // namespace clue_b200

namespace clue_b200 {
namespace {

// Centroid of cluster c, dimension d (reference utils/detail/cluster_centroid.hpp:39-65): the
// cluster's coordinates summed from 0 in ascending point order (the CSR of clue_get_clusters
// lists a cluster's points that way) with separately rounded FP32 adds, divided by the size as
// a float.  One thread per (cluster, dimension); the sums are sequential so the bits match
// the reference's host loop.
__global__ void __launch_bounds__(256) k_centroids(int ndim, int n, int n_clusters, const float* __restrict__ coords,
                                                   const int32_t* __restrict__ offsets,
                                                   const int32_t* __restrict__ points, float* __restrict__ centroids,
                                                   int32_t* __restrict__ sizes) {
  const int stride = gridDim.x * blockDim.x;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n_clusters * ndim; t += stride) {
    const int c = t / ndim, d = t - c * ndim;
    const int b = offsets[c], e = offsets[c + 1];
    const float* x = coords + (size_t)d * n;
    float acc = 0.0f;
    for (int q = b; q < e; ++q) acc = fadd(acc, __ldg(x + points[q]));
    centroids[(size_t)c * ndim + d] = fdiv(acc, (float)(e - b));
    if (sizes && d == 0) sizes[c] = e - b;
  }
}

}  // namespace
}  // namespace clue_b200

using namespace clue_b200;

extern "C" {

clue_status clue_cluster_centroids(clue_context ctx, int32_t ndim, int32_t n, const float* coords,
                                   const int32_t* cluster_index, int32_t capacity, float* centroids,
                                   int32_t* sizes, int32_t* n_clusters_out, void* stream) {
  if (!ctx || !coords || !cluster_index || (!centroids && capacity > 0) || n <= 0 || capacity < 0 || ndim < 1 ||
      ndim > kMaxDim) {
    set_error("clue_cluster_centroids: null argument, n <= 0, capacity < 0 or ndim outside [1, 10]");
    return CLUE_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  int32_t *offsets = nullptr, *points = nullptr;
  cudaError_t e = cudaMalloc(&offsets, ((size_t)n + 1) * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc(&points, (size_t)n * sizeof(int32_t));
  if (e != cudaSuccess) {
    if (offsets) cudaFree(offsets);
    set_error(std::string("clue_cluster_centroids: ") + cudaGetErrorString(e));
    return CLUE_ERR_OUT_OF_MEMORY;
  }
  int32_t n_clusters = 0, n_clustered = 0;
  clue_status st = clue_get_clusters(ctx, n, cluster_index, offsets, points, &n_clusters, &n_clustered, stream);
  if (st == CLUE_OK && n_clusters_out) *n_clusters_out = n_clusters;
  if (st == CLUE_OK && n_clusters > capacity) {
    set_error("clue_cluster_centroids: more clusters (" + std::to_string(n_clusters) + ") than the capacity (" +
              std::to_string(capacity) + ")");
    st = CLUE_ERR_CAPACITY;
  }
  if (st == CLUE_OK && n_clusters > 0) {
    const int work = n_clusters * ndim;
    k_centroids<<<std::max(1, std::min((work + 255) / 256, 148 * 16)), 256, 0, s>>>(
        ndim, n, n_clusters, coords, offsets, points, centroids, sizes);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the temporaries are freed below
    if (e != cudaSuccess) {
      set_error(std::string("clue_cluster_centroids: ") + cudaGetErrorString(e));
      st = CLUE_ERR_CUDA;
    }
  }
  cudaFree(offsets);
  cudaFree(points);
  return st;
}

clue_status clue_silhouette(clue_context ctx, int32_t ndim, int32_t n, const float* coords,
                            const int32_t* cluster_index, float* per_point, float* mean, void* stream) {
  if (!ctx || !coords || !cluster_index || n <= 0 || ndim < 1 || ndim > kMaxDim) {
    set_error("clue_silhouette: null argument, n <= 0 or ndim outside [1, 10]");
    return CLUE_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  int32_t *offsets = nullptr, *points = nullptr, *scid = nullptr;
  float *sc = nullptr, *score = per_point;
  auto release = [&]() {
    if (offsets) cudaFree(offsets);
    if (points) cudaFree(points);
    if (scid) cudaFree(scid);
    if (sc) cudaFree(sc);
    if (score && score != per_point) cudaFree(score);
  };
  cudaError_t e = cudaMalloc(&offsets, ((size_t)n + 1) * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc(&points, (size_t)n * sizeof(int32_t));
  if (e == cudaSuccess && !score) e = cudaMalloc(&score, (size_t)n * sizeof(float));
  if (e != cudaSuccess) {
    release();
    set_error(std::string("clue_silhouette: ") + cudaGetErrorString(e));
    return CLUE_ERR_OUT_OF_MEMORY;
  }
  int32_t n_clusters = 0, n_clustered = 0;
  clue_status st = clue_get_clusters(ctx, n, cluster_index, offsets, points, &n_clusters, &n_clustered, stream);
  if (st == CLUE_OK && n_clustered > 0) {
    e = cudaMalloc(&sc, (size_t)ndim * n_clustered * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&scid, (size_t)n_clustered * sizeof(int32_t));
    if (e != cudaSuccess) {
      set_error(std::string("clue_silhouette: ") + cudaGetErrorString(e));
      st = CLUE_ERR_OUT_OF_MEMORY;
    }
  }
  if (st == CLUE_OK) {
    const int blocks = std::max(1, std::min((n_clustered + 255) / 256, 148 * 16));
    if (n_clustered > 0)
      k_sil_gather<<<blocks, 256, 0, s>>>(ndim, n, n_clustered, coords, cluster_index, points, sc, scid);
    switch (ndim) {
      case 1: launch_silhouette<1>(n, n_clustered, coords, cluster_index, offsets, sc, scid, score, s); break;
      case 2: launch_silhouette<2>(n, n_clustered, coords, cluster_index, offsets, sc, scid, score, s); break;
      case 3: launch_silhouette<3>(n, n_clustered, coords, cluster_index, offsets, sc, scid, score, s); break;
      case 4: launch_silhouette<4>(n, n_clustered, coords, cluster_index, offsets, sc, scid, score, s); break;
      case 5: launch_silhouette<5>(n, n_clustered, coords, cluster_index, offsets, sc, scid, score, s); break;
      case 6: launch_silhouette<6>(n, n_clustered, coords, cluster_index, offsets, sc, scid, score, s); break;
      case 7: launch_silhouette<7>(n, n_clustered, coords, cluster_index, offsets, sc, scid, score, s); break;
      case 8: launch_silhouette<8>(n, n_clustered, coords, cluster_index, offsets, sc, scid, score, s); break;
      case 9: launch_silhouette<9>(n, n_clustered, coords, cluster_index, offsets, sc, scid, score, s); break;
      default: launch_silhouette<10>(n, n_clustered, coords, cluster_index, offsets, sc, scid, score, s); break;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      set_error(std::string("clue_silhouette: ") + cudaGetErrorString(e));
      st = CLUE_ERR_CUDA;
    }
  }
  if (st == CLUE_OK && mean) {
    // the average in index order over the points of clusters with at least two points, in
    // FP32 like the reference's reduce
    std::vector<float> h(n);
    std::vector<int32_t> lab(n), hoff((size_t)n_clusters + 1);
    e = cudaMemcpyAsync(h.data(), score, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(lab.data(), cluster_index, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(hoff.data(), offsets, ((size_t)n_clusters + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      set_error(std::string("clue_silhouette: ") + cudaGetErrorString(e));
      st = CLUE_ERR_CUDA;
    } else {
      float acc = 0.0f;
      int64_t cnt = 0;
      for (int i = 0; i < n; ++i) {
        const int c = lab[i];
        if (c < 0 || hoff[c + 1] - hoff[c] < 2) continue;
        acc += h[i];
        ++cnt;
      }
      *mean = acc / (float)cnt;
    }
  }
  if (st == CLUE_OK && !mean) {
    e = cudaStreamSynchronize(s);  // the temporaries are freed below
    if (e != cudaSuccess) st = CLUE_ERR_CUDA;
  }
  release();
  return st;
}

}  // extern "C"
