// cluster_centroid.hpp -- centroids of clusters (reference:
// include/CLUEstering/utils/cluster_centroid.hpp and utils/detail/cluster_centroid.hpp:12-65):
// the unweighted mean of the coordinates of a cluster's points, summed in point order in FP32;
// on the host from PointsHost, or on the GPU from PointsDevice.
#pragma once

#include "CLUEstering/utils/get_clusters.hpp"

#include <array>
#include <cstddef>
#include <memory>
#include <stdexcept>
#include <vector>

namespace clue {

  template <std::size_t Ndim>
  using Centroid = std::array<float, Ndim>;
  template <std::size_t Ndim>
  using Centroids = std::vector<Centroid<Ndim>>;

  template <std::size_t Ndim>
  inline Centroid<Ndim> cluster_centroid(const PointsHost<Ndim>& points, std::size_t cluster_id) {
    const auto clusters = get_clusters(points);
    const auto size = clusters.count(static_cast<int32_t>(cluster_id));
    Centroid<Ndim> centroid{};
    auto ids = points.clusterIndexes();
    for (std::size_t d = 0; d < Ndim; ++d) {
      auto coords = points.coords(d);
      for (int i = 0; i < points.size(); ++i)
        if (ids[i] >= 0 && static_cast<std::size_t>(ids[i]) == cluster_id) centroid[d] += coords[i];
      centroid[d] /= static_cast<float>(size);
    }
    return centroid;
  }

  template <std::size_t Ndim>
  inline Centroids<Ndim> cluster_centroids(const PointsHost<Ndim>& points) {
    const auto clusters = get_clusters(points);
    Centroids<Ndim> centroids(clusters.size(), Centroid<Ndim>{});
    auto ids = points.clusterIndexes();
    for (std::size_t d = 0; d < Ndim; ++d) {
      auto coords = points.coords(d);
      for (int i = 0; i < points.size(); ++i)
        if (ids[i] >= 0) centroids[ids[i]][d] += coords[i];
      for (std::size_t c = 0; c < centroids.size(); ++c)
        centroids[c][d] /= static_cast<float>(clusters.count(static_cast<int32_t>(c)));
    }
    return centroids;
  }

  // The same centroids computed on the GPU (clue_cluster_centroids) from device points and their
  // labels, bit for bit equal to cluster_centroids(points) on a host copy.  Coordinates that are
  // not one contiguous SoA block are copied into one first.
  template <concepts::Queue TQueue, std::size_t Ndim>
  inline Centroids<Ndim> cluster_centroids(TQueue& queue, const PointsDevice<DevType<TQueue>, Ndim>& points) {
    const int32_t n = points.size();
    const int dev = queue.getDevice().id;
    const float* base = points.coords(0).data();
    bool contiguous = true;
    for (std::size_t d = 1; d < Ndim; ++d) contiguous = contiguous && points.coords(d).data() == base + d * n;
    void* tmp = nullptr;
    if (!contiguous) {
      detail::check(clue_device_alloc(dev, Ndim * (std::size_t)n * sizeof(float), &tmp));
      for (std::size_t d = 0; d < Ndim; ++d)
        detail::check(clue_memcpy_dtod(static_cast<float*>(tmp) + d * n, points.coords(d).data(),
                                       (std::size_t)n * sizeof(float), queue.stream()));
      base = static_cast<const float*>(tmp);
    }
    std::unique_ptr<void, clue_status (*)(void*)> guard(tmp, clue_device_free);
    static thread_local std::unique_ptr<clue_context_s, clue_status (*)(clue_context)> ctx(nullptr, clue_context_destroy);
    static thread_local int32_t ctx_dev = -1;
    if (!ctx || ctx_dev != dev) {
      clue_context c = nullptr;
      detail::check(clue_context_create(dev, &c));
      ctx.reset(c);
      ctx_dev = dev;
    }
    // a first call sizes the output (CLUE_ERR_CAPACITY reports the cluster count)
    int32_t ncl = 0;
    void* dcen = nullptr;
    const clue_status probe = clue_cluster_centroids(ctx.get(), static_cast<int32_t>(Ndim), n, base,
                                                     points.clusterIndexes().data(), 0, nullptr, nullptr, &ncl,
                                                     queue.stream());
    if (probe != CLUE_OK && probe != CLUE_ERR_CAPACITY) detail::check(probe);
    Centroids<Ndim> out(static_cast<std::size_t>(ncl), Centroid<Ndim>{});
    if (ncl == 0) return out;
    detail::check(clue_device_alloc(dev, (std::size_t)ncl * Ndim * sizeof(float), &dcen));
    std::unique_ptr<void, clue_status (*)(void*)> guard_c(dcen, clue_device_free);
    detail::check(clue_cluster_centroids(ctx.get(), static_cast<int32_t>(Ndim), n, base, points.clusterIndexes().data(),
                                         ncl, static_cast<float*>(dcen), nullptr, &ncl, queue.stream()));
    detail::check(clue_memcpy_dtoh(out.data(), dcen, (std::size_t)ncl * Ndim * sizeof(float), queue.stream()));
    detail::check(clue_stream_synchronize(queue.stream()));
    return out;
  }

}  // namespace clue
