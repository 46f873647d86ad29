// scores.hpp -- silhouette score of clustered points (reference:
// include/CLUEstering/utils/detail/scores.hpp:17-99): for a point i of a cluster with at least
// two points, a = mean Euclidean distance to the other points of its cluster, b = the smallest
// mean distance to the points of another cluster, s = (b - a) / max(a, b); silhouette(points)
// averages s over clustered points of clusters with at least two points.  Distances are
// sqrt(sum (l - r)^2) accumulated in dimension order in FP32, as in the reference.
#pragma once

#include "CLUEstering/utils/get_clusters.hpp"

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <limits>
#include <memory>
#include <vector>

namespace clue {

  namespace detail {
    template <std::size_t Ndim>
    inline float euclid(const PointsHost<Ndim>& p, int i, int j) {
      float s = 0.f;
      for (std::size_t d = 0; d < Ndim; ++d) {
        const float t = p.view().coords[d][i] - p.view().coords[d][j];
        s += t * t;
      }
      return std::sqrt(s);
    }

    template <std::size_t Ndim>
    inline float silhouette(const HostAssociationMap& clusters, const PointsHost<Ndim>& points, int point) {
      const int own = points.view().cluster_index[point];
      float a = 0.f;
      for (auto it = clusters.lower_bound(own); it != clusters.upper_bound(own); ++it)
        if (*it != point) a += euclid(points, point, *it);
      a /= static_cast<float>(clusters.count(own) - 1);
      float b = std::numeric_limits<float>::max();
      for (int c = 0; c < static_cast<int>(clusters.size()); ++c) {
        if (c == own) continue;
        float s = 0.f;
        for (auto it = clusters.lower_bound(c); it != clusters.upper_bound(c); ++it) s += euclid(points, point, *it);
        s /= static_cast<float>(clusters.count(c));
        b = std::min(b, s);
      }
      return (b - a) / std::max(a, b);
    }
  }  // namespace detail

  template <std::size_t Ndim>
  inline float silhouette(const PointsHost<Ndim>& points, int point) {
    const auto clusters = get_clusters(points);
    return detail::silhouette<Ndim>(clusters, points, point);
  }

  template <std::size_t Ndim>
  inline float silhouette(const PointsHost<Ndim>& points) {
    const auto clusters = get_clusters(points);
    float sum = 0.f;
    std::size_t count = 0;
    for (int i = 0; i < points.size(); ++i) {
      const int c = points.view().cluster_index[i];
      if (c == -1 || clusters.count(c) < 2) continue;
      sum += detail::silhouette<Ndim>(clusters, points, i);
      ++count;
    }
    return sum / static_cast<float>(count);
  }

  // The same score computed on the GPU (clue_silhouette) from device points and their labels,
  // bit for bit equal to silhouette(points) on a host copy.  Coordinates that are not one
  // contiguous SoA block are copied into one first.
  template <concepts::Queue TQueue, std::size_t Ndim>
  inline float silhouette(TQueue& queue, const PointsDevice<DevType<TQueue>, Ndim>& points) {
    const int32_t n = points.size();
    const float* base = points.coords(0).data();
    bool contiguous = true;
    for (std::size_t d = 1; d < Ndim; ++d) contiguous = contiguous && points.coords(d).data() == base + d * n;
    void* tmp = nullptr;
    if (!contiguous) {
      detail::check(clue_device_alloc(queue.getDevice().id, Ndim * (std::size_t)n * sizeof(float), &tmp));
      for (std::size_t d = 0; d < Ndim; ++d)
        detail::check(clue_memcpy_dtod(static_cast<float*>(tmp) + d * n, points.coords(d).data(),
                                       (std::size_t)n * sizeof(float), queue.stream()));
      base = static_cast<const float*>(tmp);
    }
    std::unique_ptr<void, clue_status (*)(void*)> guard(tmp, clue_device_free);
    static thread_local std::unique_ptr<clue_context_s, clue_status (*)(clue_context)> ctx(nullptr, clue_context_destroy);
    static thread_local int32_t ctx_dev = -1;
    if (!ctx || ctx_dev != queue.getDevice().id) {
      clue_context c = nullptr;
      detail::check(clue_context_create(queue.getDevice().id, &c));
      ctx.reset(c);
      ctx_dev = queue.getDevice().id;
    }
    float mean = 0.f;
    detail::check(clue_silhouette(ctx.get(), static_cast<int32_t>(Ndim), n, base, points.clusterIndexes().data(), nullptr,
                                  &mean, queue.stream()));
    return mean;
  }

}  // namespace clue
