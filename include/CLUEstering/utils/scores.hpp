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

}  // namespace clue
