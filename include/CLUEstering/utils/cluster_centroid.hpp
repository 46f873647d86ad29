// cluster_centroid.hpp -- centroids of clusters (reference:
// include/CLUEstering/utils/cluster_centroid.hpp and utils/detail/cluster_centroid.hpp:12-65):
// the unweighted mean of the coordinates of a cluster's points, summed in point order in FP32.
#pragma once

#include "CLUEstering/utils/get_clusters.hpp"

#include <array>
#include <cstddef>
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

}  // namespace clue
