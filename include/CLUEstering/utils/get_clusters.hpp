// get_clusters.hpp -- cluster -> points maps of clustered points
// (reference: include/CLUEstering/utils/get_clusters.hpp:21-36).  The host overload builds a
// HostAssociationMap; the device overload builds a DevAssociationMap on the GPU
// (clue_get_clusters) and throws std::invalid_argument when no point is clustered.
#pragma once

#include "CLUEstering/data_structures/AssociationMap.hpp"
#include "CLUEstering/data_structures/Points.hpp"

#include <algorithm>
#include <cstddef>
#include <span>

namespace clue {

  template <std::size_t Ndim>
  inline HostAssociationMap get_clusters(const PointsHost<Ndim>& points) {
    auto ids = points.clusterIndexes();
    const auto clustered = std::ranges::count_if(ids, [](int c) { return c > -1; });
    return internal::make_associator(std::span<const int32_t>(ids.data(), ids.size()), static_cast<int32_t>(clustered));
  }

  template <concepts::Queue TQueue, std::size_t Ndim>
  inline DevAssociationMap get_clusters(TQueue& queue, const PointsDevice<DevType<TQueue>, Ndim>& points) {
    auto ids = points.clusterIndexes();
    return internal::make_associator(queue, std::span<const int32_t>(ids.data(), ids.size()));
  }

}  // namespace clue
