// ClusterProperties.hpp -- number of clusters, cluster -> points map and cluster sizes of a
// clustered set of points (reference: include/CLUEstering/data_structures/ClusterProperties.hpp).
#pragma once

#include "CLUEstering/data_structures/AssociationMap.hpp"

#include <algorithm>
#include <cstddef>
#include <span>
#include <vector>

namespace clue {

  class ClusterProperties {
  public:
    explicit ClusterProperties(std::span<const int> cluster_indexes)
        : m_nclusters(compute_nclusters(cluster_indexes)),
          m_clusters(static_cast<std::size_t>(
                         std::ranges::count_if(cluster_indexes, [](int c) { return c >= 0; })),
                     m_nclusters) {
      m_clusters.fill(cluster_indexes);
      m_cluster_sizes.resize(m_nclusters);
      for (std::size_t c = 0; c < m_nclusters; ++c) m_cluster_sizes[c] = m_clusters.count(static_cast<int32_t>(c));
    }
    const std::size_t& n_clusters() const { return m_nclusters; }
    const HostAssociationMap& clusters() const { return m_clusters; }
    const std::vector<std::size_t>& cluster_sizes() const { return m_cluster_sizes; }

    // max label + 1 (reference: utils/detail/get_cluster_properties.hpp)
    static std::size_t compute_nclusters(std::span<const int> cluster_indexes) {
      int mx = -1;
      for (int c : cluster_indexes) mx = std::max(mx, c);
      return static_cast<std::size_t>(mx + 1);
    }

  private:
    std::size_t m_nclusters;
    HostAssociationMap m_clusters;
    std::vector<std::size_t> m_cluster_sizes;
  };

}  // namespace clue
