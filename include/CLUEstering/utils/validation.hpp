// validation.hpp -- compare two clusterings of the same points by their cluster count and their
// multiset of cluster sizes (reference: include/CLUEstering/utils/validation.hpp:13-24).  Labels
// may differ: a relabelled copy of a clustering validates against it.
#pragma once

#include "CLUEstering/data_structures/Points.hpp"

#include <algorithm>
#include <cstddef>
#include <vector>

namespace clue {

  template <std::size_t Ndim>
  inline bool validate_results(PointsHost<Ndim>& results, PointsHost<Ndim>& truth) {
    if (results.n_clusters() != truth.n_clusters()) return false;
    std::vector<std::size_t> a = results.cluster_sizes();
    std::vector<std::size_t> b = truth.cluster_sizes();
    std::ranges::sort(a);
    std::ranges::sort(b);
    return a == b;
  }

}  // namespace clue
