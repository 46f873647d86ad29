// Clusterer.hpp -- clue::Clusterer<TQueue, N>, the user-facing entry of the CLUE pipeline.
//
// Same constructors, defaults, overloads and exceptions as the reference
// (include/CLUEstering/core/Clusterer.hpp:84-207, core/detail/Clusterer.hpp:20-48):
//   * Clusterer(queue, Dim<N>, dc, rhoc, dm = dc, seed_dc = dc, pPBin = 128) throws
//     std::invalid_argument unless dc > 0, rhoc >= 0, dm > 0, seed_dc > 0, pPBin > 0;
//   * make_clusters(queue, h), make_clusters(h), make_clusters(queue, h, d),
//     make_clusters(queue, d), each with (metric = EuclideanMetric<N>{},
//     kernel = FlatKernel{.5f}, block_size = 256); every call waits for its results;
//   * setWrappedCoordinates(range | ints...), getClusters(h), getClusters(queue, d).
// The work runs in libclue_b200 (clue_make_clusters).  block_size is accepted and ignored: the
// library picks its own launch shapes.  The seed list keeps the reference's capacity history
// (internal/SeedArray.hpp:33-41 with core/detail/SetupSeeds.hpp:10-20): capacity =
// max(previous capacity, points without a nearest higher); seeds past it are dropped.
#pragma once

#include "CLUEstering/core/ConvolutionalKernel.hpp"
#include "CLUEstering/core/DistanceMetrics.hpp"
#include "CLUEstering/data_structures/Points.hpp"
#include "CLUEstering/utils/get_clusters.hpp"

#include <algorithm>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <optional>
#include <ranges>
#include <stdexcept>
#include <type_traits>

namespace clue {

  namespace concepts {
    template <typename K>
    concept convolutional_kernel = requires(const K& k) {
      { k.c() } -> std::convertible_to<const clue_kernel&>;
    };
  }  // namespace concepts

  template <concepts::Queue TQueue, std::size_t Ndim>
  class Clusterer {
    static_assert(Ndim >= 1 && Ndim <= CLUE_MAX_DIM, "libclue_b200 clusters 1 to 10 dimensions");
    using TPointsHost = PointsHost<Ndim>;
    using TDev = DevType<TQueue>;
    using TPointsDevice = PointsDevice<TDev, Ndim>;

  public:
    Clusterer(TQueue& queue, Dim<Ndim>, float dc, float rhoc, std::optional<float> dm = std::nullopt,
              std::optional<float> seed_dc = std::nullopt, int pPBin = 128)
        : m_device(queue.getDevice()) {
      setParameters(dc, rhoc, dm, seed_dc, pPBin);
    }

    void setParameters(float dc, float rhoc, std::optional<float> dm = std::nullopt,
                       std::optional<float> seed_dc = std::nullopt, int pPBin = 128) {
      if (dc <= 0.f || rhoc < 0.f || dm.value_or(dc) <= 0.f || seed_dc.value_or(dc) <= 0.f || pPBin <= 0)
        throw std::invalid_argument("Invalid clustering parameters. The parameters must be positive.");
      m_dc = dc;
      m_rhoc = rhoc;
      m_dm = dm.value_or(dc);
      m_seed_dc = seed_dc.value_or(dc);
      m_pointsPerTile = pPBin;
    }

    template <typename Kernel = FlatKernel, concepts::distance_metric<Ndim> DistanceMetric = EuclideanMetric<Ndim>>
    void make_clusters(TQueue& queue, TPointsHost& h_points, const DistanceMetric& metric = EuclideanMetric<Ndim>{},
                       const Kernel& kernel = FlatKernel{.5f}, std::size_t block_size = 256) {
      (void)block_size;
      if (detail::contiguous(h_points.view())) {
        // Host SoA straight through the library's pinned staging buffers.
        clue_outputs out{h_points.view().cluster_index, nullptr, nullptr, nullptr, nullptr};
        run(queue, metric.c(), kernel.c(), h_points.view().coords[0], h_points.view().weight, out, h_points.size(),
            CLUE_MEM_HOST);
        h_points.mark_clustered();
        return;
      }
      Device dev = queue.getDevice();
      TPointsDevice d_points(dev, Dim<Ndim>{}, h_points.size());
      make_clusters(queue, h_points, d_points, metric, kernel, block_size);
    }

    template <typename Kernel = FlatKernel, concepts::distance_metric<Ndim> DistanceMetric = EuclideanMetric<Ndim>>
    void make_clusters(TPointsHost& h_points, const DistanceMetric& metric = EuclideanMetric<Ndim>{},
                       const Kernel& kernel = FlatKernel{.5f}, std::size_t block_size = 256) {
      auto& queue = get_queue(DevicePool::deviceAt(0u));
      make_clusters(queue, h_points, metric, kernel, block_size);
    }

    template <typename Kernel = FlatKernel, concepts::distance_metric<Ndim> DistanceMetric = EuclideanMetric<Ndim>>
    void make_clusters(TQueue& queue, TPointsHost& h_points, TPointsDevice& dev_points,
                       const DistanceMetric& metric = EuclideanMetric<Ndim>{}, const Kernel& kernel = FlatKernel{.5f},
                       std::size_t block_size = 256) {
      copyToDevice(queue, dev_points, h_points);
      make_clusters(queue, dev_points, metric, kernel, block_size);
      copyToHost(queue, h_points, dev_points);
      h_points.mark_clustered();
    }

    template <typename Kernel = FlatKernel, concepts::distance_metric<Ndim> DistanceMetric = EuclideanMetric<Ndim>>
    void make_clusters(TQueue& queue, TPointsDevice& dev_points, const DistanceMetric& metric = EuclideanMetric<Ndim>{},
                       const Kernel& kernel = FlatKernel{.5f}, std::size_t block_size = 256) {
      (void)block_size;
      auto& v = dev_points.view();
      clue_outputs out{v.cluster_index, v.is_seed, v.rho, v.nearest_higher, v.delta};
      const float* coords = dev_points.soa_coords(queue);
      const clue_run_info info = run(queue, metric.c(), kernel.c(), coords, v.weight, out, dev_points.size(), CLUE_MEM_DEVICE);
      dev_points.mark_clustered(static_cast<std::size_t>(info.n_clusters));
    }

    template <std::ranges::contiguous_range TRange>
      requires std::integral<std::ranges::range_value_t<TRange>>
    void setWrappedCoordinates(const TRange& wrapped_coordinates) {
      m_wrapped = {};
      const auto k = std::min<std::size_t>(std::ranges::size(wrapped_coordinates), Ndim);
      for (std::size_t d = 0; d < k; ++d) m_wrapped[d] = static_cast<uint8_t>(std::ranges::data(wrapped_coordinates)[d]);
    }
    template <std::integral... TArgs>
    void setWrappedCoordinates(TArgs... wrapped_coordinates) {
      m_wrapped = {static_cast<uint8_t>(wrapped_coordinates)...};
    }

    auto getClusters(const TPointsHost& h_points) { return get_clusters(h_points); }
    auto getClusters(TQueue& queue, const TPointsDevice& d_points) { return get_clusters(queue, d_points); }

    // Information on the last run (seeds, clusters, dropped seeds, grid shape).
    const clue_run_info& lastRunInfo() const { return m_info; }

  private:
    clue_run_info run(TQueue& queue, const clue_metric& metric, const clue_kernel& kernel, const float* coords,
                      const float* weight, const clue_outputs& out, int32_t n, int32_t memory) {
      if (!m_ctx || m_ctx_device != queue.getDevice().id) {
        clue_context c = nullptr;
        detail::check(clue_context_create(queue.getDevice().id, &c));
        m_ctx = std::shared_ptr<clue_context_s>(c, [](clue_context p) { clue_context_destroy(p); });
        m_ctx_device = queue.getDevice().id;
      }
      clue_params p{};
      p.dc = m_dc;
      p.rhoc = m_rhoc;
      p.dm = m_dm;
      p.seed_dc = m_seed_dc;
      p.points_per_tile = m_pointsPerTile;
      for (std::size_t d = 0; d < Ndim; ++d) p.wrapped[d] = m_wrapped[d];
      p.seed_capacity = m_seed_capacity;
      p.tiebreak = CLUE_TIE_REFERENCE;
      p.flags = 0;
      clue_run_info info{};
      detail::check(clue_make_clusters(m_ctx.get(), &p, &kernel, &metric, static_cast<int32_t>(Ndim), n, coords, weight,
                                       &out, memory, queue.stream(), &info));
      if (info.seed_capacity_used > m_seed_capacity) m_seed_capacity = info.seed_capacity_used;
      m_info = info;
      return info;
    }

    Device m_device;
    float m_dc = 0.f, m_rhoc = 0.f, m_dm = 0.f, m_seed_dc = 0.f;
    int m_pointsPerTile = 128;
    std::array<uint8_t, Ndim> m_wrapped{};
    int64_t m_seed_capacity = 0;
    std::shared_ptr<clue_context_s> m_ctx;
    int32_t m_ctx_device = -1;
    clue_run_info m_info{};
  };

  template <concepts::Queue Q, std::size_t N>
  Clusterer(Q&, Dim<N>, float, float) -> Clusterer<std::remove_cvref_t<Q>, N>;
  template <concepts::Queue Q, std::size_t N>
  Clusterer(Q&, Dim<N>, float, float, std::optional<float>) -> Clusterer<std::remove_cvref_t<Q>, N>;
  template <concepts::Queue Q, std::size_t N>
  Clusterer(Q&, Dim<N>, float, float, std::optional<float>, std::optional<float>) -> Clusterer<std::remove_cvref_t<Q>, N>;
  template <concepts::Queue Q, std::size_t N>
  Clusterer(Q&, Dim<N>, float, float, std::optional<float>, std::optional<float>, int)
      -> Clusterer<std::remove_cvref_t<Q>, N>;

}  // namespace clue
