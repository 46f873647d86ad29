// DistanceMetrics.hpp -- the six distance metrics of the reference
// (include/CLUEstering/core/DistanceMetrics.hpp:17-258) with the same constructors and call
// operator on Point<N> = std::array<float, N + 1> (the last element, the weight, is ignored).
// The arithmetic runs in libclue_b200 (same operation order on host and device).
#pragma once

#include "CLUEstering/detail/Runtime.hpp"

#include <array>
#include <concepts>
#include <cstddef>

namespace clue {

  template <std::size_t Ndim>
  using Point = std::array<float, Ndim + 1>;

  namespace detail {
    template <std::size_t Ndim>
    class MetricBase {
    public:
      float operator()(const Point<Ndim>& lhs, const Point<Ndim>& rhs) const {
        return clue_metric_eval(&m_m, static_cast<int32_t>(Ndim), lhs.data(), rhs.data());
      }
      const clue_metric& c() const { return m_m; }

    protected:
      explicit MetricBase(int32_t type) : m_m{} { m_m.type = type; }
      template <typename R>
      void set(const R& values) {
        std::size_t d = 0;
        for (auto v : values)
          if (d < Ndim) m_m.par[d++] = static_cast<float>(v);
      }
      clue_metric m_m;
    };
  }  // namespace detail

  template <std::size_t Ndim>
  class EuclideanMetric : public detail::MetricBase<Ndim> {
  public:
    EuclideanMetric() : detail::MetricBase<Ndim>(CLUE_METRIC_EUCLIDEAN) {}
  };

  template <std::size_t Ndim>
  class WeightedEuclideanMetric : public detail::MetricBase<Ndim> {
  public:
    template <std::floating_point... TValues>
      requires(sizeof...(TValues) == Ndim)
    WeightedEuclideanMetric(TValues... weights) : detail::MetricBase<Ndim>(CLUE_METRIC_WEIGHTED_EUCLIDEAN) {
      this->set(std::array<float, Ndim>{static_cast<float>(weights)...});
    }
    WeightedEuclideanMetric(const std::array<float, Ndim>& weights)
        : detail::MetricBase<Ndim>(CLUE_METRIC_WEIGHTED_EUCLIDEAN) {
      this->set(weights);
    }
  };

  template <std::size_t Ndim>
  class PeriodicEuclideanMetric : public detail::MetricBase<Ndim> {
  public:
    // period 0 marks a non-periodic coordinate
    PeriodicEuclideanMetric(const std::array<float, Ndim>& periods)
        : detail::MetricBase<Ndim>(CLUE_METRIC_PERIODIC_EUCLIDEAN) {
      this->set(periods);
    }
  };

  template <std::size_t Ndim>
  class ManhattanMetric : public detail::MetricBase<Ndim> {
  public:
    ManhattanMetric() : detail::MetricBase<Ndim>(CLUE_METRIC_MANHATTAN) {}
  };

  template <std::size_t Ndim>
  class ChebyshevMetric : public detail::MetricBase<Ndim> {
  public:
    ChebyshevMetric() : detail::MetricBase<Ndim>(CLUE_METRIC_CHEBYSHEV) {}
  };

  template <std::size_t Ndim>
  class WeightedChebyshevMetric : public detail::MetricBase<Ndim> {
  public:
    template <std::floating_point... TValues>
      requires(sizeof...(TValues) == Ndim)
    WeightedChebyshevMetric(TValues... weights) : detail::MetricBase<Ndim>(CLUE_METRIC_WEIGHTED_CHEBYSHEV) {
      this->set(std::array<float, Ndim>{static_cast<float>(weights)...});
    }
    WeightedChebyshevMetric(const std::array<float, Ndim>& weights)
        : detail::MetricBase<Ndim>(CLUE_METRIC_WEIGHTED_CHEBYSHEV) {
      this->set(weights);
    }
  };

  namespace metrics {
    template <std::size_t Ndim>
    using Euclidean = clue::EuclideanMetric<Ndim>;
    template <std::size_t Ndim>
    using WeightedEuclidean = clue::WeightedEuclideanMetric<Ndim>;
    template <std::size_t Ndim>
    using PeriodicEuclidean = clue::PeriodicEuclideanMetric<Ndim>;
    template <std::size_t Ndim>
    using Manhattan = clue::ManhattanMetric<Ndim>;
    template <std::size_t Ndim>
    using Chebyshev = clue::ChebyshevMetric<Ndim>;
    template <std::size_t Ndim>
    using WeightedChebyshev = clue::WeightedChebyshevMetric<Ndim>;
  }  // namespace metrics

  namespace concepts {
    template <typename TMetric, std::size_t Ndim>
    concept distance_metric = requires(TMetric&& metric) {
      { metric(std::array<float, Ndim + 1>{}, std::array<float, Ndim + 1>{}) } -> std::same_as<float>;
      { metric.c() } -> std::convertible_to<const clue_metric&>;
    };
  }  // namespace concepts

}  // namespace clue
