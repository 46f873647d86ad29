// Points.hpp -- PointsHost<N> and PointsDevice<TDev, N>, the SoA point containers of the
// clue:: API, and copyToHost / copyToDevice between them.
//
// Constructors, accessors and exceptions follow the reference
// (include/CLUEstering/data_structures/PointsHost.hpp:72-206,
//  data_structures/PointsDevice.hpp:129-253, data_structures/internal/PointsCommon.hpp:15-87):
//   * coordinates are SoA, coords(d)[i]; weights(); clusterIndexes();
//   * a container built from caller buffers does not own them; the one-argument forms
//     allocate one buffer (host: coords, weight, cluster_index; device: the same plus
//     is_seed, rho, nearest_higher, in the reference's order);
//   * n <= 0 throws std::invalid_argument, coords(d >= N) and operator[] past the end throw
//     std::out_of_range, copies between containers of different sizes throw
//     std::invalid_argument.
// PointsDevice also holds delta (distance to the nearest higher), which the reference declares
// but never defines.  Device memory comes from libclue_b200 (clue_device_alloc).
#pragma once

#include "CLUEstering/data_structures/ClusterProperties.hpp"
#include "CLUEstering/detail/Runtime.hpp"

#include <array>
#include <cfloat>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <optional>
#include <ranges>
#include <span>
#include <stdexcept>
#include <tuple>
#include <type_traits>
#include <vector>

namespace clue {

  template <std::size_t Ndim>
  struct PointsView {
    std::array<float*, Ndim> coords{};
    float* weight = nullptr;
    int* cluster_index = nullptr;
    int* is_seed = nullptr;
    float* rho = nullptr;
    int* nearest_higher = nullptr;
    float* delta = nullptr;
    int32_t n = 0;
  };

  namespace detail {
    inline int32_t checked_size(int32_t n, const char* who) {
      if (n <= 0)
        throw std::invalid_argument(std::string("Number of points passed to ") + who +
                                    " constructor must be positive.");
      return n;
    }

    struct DeviceBuffer {
      std::shared_ptr<void> mem;
      static DeviceBuffer make(Device dev, std::size_t bytes) {
        void* p = nullptr;
        check(clue_device_alloc(dev.id, bytes, &p));
        return DeviceBuffer{std::shared_ptr<void>(p, [](void* q) { clue_device_free(q); })};
      }
      std::byte* data() const { return static_cast<std::byte*>(mem.get()); }
    };

    // Coordinates are laid out as one SoA block when coords[d] == coords[0] + d * n.
    template <std::size_t Ndim>
    inline bool contiguous(const PointsView<Ndim>& v) {
      for (std::size_t d = 1; d < Ndim; ++d)
        if (v.coords[d] != v.coords[0] + d * static_cast<std::size_t>(v.n)) return false;
      return true;
    }
  }  // namespace detail

  // ---------------------------------------------------------------------------------------
  template <std::size_t Ndim>
  class PointsHost {
  public:
    class Point {
    public:
      Point(const std::array<float, Ndim>& coordinates, float weight, int cluster_index)
          : m_coordinates(coordinates), m_weight(weight), m_clusterIndex(cluster_index) {}
      float operator[](std::size_t dim) const {
        if (dim >= Ndim) throw std::out_of_range("Point coordinate index out of range");
        return m_coordinates[dim];
      }
      float weight() const { return m_weight; }
      int cluster_index() const { return m_clusterIndex; }

    private:
      std::array<float, Ndim> m_coordinates;
      float m_weight;
      int m_clusterIndex;
    };

    static std::size_t soa_bytes(int32_t n) {
      return ((Ndim + 1) * sizeof(float) + sizeof(int)) * static_cast<std::size_t>(n);
    }

    PointsHost(Dim<Ndim>, int32_t n_points) : m_size(detail::checked_size(n_points, "PointsHost")) {
      m_owned.resize(soa_bytes(n_points));
      partition(m_owned.data());
    }
    PointsHost(Dim<Ndim>, int32_t n_points, std::span<std::byte> buffer)
        : m_size(detail::checked_size(n_points, "PointsHost")) {
      if (buffer.size() < soa_bytes(n_points)) throw std::invalid_argument("PointsHost buffer too small");
      partition(buffer.data());
    }
    // input: coordinates then weights, SoA ((Ndim + 1) * n floats); output: n cluster indexes
    PointsHost(Dim<Ndim>, int32_t n_points, std::span<float> input, std::span<int> output)
        : m_size(detail::checked_size(n_points, "PointsHost")) {
      wire(input.data(), input.data() + Ndim * static_cast<std::size_t>(n_points), output.data());
    }
    PointsHost(Dim<Ndim>, int32_t n_points, std::span<float> coordinates, std::span<float> weights,
               std::span<int> output)
        : m_size(detail::checked_size(n_points, "PointsHost")) {
      wire(coordinates.data(), weights.data(), output.data());
    }
    PointsHost(Dim<Ndim>, int32_t n_points, float* input, int* output)
        : m_size(detail::checked_size(n_points, "PointsHost")) {
      wire(input, input + Ndim * static_cast<std::size_t>(n_points), output);
    }
    PointsHost(Dim<Ndim>, int32_t n_points, float* coordinates, float* weights, int* output)
        : m_size(detail::checked_size(n_points, "PointsHost")) {
      wire(coordinates, weights, output);
    }
    // One buffer per coordinate, then the weights, then the cluster indexes.
    template <concepts::Pointer... TBuffers>
      requires(sizeof...(TBuffers) == Ndim + 2 and Ndim > 1)
    PointsHost(Dim<Ndim>, int32_t n_points, TBuffers... buffers)
        : m_size(detail::checked_size(n_points, "PointsHost")) {
      wire_each(std::make_tuple(buffers...), std::make_index_sequence<Ndim>{});
    }
    template <std::ranges::contiguous_range... TBuffers>
      requires(sizeof...(TBuffers) == Ndim + 2 and Ndim > 1)
    PointsHost(Dim<Ndim>, int32_t n_points, TBuffers&&... buffers)
        : m_size(detail::checked_size(n_points, "PointsHost")) {
      wire_each(std::make_tuple(std::ranges::data(buffers)...), std::make_index_sequence<Ndim>{});
    }

    PointsHost(const PointsHost&) = delete;
    PointsHost& operator=(const PointsHost&) = delete;
    PointsHost(PointsHost&&) = default;
    PointsHost& operator=(PointsHost&&) = default;
    ~PointsHost() = default;

    int32_t size() const { return m_size; }
    std::span<const float> coords(std::size_t dim) const {
      check_dim(dim);
      return {m_view.coords[dim], static_cast<std::size_t>(m_size)};
    }
    std::span<float> coords(std::size_t dim) {
      check_dim(dim);
      return {m_view.coords[dim], static_cast<std::size_t>(m_size)};
    }
    std::span<const float> weights() const { return {m_view.weight, static_cast<std::size_t>(m_size)}; }
    std::span<float> weights() { return {m_view.weight, static_cast<std::size_t>(m_size)}; }
    std::span<const int> clusterIndexes() const { return {m_view.cluster_index, static_cast<std::size_t>(m_size)}; }
    std::span<int> clusterIndexes() { return {m_view.cluster_index, static_cast<std::size_t>(m_size)}; }
    bool clustered() const { return m_clustered; }
    const PointsView<Ndim>& view() const { return m_view; }
    PointsView<Ndim>& view() { return m_view; }

    Point operator[](std::size_t idx) const {
      if (idx >= static_cast<std::size_t>(m_size)) throw std::out_of_range("Index out of range in PointsHost::operator[]");
      std::array<float, Ndim> c;
      for (std::size_t d = 0; d < Ndim; ++d) c[d] = m_view.coords[d][idx];
      return Point(c, m_view.weight[idx], m_view.cluster_index[idx]);
    }

    // Lazily computed from the cluster indexes and cached until the next clustering.
    const std::size_t& n_clusters() { return properties().n_clusters(); }
    const HostAssociationMap& clusters() { return properties().clusters(); }
    const std::vector<std::size_t>& cluster_sizes() { return properties().cluster_sizes(); }
    const ClusterProperties& cluster_properties() { return properties(); }

    // Marks the points as clustered (the library does this after make_clusters; read_output too).
    void mark_clustered() {
      m_clustered = true;
      m_properties.reset();
    }

  private:
    void check_dim(std::size_t dim) const {
      if (dim >= Ndim) throw std::out_of_range("Dimension out of range in call to coords.");
    }
    const ClusterProperties& properties() {
      if (!m_clustered) throw std::logic_error("points have not been clustered");
      if (!m_properties) m_properties.emplace(clusterIndexes());
      return *m_properties;
    }
    void partition(std::byte* b) {
      auto* f = reinterpret_cast<float*>(b);
      wire(f, f + Ndim * static_cast<std::size_t>(m_size), reinterpret_cast<int*>(f + (Ndim + 1) * static_cast<std::size_t>(m_size)));
    }
    void wire(float* coords, float* weight, int* out) {
      for (std::size_t d = 0; d < Ndim; ++d) m_view.coords[d] = coords + d * static_cast<std::size_t>(m_size);
      m_view.weight = weight;
      m_view.cluster_index = out;
      m_view.n = m_size;
    }
    template <typename Tuple, std::size_t... D>
    void wire_each(const Tuple& t, std::index_sequence<D...>) {
      ((m_view.coords[D] = reinterpret_cast<float*>(std::get<D>(t))), ...);
      m_view.weight = reinterpret_cast<float*>(std::get<Ndim>(t));
      m_view.cluster_index = reinterpret_cast<int*>(std::get<Ndim + 1>(t));
      m_view.n = m_size;
    }

    PointsView<Ndim> m_view;
    std::vector<std::byte> m_owned;
    int32_t m_size;
    bool m_clustered = false;
    std::optional<ClusterProperties> m_properties;
  };

  // ---------------------------------------------------------------------------------------
  template <typename TDev, std::size_t Ndim>
  class PointsDevice {
  public:
    // Reference layout of the one-buffer form: coords, weight, cluster_index, is_seed, rho,
    // nearest_higher (data_structures/detail/PointsDevice.hpp:20-45).
    static std::size_t soa_bytes(int32_t n) {
      return ((Ndim + 2) * sizeof(float) + 3 * sizeof(int)) * static_cast<std::size_t>(n);
    }

    PointsDevice(TDev& device, Dim<Ndim>, int32_t n_points)
        : m_dev(device), m_size(detail::checked_size(n_points, "PointsDevice")) {
      m_buffer = detail::DeviceBuffer::make(device, soa_bytes(n_points) + sizeof(float) * (std::size_t)n_points);
      partition_full(m_buffer.data());
      m_view.delta = reinterpret_cast<float*>(m_buffer.data() + soa_bytes(n_points));
    }
    PointsDevice(TDev& device, Dim<Ndim>, int32_t n_points, std::span<std::byte> buffer)
        : m_dev(device), m_size(detail::checked_size(n_points, "PointsDevice")) {
      if (buffer.size() < soa_bytes(n_points)) throw std::invalid_argument("PointsDevice buffer too small");
      partition_full(buffer.data());
      m_buffer = detail::DeviceBuffer::make(device, sizeof(float) * (std::size_t)n_points);
      m_view.delta = reinterpret_cast<float*>(m_buffer.data());
    }
    PointsDevice(TDev& device, Dim<Ndim>, int32_t n_points, std::span<float> input, std::span<int> output)
        : m_dev(device), m_size(detail::checked_size(n_points, "PointsDevice")) {
      wire(input.data(), input.data() + Ndim * (std::size_t)n_points, output.data());
    }
    PointsDevice(TDev& device, Dim<Ndim>, int32_t n_points, std::span<float> coordinates,
                 std::span<float> weights, std::span<int> output)
        : m_dev(device), m_size(detail::checked_size(n_points, "PointsDevice")) {
      wire(coordinates.data(), weights.data(), output.data());
    }
    PointsDevice(TDev& device, Dim<Ndim>, int32_t n_points, float* input, int* output)
        : m_dev(device), m_size(detail::checked_size(n_points, "PointsDevice")) {
      wire(input, input + Ndim * (std::size_t)n_points, output);
    }
    PointsDevice(TDev& device, Dim<Ndim>, int32_t n_points, float* coordinates, float* weights, int* output)
        : m_dev(device), m_size(detail::checked_size(n_points, "PointsDevice")) {
      wire(coordinates, weights, output);
    }
    template <concepts::Pointer... TBuffers>
      requires(sizeof...(TBuffers) == Ndim + 2 and Ndim > 1)
    PointsDevice(TDev& device, Dim<Ndim>, int32_t n_points, TBuffers... buffers)
        : m_dev(device), m_size(detail::checked_size(n_points, "PointsDevice")) {
      auto t = std::make_tuple(buffers...);
      wire_each(t, std::make_index_sequence<Ndim>{});
    }

    PointsDevice(const PointsDevice&) = delete;
    PointsDevice& operator=(const PointsDevice&) = delete;
    PointsDevice(PointsDevice&&) = default;
    PointsDevice& operator=(PointsDevice&&) = default;
    ~PointsDevice() = default;

    int32_t size() const { return m_size; }
    // Spans over DEVICE memory.
    std::span<const float> coords(std::size_t dim) const {
      check_dim(dim);
      return {m_view.coords[dim], (std::size_t)m_size};
    }
    std::span<float> coords(std::size_t dim) {
      check_dim(dim);
      return {m_view.coords[dim], (std::size_t)m_size};
    }
    std::span<const float> weights() const { return {m_view.weight, (std::size_t)m_size}; }
    std::span<float> weights() { return {m_view.weight, (std::size_t)m_size}; }
    std::span<const int> clusterIndexes() const { return {m_view.cluster_index, (std::size_t)m_size}; }
    std::span<int> clusterIndexes() { return {m_view.cluster_index, (std::size_t)m_size}; }
    bool clustered() const { return m_clustered; }
    const PointsView<Ndim>& view() const { return m_view; }
    PointsView<Ndim>& view() { return m_view; }
    std::span<const float> rho() const { return {m_view.rho, (std::size_t)m_size}; }
    std::span<float> rho() { return {m_view.rho, (std::size_t)m_size}; }
    std::span<const float> delta() const { return {m_view.delta, (std::size_t)m_size}; }
    std::span<float> delta() { return {m_view.delta, (std::size_t)m_size}; }
    std::span<const int> nearestHigher() const { return {m_view.nearest_higher, (std::size_t)m_size}; }
    std::span<int> nearestHigher() { return {m_view.nearest_higher, (std::size_t)m_size}; }
    std::span<const int> isSeed() const { return {m_view.is_seed, (std::size_t)m_size}; }
    std::span<int> isSeed() { return {m_view.is_seed, (std::size_t)m_size}; }
    Device device() const { return m_dev; }

    // Clusters of the last clustering (max label + 1); read from the device once and cached.
    const std::size_t& n_clusters() {
      if (!m_clustered) throw std::logic_error("points have not been clustered");
      if (!m_nclusters) {
        std::vector<int> h(m_size);
        detail::check(clue_memcpy_dtoh(h.data(), m_view.cluster_index, h.size() * sizeof(int), nullptr));
        m_nclusters = ClusterProperties::compute_nclusters(h);
      }
      return *m_nclusters;
    }

    // Marks the points as clustered with a known cluster count (the Clusterer does this).
    void mark_clustered(std::optional<std::size_t> nclusters = std::nullopt) {
      m_clustered = true;
      m_nclusters = nclusters;
    }

    // A device pointer to the coordinates as one SoA block, gathering them into internal
    // scratch when the caller gave one buffer per coordinate.
    template <concepts::Queue TQueue>
    const float* soa_coords(TQueue& queue) {
      if (detail::contiguous(m_view)) return m_view.coords[0];
      const std::size_t n = (std::size_t)m_size;
      if (!m_gather.mem) m_gather = detail::DeviceBuffer::make(m_dev, Ndim * n * sizeof(float));
      auto* dst = reinterpret_cast<float*>(m_gather.data());
      for (std::size_t d = 0; d < Ndim; ++d)
        detail::check(clue_memcpy_dtod(dst + d * n, m_view.coords[d], n * sizeof(float), queue.stream()));
      return dst;
    }

  private:
    void check_dim(std::size_t dim) const {
      if (dim >= Ndim) throw std::out_of_range("Dimension out of range in call to coords.");
    }
    void partition_full(std::byte* b) {
      const std::size_t n = (std::size_t)m_size;
      auto* f = reinterpret_cast<float*>(b);
      for (std::size_t d = 0; d < Ndim; ++d) m_view.coords[d] = f + d * n;
      m_view.weight = f + Ndim * n;
      m_view.cluster_index = reinterpret_cast<int*>(f + (Ndim + 1) * n);
      m_view.is_seed = reinterpret_cast<int*>(f + (Ndim + 2) * n);
      m_view.rho = f + (Ndim + 3) * n;
      m_view.nearest_higher = reinterpret_cast<int*>(f + (Ndim + 4) * n);
      m_view.n = m_size;
    }
    // Caller buffers for coords / weight / cluster_index; is_seed, rho, nearest_higher and
    // delta in one internal buffer (reference: 3 * n * 4 bytes, here 4 * n * 4 with delta).
    void alloc_internal() {
      const std::size_t n = (std::size_t)m_size;
      m_buffer = detail::DeviceBuffer::make(m_dev, 4 * n * sizeof(float));
      auto* f = reinterpret_cast<float*>(m_buffer.data());
      m_view.is_seed = reinterpret_cast<int*>(f);
      m_view.rho = f + n;
      m_view.nearest_higher = reinterpret_cast<int*>(f + 2 * n);
      m_view.delta = f + 3 * n;
      m_view.n = m_size;
    }
    void wire(float* coords, float* weight, int* out) {
      for (std::size_t d = 0; d < Ndim; ++d) m_view.coords[d] = coords + d * (std::size_t)m_size;
      m_view.weight = weight;
      m_view.cluster_index = out;
      alloc_internal();
    }
    template <typename Tuple, std::size_t... D>
    void wire_each(const Tuple& t, std::index_sequence<D...>) {
      ((m_view.coords[D] = reinterpret_cast<float*>(std::get<D>(t))), ...);
      m_view.weight = reinterpret_cast<float*>(std::get<Ndim>(t));
      m_view.cluster_index = reinterpret_cast<int*>(std::get<Ndim + 1>(t));
      alloc_internal();
    }

    Device m_dev;
    PointsView<Ndim> m_view;
    detail::DeviceBuffer m_buffer;
    detail::DeviceBuffer m_gather;
    int32_t m_size;
    bool m_clustered = false;
    std::optional<std::size_t> m_nclusters;
  };

  template <typename TDev, std::size_t N>
  PointsDevice(TDev&, Dim<N>, int32_t) -> PointsDevice<std::remove_cvref_t<TDev>, N>;
  template <typename TDev, std::size_t N, typename... TArgs>
  PointsDevice(TDev&, Dim<N>, int32_t, TArgs&&...) -> PointsDevice<std::remove_cvref_t<TDev>, N>;

  // ---- copies (reference: data_structures/PointsDevice.hpp:19-107) -----------------------
  template <concepts::Queue TQueue, std::size_t Ndim>
  inline void copyToHost(TQueue& queue, PointsHost<Ndim>& h_points, const PointsDevice<DevType<TQueue>, Ndim>& d_points) {
    if (h_points.size() != d_points.size())
      throw std::invalid_argument("Host and device points have different sizes.");
    const std::size_t n = (std::size_t)h_points.size();
    for (std::size_t d = 0; d < Ndim; ++d)
      detail::check(clue_memcpy_dtoh(h_points.view().coords[d], d_points.view().coords[d], n * sizeof(float), queue.stream()));
    detail::check(clue_memcpy_dtoh(h_points.view().weight, d_points.view().weight, n * sizeof(float), queue.stream()));
    detail::check(clue_memcpy_dtoh(h_points.view().cluster_index, d_points.view().cluster_index, n * sizeof(int), queue.stream()));
    queue.wait();
    if (d_points.clustered()) h_points.mark_clustered();
  }
  template <concepts::Queue TQueue, std::size_t Ndim>
  inline auto copyToHost(TQueue& queue, const PointsDevice<DevType<TQueue>, Ndim>& d_points) {
    PointsHost<Ndim> h(Dim<Ndim>{}, d_points.size());
    copyToHost(queue, h, d_points);
    return h;
  }
  template <concepts::Queue TQueue, std::size_t Ndim>
  inline void copyToDevice(TQueue& queue, PointsDevice<DevType<TQueue>, Ndim>& d_points, const PointsHost<Ndim>& h_points) {
    if (h_points.size() != d_points.size())
      throw std::invalid_argument("Host and device points have different sizes.");
    const std::size_t n = (std::size_t)h_points.size();
    for (std::size_t d = 0; d < Ndim; ++d)
      detail::check(clue_memcpy_htod(d_points.view().coords[d], h_points.view().coords[d], n * sizeof(float), queue.stream()));
    detail::check(clue_memcpy_htod(d_points.view().weight, h_points.view().weight, n * sizeof(float), queue.stream()));
    queue.wait();
  }
  template <concepts::Queue TQueue, std::size_t Ndim>
  inline auto copyToDevice(TQueue& queue, const PointsHost<Ndim>& h_points) {
    Device dev = queue.getDevice();
    PointsDevice<Device, Ndim> d(dev, Dim<Ndim>{}, h_points.size());
    copyToDevice(queue, d, h_points);
    return d;
  }

}  // namespace clue
