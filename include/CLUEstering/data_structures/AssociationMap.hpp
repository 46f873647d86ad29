// AssociationMap.hpp -- key -> values map in CSR form (offsets[keys + 1], indexes[values]).
//
// Same interface as the reference's AssociationMapBase
// (include/CLUEstering/data_structures/detail/AssociationMapBase.hpp:50-110): size, extents,
// begin/end, count, contains, lower_bound, upper_bound, equal_range and extract, with
// std::out_of_range for keys outside [0, size()).  HostAssociationMap lives in host memory;
// DevAssociationMap holds the CSR in device memory (built by clue_get_clusters) and hands out
// raw device pointers plus a host copy.
#pragma once

#include "CLUEstering/detail/Runtime.hpp"

#include <algorithm>
#include <cstdint>
#include <memory>
#include <span>
#include <stdexcept>
#include <utility>
#include <vector>

namespace clue {

  struct AssociationMapExtents {
    std::size_t values = 0;
    std::size_t keys = 0;
  };

  class HostAssociationMap {
  public:
    using key_type = int32_t;
    using mapped_type = int32_t;
    using size_type = std::size_t;
    using iterator = mapped_type*;
    using const_iterator = const mapped_type*;
    struct Containers {
      const std::vector<key_type>& keys;
      const std::vector<mapped_type>& values;
    };

    HostAssociationMap(size_type nelements, size_type nbins)
        : m_indexes(nelements), m_offsets(nbins + 1, 0), m_extents{nelements, nbins} {}
    HostAssociationMap(std::vector<key_type> offsets, std::vector<mapped_type> indexes)
        : m_indexes(std::move(indexes)), m_offsets(std::move(offsets)) {
      m_extents = {m_indexes.size(), m_offsets.empty() ? 0 : m_offsets.size() - 1};
    }

    // Counting sort of the associations (key -1 is skipped); values ascend inside a key
    // (reference: data_structures/AssociationMap.hpp:53-74).
    void fill(std::span<const key_type> associations) {
      std::vector<key_type> next(m_extents.keys + 1, 0);
      for (auto k : associations)
        if (k >= 0) ++next[k + 1];
      for (size_type k = 0; k < m_extents.keys; ++k) next[k + 1] += next[k];
      std::copy(next.begin(), next.end(), m_offsets.begin());
      for (size_type i = 0; i < associations.size(); ++i)
        if (associations[i] >= 0) m_indexes[next[associations[i]]++] = static_cast<mapped_type>(i);
    }

    size_type size() const { return m_extents.keys; }
    AssociationMapExtents extents() const { return m_extents; }

    iterator begin() { return m_indexes.data(); }
    const_iterator begin() const { return m_indexes.data(); }
    const_iterator cbegin() const { return m_indexes.data(); }
    iterator end() { return m_indexes.data() + m_offsets[m_extents.keys]; }
    const_iterator end() const { return m_indexes.data() + m_offsets[m_extents.keys]; }
    const_iterator cend() const { return end(); }

    size_type count(key_type key) const {
      check(key, "count");
      return static_cast<size_type>(m_offsets[key + 1] - m_offsets[key]);
    }
    bool contains(key_type key) const {
      check(key, "contains");
      return m_offsets[key + 1] > m_offsets[key];
    }
    iterator lower_bound(key_type key) {
      check(key, "lower_bound");
      return m_indexes.data() + m_offsets[key];
    }
    const_iterator lower_bound(key_type key) const {
      check(key, "lower_bound");
      return m_indexes.data() + m_offsets[key];
    }
    iterator upper_bound(key_type key) {
      check(key, "upper_bound");
      return m_indexes.data() + m_offsets[key + 1];
    }
    const_iterator upper_bound(key_type key) const {
      check(key, "upper_bound");
      return m_indexes.data() + m_offsets[key + 1];
    }
    std::pair<iterator, iterator> equal_range(key_type key) { return {lower_bound(key), upper_bound(key)}; }
    std::pair<const_iterator, const_iterator> equal_range(key_type key) const {
      return {lower_bound(key), upper_bound(key)};
    }
    Containers extract() const { return Containers{m_offsets, m_indexes}; }

  private:
    void check(key_type key, const char* what) const {
      if (key < 0 || key >= static_cast<key_type>(m_extents.keys))
        throw std::out_of_range(std::string("AssociationMap::") + what + " key out of range");
    }
    std::vector<mapped_type> m_indexes;
    std::vector<key_type> m_offsets;
    AssociationMapExtents m_extents;
  };

  // CSR in device memory.  offsets() holds size() + 1 entries, indexes() extents().values.
  class DevAssociationMap {
  public:
    using key_type = int32_t;
    using mapped_type = int32_t;
    using size_type = std::size_t;

    DevAssociationMap(Device dev, size_type nelements, size_type nbins) : m_dev(dev), m_extents{nelements, nbins} {
      void* p = nullptr;
      detail::check(clue_device_alloc(dev.id, (nelements + nbins + 1) * sizeof(int32_t), &p));
      m_buf = std::shared_ptr<void>(p, [](void* q) { clue_device_free(q); });
    }
    size_type size() const { return m_extents.keys; }
    AssociationMapExtents extents() const { return m_extents; }
    key_type* offsets() const { return static_cast<key_type*>(m_buf.get()); }
    mapped_type* indexes() const { return offsets() + m_extents.keys + 1; }
    Device device() const { return m_dev; }

    // The same map in host memory (synchronises the queue).
    template <concepts::Queue TQueue>
    HostAssociationMap toHost(TQueue& queue) const {
      std::vector<key_type> off(m_extents.keys + 1);
      std::vector<mapped_type> idx(m_extents.values);
      detail::check(clue_memcpy_dtoh(off.data(), offsets(), off.size() * sizeof(key_type), queue.stream()));
      if (!idx.empty())
        detail::check(clue_memcpy_dtoh(idx.data(), indexes(), idx.size() * sizeof(mapped_type), queue.stream()));
      queue.wait();
      return HostAssociationMap(std::move(off), std::move(idx));
    }

  private:
    Device m_dev;
    AssociationMapExtents m_extents;
    std::shared_ptr<void> m_buf;
  };

  namespace internal {
    // Host map with keys 0..max(association) (reference: internal/MakeAssociator.hpp:35-42).
    inline HostAssociationMap make_associator(std::span<const int32_t> associations, int32_t elements) {
      if (associations.empty())
        throw std::invalid_argument("make_associator: elements and associations must be non-zero");
      const int32_t bins = *std::ranges::max_element(associations) + 1;
      HostAssociationMap map(static_cast<std::size_t>(std::max(elements, 0)), static_cast<std::size_t>(std::max(bins, 0)));
      map.fill(associations);
      return map;
    }
    inline HostAssociationMap make_associator(std::span<int32_t> associations, int32_t elements) {
      return make_associator(std::span<const int32_t>(associations.data(), associations.size()), elements);
    }

    // Device map from device labels (reference: internal/MakeAssociator.hpp:11-34): throws
    // std::invalid_argument when no label is >= 0, like the reference.
    template <concepts::Queue TQueue>
    inline DevAssociationMap make_associator(TQueue& queue, std::span<const int32_t> d_associations) {
      if (d_associations.empty())
        throw std::invalid_argument("make_associator: elements and associations must be non-zero");
      const auto n = static_cast<int32_t>(d_associations.size());
      // Scratch CSR sized for the worst case, then trimmed into the returned map.
      void* tmp = nullptr;
      detail::check(clue_device_alloc(queue.getDevice().id, (2 * (std::size_t)n + 1) * sizeof(int32_t), &tmp));
      std::unique_ptr<void, clue_status (*)(void*)> guard(tmp, clue_device_free);
      auto* off = static_cast<int32_t*>(tmp);
      auto* pts = off + n + 1;
      static thread_local std::unique_ptr<clue_context_s, clue_status (*)(clue_context)> ctx(nullptr, clue_context_destroy);
      static thread_local int32_t ctx_dev = -1;
      if (!ctx || ctx_dev != queue.getDevice().id) {
        clue_context c = nullptr;
        detail::check(clue_context_create(queue.getDevice().id, &c));
        ctx.reset(c);
        ctx_dev = queue.getDevice().id;
      }
      int32_t nclusters = 0, nclustered = 0;
      detail::check(clue_get_clusters(ctx.get(), n, d_associations.data(), off, pts, &nclusters, &nclustered,
                                      queue.stream()));
      if (nclustered == 0)
        throw std::invalid_argument("make_associator: elements and associations must be non-zero");
      DevAssociationMap map(queue.getDevice(), (std::size_t)nclustered, (std::size_t)nclusters);
      detail::check(clue_memcpy_dtod(map.offsets(), off, ((std::size_t)nclusters + 1) * sizeof(int32_t), queue.stream()));
      detail::check(clue_memcpy_dtod(map.indexes(), pts, (std::size_t)nclustered * sizeof(int32_t), queue.stream()));
      queue.wait();
      return map;
    }
  }  // namespace internal

}  // namespace clue
