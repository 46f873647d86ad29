// Runtime.hpp -- devices, queues, dimensions and error mapping of the clue:: C++ API.
//
// Header-only layer over the C ABI of libclue_b200 (include/clue_b200.h).  It mirrors the
// host-side vocabulary of the reference (include/CLUEstering/detail/Dim.hpp,
// detail/concepts.hpp, internal/alpaka/devices.hpp:108-132, utils/get_queue.hpp:14-27): a
// Queue is a CUDA stream on one device, DevicePool enumerates the CUDA devices.
#pragma once

#include <clue_b200.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>

namespace clue {

  template <std::size_t N>
  struct Dim {
    constexpr static std::size_t size = N;
  };

  namespace detail {
    // Status codes back onto the reference's host exception types.
    inline void check(clue_status s) {
      if (s == CLUE_OK) return;
      std::string msg = clue_last_error();
      if (msg.empty()) msg = clue_status_string(s);
      switch (s) {
        case CLUE_ERR_INVALID_ARG:
        case CLUE_ERR_NONFINITE:
          throw std::invalid_argument(msg);
        case CLUE_ERR_OUT_OF_RANGE:
          throw std::out_of_range(msg);
        default:
          throw std::runtime_error(msg);
      }
    }
  }  // namespace detail

  class Queue;

  // One CUDA device.
  struct Device {
    int32_t id = 0;
    // A new queue (CUDA stream) on this device.
    Queue makeQueue() const;
    friend bool operator==(const Device& a, const Device& b) { return a.id == b.id; }
  };

  // The CUDA devices of the machine (reference: internal/alpaka/devices.hpp DevicePool).
  class DevicePool {
  public:
    static std::size_t size() {
      int32_t c = 0;
      if (clue_device_count(&c) != CLUE_OK) return 0;
      return static_cast<std::size_t>(c);
    }
    static Device deviceAt(std::size_t i) {
      if (i >= size()) throw std::runtime_error("No device with index " + std::to_string(i));
      return Device{static_cast<int32_t>(i)};
    }
  };

  // A stream on one device; work enqueued by the library on a queue is ordered.
  class Queue {
  public:
    explicit Queue(Device dev = Device{}) : m_dev(dev) {
      void* s = nullptr;
      detail::check(clue_stream_create(dev.id, &s));
      m_stream = std::shared_ptr<void>(s, [](void* p) { clue_stream_destroy(p); });
    }
    Device getDevice() const { return m_dev; }
    void* stream() const { return m_stream.get(); }
    void wait() const { detail::check(clue_stream_synchronize(m_stream.get())); }

  private:
    Device m_dev;
    std::shared_ptr<void> m_stream;
  };

  inline Queue Device::makeQueue() const { return Queue(*this); }

  // Static queue per device (reference: utils/get_queue.hpp:14-27, a function-local static).
  inline Queue& get_queue(Device dev) {
    static Queue* queues[64] = {};
    if (dev.id < 0 || dev.id >= 64) throw std::out_of_range("device id out of range");
    if (!queues[dev.id]) queues[dev.id] = new Queue(dev);
    return *queues[dev.id];
  }
  template <typename T>
    requires std::is_integral_v<T>
  inline Queue& get_queue(T id) {
    return get_queue(DevicePool::deviceAt(static_cast<std::size_t>(id)));
  }

  template <typename T>
  using DevType = Device;

  namespace concepts {
    template <class T>
    concept Queue = std::is_same_v<std::remove_cvref_t<T>, ::clue::Queue>;
    template <typename T>
    concept Pointer = std::is_pointer_v<T>;
  }  // namespace concepts

}  // namespace clue
