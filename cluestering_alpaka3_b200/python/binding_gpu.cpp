// Python module with the reference's backend-module interface
// (CLUEstering/BindingModules/serial/binding_cpu.cpp:18-240 and cuda/binding_gpu_cuda.cpp in the
// reference): listDevices(backend) and mainRun(dc, rhoc, dm, seed_dc, pPBin, wrapped, data,
// results, kernel, Ndim, n_points, block_size, device_id) for the three kernel types.
// data is the (Ndim + 1) x n float32 SoA block (coordinates, then weights); results receives
// the n cluster indexes.  The module name is set at build time (CLUE_MODULE_NAME): built as
// CLUE_GPU_CUDA it stands in for the reference's CUDA backend module, built as CLUE_GPU_B200 it
// is the library's own backend name.  The work runs in libclue_b200 through the clue:: C++ API,
// as the reference's run<N> (CLUEstering/BindingModules/Run.hpp:7-28) does through alpaka.
#include "CLUEstering/CLUEstering.hpp"

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cstdint>
#include <iostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#ifndef CLUE_MODULE_NAME
#define CLUE_MODULE_NAME CLUE_GPU_B200
#endif

namespace py = pybind11;

namespace {

  void listDevices(const std::string& backend) {
    const auto n = clue::DevicePool::size();
    if (n == 0) {
      std::cout << "No devices found for the " << backend << " backend." << std::endl;
      return;
    }
    std::cout << backend << " devices found: \n";
    for (std::size_t i = 0; i < n; ++i) std::cout << '\t' << "device " << i << ": CUDA device " << i << '\n';
  }

  template <std::size_t Ndim, typename Kernel>
  void run(float dc, float rhoc, float dm, float seed_dc, int pPBin, std::vector<uint8_t>&& wrapped, float* data,
           int* results, int32_t n_points, const Kernel& kernel, clue::Queue& queue, std::size_t block_size) {
    auto dim = clue::Dim<Ndim>{};
    clue::Clusterer algo(queue, dim, dc, rhoc, dm, seed_dc, pPBin);
    algo.setWrappedCoordinates(wrapped);
    clue::PointsHost h_points(dim, n_points, data, results);
    algo.make_clusters(queue, h_points, clue::EuclideanMetric<Ndim>{}, kernel, block_size);
  }

  template <typename Kernel, std::size_t... N>
  bool dispatch(int ndim, std::index_sequence<N...>, float dc, float rhoc, float dm, float seed_dc, int pPBin,
                std::vector<uint8_t>& wrapped, float* data, int* results, int32_t n_points, const Kernel& kernel,
                clue::Queue& queue, std::size_t block_size) {
    return ((ndim == int(N + 1) ? (run<N + 1, Kernel>(dc, rhoc, dm, seed_dc, pPBin, std::move(wrapped), data, results,
                                                       n_points, kernel, queue, block_size),
                                   true)
                                : false) ||
            ...);
  }

  template <typename Kernel>
  void mainRun(float dc, float rhoc, float dm, float seed_dc, int pPBin, std::vector<uint8_t> wrapped,
               py::array_t<float> data, py::array_t<int> results, const Kernel& kernel, int Ndim, int32_t n_points,
               std::size_t block_size, std::size_t device_id) {
    auto rData = data.request();
    auto rResults = results.request();
    if (n_points > 0 && (rData.size < (py::ssize_t)(Ndim + 1) * n_points || rResults.size < n_points))
      throw std::invalid_argument("data must hold (Ndim + 1) * n_points floats and results n_points ints");
    auto* pData = static_cast<float*>(rData.ptr);
    auto* pResults = static_cast<int*>(rResults.ptr);
    auto& queue = clue::get_queue(device_id);
    py::gil_scoped_release release;
    if (!dispatch<Kernel>(Ndim, std::make_index_sequence<10>{}, dc, rhoc, dm, seed_dc, pPBin, wrapped, pData, pResults,
                          n_points, kernel, queue, block_size))
      std::cout << "This library only works up to 10 dimensions\n";
  }

}  // namespace

PYBIND11_MODULE(CLUE_MODULE_NAME, m) {
  m.doc() = "Binding of the CLUE algorithm running on NVIDIA B200 GPUs (libclue_b200)";
  m.def("listDevices", &listDevices, "List the available devices for the backend");
  m.def("mainRun", &mainRun<clue::FlatKernel>, "mainRun");
  m.def("mainRun", &mainRun<clue::ExponentialKernel>, "mainRun");
  m.def("mainRun", &mainRun<clue::GaussianKernel>, "mainRun");
}
