// Python module CLUE_Convolutional_Kernels with the reference's kernel classes
// (CLUEstering/BindingModules/binding_kernels.cpp): FlatKernel(flat),
// ExponentialKernel(avg, amplitude), GaussianKernel(avg, std, amplitude); the constructors
// raise ValueError on invalid parameters (std::invalid_argument).
#include "CLUEstering/core/ConvolutionalKernel.hpp"

#include <pybind11/pybind11.h>

PYBIND11_MODULE(CLUE_Convolutional_Kernels, m) {
  m.doc() = "FlatKernel, ExponentialKernel and GaussianKernel for the density sums of libclue_b200.";
  pybind11::class_<clue::FlatKernel>(m, "FlatKernel").def(pybind11::init<float>());
  pybind11::class_<clue::ExponentialKernel>(m, "ExponentialKernel").def(pybind11::init<float, float>());
  pybind11::class_<clue::GaussianKernel>(m, "GaussianKernel").def(pybind11::init<float, float, float>());
}
