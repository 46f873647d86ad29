// ConvolutionalKernel.hpp -- the density kernels of the reference
// (include/CLUEstering/core/ConvolutionalKernel.hpp:14-85,
//  core/detail/ConvolutionalKernel.hpp:10-65): same constructors and throwing rules, except
// that GaussianKernel accepts a mean of 0 (the benchmark configuration uses it).
#pragma once

#include "CLUEstering/detail/Runtime.hpp"

namespace clue {

  class FlatKernel {
  public:
    FlatKernel(float flat) : m_k{CLUE_KERNEL_FLAT, {flat, 0.f, 0.f}} { detail::check(clue_check_kernel(&m_k)); }
    // Kernel value for points i and j at distance dist (1 for i == j).
    float operator()(float dist, int i, int j) const { return clue_kernel_eval(&m_k, dist, i, j); }
    const clue_kernel& c() const { return m_k; }

  private:
    clue_kernel m_k;
  };

  class ExponentialKernel {
  public:
    ExponentialKernel(float exp_avg, float exp_amplitude)
        : m_k{CLUE_KERNEL_EXPONENTIAL, {exp_avg, exp_amplitude, 0.f}} {
      detail::check(clue_check_kernel(&m_k));
    }
    float operator()(float dist, int i, int j) const { return clue_kernel_eval(&m_k, dist, i, j); }
    const clue_kernel& c() const { return m_k; }

  private:
    clue_kernel m_k;
  };

  class GaussianKernel {
  public:
    GaussianKernel(float gaus_avg, float gaus_std, float gaus_amplitude)
        : m_k{CLUE_KERNEL_GAUSSIAN, {gaus_avg, gaus_std, gaus_amplitude}} {
      detail::check(clue_check_kernel(&m_k));
    }
    float operator()(float dist, int i, int j) const { return clue_kernel_eval(&m_k, dist, i, j); }
    const clue_kernel& c() const { return m_k; }

  private:
    clue_kernel m_k;
  };

}  // namespace clue
