// TEST INFRASTRUCTURE ONLY. Stand-in for octotiger/cuda_util/cuda_scheduler.hpp
// (HPX, taylor<>, buffer sizes) when oracle/build_ref_gpu.sh compiles the
// reference's CUDA interaction kernels: they need only the stencil byte size.
#pragma once
#include <cstddef>

#include "octotiger/common_kernel/interaction_constants.hpp"
namespace octotiger {
namespace fmm {
constexpr std::size_t full_stencil_size = FULL_STENCIL_SIZE * sizeof(double);
}
}   // namespace octotiger
