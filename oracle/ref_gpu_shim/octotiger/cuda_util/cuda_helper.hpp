// TEST INFRASTRUCTURE ONLY. Stand-in for octotiger/cuda_util/cuda_helper.hpp
// (HPX CUDA executors, CPPuddle stream pools) when oracle/build_ref_gpu.sh
// compiles the reference's own CUDA interaction kernels: only the names their
// launch helpers mention are declared; those helpers are never called.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
namespace hpx {
namespace cuda {
namespace experimental {
struct cuda_executor {};
}   // namespace experimental
}   // namespace cuda
template <class... A>
void apply(A&&...) {}
}   // namespace hpx
template <class E>
struct round_robin_pool {};
using pool_strategy = round_robin_pool<hpx::cuda::experimental::cuda_executor>;
template <class E, class S>
struct stream_interface {
    E interface;
};
