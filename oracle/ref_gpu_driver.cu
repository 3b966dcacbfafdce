// TEST INFRASTRUCTURE ONLY. The reference's own CUDA interaction kernels
// (cuda_multipole_interactions_kernel_rho / _non_rho with their block-sum
// kernels, src/multipole_interactions/legacy/multipole_cuda_kernel.cpp:40-145
// and :331-436; cuda_p2p_interactions_kernel with cuda_sum_p2p_results,
// src/monopole_interactions/legacy/monopole_cuda_kernel.cpp:38-150), compiled
// in place from the Octo-Tiger source tree by oracle/build_ref_gpu.sh (nothing
// of them is copied here) with stand-ins for the HPX / CPPuddle headers
// (oracle/ref_gpu_shim) and the stencil generators of the reference
// (src/*/util/calculate_stencil.cpp, with the opts() stand-in of
// oracle/ref_shim). This file adds only a C entry per kernel sequence with the
// launch shapes of the reference's launchers
// (src/multipole_interactions/legacy/cuda_multipole_interaction_interface.cpp:192-217,
// src/monopole_interactions/legacy/cuda_monopole_interaction_interface.cpp:140-150)
// and the constant-memory set-up of src/cuda_util/cuda_scheduler.cpp:36-87.
// Used by the GPU tests (bit-identical to the oracle with --fmad=false) and by
// tests/reference_gpu_timing.py; never linked into libotfmm.so.
#include <memory>

#include "octotiger/options.hpp"   // stand-in: opts().theta

static otfmm_ref_opts g_opts{0.5};
otfmm_ref_opts& opts() { return g_opts; }

#include "src/monopole_interactions/util/calculate_stencil.cpp"
#include "src/multipole_interactions/util/calculate_stencil.cpp"
#include "src/multipole_interactions/legacy/multipole_cuda_kernel.cpp"
#include "src/monopole_interactions/legacy/monopole_cuda_kernel.cpp"

namespace ofmm = octotiger::fmm;

extern "C" {

// Stencil masks and monopole constants of opening angle theta into the
// kernels' constant memory on the current device.
int refgpu_init(double theta) {
    g_opts.theta = theta;
    const auto sup = ofmm::multipole_interactions::calculate_stencil();
    const auto mp = ofmm::multipole_interactions::calculate_stencil_masks(sup);
    const auto p2p = ofmm::monopole_interactions::calculate_stencil();
    const auto pm = ofmm::monopole_interactions::calculate_stencil_masks(p2p.first);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -4;
    auto p2p_masks = std::make_unique<bool[]>(ofmm::FULL_STENCIL_SIZE);
    auto four = std::make_unique<double[]>(4 * ofmm::FULL_STENCIL_SIZE);
    for (size_t i = 0; i < ofmm::FULL_STENCIL_SIZE; ++i) {
        p2p_masks[i] = pm.first[i];
        for (int k = 0; k < 4; ++k) four[4 * i + k] = pm.second[i][k];
    }
    ofmm::monopole_interactions::init_stencil(dev, std::move(p2p_masks), std::move(four));
    auto masks = std::make_unique<bool[]>(ofmm::FULL_STENCIL_SIZE);
    auto inner = std::make_unique<bool[]>(ofmm::FULL_STENCIL_SIZE);
    for (size_t i = 0; i < ofmm::FULL_STENCIL_SIZE; ++i) {
        masks[i] = mp.first[i];
        inner[i] = mp.second[i];
    }
    ofmm::multipole_interactions::init_stencil(dev, std::move(masks), std::move(inner));
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -4;
}

// Doubles of the per-block partial results the multipole kernel writes
// (one slab of L and of L_c per stencil column block).
size_t refgpu_m2l_scratch_doubles(void) {
    return (size_t)ofmm::NUMBER_MULTIPOLE_BLOCKS * ofmm::NUMBER_MULTIPOLE_BLOCKS *
           (ofmm::NUMBER_POT_EXPANSIONS + ofmm::NUMBER_ANG_CORRECTIONS);
}
size_t refgpu_p2p_scratch_doubles(void) {
    return (size_t)ofmm::NUMBER_P2P_BLOCKS * ofmm::NUMBER_POT_EXPANSIONS_SMALL;
}

// One multipole (M2L) call on the reference's SoA buffers (device pointers):
// mon[5832], com[3][5851], M[20][5851] in; L[20][531], L_c[3][531] out;
// scratch of refgpu_m2l_scratch_doubles() doubles.
int refgpu_m2l(const double* mon, const double* com, const double* M, double* scratch, double* L, double* Lc,
               double theta, int rho, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    int blocks = ofmm::NUMBER_MULTIPOLE_BLOCKS * ofmm::NUMBER_MULTIPOLE_BLOCKS;
    double* tmp_exp = scratch;
    double* tmp_corr = scratch + (size_t)blocks * ofmm::NUMBER_POT_EXPANSIONS;
    const dim3 grid(INX, ofmm::NUMBER_MULTIPOLE_BLOCKS, ofmm::NUMBER_MULTIPOLE_BLOCKS), block(1, INX, INX);
    const dim3 grid_sum_exp(1, 20, INX), grid_sum_corr(1, 3, INX);
    if (rho) {
        ofmm::multipole_interactions::cuda_multipole_interactions_kernel_rho<<<grid, block, 0, s>>>(
            mon, com, M, tmp_exp, tmp_corr, theta, false);
        ofmm::multipole_interactions::cuda_sum_multipole_potential_expansions_results<<<grid_sum_exp, block, 0, s>>>(
            blocks, tmp_exp, L);
        ofmm::multipole_interactions::cuda_sum_multipole_angular_corrections_results<<<grid_sum_corr, block, 0, s>>>(
            blocks, tmp_corr, Lc);
    } else {
        ofmm::multipole_interactions::cuda_multipole_interactions_kernel_non_rho<<<grid, block, 0, s>>>(
            mon, com, M, tmp_exp, theta, false);
        ofmm::multipole_interactions::cuda_sum_multipole_potential_expansions_results<<<grid_sum_exp, block, 0, s>>>(
            blocks, tmp_exp, L);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

// One monopole (P2P) call: mon[5832] in, L4[4][531] out, scratch of
// refgpu_p2p_scratch_doubles() doubles.
int refgpu_p2p(const double* mon, double* scratch, double* L4, double theta, double dx, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const dim3 grid(1, ofmm::NUMBER_P2P_BLOCKS, INX), block(1, INX, INX), grid_sum(1, 1, INX);
    ofmm::monopole_interactions::cuda_p2p_interactions_kernel<<<grid, block, 0, s>>>(mon, scratch, theta, dx);
    ofmm::monopole_interactions::cuda_sum_p2p_results<<<grid_sum, block, 0, s>>>(scratch, L4);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

}   // extern "C"
