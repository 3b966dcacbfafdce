// Copies between page-locked, device-mapped host buffers and the device pool
// done by the SMs instead of the copy engines, for otfmm_batch_host: one
// launch per pool chunk moves the scattered records (the moments of the
// refined subgrids, the centres of mass the kernels read, the outputs of
// refined and leaf subgrids) that would otherwise take one DMA copy per run of
// consecutive subgrids, or move more bytes.
// Part of libotfmm.so; included once, in order, by otfmm.cu (one translation unit).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "layout.cuh"

namespace otfmm {

// Small CTAs with few registers, so that one fits an SM beside a multipole
// tile CTA; every thread keeps four 16-byte loads in flight.
constexpr int HC_THREADS = 128;
constexpr int HC_INFLIGHT = 4;

// Copies n2 double2 from src to dst with the CTA's threads, HC_INFLIGHT loads
// of a thread in flight.
__device__ __forceinline__ void cta_copy(double2* __restrict__ dst, const double2* __restrict__ src, int n2) {
    for (int b = 0; b < n2; b += HC_THREADS * HC_INFLIGHT) {
        double2 v[HC_INFLIGHT];
#pragma unroll
        for (int k = 0; k < HC_INFLIGHT; ++k) {
            const int j = b + k * HC_THREADS + threadIdx.x;
            if (j < n2) v[k] = src[j];
        }
#pragma unroll
        for (int k = 0; k < HC_INFLIGHT; ++k) {
            const int j = b + k * HC_THREADS + threadIdx.x;
            if (j < n2) dst[j] = v[k];
        }
    }
}

// Upload of pool chunk [a, a + n) from the mapped host pool (one CTA per
// subgrid): the 20 x 512 moments of a refined subgrid, and the centres of mass
// of the subgrids flagged in needs_com.
__global__ void __launch_bounds__(HC_THREADS) gather_pool_kernel(const double* __restrict__ host_M,
                                                                 const double* __restrict__ host_com,
                                                                 double* __restrict__ dev_M, double* __restrict__ dev_com,
                                                                 const uint8_t* __restrict__ is_leaf,
                                                                 const uint8_t* __restrict__ needs_com, int a) {
    const size_t i = (size_t)a + blockIdx.x;
    if (!is_leaf[i])
        cta_copy(reinterpret_cast<double2*>(dev_M + i * 20 * NCELL),
                 reinterpret_cast<const double2*>(host_M + i * 20 * NCELL), 10 * NCELL);
    if (needs_com[i])
        cta_copy(reinterpret_cast<double2*>(dev_com + i * 3 * NCELL),
                 reinterpret_cast<const double2*>(host_com + i * 3 * NCELL), 3 * NCELL / 2);
}

// Download of pool chunk [a, a + n): L[0..19] of a refined subgrid, L[0..3] of
// a leaf (its L[4..19] are left as the caller set them), and L_c of the
// subgrids flagged in writes_lc (refined ones, leaves with a refined
// neighbour; the others' L_c is left as the caller set it), from the device
// into the mapped host outputs (one CTA per subgrid).
__global__ void __launch_bounds__(HC_THREADS) scatter_outputs_kernel(const double* __restrict__ dev_L,
                                                                     const double* __restrict__ dev_Lc,
                                                                     double* __restrict__ host_L,
                                                                     double* __restrict__ host_Lc,
                                                                     const uint8_t* __restrict__ is_leaf,
                                                                     const uint8_t* __restrict__ writes_lc, int a) {
    const size_t i = (size_t)a + blockIdx.x;
    const int ncomp = is_leaf[i] ? 4 : 20;
    cta_copy(reinterpret_cast<double2*>(host_L + i * 20 * NCELL),
             reinterpret_cast<const double2*>(dev_L + i * 20 * NCELL), ncomp * NCELL / 2);
    if (writes_lc[i])
        cta_copy(reinterpret_cast<double2*>(host_Lc + i * 3 * NCELL),
                 reinterpret_cast<const double2*>(dev_Lc + i * 3 * NCELL), 3 * NCELL / 2);
}

}   // namespace otfmm
