// Per-subgrid entry points on the reference's SoA halo buffers, and the
// device-side staging of those buffers from the resident pool.
// Part of libotfmm.so; included once, in order, by otfmm.cu (one translation unit).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/otfmm.h"
#include "pair_math.cuh"
#include "m2l_tiles.cuh"

namespace otfmm {

struct SoaArgs {
    const double* mon;
    const double* M;
    const double* com;
    double* L;
    double* Lc;
    Tables t;
};

template <int PREC, bool RHO, bool ROOT>
__global__ void __launch_bounds__(THREADS, 1) soa_m2l_kernel(SoaArgs a) {
    extern __shared__ double sm[];
    const int x0 = TILE_X * blockIdx.x;
    OutPtr out{a.L, a.Lc, CLU, false};
    if (ROOT) {
        for (int r = threadIdx.x; r < NCELL; r += blockDim.x) {
            const int f = ((r >> 6) + INX - PAD_OFF) * PSTRIDE * PSTRIDE + (((r >> 3) & 7) + INX - PAD_OFF) * PSTRIDE +
                          ((r & 7) + INX - PAD_OFF);
            for (int q = 0; q < NCOMP; ++q)
                sm[q * NCELL + r] = (q < 20) ? a.M[q * CL + f] * stage_scale<PREC>(q) : a.com[(q - 20) * CL + f];
        }
        __syncthreads();
        root_tile<PREC, RHO>(sm, x0, a.t, out);
    } else {
        stage_region_soa<PREC>(sm, x0, a.mon, a.M, a.com);
        __syncthreads();
        m2l_tile<PREC, RHO>(sm, x0, a.t, 0u, a.mon, out);
    }
}

// Per-subgrid P2P on the reference's staged mon[5832] (one thread per cell).
template <int PREC>
__global__ void soa_p2p_kernel(const double* __restrict__ mon, double dx, double* __restrict__ L4, Tables t) {
    const int cu = blockIdx.x * blockDim.x + threadIdx.x;
    if (cu >= NCELL) return;
    const int cx = cu >> 6, cy = (cu >> 3) & 7, cz = cu & 7;
    const int p = ((cx & 1) << 2) | ((cy & 1) << 1) | (cz & 1);
    const int n = t.count[p];
    const int2* ent = t.entries + p * MAX_ENTRIES;
    const double dc0 = __ddiv_rn(1.0, dx), dc1 = __ddiv_rn(-1.0, dx);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int e = 0; e < n; ++e) {
        const int y = __ldg(&ent[e].y);
        const int ax = cx + entry_sx(y), ay = cy + entry_sy(y), az = cz + entry_sz(y);
        const double m = mon[(ax + INX - PAD_OFF) * PSTRIDE * PSTRIDE + (ay + INX - PAD_OFF) * PSTRIDE + (az + INX - PAD_OFF)];
        const double* four = c_four[entry_sidx(y)];
        if (PREC == PREC_EXACT) {
            const double ms = __dmul_rn(m, dc0);
            acc[0] = __dadd_rn(acc[0], __dmul_rn(four[0], ms));
            for (int q = 1; q < 4; ++q) acc[q] = __dadd_rn(acc[q], __dmul_rn(__dmul_rn(four[q], ms), dc1));
        } else {
            const double ms = m * dc0;
            acc[0] = fma(four[0], ms, acc[0]);
            for (int q = 1; q < 4; ++q) acc[q] = fma(four[q], ms * dc1, acc[q]);
        }
    }
    for (int q = 0; q < 4; ++q) L4[q * CLU + cu] = acc[q];
}

// Per-subgrid P2M against one refined neighbour slab (update_neighbor_input layout).
template <int PREC, bool RHO>
__global__ void soa_p2m_kernel(int d, const double* __restrict__ nM, const double* __restrict__ ncom,
                               const double* __restrict__ icom, double* L4, double* Lc, Tables t) {
    const int cu = blockIdx.x * blockDim.x + threadIdx.x;
    if (cu >= NCELL) return;
    const int r = d < 13 ? d : d + 1;
    const int o[3] = {r % 3 - 1, (r / 3) % 3 - 1, r / 9 - 1};
    int s[3], e[3], sz[3];
    for (int a = 0; a < 3; ++a) {
        s[a] = (o[a] == -1) ? INX - SMAX : 0;
        e[a] = (o[a] == 1) ? SMAX : INX;
        sz[a] = e[a] - s[a];
    }
    const int stride = sz[0] * sz[1] * sz[2] + 19;
    const int cx = cu >> 6, cy = (cu >> 3) & 7, cz = cu & 7;
    const int p = ((cx & 1) << 2) | ((cy & 1) << 1) | (cz & 1);
    const int n = t.count[p];
    const int2* ent = t.entries + p * MAX_ENTRIES;
    double X[3], acc[4], corr[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < 3; ++a) X[a] = icom[a * CLU + cu];
    for (int q = 0; q < 4; ++q) acc[q] = L4[q * CLU + cu];
    if (RHO)
        for (int a = 0; a < 3; ++a) corr[a] = Lc[a * CLU + cu];
    bool any = false;
    for (int en = 0; en < n; ++en) {
        const int y = __ldg(&ent[en].y);
        const int ax = cx + entry_sx(y), ay = cy + entry_sy(y), az = cz + entry_sz(y);
        if (raw_dir(ax, ay, az) != r) continue;
        const int lx = (ax & 7) - s[0], ly = (ay & 7) - s[1], lz = (az & 7) - s[2];
        if (lx < 0 || ly < 0 || lz < 0 || lx >= sz[0] || ly >= sz[1] || lz >= sz[2]) continue;
        const int f = lx * (sz[1] * sz[2]) + ly * sz[2] + lz;
        double Y[3], mp[20];
        for (int a = 0; a < 3; ++a) Y[a] = ncom[a * stride + f];
        for (int q = 0; q < 20; ++q) mp[q] = nM[q * stride + f] * stage_scale<PREC>(q);
        if (PREC == PREC_EXACT)
            exact_p2m_pair<RHO>(X, Y, mp, acc, corr);
        else
            fast_p2m_pair<RHO>(X, Y, mp, acc, corr);
        any = true;
    }
    (void)any;
    for (int q = 0; q < 4; ++q) L4[q * CLU + cu] = acc[q];
    if (RHO)
        for (int a = 0; a < 3; ++a) Lc[a * CLU + cu] = corr[a];
}


// Device restatement of the reference's halo staging for the per-subgrid
// entry points, from the resident pool: multipole update_input
// (multipole_interaction_interface.hpp:88-281) into mon[5832], M[20][5851],
// com[3][5851] (own and refined cells: moments and centres of mass; leaf
// neighbours: mass at the cell centre; empty directions and the root's halo:
// zeros), or monopole update_input (monopole_interaction_interface.hpp:64-143)
// into mon[5832] (own and leaf cells' masses). One thread per padded entry.
__global__ void stage_soa_kernel(const double* __restrict__ M, const double* __restrict__ com,
                                 const double* __restrict__ mon, const uint8_t* __restrict__ is_leaf,
                                 otfmm_work_item it, double* mon_out, double* M_out, double* com_out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    const bool leaf_item = (it.kind == OTFMM_KIND_LEAF);
    if (f >= CL) return;
    if (f >= ENTRIES) {   // SoA padding tail of the component arrays
        if (!leaf_item) {
            for (int q = 0; q < 20; ++q) M_out[q * CL + f] = 0.0;
            for (int a = 0; a < 3; ++a) com_out[a * CL + f] = 0.0;
        }
        return;
    }
    const int ax = f / (PSTRIDE * PSTRIDE) - (INX - PAD_OFF), ay = (f / PSTRIDE) % PSTRIDE - (INX - PAD_OFF),
              az = f % PSTRIDE - (INX - PAD_OFF);
    const int raw = raw_dir(ax, ay, az);
    const bool centre = (raw == 13);
    const int src = centre ? it.subgrid
                           : (it.kind == OTFMM_KIND_M2L_ROOT ? -1 : it.neighbors[raw < 13 ? raw : raw - 1]);
    const int u = (ax & 7) * 64 + (ay & 7) * 8 + (az & 7);
    if (leaf_item) {
        mon_out[f] = (src >= 0 && (centre || is_leaf[src])) ? mon[(size_t)src * NCELL + u] : 0.0;
        return;
    }
    double m0 = 0.0, c[3] = {0.0, 0.0, 0.0};
    bool moments = false;
    if (src >= 0) {
        if (centre || !is_leaf[src]) {
            moments = true;
            for (int a = 0; a < 3; ++a) c[a] = com[((size_t)src * 3 + a) * NCELL + u];
        } else {
            m0 = mon[(size_t)src * NCELL + u];
            const int ip[3] = {ax + INX, ay + INX, az + INX};
            for (int a = 0; a < 3; ++a)
                c[a] = __dsub_rn(__dadd_rn(__dmul_rn((double)ip[a], it.dx), it.xbase[a]), __dmul_rn((double)INX, it.dx));
        }
    }
    mon_out[f] = m0;
    for (int q = 0; q < 20; ++q) M_out[q * CL + f] = moments ? M[((size_t)src * 20 + q) * NCELL + u] : 0.0;
    for (int a = 0; a < 3; ++a) com_out[a * CL + f] = c[a];
}

// Slab of refined neighbour nb in direction d for the per-subgrid P2M entry
// point (update_neighbor_input, p2m_interaction_interface.hpp:102-160): the
// cells within reach, component-major with stride size + 19.
__global__ void stage_p2m_kernel(const double* __restrict__ M, const double* __restrict__ com, int nb, int d,
                                 double* nM, double* ncom) {
    const int r = d < 13 ? d : d + 1;
    const int o[3] = {r % 3 - 1, (r / 3) % 3 - 1, r / 9 - 1};
    int s[3], sz[3];
    for (int a = 0; a < 3; ++a) {
        s[a] = (o[a] == -1) ? INX - SMAX : 0;
        sz[a] = ((o[a] == 1) ? SMAX : INX) - s[a];
    }
    const int size = sz[0] * sz[1] * sz[2], stride = size + 19;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= stride) return;
    if (f >= size) {
        for (int q = 0; q < 20; ++q) nM[q * stride + f] = 0.0;
        for (int a = 0; a < 3; ++a) ncom[a * stride + f] = 0.0;
        return;
    }
    const int x = f / (sz[1] * sz[2]) + s[0], y = (f / sz[2]) % sz[1] + s[1], z = f % sz[2] + s[2];
    const int u = x * 64 + y * 8 + z;
    for (int q = 0; q < 20; ++q) nM[q * stride + f] = M[((size_t)nb * 20 + q) * NCELL + u];
    for (int a = 0; a < 3; ++a) ncom[a * stride + f] = com[((size_t)nb * 3 + a) * NCELL + u];
}

}   // namespace otfmm
