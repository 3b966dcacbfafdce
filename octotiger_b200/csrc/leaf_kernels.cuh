// Leaf subgrids: P2P over the leaf's own and leaf neighbours' masses and P2M
// against refined neighbours, as persistent batched kernels.
// Part of libotfmm.so; included once, in order, by otfmm.cu (one translation unit).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/otfmm.h"
#include "pair_math.cuh"
#include "layout.cuh"

namespace otfmm {

// Leaf items: P2P (p2p_kernel_impl, monopole kokkos_kernel.hpp:143-320) over
// the masses of the leaf and its leaf neighbours; refined and empty
// neighbours are staged as zero mass (update_input,
// monopole_interaction_interface.hpp:82-87), which adds exact zeros, so the
// sweep has no branch. Writes L0..L3 only, like the reference's monopole path
// (L4..L19 and L_c of a leaf are left as the caller zeroed them; the P2M
// kernel adds the refined-neighbour part afterwards).
// Persistent: each CTA stages the per-parity offset/constant table once and
// then walks the leaf list with a grid stride (every leaf costs the same).
constexpr int P2P_CTAS_PER_SM = 2;
constexpr int P2P_THREADS = 256;   // 8 warps: one per parity class, two cells per thread
constexpr int P2P_TABLE_BYTES = 8 * MAX_ENTRIES * (4 * 8 + 4);
constexpr int P2P_SMEM_BYTES = P_SMEM_DOUBLES * 8 + P2P_TABLE_BYTES;

template <int PREC>
__global__ void __launch_bounds__(P2P_THREADS, P2P_CTAS_PER_SM) p2p_batch_kernel(BatchArgs a) {
    extern __shared__ double dyn[];
    double* pm = dyn;                                                      // mass region
    double4* s_four = reinterpret_cast<double4*>(dyn + P_SMEM_DOUBLES);   // [8][MAX_ENTRIES]
    int* s_delta = reinterpret_cast<int*>(s_four + 8 * MAX_ENTRIES);       // [8][MAX_ENTRIES]
    __shared__ ItemInfo it;
    for (int e = threadIdx.x; e < 8 * MAX_ENTRIES; e += blockDim.x) {
        const int p = e / MAX_ENTRIES, k = e % MAX_ENTRIES;
        if (k < a.t.count[p]) {
            const int2 en = a.t.entries_p2p[e];
            s_delta[e] = en.x;
            s_four[e] = make_double4(c_four[en.y][0], c_four[en.y][1], c_four[en.y][2], c_four[en.y][3]);
        }
    }
    // thread -> two cells: warp w owns parity class w (64 cells); lane covers
    // sub-lattice x' = i and i + 2 at (j, k), so each table read serves two pairs
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int p = w;
    const int i = lane >> 4, j = (lane >> 2) & 3, k = lane & 3;
    const int px = (p >> 2) & 1, py = (p >> 1) & 1, pz = p & 1;
    const int cy = py + 2 * j, cz = pz + 2 * k;
    const int cxa = px + 2 * i, cxb = px + 2 * (i + 2);
    const int lane_off = i * P_XS + j * P_RS + k;
    constexpr int OFF_B = 2 * P_XS;   // second cell: two sub-lattice planes further in x
    const int n = a.t.count[p];
    const double4* four = s_four + p * MAX_ENTRIES;
    const int* delta = s_delta + p * MAX_ENTRIES;
    const int nleaf = a.wl.counts[WL_LEAF];
    for (int kk = blockIdx.x; kk < nleaf; kk += gridDim.x) {
        __syncthreads();   // previous leaf's readers are done with pm / it
        load_item(a, a.wl.leaf[kk], it);
        const double dc0 = __ddiv_rn(1.0, it.dx), dc1 = __ddiv_rn(-1.0, it.dx);
        for (int r = threadIdx.x; r < P_REG * P_REG * P_REG; r += blockDim.x) {
            const int ax = r / (P_REG * P_REG) - 2, ay = (r / P_REG) % P_REG - 2, az = r % P_REG - 2;
            const int raw = raw_dir(ax, ay, az);
            const int src = (raw == 13) ? it.subgrid : it.nb[raw < 13 ? raw : raw - 1];
            double m = 0.0;
            if (src >= 0 && (raw == 13 || a.is_leaf[src]))
                m = a.mon[(size_t)src * NCELL + (ax & 7) * 64 + (ay & 7) * 8 + (az & 7)];
            if (PREC != PREC_EXACT) m *= dc0;   // 1/dx folded into the staged mass
            const int cls = ((ax & 1) << 2) | ((ay & 1) << 1) | (az & 1);
            pm[cls * P_CLS + ((ax + 2) >> 1) * P_XS + ((ay + 2) >> 1) * P_RS + ((az + 2) >> 1)] = m;
        }
        __syncthreads();
        double ga[4] = {0.0, 0.0, 0.0, 0.0}, gb[4] = {0.0, 0.0, 0.0, 0.0};
        if (PREC == PREC_EXACT) {
            for (int e = 0; e < n; ++e) {
                const double4 f = four[e];
                const int d = delta[e] + lane_off;
                const double ma = __dmul_rn(pm[d], dc0), mb = __dmul_rn(pm[d + OFF_B], dc0);
                ga[0] = __dadd_rn(ga[0], __dmul_rn(f.x, ma));
                ga[1] = __dadd_rn(ga[1], __dmul_rn(__dmul_rn(f.y, ma), dc1));
                ga[2] = __dadd_rn(ga[2], __dmul_rn(__dmul_rn(f.z, ma), dc1));
                ga[3] = __dadd_rn(ga[3], __dmul_rn(__dmul_rn(f.w, ma), dc1));
                gb[0] = __dadd_rn(gb[0], __dmul_rn(f.x, mb));
                gb[1] = __dadd_rn(gb[1], __dmul_rn(__dmul_rn(f.y, mb), dc1));
                gb[2] = __dadd_rn(gb[2], __dmul_rn(__dmul_rn(f.z, mb), dc1));
                gb[3] = __dadd_rn(gb[3], __dmul_rn(__dmul_rn(f.w, mb), dc1));
            }
        } else {
#pragma unroll 4
            for (int e = 0; e < n; ++e) {
                const double4 f = four[e];
                const int d = delta[e] + lane_off;
                const double ma = pm[d], mb = pm[d + OFF_B];
                ga[0] = fma(f.x, ma, ga[0]);
                ga[1] = fma(f.y, ma, ga[1]);
                ga[2] = fma(f.z, ma, ga[2]);
                ga[3] = fma(f.w, ma, ga[3]);
                gb[0] = fma(f.x, mb, gb[0]);
                gb[1] = fma(f.y, mb, gb[1]);
                gb[2] = fma(f.z, mb, gb[2]);
                gb[3] = fma(f.w, mb, gb[3]);
            }
#pragma unroll
            for (int q = 1; q < 4; ++q) {
                ga[q] *= dc1;
                gb[q] *= dc1;
            }
        }
        double* L = a.L + (size_t)it.subgrid * 20 * NCELL;
        double* Lc = a.Lc + (size_t)it.subgrid * 3 * NCELL;
        const int cfa = cxa * 64 + cy * 8 + cz, cfb = cxb * 64 + cy * 8 + cz;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            L[q * NCELL + cfa] = ga[q];
            L[q * NCELL + cfb] = gb[q];
        }
        (void)Lc;   // L4..L19 and L_c of a leaf are not written here (see otfmm_batch)
    }
}

// Leaf items, P2P in the fast FP64 form (T = double) or the FP32 split form
// (T = float, FP32 partial sums promoted to FP64 every CHUNK partners):
// persistent, one CTA of 1024 threads per SM made of 4 groups of 8 warps.
// Every group solves one leaf at a time (warp = parity class, two cells per
// thread, the partner mass of each stencil entry read from the staged
// region); the 4 groups share one copy of the per-parity delta and monopole
// constant table, and synchronise among themselves with named barriers.
constexpr int P2_GROUPS = 4;
constexpr int P2_THREADS = 256 * P2_GROUPS;
template <class T>
struct P2Vec;
template <>
struct P2Vec<double> {
    using type = double4;
};
template <>
struct P2Vec<float> {
    using type = float4;
};
template <class T>
constexpr int p2_smem_bytes() {
    return 8 * MAX_ENTRIES * (int)(sizeof(typename P2Vec<T>::type) + sizeof(int)) +
           P2_GROUPS * P_SMEM_DOUBLES * (int)sizeof(T);
}
static_assert(p2_smem_bytes<double>() <= 232448 - 1024, "FP64 P2P groups fit");

__device__ __forceinline__ void group_sync(int g) {
    asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(256) : "memory");
}

template <class T, int CHUNK>
__global__ void __launch_bounds__(P2_THREADS, 1) p2p_leaf_kernel(BatchArgs a) {
    using V4 = typename P2Vec<T>::type;
    extern __shared__ __align__(16) unsigned char p2_dyn[];
    V4* s_four = reinterpret_cast<V4*>(p2_dyn);
    int* s_delta = reinterpret_cast<int*>(p2_dyn + 8 * MAX_ENTRIES * sizeof(V4));
    T* regions = reinterpret_cast<T*>(p2_dyn + 8 * MAX_ENTRIES * (sizeof(V4) + sizeof(int)));
    __shared__ ItemInfo its[P2_GROUPS];
    const int nleaf = a.wl.counts[WL_LEAF];
    if (blockIdx.x * P2_GROUPS >= nleaf) return;   // no leaf for this CTA (uniform for the block)
    // per-parity monopole constants and deltas, prebuilt in stencil order at context creation
    for (int e = threadIdx.x; e < 8 * MAX_ENTRIES; e += blockDim.x) {
        const double4 f = a.t.p2p_four[e];
        s_four[e] = V4{(T)f.x, (T)f.y, (T)f.z, (T)f.w};
        s_delta[e] = a.t.entries_p2p[e].x;
    }
    __syncthreads();
    const int g = threadIdx.x >> 8, tid = threadIdx.x & 255;
    T* pm = regions + g * P_SMEM_DOUBLES;
    ItemInfo& it = its[g];
    const int p = tid >> 5, lane = tid & 31;
    const int i = lane >> 4, j = (lane >> 2) & 3, k = lane & 3;
    const int px = (p >> 2) & 1, py = (p >> 1) & 1, pz = p & 1;
    const int cy = py + 2 * j, cz = pz + 2 * k;
    const int cxa = px + 2 * i, cxb = px + 2 * (i + 2);
    const int lane_off = i * P_XS + j * P_RS + k;
    constexpr int OFF_B = 2 * P_XS;   // second cell: two sub-lattice planes further in x
    const int n = a.t.count[p];
    const V4* four = s_four + p * MAX_ENTRIES;
    const int* delta = s_delta + p * MAX_ENTRIES;
    for (int kk = blockIdx.x * P2_GROUPS + g; kk < nleaf; kk += gridDim.x * P2_GROUPS) {
        group_sync(g);   // the group's previous leaf is done with pm / it
        if (tid == 0) {
            const otfmm_work_item& w = a.items[a.wl.leaf[kk]];
            it.subgrid = w.subgrid;
            it.dx = w.dx;
            for (int d = 0; d < 26; ++d) it.nb[d] = w.neighbors[d];
        }
        group_sync(g);
        const double dc0 = 1.0 / it.dx;
        for (int r = tid; r < P_REG * P_REG * P_REG; r += 256) {
            const int ax = r / (P_REG * P_REG) - 2, ay = (r / P_REG) % P_REG - 2, az = r % P_REG - 2;
            const int raw = raw_dir(ax, ay, az);
            const int src = (raw == 13) ? it.subgrid : it.nb[raw < 13 ? raw : raw - 1];
            double m = 0.0;
            if (src >= 0 && (raw == 13 || a.is_leaf[src]))
                m = a.mon[(size_t)src * NCELL + (ax & 7) * 64 + (ay & 7) * 8 + (az & 7)];
            const int cls = ((ax & 1) << 2) | ((ay & 1) << 1) | (az & 1);
            pm[cls * P_CLS + ((ax + 2) >> 1) * P_XS + ((ay + 2) >> 1) * P_RS + ((az + 2) >> 1)] = (T)(m * dc0);
        }
        group_sync(g);
        double ga[4] = {0.0, 0.0, 0.0, 0.0}, gb[4] = {0.0, 0.0, 0.0, 0.0};
        if (sizeof(T) == 8) {
#pragma unroll 4
            for (int e = 0; e < n; ++e) {
                const V4 f = four[e];
                const int d = delta[e] + lane_off;
                const double ma = pm[d], mb = pm[d + OFF_B];
                ga[0] = fma((double)f.x, ma, ga[0]);
                ga[1] = fma((double)f.y, ma, ga[1]);
                ga[2] = fma((double)f.z, ma, ga[2]);
                ga[3] = fma((double)f.w, ma, ga[3]);
                gb[0] = fma((double)f.x, mb, gb[0]);
                gb[1] = fma((double)f.y, mb, gb[1]);
                gb[2] = fma((double)f.z, mb, gb[2]);
                gb[3] = fma((double)f.w, mb, gb[3]);
            }
        } else {
#pragma unroll 1
            for (int e0 = 0; e0 < n; e0 += CHUNK) {
                const int e1 = min(e0 + CHUNK, n);
                float fa[4] = {0.f, 0.f, 0.f, 0.f}, fb[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 4
                for (int e = e0; e < e1; ++e) {
                    const V4 f = four[e];
                    const int d = delta[e] + lane_off;
                    const float ma = (float)pm[d], mb = (float)pm[d + OFF_B];
                    fa[0] = fmaf((float)f.x, ma, fa[0]);
                    fa[1] = fmaf((float)f.y, ma, fa[1]);
                    fa[2] = fmaf((float)f.z, ma, fa[2]);
                    fa[3] = fmaf((float)f.w, ma, fa[3]);
                    fb[0] = fmaf((float)f.x, mb, fb[0]);
                    fb[1] = fmaf((float)f.y, mb, fb[1]);
                    fb[2] = fmaf((float)f.z, mb, fb[2]);
                    fb[3] = fmaf((float)f.w, mb, fb[3]);
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    ga[q] += (double)fa[q];
                    gb[q] += (double)fb[q];
                }
            }
        }
        const double dc1 = -dc0;
#pragma unroll
        for (int q = 1; q < 4; ++q) {
            ga[q] *= dc1;
            gb[q] *= dc1;
        }
        double* L = a.L + (size_t)it.subgrid * 20 * NCELL;
        const int cfa = cxa * 64 + cy * 8 + cz, cfb = cxb * 64 + cy * 8 + cz;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            L[q * NCELL + cfa] = ga[q];
            L[q * NCELL + cfb] = gb[q];
        }
    }
}

// Leaf items with refined neighbours: P2M (p2m_kernel_impl_rho / _non_rho,
// monopole kokkos_kernel.hpp:517-942) after P2P: one CTA per leaf of the P2M
// work list (grid stride). The refined directions are taken one after the
// other in direction order, like the reference's one launch per refined
// neighbour; within a direction only the cells that have partners there
// work, ordered by their partner count (a table built at context creation),
// so the lanes of a warp run loops of similar length. The exact form visits a
// cell's entries of that direction in stencil order on one lane; the fast
// form spreads them over F lanes (as many as the CTA holds, up to 16) and
// sums the F partial results in a fixed butterfly order. The per-cell sums
// live in shared memory between directions. Partner moments come through L1/L2.
template <int PREC, bool RHO>
__global__ void __launch_bounds__(P_THREADS) p2m_batch_kernel(BatchArgs a) {
    __shared__ ItemInfo it;
    __shared__ double s_acc[7][NCELL];   // L0..L3, then L_c x, y, z
    constexpr int P64 = (PREC == PREC_EXACT) ? PREC_EXACT : PREC_FAST;
    const int np2m = a.wl.counts[WL_P2M];
    for (int kk = blockIdx.x; kk < np2m; kk += gridDim.x) {
        __syncthreads();   // `it` and s_acc are reused
        load_item(a, a.wl.p2m[kk], it);
        uint32_t refmask = 0;
        for (int d = 0; d < 26; ++d) {
            const int nb = it.nb[d];
            if (nb >= 0 && !a.is_leaf[nb]) refmask |= 1u << (d < 13 ? d : d + 1);
        }
        const size_t sub = (size_t)it.subgrid;
        double* L = a.L + sub * 20 * NCELL;
        double* Lc = a.Lc + sub * 3 * NCELL;
        for (int cu = threadIdx.x; cu < NCELL; cu += blockDim.x) {
#pragma unroll
            for (int q = 0; q < 4; ++q) s_acc[q][cu] = L[q * NCELL + cu];
#pragma unroll
            for (int q = 4; q < 7; ++q) s_acc[q][cu] = 0.0;
        }
        for (uint32_t rm = refmask; rm; rm &= rm - 1) {
            const int raw = __ffs(rm) - 1;
            __syncthreads();   // the previous direction's sums are in place
            const size_t nb = (size_t)it.nb[raw < 13 ? raw : raw - 1];
            const double* __restrict__ nM = a.M + nb * 20 * NCELL;
            const double* __restrict__ ncom = a.com + nb * 3 * NCELL;
            const int t0 = __ldg(a.t.p2m_perm_start + raw), nt = __ldg(a.t.p2m_perm_start + raw + 1) - t0;
            // F lanes share a cell's entries of this direction (fast form; F divides 32);
            // the exact form keeps one lane per cell and the stencil order
            int F = 1;
            if (P64 != PREC_EXACT)
                while (F < a.p2m_lanes && nt * 2 * F <= (int)blockDim.x) F <<= 1;
            const int tgt = threadIdx.x / F, f = threadIdx.x % F;
            const bool active = tgt < nt;
            const int cu = active ? __ldg(a.t.p2m_perm + t0 + tgt) : 0;
            double X[3], acc[4], corr[3];
#pragma unroll
            for (int q = 0; q < 3; ++q) X[q] = __ldg(a.com + (sub * 3 + q) * NCELL + cu);
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[q] = (P64 == PREC_EXACT && active) ? s_acc[q][cu] : 0.0;
#pragma unroll
            for (int q = 0; q < 3; ++q) corr[q] = (P64 == PREC_EXACT && active) ? s_acc[4 + q][cu] : 0.0;
            const int beg = active ? __ldg(a.t.p2m_start + cu * 28 + raw) : 0;
            const int end = active ? __ldg(a.t.p2m_start + cu * 28 + raw + 1) : 0;
#pragma unroll 1
            for (int q = beg + f; q < end; q += F) {
                const int u = __ldg(a.t.p2m_list + q);
                double Y[3], mp[20];
#pragma unroll
                for (int c = 0; c < 3; ++c) Y[c] = __ldg(ncom + c * NCELL + u);
#pragma unroll
                for (int c = 0; c < 20; ++c) mp[c] = __ldg(nM + c * NCELL + u) * stage_scale<P64>(c);
                if (P64 == PREC_EXACT)
                    exact_p2m_pair<RHO>(X, Y, mp, acc, corr);
                else
                    fast_p2m_pair<RHO>(X, Y, mp, acc, corr);
            }
            if (P64 != PREC_EXACT) {
                // fixed-order butterfly over the F lanes of each cell
                for (int o = F >> 1; o > 0; o >>= 1) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
#pragma unroll
                    for (int q = 0; q < 3; ++q) corr[q] += __shfl_xor_sync(0xffffffffu, corr[q], o);
                }
                if (active && f == 0) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) s_acc[q][cu] += acc[q];
#pragma unroll
                    for (int q = 0; q < 3; ++q) s_acc[4 + q][cu] += corr[q];
                }
            } else if (active) {
#pragma unroll
                for (int q = 0; q < 4; ++q) s_acc[q][cu] = acc[q];
#pragma unroll
                for (int q = 0; q < 3; ++q) s_acc[4 + q][cu] = corr[q];
            }
        }
        __syncthreads();
        for (int cu = threadIdx.x; cu < NCELL; cu += blockDim.x) {
#pragma unroll
            for (int q = 0; q < 4; ++q) L[q * NCELL + cu] = s_acc[q][cu];
            // L_c of a leaf with a refined neighbour: the P2M correction (zero for DRHODT)
#pragma unroll
            for (int q = 0; q < 3; ++q) Lc[q * NCELL + cu] = RHO ? s_acc[4 + q][cu] : 0.0;
        }
    }
}

// Fast-form P2M with every refined direction of a leaf in flight at once:
// one CTA per leaf of the P2M work list (grid stride). The work of a leaf is
// the list of (direction, cell, lane) slots of its refined directions, F lanes
// per cell (F = the tuning's P2M lane count), walked in rounds of the CTA's
// threads; the F lanes of a cell sum their partners' contributions in a fixed
// butterfly order into one partial per (direction, cell) in shared memory.
// After one barrier every cell adds its partials to its P2P result in direction
// order. Deterministic; no barrier between directions.
template <bool RHO>
__global__ void __launch_bounds__(P_THREADS) p2m_fast_kernel(BatchArgs a) {
    extern __shared__ double s_part[];   // [groups][7]: L0..L3, L_c x, y, z
    __shared__ ItemInfo it;
    __shared__ int s_dir[27], s_cum[28];
    __shared__ int s_ndir;
    const int F = a.p2m_lanes;
    const int np2m = a.wl.counts[WL_P2M];
    for (int kk = blockIdx.x; kk < np2m; kk += gridDim.x) {
        __syncthreads();   // `it`, the direction list and s_part are reused
        load_item(a, a.wl.p2m[kk], it);
        if (threadIdx.x == 0) {
            int n = 0, cum = 0;
            for (int d = 0; d < 26; ++d) {
                const int nb = it.nb[d];
                if (nb >= 0 && !a.is_leaf[nb]) {
                    const int r = d < 13 ? d : d + 1;
                    s_dir[n] = r;
                    s_cum[n] = cum;
                    cum += (a.t.p2m_perm_start[r + 1] - a.t.p2m_perm_start[r]) * F;
                    ++n;
                }
            }
            s_cum[n] = cum;
            s_ndir = n;
        }
        __syncthreads();
        const int ndir = s_ndir, total = s_cum[ndir];
        const size_t sub = (size_t)it.subgrid;
        for (int g0 = 0; g0 < total; g0 += blockDim.x) {
            const int g = g0 + threadIdx.x;
            double acc[4] = {0.0, 0.0, 0.0, 0.0}, corr[3] = {0.0, 0.0, 0.0};
            int k = 0;
            if (g < total) {
                while (s_cum[k + 1] <= g) ++k;
                const int r = s_dir[k];
                const int local = g - s_cum[k], tgt = local / F, f = local % F;
                const int cu = __ldg(a.t.p2m_perm + a.t.p2m_perm_start[r] + tgt);
                const size_t nb = (size_t)it.nb[r < 13 ? r : r - 1];
                const double* __restrict__ nM = a.M + nb * 20 * NCELL;
                const double* __restrict__ ncom = a.com + nb * 3 * NCELL;
                double X[3];
#pragma unroll
                for (int q = 0; q < 3; ++q) X[q] = __ldg(a.com + (sub * 3 + q) * NCELL + cu);
                const int beg = __ldg(a.t.p2m_start + cu * 28 + r), end = __ldg(a.t.p2m_start + cu * 28 + r + 1);
#pragma unroll 1
                for (int q = beg + f; q < end; q += F) {
                    const int u = __ldg(a.t.p2m_list + q);
                    double Y[3], mp[20];
#pragma unroll
                    for (int c = 0; c < 3; ++c) Y[c] = __ldg(ncom + c * NCELL + u);
#pragma unroll
                    for (int c = 0; c < 20; ++c) mp[c] = __ldg(nM + c * NCELL + u) * stage_scale<PREC_FAST>(c);
                    fast_p2m_pair<RHO>(X, Y, mp, acc, corr);
                }
            }
            // F lanes of a cell are aligned within the warp (F divides 32, every
            // direction's slot count is a multiple of F)
            for (int o = F >> 1; o > 0; o >>= 1) {
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
#pragma unroll
                for (int q = 0; q < 3; ++q) corr[q] += __shfl_xor_sync(0xffffffffu, corr[q], o);
            }
            if (g < total && (g % F) == 0) {
                double* part = s_part + (size_t)(g / F) * 7;
#pragma unroll
                for (int q = 0; q < 4; ++q) part[q] = acc[q];
#pragma unroll
                for (int q = 0; q < 3; ++q) part[4 + q] = corr[q];
            }
        }
        __syncthreads();
        double* L = a.L + sub * 20 * NCELL;
        double* Lc = a.Lc + sub * 3 * NCELL;
        for (int cu = threadIdx.x; cu < NCELL; cu += blockDim.x) {
            double acc[4], corr[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[q] = L[q * NCELL + cu];
            for (int k = 0; k < ndir; ++k) {
                const int t = __ldg(a.t.p2m_slot + s_dir[k] * NCELL + cu);
                if (t < 0) continue;
                const double* part = s_part + (size_t)(s_cum[k] / F + t) * 7;
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[q] += part[q];
#pragma unroll
                for (int q = 0; q < 3; ++q) corr[q] += part[4 + q];
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) L[q * NCELL + cu] = acc[q];
#pragma unroll
            for (int q = 0; q < 3; ++q) Lc[q * NCELL + cu] = RHO ? corr[q] : 0.0;
        }
    }
}

}   // namespace otfmm
