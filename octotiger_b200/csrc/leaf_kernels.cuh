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
            if (raw == 13 || ((it.leafmask >> raw) & 1u))
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

// Leaf items, P2P over the partner box (fast FP64 form T = double; FP32 split
// form T = float, FP32 partial sums promoted to FP64 every ROWS partner rows of
// 6). With a stencil of coarse reach 1 the partners of a cell are the cells of
// the 3x3x3 coarse cells around its own, a 6x6x6 box shared by the 8 cells of a
// coarse cell. One CTA of 128 threads per leaf (CTAs take leaves from an atomic counter):
// warp w takes the cells of x/y parity (w >> 1, w & 1); lane (Cx, Cy, c) the
// four cells (2 Cx + px, 2 Cy + py, z), z in {2c, 2c + 1, 2c + 4, 2c + 5}.
// A partner mass read from shared memory serves two of them (the two cells of
// a coarse cell), a monopole constant (one warp-uniform read) two as well (the
// two cells of one parity). FULL: every parity has the whole box in its stencil
// and the constants come from the 7^3 table of offsets; otherwise from the
// per-parity box tables, zero where an offset is off the stencil.
template <class T>
struct BoxLayout;
template <>
struct BoxLayout<float> {   // float2 reads: the 16 lanes of a half-warp hit distinct 8-byte slots
    static constexpr int RYS = 18, RXS = 216;
    using V2 = float2;
};
template <>
struct BoxLayout<double> {   // double2 reads: the 8 lanes of a quarter-warp hit distinct 16-byte slots
    static constexpr int RYS = 14, RXS = 168;
    using V2 = double2;
};
constexpr int BOX_THREADS = 128;
constexpr int BOX_CUBE = 343;
constexpr int BOX_CELLS = 216;
template <class T, bool FULL>
constexpr int box_smem_bytes() {
    return (FULL ? BOX_CUBE : 8 * BOX_CELLS) * (int)sizeof(typename P2Vec<T>::type) +
           P_REG * BoxLayout<T>::RXS * (int)sizeof(T);
}
static_assert(11 * BoxLayout<float>::RYS + 12 <= BoxLayout<float>::RXS &&
                  11 * BoxLayout<double>::RYS + 12 <= BoxLayout<double>::RXS,
              "box region rows fit their planes");

// f[0..3] += q * m: FP32 as two packed FMAs (x, y) and (z, w); FP64 as four.
__device__ __forceinline__ void box_fma4(const float4& q, float m, float f[4]) {
    const float2 mm = make_float2(m, m);
    const float2 lo = __ffma2_rn(make_float2(q.x, q.y), mm, make_float2(f[0], f[1]));
    const float2 hi = __ffma2_rn(make_float2(q.z, q.w), mm, make_float2(f[2], f[3]));
    f[0] = lo.x;
    f[1] = lo.y;
    f[2] = hi.x;
    f[3] = hi.y;
}
__device__ __forceinline__ void box_fma4(const double4& q, double m, double f[4]) {
    f[0] = fma(q.x, m, f[0]);
    f[1] = fma(q.y, m, f[1]);
    f[2] = fma(q.z, m, f[2]);
    f[3] = fma(q.w, m, f[3]);
}

// Five CTAs per SM (96 registers; the box P2P of the AMR polytrope: 0.116 against
// 0.124 ms with four), four for the split form's 18-partner chunks, whose
// extra promotions would spill at 96 registers.
template <class T, int ROWS>
constexpr int box_ctas_per_sm() { return (sizeof(T) == 4 && ROWS == 3) ? 4 : 5; }

template <class T, bool FULL, int ROWS>
__global__ void __launch_bounds__(BOX_THREADS, box_ctas_per_sm<T, ROWS>()) p2p_box_kernel(BatchArgs a) {
    using V4 = typename P2Vec<T>::type;
    using V2 = typename BoxLayout<T>::V2;
    constexpr int RYS = BoxLayout<T>::RYS, RXS = BoxLayout<T>::RXS;
    constexpr int NT = FULL ? BOX_CUBE : 8 * BOX_CELLS;
    extern __shared__ __align__(16) unsigned char bx_dyn[];
    V4* s_four = reinterpret_cast<V4*>(bx_dyn);
    T* reg = reinterpret_cast<T*>(bx_dyn + NT * sizeof(V4));
    __shared__ ItemInfo it;
    const int nleaf = a.wl.counts[WL_LEAF];
    if (blockIdx.x >= nleaf) return;   // uniform for the block
    const double4* src4 = FULL ? a.t.p2p_cube : a.t.p2p_box;
    for (int e = threadIdx.x; e < NT; e += BOX_THREADS) {
        const double4 f = src4[e];
        s_four[e] = V4{(T)f.x, (T)f.y, (T)f.z, (T)f.w};
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int px = w >> 1, py = w & 1;
    const int c = lane & 1, Cy = (lane >> 1) & 3, Cx = lane >> 3;
    // constants of the cells of z parity 0 (qa) and 1 (qb) for box row (i, j):
    // FULL: qa[k] = cube[base(i, j) + k + 1], qb[k] = cube[base(i, j) + k]
    const V4* tab_a = FULL ? s_four + (1 - px) * 49 + (1 - py) * 7 : s_four + (4 * px + 2 * py) * BOX_CELLS;
    const V4* tab_b = FULL ? tab_a : tab_a + BOX_CELLS;
    const int lane_off = (2 * Cx) * RXS + (2 * Cy) * RYS + 2 * c;
    __shared__ int s_next;
    for (;;) {
        __syncthreads();   // the previous leaf is done with `reg` and `it`
        if (threadIdx.x == 0) s_next = atomicAdd(a.wl.counts + WL_LEAF_NEXT, 1);
        __syncthreads();
        const int kk = s_next;
        if (kk >= nleaf) break;
        load_item(a, a.wl.leaf[kk], it);
        const double dc0 = 1.0 / it.dx;
        const uint32_t lm = it.leafmask | (1u << 13);   // the leaf itself and its leaf neighbours
        const size_t own = (size_t)it.subgrid;
        // masses / dx of the cells -2..9 per axis (the leaf and its leaf neighbours;
        // zeros elsewhere), seven loads of a thread in flight at a time
        constexpr int NR = P_REG * P_REG * P_REG, NB = 7;
#pragma unroll 1
        for (int r0 = 0; r0 < NR; r0 += NB * BOX_THREADS) {
            double v[NB];
#pragma unroll
            for (int t = 0; t < NB; ++t) {
                const int r = r0 + threadIdx.x + t * BOX_THREADS;
                v[t] = 0.0;
                if (r < NR) {
                    const int ax = r / (P_REG * P_REG) - 2, ay = (r / P_REG) % P_REG - 2, az = r % P_REG - 2;
                    const int raw = raw_dir(ax, ay, az);
                    if ((lm >> raw) & 1u) {
                        const size_t src = (raw == 13) ? own : (size_t)it.nb[raw < 13 ? raw : raw - 1];
                        v[t] = __ldg(a.mon + src * NCELL + (ax & 7) * 64 + (ay & 7) * 8 + (az & 7));
                    }
                }
            }
#pragma unroll
            for (int t = 0; t < NB; ++t) {
                const int r = r0 + threadIdx.x + t * BOX_THREADS;
                if (r < NR) {
                    const int rx = r / (P_REG * P_REG), ry = (r / P_REG) % P_REG, rz = r % P_REG;
                    reg[rx * RXS + ry * RYS + rz] = (T)(v[t] * dc0);
                }
            }
        }
        __syncthreads();
        double g[4][4];
        T f[4][4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                g[u][q] = 0.0;
                f[u][q] = (T)0;
            }
#pragma unroll 1
        for (int i = 0; i < 6; ++i) {
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                // partner masses of box row (i, j): m[k] for cells 2c, 2c + 1 and m[k + 4] for 2c + 4, 2c + 5
                const T* row = reg + lane_off + i * RXS + j * RYS;
                T m[10];
#pragma unroll
                for (int h = 0; h < 5; ++h) {
                    const V2 v = *reinterpret_cast<const V2*>(row + 2 * h);
                    m[2 * h] = v.x;
                    m[2 * h + 1] = v.y;
                }
                const int b = FULL ? i * 49 + j * 7 : (i * 6 + j) * 6;
                V4 qa[6], qb[6];
                if (FULL) {
                    V4 q7[7];
#pragma unroll
                    for (int k = 0; k < 7; ++k) q7[k] = tab_a[b + k];
#pragma unroll
                    for (int k = 0; k < 6; ++k) {
                        qa[k] = q7[k + 1];
                        qb[k] = q7[k];
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 6; ++k) {
                        qa[k] = tab_a[b + k];
                        qb[k] = tab_b[b + k];
                    }
                }
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    const T mA = m[k], mC = m[k + 4];
                    box_fma4(qa[k], mA, f[0]);
                    box_fma4(qb[k], mA, f[1]);
                    box_fma4(qa[k], mC, f[2]);
                    box_fma4(qb[k], mC, f[3]);
                }
                if constexpr (sizeof(T) == 4) {
                    if ((j % ROWS) != ROWS - 1) continue;
#pragma unroll
                    for (int u = 0; u < 4; ++u)
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            g[u][q] += (double)f[u][q];
                            f[u][q] = (T)0;
                        }
                }
            }
        }
        if constexpr (sizeof(T) == 8) {
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int q = 0; q < 4; ++q) g[u][q] = (double)f[u][q];
        }
        const double dc1 = -dc0;
        double* L = a.L + (size_t)it.subgrid * 20 * NCELL;
        const int cxy = (2 * Cx + px) * 64 + (2 * Cy + py) * 8;
        const int zc[4] = {2 * c, 2 * c + 1, 2 * c + 4, 2 * c + 5};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            L[cxy + zc[u]] = g[u][0];
#pragma unroll
            for (int q = 1; q < 4; ++q) L[q * NCELL + cxy + zc[u]] = g[u][q] * dc1;
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
        const uint32_t refmask = it.nbmask & ~it.leafmask;
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
#pragma unroll 2
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

// Fast-form P2M by coarse cell (reach 1). The partners of a leaf cell in a
// refined neighbour are the neighbour's cells inside the 3x3x3 coarse cells
// around the cell's coarse cell, one list shared by the 8 cells of a coarse
// cell, all inside the neighbour's slab next to the leaf (2 cells deep across
// each shared face). Per leaf the refined directions are taken in rounds (in
// raw-direction order, as many as fit the shared-memory budget): the round's
// slabs are staged in shared memory (scaled moments and centres of mass), then
// its units - 4 coarse cells of one direction - go to the warps, one lane per
// cell (lane = 8 x slot + cell of the coarse cell), so the 8 lanes of a coarse
// cell read each partner together. A direction's partner lists are cut in
// parts of at most PC_PART partners (the same number of parts for all its
// units), so that face units (72 partners) and corner units (8) make work
// items of similar length. Each (item, cell) partial goes to shared memory; at
// the end of the round every cell adds the round's partials to L (and L_c) in
// direction, then part order. One CTA per leaf of the P2M work list (taken
// from an atomic counter).
constexpr int PC_THREADS = 256;
constexpr int PC_PART = 24;               // partners of one work item (a unit's list is cut in parts)
constexpr int PC_ROUND_ITEMS = 24;        // partials of one round: 24 x 32 x 7 doubles
constexpr int PC_ROUND_CELLS = 320;       // staged slab cells of one round: 23 doubles each
constexpr int PC_SMEM_BYTES = (PC_ROUND_ITEMS * 32 * 7 + 23 * PC_ROUND_CELLS) * 8;
__device__ __forceinline__ void pc_slab_shape(int r, int lo[3], int n[3]) {
    const int o[3] = {r % 3 - 1, (r / 3) % 3 - 1, r / 9 - 1};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        lo[d] = (o[d] == -1) ? INX - 2 : 0;
        n[d] = (o[d] == 0) ? INX : 2;
    }
}

template <bool RHO>
__global__ void __launch_bounds__(PC_THREADS, 2) p2m_coarse_kernel(BatchArgs a) {
    extern __shared__ double s_pc[];
    double* part = s_pc;                              // [round items][32 lanes][7]: L0..L3, L_c x, y, z
    double* slab = s_pc + PC_ROUND_ITEMS * 32 * 7;    // [23][PC_ROUND_CELLS]: 20 scaled moments, centre of mass
    __shared__ ItemInfo it;
    __shared__ int s_next, s_nr;
    __shared__ int8_t s_rdir[27];                     // the round's directions, in order
    __shared__ int s_rcell[28], s_ritem[28];          // their first slab cell / work item in the round
    const int np2m = a.wl.counts[WL_P2M];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for (;;) {
        __syncthreads();   // `it` and the round tables are reused
        if (threadIdx.x == 0) s_next = atomicAdd(a.wl.counts + WL_P2M_NEXT, 1);
        __syncthreads();
        const int kk = s_next;
        if (kk >= np2m) break;
        load_item(a, a.wl.p2m[kk], it);
        const uint32_t refmask = it.nbmask & ~it.leafmask;
        const size_t sub = (size_t)it.subgrid;
        double* L = a.L + sub * 20 * NCELL;
        double* Lc = a.Lc + sub * 3 * NCELL;
        bool first_round = true;
        for (int r0 = 0; r0 < 27;) {
            if (threadIdx.x == 0) {
                // the next round: directions from r0 on while slabs and units fit
                int n = 0, cells = 0, items = 0, r = r0;
                for (; r < 27; ++r) {
                    if (!((refmask >> r) & 1u)) continue;
                    int lo[3], sz[3];
                    pc_slab_shape(r, lo, sz);
                    const int c = sz[0] * sz[1] * sz[2];
                    const int w = (a.t.pc_unit_start[r + 1] - a.t.pc_unit_start[r]) * a.t.pc_parts[r];
                    if (n > 0 && (cells + c > PC_ROUND_CELLS || items + w > PC_ROUND_ITEMS)) break;
                    s_rdir[n] = (int8_t)r;
                    s_rcell[n] = cells;
                    s_ritem[n] = items;
                    cells += c;
                    items += w;
                    ++n;
                }
                s_rcell[n] = cells;
                s_ritem[n] = items;
                s_nr = n;
                s_next = r;   // where the following round starts
            }
            __syncthreads();
            const int nr = s_nr;
            r0 = s_next;
            // stage the round's slabs
            for (int t = threadIdx.x; t < s_rcell[nr]; t += blockDim.x) {
                int k = 0;
                while (s_rcell[k + 1] <= t) ++k;
                const int r = s_rdir[k], idx = t - s_rcell[k];
                int lo[3], sz[3];
                pc_slab_shape(r, lo, sz);
                const int x = lo[0] + idx / (sz[1] * sz[2]), y = lo[1] + (idx / sz[2]) % sz[1], z = lo[2] + idx % sz[2];
                const int u = x * 64 + y * 8 + z;
                const size_t nb = (size_t)it.nb[r < 13 ? r : r - 1];
#pragma unroll
                for (int c = 0; c < 20; ++c)
                    slab[c * PC_ROUND_CELLS + t] = __ldg(a.M + (nb * 20 + c) * NCELL + u) * stage_scale<PREC_FAST>(c);
#pragma unroll
                for (int q = 0; q < 3; ++q) slab[(20 + q) * PC_ROUND_CELLS + t] = __ldg(a.com + (nb * 3 + q) * NCELL + u);
            }
            __syncthreads();
            // the round's work items: (unit, part) of each direction
            for (int wi = warp; wi < s_ritem[nr]; wi += nwarps) {
                int k = 0;
                while (s_ritem[k + 1] <= wi) ++k;
                const int r = s_rdir[k], np = a.t.pc_parts[r];
                const int unit = (wi - s_ritem[k]) / np, pt = (wi - s_ritem[k]) % np;
                const int slot = 4 * unit + (lane >> 3), ci = lane & 7;
                const int C = __ldg(a.t.pc_coarse + 4 * a.t.pc_unit_start[r] + slot);
                double acc[4] = {0.0, 0.0, 0.0, 0.0}, corr[3] = {0.0, 0.0, 0.0};
                if (C >= 0) {
                    const int cu = (2 * (C >> 4) + (ci & 1)) * 64 + (2 * ((C >> 2) & 3) + ((ci >> 1) & 1)) * 8 +
                                   (2 * (C & 3) + (ci >> 2));
                    double X[3];
#pragma unroll
                    for (int q = 0; q < 3; ++q) X[q] = __ldg(a.com + (sub * 3 + q) * NCELL + cu);
                    const int2 be = __ldg(a.t.pc_range + r * 64 + C);
                    const double* sl = slab + s_rcell[k];
                    const int q1 = min(be.y, be.x + (pt + 1) * PC_PART);
#pragma unroll 1
                    for (int q = be.x + pt * PC_PART; q < q1; ++q) {
                        const int v = __ldg(a.t.pc_list + q);
                        double Y[3], mp[20];
#pragma unroll
                        for (int c = 0; c < 3; ++c) Y[c] = sl[(20 + c) * PC_ROUND_CELLS + v];
#pragma unroll
                        for (int c = 0; c < 20; ++c) mp[c] = sl[c * PC_ROUND_CELLS + v];
                        fast_p2m_pair<RHO>(X, Y, mp, acc, corr);
                    }
                }
                double* pp = part + ((size_t)wi * 32 + lane) * 7;
#pragma unroll
                for (int q = 0; q < 4; ++q) pp[q] = acc[q];
#pragma unroll
                for (int q = 0; q < 3; ++q) pp[4 + q] = corr[q];
            }
            __syncthreads();
            // every cell adds the round's partials in direction, then part order
            for (int cu = threadIdx.x; cu < NCELL; cu += blockDim.x) {
                const int cx = cu >> 6, cy = (cu >> 3) & 7, cz = cu & 7;
                const int C = (cx >> 1) * 16 + (cy >> 1) * 4 + (cz >> 1);
                const int ci = (cx & 1) | ((cy & 1) << 1) | ((cz & 1) << 2);
                double acc[4], corr[3];
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[q] = L[q * NCELL + cu];
#pragma unroll
                for (int q = 0; q < 3; ++q) corr[q] = first_round ? 0.0 : Lc[q * NCELL + cu];
                for (int k = 0; k < nr; ++k) {
                    const int sl = __ldg(a.t.pc_slot + s_rdir[k] * 64 + C);
                    if (sl < 0) continue;
                    const int np = a.t.pc_parts[s_rdir[k]];
                    for (int pt = 0; pt < np; ++pt) {
                        const double* pp =
                            part + ((size_t)(s_ritem[k] + (sl >> 2) * np + pt) * 32 + (sl & 3) * 8 + ci) * 7;
#pragma unroll
                        for (int q = 0; q < 4; ++q) acc[q] += pp[q];
#pragma unroll
                        for (int q = 0; q < 3; ++q) corr[q] += pp[4 + q];
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) L[q * NCELL + cu] = acc[q];
#pragma unroll
                for (int q = 0; q < 3; ++q) Lc[q * NCELL + cu] = RHO ? corr[q] : 0.0;
            }
            first_round = false;
            __syncthreads();   // partials, slabs and the round tables are reused
            if (nr == 0) break;
        }
    }
}

// Fast-form P2M with every refined direction of a leaf in flight at once:
// one CTA per leaf of the P2M work list (taken from an atomic counter). The work of a leaf is
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
    __shared__ int s_next;
    const int F = a.p2m_lanes;
    const int np2m = a.wl.counts[WL_P2M];
    for (;;) {
        __syncthreads();   // `it`, the direction list and s_part are reused
        if (threadIdx.x == 0) s_next = atomicAdd(a.wl.counts + WL_P2M_NEXT, 1);
        __syncthreads();
        const int kk = s_next;
        if (kk >= np2m) break;
        load_item(a, a.wl.p2m[kk], it);
        if (threadIdx.x == 0) {
            int n = 0, cum = 0;
            const uint32_t refmask = it.nbmask & ~it.leafmask;
            for (int d = 0; d < 26; ++d) {
                const int r = d < 13 ? d : d + 1;
                if ((refmask >> r) & 1u) {
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
#pragma unroll 2
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
