// Kernels for opening angles below 0.5 (coarse reach 2: partners up to five
// cells away, theta >= 0.34). The halo of a tile no longer fits in shared
// memory as a whole; partners are staged plane by plane or read from the
// buffers, in the reference's stencil order:
//   * m2l_r2_kernel: multipole tiles of refined items, partner x-planes
//     staged one by one in shared memory;
//   * p2p_r2_kernel: P2P of leaves from the pool;
//   * soa_m2l_r2_kernel: the per-subgrid entry point on the reference's 18^3
//     SoA buffers.
// Root tiles and P2M use the reach-independent kernels.
// Part of libotfmm.so; included once, in order, by otfmm.cu (one translation unit).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/otfmm.h"
#include "pair_math.cuh"
#include "layout.cuh"
#include "m2l_tiles.cuh"
#include "soa_kernels.cuh"

namespace otfmm {

// Multipole tiles (half a subgrid, 256 threads; warp = parity class) of
// refined and root items, persistent over the same tile counter as
// m2l_batch_kernel. A tile's partners lie in the 12 x-planes x0-4 .. x0+7 of
// 16 x 16 cells (y, z in -4 .. 11); the planes are staged one after the other
// in shared memory (what update_input stages at those positions:
// multipole_interaction_interface.hpp:88-281) and every target cell walks the
// entries of its parity class with sx = plane - cx. Increasing planes mean
// increasing sx, and the entries of one sx are in stencil order, so each cell
// accumulates in the reference's order. Root tiles stage their own cells
// (reach-independent root stencil).
constexpr int PL_RS = 12;                     // z' row: 8 cells + 4 pad (half-warps conflict-free)
constexpr int PL_COMP = 8 * PL_RS;            // one component of one (y, z) parity class
constexpr int PL_CLS = NCOMP * PL_COMP;       // 2208 doubles
constexpr int PL_DOUBLES = 4 * PL_CLS;        // 8832 doubles = 70,656 bytes
constexpr int PL_SMEM_BYTES = (ROOT_SMEM_DOUBLES > PL_DOUBLES ? ROOT_SMEM_DOUBLES : PL_DOUBLES) * 8;
static_assert(PL_RS % 16 == 12, "plane rows keep (j, k) half-warps conflict-free");

template <int PREC, bool RHO>
__global__ void __launch_bounds__(THREADS, 1) m2l_r2_kernel(BatchArgs a) {
    extern __shared__ double sm[];
    __shared__ ItemInfo it;
    __shared__ int tile;
    constexpr int RU = root_units<PREC>();
    const int nroot = a.wl.counts[WL_ROOT], nm2l = a.wl.counts[WL_M2L];
    const int total = RU * nroot + 2 * nm2l;
    for (;;) {
        if (threadIdx.x == 0) tile = atomicAdd(a.wl.counts + WL_M2L_NEXT, 1);
        __syncthreads();
        const int t = tile;
        if (t >= total) break;
        const int item_idx = (t < RU * nroot) ? a.wl.root[t / RU] : a.wl.m2l[(t - RU * nroot) >> 1];
        load_item(a, item_idx, it);
        const int x0 = TILE_X * (t & 1);
        const size_t sub = (size_t)it.subgrid;
        OutPtr out{a.L + sub * 20 * NCELL, a.Lc + sub * 3 * NCELL, NCELL, true};
        if (it.kind == OTFMM_KIND_M2L_ROOT) {
            for (int r = threadIdx.x; r < NCELL; r += blockDim.x)
                for (int q = 0; q < NCOMP; ++q)
                    sm[q * NCELL + r] = (q < 20) ? a.M[(sub * 20 + q) * NCELL + r] * stage_scale<PREC>(q)
                                                 : a.com[(sub * 3 + (q - 20)) * NCELL + r];
            __syncthreads();
            if (PREC == PREC_EXACT)
                root_tile<PREC, RHO>(sm, x0, a.t, out);
            else
                root_unit_fast<RHO, THREADS / 32>(sm, t % RU, a.t, out);
            __syncthreads();   // shared memory and `it` are reused by the next tile
            continue;
        }
        const uint32_t monomask = it.leafmask;   // leaf neighbours, by raw direction
        const CellMap c = cell_map(x0);
        const int cu = c.cx * 64 + c.cy * 8 + c.cz;
        const int lane_off = c.j * PL_RS + c.k;
        double X[3], mc[20], acc[20], corr[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int q = 0; q < 3; ++q) X[q] = a.com[(sub * 3 + q) * NCELL + cu];
#pragma unroll
        for (int q = 0; q < 20; ++q) {
            mc[q] = a.M[(sub * 20 + q) * NCELL + cu] * stage_scale<PREC>(q);
            acc[q] = 0.0;
        }
        const double inv_m0 = 1.0 / mc[0];
        const int2* ent = a.t.entries_r2 + c.p * MAX_ENTRIES_R2;
        const int* sxs = a.t.r2_sx_start + c.p * 12;
        for (int plane = x0 - 4; plane <= x0 + 7; ++plane) {
            __syncthreads();   // the previous plane is consumed
            {
                // stage plane `plane`: one cell per thread
                const int r = threadIdx.x;
                const int ax = plane, ay = (r >> 4) - 4, az = (r & 15) - 4;
                const int raw = raw_dir(ax, ay, az);
                const int src = (raw == 13) ? it.subgrid : it.nb[raw < 13 ? raw : raw - 1];
                const int u = (ax & 7) * 64 + (ay & 7) * 8 + (az & 7);
                double v[NCOMP];
                if (src < 0) {
#pragma unroll
                    for (int q = 0; q < NCOMP; ++q) v[q] = 0.0;
                } else if ((it.leafmask >> raw) & 1u) {
                    v[0] = a.mon[(size_t)src * NCELL + u];
#pragma unroll
                    for (int q = 1; q < 20; ++q) v[q] = 0.0;
                    const int ip[3] = {ax + INX, ay + INX, az + INX};
#pragma unroll
                    for (int q = 0; q < 3; ++q)
                        v[20 + q] = __dsub_rn(__dadd_rn(__dmul_rn((double)ip[q], it.dx), it.xbase[q]),
                                              __dmul_rn((double)INX, it.dx));
                } else {
#pragma unroll
                    for (int q = 0; q < 20; ++q) v[q] = a.M[((size_t)src * 20 + q) * NCELL + u] * stage_scale<PREC>(q);
#pragma unroll
                    for (int q = 0; q < 3; ++q) v[20 + q] = a.com[((size_t)src * 3 + q) * NCELL + u];
                }
                const int base = (((ay & 1) << 1) | (az & 1)) * PL_CLS + ((ay + 4) >> 1) * PL_RS + ((az + 4) >> 1);
#pragma unroll
                for (int q = 0; q < NCOMP; ++q) sm[base + q * PL_COMP] = v[q];
            }
            __syncthreads();
            const int sx = plane - c.cx;
            if (sx < -SMAX || sx > SMAX) continue;
            const int e1 = sxs[sx + SMAX + 1];
#pragma unroll 1
            for (int e = sxs[sx + SMAX]; e < e1; ++e) {
                const int2 en = __ldg(ent + e);
                const int pb = en.x + lane_off;
                double Y[3];
#pragma unroll
                for (int q = 0; q < 3; ++q) Y[q] = sm[pb + (20 + q) * PL_COMP];
                if (entry_flags(en.y) & F_FAR) {
                    double mp[20];
#pragma unroll
                    for (int q = 0; q < 20; ++q) mp[q] = sm[pb + q * PL_COMP];
                    if (PREC == PREC_EXACT)
                        exact_m2l_pair<RHO>(X, Y, mp, mc, acc, corr);
                    else
                        fast_m2l_pair<RHO>(X, Y, mp, mc + 10, inv_m0, acc, corr);
                } else {
                    // monopole-only offsets: only leaf partners carry mass
                    const int ay = c.cy + entry_sy(en.y), az = c.cz + entry_sz(en.y);
                    if (!((monomask >> raw_dir(plane, ay, az)) & 1u)) continue;
                    const double m0 = sm[pb];
                    if (PREC == PREC_EXACT) {
                        double mp[20];
                        mp[0] = m0;
#pragma unroll
                        for (int q = 1; q < 20; ++q) mp[q] = 0.0;
                        exact_m2l_pair<RHO>(X, Y, mp, mc, acc, corr);
                    } else {
                        fast_m2l_mass_pair<RHO>(X, Y, m0, mc + 10, inv_m0, acc, corr);
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 20; ++q) out.L[q * out.stride + cu] = acc[q];
        write_lc<RHO>(out, cu, corr);
        __syncthreads();   // shared memory and `it` are reused by the next tile
    }
}

// The RHO multipole tiles of theta < 0.5 in the fused FP32-split form
// (m2l_split_fz_kernel's arithmetic on m2l_r2_kernel's plane streaming): the
// 12 partner x-planes of a tile are staged one after the other, per (y, z)
// parity class in rows of 12 (8 cells + 4 pad, so a quarter-warp (k, two j)
// reads distinct 16-byte slots): FP32 float4 (Q0..Q3) (Q4,Q5,-O0,-O1)
// (-O2..-O5) (-O6..-O9) and FP64 double2 (Px,Py) (Pz,m0) (O0,O1) .. (O8,O9),
// everything in units of dx. Each thread serves one target cell and, for its
// pairs in the plane, builds the FP32 tensor and contraction and the FP64
// correction L_c in one instruction stream (promoted to FP64 every 16 pairs).
// Root tiles run the fast FP64 form.
constexpr int R2S_COMP = 8 * PL_RS;                 // 96 cells of one (y, z) parity class
constexpr int R2S_F_CLS = 4 * R2S_COMP;             // float4 per class
constexpr int R2S_D_CLS = 7 * R2S_COMP;             // double2 per class
constexpr int R2S_F_BYTES = 4 * R2S_F_CLS * 16;     // 24,576
constexpr int R2S_SMEM_BYTES = R2S_F_BYTES + 4 * R2S_D_CLS * 16;   // 24,576 + 43,008 = 67,584
constexpr int R2S_SMEM_ALLOC = R2S_SMEM_BYTES > ROOT_SMEM_DOUBLES * 8 ? R2S_SMEM_BYTES : ROOT_SMEM_DOUBLES * 8;
static_assert(PL_RS % 8 == 4, "rows of 12 sixteen-byte slots: quarter-warps (k, two j) conflict-free");

__global__ void __launch_bounds__(THREADS, 1) m2l_r2_split_kernel(BatchArgs a) {
    extern __shared__ __align__(16) unsigned char r2s_dyn[];
    float4* sf = reinterpret_cast<float4*>(r2s_dyn);
    double2* sb = reinterpret_cast<double2*>(r2s_dyn + R2S_F_BYTES);
    __shared__ ItemInfo it;
    __shared__ int tile;
    constexpr int RU = ROOT_UNITS_FAST;
    const int nroot = a.wl.counts[WL_ROOT], nm2l = a.wl.counts[WL_M2L];
    const int total = RU * nroot + 2 * nm2l;
    for (;;) {
        if (threadIdx.x == 0) tile = atomicAdd(a.wl.counts + WL_M2L_NEXT, 1);
        __syncthreads();
        const int t = tile;
        if (t >= total) break;
        const int item_idx = (t < RU * nroot) ? a.wl.root[t / RU] : a.wl.m2l[(t - RU * nroot) >> 1];
        load_item(a, item_idx, it);
        const int x0 = TILE_X * (t & 1);
        const size_t sub = (size_t)it.subgrid;
        OutPtr out{a.L + sub * 20 * NCELL, a.Lc + sub * 3 * NCELL, NCELL, true};
        if (it.kind == OTFMM_KIND_M2L_ROOT) {
            double* sm = reinterpret_cast<double*>(r2s_dyn);
            for (int r = threadIdx.x; r < NCELL; r += blockDim.x)
                for (int q = 0; q < NCOMP; ++q)
                    sm[q * NCELL + r] = (q < 20) ? a.M[(sub * 20 + q) * NCELL + r] * stage_scale<PREC_FAST>(q)
                                                 : a.com[(sub * 3 + (q - 20)) * NCELL + r];
            __syncthreads();
            root_unit_fast<true, THREADS / 32>(sm, t % RU, a.t, out);
            __syncthreads();   // shared memory and `it` are reused by the next tile
            continue;
        }
        const uint32_t monomask = it.leafmask;
        const CellMap c = cell_map(x0);
        const int cu = c.cx * 64 + c.cy * 8 + c.cz;
        const int lane_off = c.j * PL_RS + c.k;
        const double inv_dx = 1.0 / it.dx, inv2 = inv_dx * inv_dx, inv3 = inv2 * inv_dx;
        const double Pc0 = (a.com[(sub * 3 + 0) * NCELL + cu] - it.xbase[0]) * inv_dx;
        const double Pc1 = (a.com[(sub * 3 + 1) * NCELL + cu] - it.xbase[1]) * inv_dx;
        const double Pc2 = (a.com[(sub * 3 + 2) * NCELL + cu] - it.xbase[2]) * inv_dx;
        FzLc z;
#pragma unroll
        for (int q = 0; q < 3; ++q) z.La[q] = z.Lb[q] = 0.0;
        z.V = 0.0;
#pragma unroll
        for (int q = 0; q < 6; ++q) z.W[q] = 0.0;
        double acc[20];
        float accf[20], ext = 0.0f;
#pragma unroll
        for (int q = 0; q < 20; ++q) {
            acc[q] = 0.0;
            accf[q] = 0.0f;
        }
        int in_chunk = 0;
        const int2* ent = a.t.entries_r2s + c.p * MAX_ENTRIES_R2;
        const int* sxs = a.t.r2_sx_start + c.p * 12;
        const int* fend = a.t.r2s_far_end + c.p * 11;
        for (int plane = x0 - 4; plane <= x0 + 7; ++plane) {
            __syncthreads();   // the previous plane is consumed
            {
                // stage plane `plane`: one cell per thread, in units of dx
                const int r = threadIdx.x;
                const int ax = plane, ay = (r >> 4) - 4, az = (r & 15) - 4;
                const int raw = raw_dir(ax, ay, az);
                const int src = (raw == 13) ? it.subgrid : it.nb[raw < 13 ? raw : raw - 1];
                const int u = (ax & 7) * 64 + (ay & 7) * 8 + (az & 7);
                double m0 = 0.0, q[6], o[10], P[3];
#pragma unroll
                for (int k = 0; k < 6; ++k) q[k] = 0.0;
#pragma unroll
                for (int k = 0; k < 10; ++k) o[k] = 0.0;
                if (src < 0) {
                    // empty direction: zero moments at the cell's own centre
                    P[0] = ax;
                    P[1] = ay;
                    P[2] = az;
                } else if ((it.leafmask >> raw) & 1u) {
                    m0 = a.mon[(size_t)src * NCELL + u];
                    const int ip[3] = {ax + INX, ay + INX, az + INX};
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const double cc = __dsub_rn(__dadd_rn(__dmul_rn((double)ip[k], it.dx), it.xbase[k]),
                                                    __dmul_rn((double)INX, it.dx));
                        P[k] = (cc - it.xbase[k]) * inv_dx;
                    }
                } else {
                    const double* Ms = a.M + (size_t)src * 20 * NCELL + u;
                    m0 = Ms[0];
#pragma unroll
                    for (int k = 0; k < 6; ++k) q[k] = Ms[(4 + k) * NCELL] * ((factor_of(4 + k) / 2.0) * inv2);
#pragma unroll
                    for (int k = 0; k < 10; ++k) o[k] = Ms[(10 + k) * NCELL] * ((factor_of(10 + k) / 6.0) * inv3);
#pragma unroll
                    for (int k = 0; k < 3; ++k) P[k] = (a.com[((size_t)src * 3 + k) * NCELL + u] - it.xbase[k]) * inv_dx;
                }
                const int cls = ((ay & 1) << 1) | (az & 1);
                const int cell = ((ay + 4) >> 1) * PL_RS + ((az + 4) >> 1);
                float4* fa = sf + cls * R2S_F_CLS + cell;
                double2* da = sb + cls * R2S_D_CLS + cell;
                fa[0] = make_float4((float)q[0], (float)q[1], (float)q[2], (float)q[3]);
                fa[R2S_COMP] = make_float4((float)q[4], (float)q[5], (float)-o[0], (float)-o[1]);
                fa[2 * R2S_COMP] = make_float4((float)-o[2], (float)-o[3], (float)-o[4], (float)-o[5]);
                fa[3 * R2S_COMP] = make_float4((float)-o[6], (float)-o[7], (float)-o[8], (float)-o[9]);
                da[0] = make_double2(P[0], P[1]);
                da[R2S_COMP] = make_double2(P[2], m0);
#pragma unroll
                for (int k = 0; k < 5; ++k) da[(2 + k) * R2S_COMP] = make_double2(o[2 * k], o[2 * k + 1]);
            }
            __syncthreads();
            const int sx = plane - c.cx;
            if (sx < -SMAX || sx > SMAX) continue;
            // the plane's full-multipole partners three at a time (the L_c chains of
            // consecutive pairs interleave in La / Lb), then the monopole-only ones;
            // FP32 sums promoted to FP64 every 15 pairs
            const int eb = sxs[sx + SMAX], ef = fend[sx + SMAX], e1 = sxs[sx + SMAX + 1];
            int e = eb;
#pragma unroll 1
            for (; e + 2 < ef; e += 3) {
                const int2 na = __ldg(ent + e), nb = __ldg(ent + e + 1), nc = __ldg(ent + e + 2);
                const int ca = na.x / PL_CLS, la = na.x - ca * PL_CLS + lane_off;
                const int cb = nb.x / PL_CLS, lb = nb.x - cb * PL_CLS + lane_off;
                const int cc = nc.x / PL_CLS, lc = nc.x - cc * PL_CLS + lane_off;
                fz_far_pair<R2S_COMP>(sb + ca * R2S_D_CLS + la, sf + ca * R2S_F_CLS + la, Pc0, Pc1, Pc2, accf, &ext,
                                      z.La, z);
                fz_far_pair<R2S_COMP>(sb + cb * R2S_D_CLS + lb, sf + cb * R2S_F_CLS + lb, Pc0, Pc1, Pc2, accf, &ext,
                                      z.Lb, z);
                fz_far_pair<R2S_COMP>(sb + cc * R2S_D_CLS + lc, sf + cc * R2S_F_CLS + lc, Pc0, Pc1, Pc2, accf, &ext,
                                      z.La, z);
                in_chunk += 3;
                if (in_chunk >= 15) {
                    in_chunk = 0;
                    accf[0] += ext;
                    ext = 0.0f;
#pragma unroll
                    for (int q = 0; q < 20; ++q) {
                        acc[q] += (double)accf[q];
                        accf[q] = 0.0f;
                    }
                }
            }
#pragma unroll 1
            for (; e < e1; ++e) {
                const int2 en = __ldg(ent + e);
                // en.x addresses the FP64 plane layout of m2l_r2_kernel: class and cell
                const int cls = en.x / PL_CLS, cell = en.x - cls * PL_CLS + lane_off;
                const double2* pb = sb + cls * R2S_D_CLS + cell;
                if (e < ef) {
                    fz_far_pair<R2S_COMP>(pb, sf + cls * R2S_F_CLS + cell, Pc0, Pc1, Pc2, accf, &ext, z.La, z);
                } else {
                    // monopole-only offsets: only leaf partners carry mass
                    const int ay = c.cy + entry_sy(en.y), az = c.cz + entry_sz(en.y);
                    if (!((monomask >> raw_dir(plane, ay, az)) & 1u)) continue;
                    fz_mass_pair(pb, R2S_COMP, Pc0, Pc1, Pc2, accf, z);
                }
                if (++in_chunk >= 15) {
                    in_chunk = 0;
                    accf[0] += ext;
                    ext = 0.0f;
#pragma unroll
                    for (int q = 0; q < 20; ++q) {
                        acc[q] += (double)accf[q];
                        accf[q] = 0.0f;
                    }
                }
            }
        }
        accf[0] += ext;
#pragma unroll
        for (int q = 0; q < 20; ++q) acc[q] += (double)accf[q];
        // the target's part of L_c: O_c / m_c against the mass-weighted geometry
        const double inv_m0 = 1.0 / a.M[(sub * 20) * NCELL + cu];
        double c_oct[10];
#pragma unroll
        for (int k = 0; k < 10; ++k)
            c_oct[k] = a.M[(sub * 20 + 10 + k) * NCELL + cu] * ((factor_of(10 + k) / 6.0) * inv3) * inv_m0;
        double corr[3];
        fz_finish_lc(z, c_oct, corr);
        const double s1 = inv_dx, s2 = s1 * inv_dx, s3 = s2 * inv_dx, s4 = s3 * inv_dx;
#pragma unroll
        for (int q = 0; q < 20; ++q) out.L[q * out.stride + cu] = acc[q] * (q == 0 ? s1 : q < 4 ? s2 : q < 10 ? s3 : s4);
#pragma unroll
        for (int q = 0; q < 3; ++q) out.Lc[q * out.stride + cu] = corr[q] * s2;
        __syncthreads();   // shared memory and `it` are reused by the next tile
    }
}

// P2P of leaves: one CTA (512 threads) per leaf, grid stride. The leaf's
// 18^3 mass halo (padding 5) is staged in shared memory first, refined and
// empty neighbours as zero mass (monopole update_input,
// monopole_interaction_interface.hpp:64-143); warp w then serves parity class
// w (two cells per thread), so the warp walks one entry list and every entry's
// constants serve two pairs.
constexpr int R2_PAD = SMAX;                  // halo width
constexpr int R2_REG = INX + 2 * R2_PAD;      // 18
constexpr int R2_ROW = R2_REG + 1;            // z rows padded to 19 doubles
constexpr int R2_PLANE = R2_REG * R2_ROW;
constexpr int R2_SMEM_BYTES = R2_REG * R2_PLANE * 8;   // 49,248 bytes
template <int PREC>
__global__ void __launch_bounds__(256) p2p_r2_kernel(BatchArgs a) {
    extern __shared__ double pm[];
    __shared__ ItemInfo it;
    // warp = parity class, two cells per thread (sub-lattice x' = i and i + 2)
    const int p = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = lane >> 4, j = (lane >> 2) & 3, k = lane & 3;
    const int cy = ((p >> 1) & 1) + 2 * j, cz = (p & 1) + 2 * k;
    const int cxa = ((p >> 2) & 1) + 2 * i, cxb = cxa + 4;
    const int own_a = (cxa + R2_PAD) * R2_PLANE + (cy + R2_PAD) * R2_ROW + (cz + R2_PAD);
    constexpr int OFF_B = 4 * R2_PLANE;
    const int n = a.t.count[p];
    const int2* ent = a.t.entries_r2 + p * MAX_ENTRIES_R2;
    const double4* four = a.t.r2_four + p * MAX_ENTRIES_R2;
    const int nleaf = a.wl.counts[WL_LEAF];
    for (int kk = blockIdx.x; kk < nleaf; kk += gridDim.x) {
        __syncthreads();   // `it` and the halo are reused
        load_item(a, a.wl.leaf[kk], it);
        for (int r = threadIdx.x; r < R2_REG * R2_REG * R2_REG; r += blockDim.x) {
            const int ax = r / (R2_REG * R2_REG) - R2_PAD, ay = (r / R2_REG) % R2_REG - R2_PAD,
                      az = r % R2_REG - R2_PAD;
            const int raw = raw_dir(ax, ay, az);
            const int src = (raw == 13) ? it.subgrid : it.nb[raw < 13 ? raw : raw - 1];
            double m = 0.0;
            if (raw == 13 || ((it.leafmask >> raw) & 1u))
                m = a.mon[(size_t)src * NCELL + (ax & 7) * 64 + (ay & 7) * 8 + (az & 7)];
            pm[(ax + R2_PAD) * R2_PLANE + (ay + R2_PAD) * R2_ROW + (az + R2_PAD)] = m;
        }
        __syncthreads();
        const double dc0 = __ddiv_rn(1.0, it.dx), dc1 = __ddiv_rn(-1.0, it.dx);
        double ga[4] = {0.0, 0.0, 0.0, 0.0}, gb[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 2
        for (int e = 0; e < n; ++e) {
            const int y = __ldg(&ent[e].y);
            const double4 f = four[e];
            const int d = own_a + entry_sx(y) * R2_PLANE + entry_sy(y) * R2_ROW + entry_sz(y);
            const double ma = pm[d], mb = pm[d + OFF_B];
            if (PREC == PREC_EXACT) {
                const double sa = __dmul_rn(ma, dc0), sb = __dmul_rn(mb, dc0);
                ga[0] = __dadd_rn(ga[0], __dmul_rn(f.x, sa));
                ga[1] = __dadd_rn(ga[1], __dmul_rn(__dmul_rn(f.y, sa), dc1));
                ga[2] = __dadd_rn(ga[2], __dmul_rn(__dmul_rn(f.z, sa), dc1));
                ga[3] = __dadd_rn(ga[3], __dmul_rn(__dmul_rn(f.w, sa), dc1));
                gb[0] = __dadd_rn(gb[0], __dmul_rn(f.x, sb));
                gb[1] = __dadd_rn(gb[1], __dmul_rn(__dmul_rn(f.y, sb), dc1));
                gb[2] = __dadd_rn(gb[2], __dmul_rn(__dmul_rn(f.z, sb), dc1));
                gb[3] = __dadd_rn(gb[3], __dmul_rn(__dmul_rn(f.w, sb), dc1));
            } else {
                const double sa = ma * dc0, sb = mb * dc0;
                ga[0] = fma(f.x, sa, ga[0]);
                ga[1] = fma(f.y, sa, ga[1]);
                ga[2] = fma(f.z, sa, ga[2]);
                ga[3] = fma(f.w, sa, ga[3]);
                gb[0] = fma(f.x, sb, gb[0]);
                gb[1] = fma(f.y, sb, gb[1]);
                gb[2] = fma(f.z, sb, gb[2]);
                gb[3] = fma(f.w, sb, gb[3]);
            }
        }
        if (PREC != PREC_EXACT)
#pragma unroll
            for (int c = 1; c < 4; ++c) {
                ga[c] *= dc1;
                gb[c] *= dc1;
            }
        double* L = a.L + (size_t)it.subgrid * 20 * NCELL;
        const int cfa = cxa * 64 + cy * 8 + cz, cfb = cxb * 64 + cy * 8 + cz;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            L[c * NCELL + cfa] = ga[c];
            L[c * NCELL + cfb] = gb[c];
        }
    }
}

// P2P of leaves at theta < 0.5 in the FP32-split form: the layout and walk of
// p2p_r2_kernel with the masses staged in FP32 already divided by dx (exact for
// dx = 2^-k), the monopole constants in FP32 and the four products of a
// (partner, cell) as two packed FMAs; the FP32 sums are promoted to FP64 every
// R2_SPLIT_CHUNK partners.
constexpr int R2_SPLIT_CHUNK = 32;
// Its FP32 halo is split by parity into 9^3 sub-lattices (rows of 12, planes
// of 112 floats): the 32 lanes of a warp (one parity class, cells two apart)
// then read 32 distinct banks (the unsplit layout gave up to 4-way conflicts).
constexpr int R2F_RS = 12, R2F_XS = 112, R2F_CLS = 9 * R2F_XS;
constexpr int R2F_SMEM_BYTES = 8 * R2F_CLS * 4;   // 32,256
// Position of halo cell (rx, ry, rz) = absolute coordinates + R2_PAD, each in [0, 17].
__host__ __device__ constexpr int r2f_index(int rx, int ry, int rz) {
    return (((rx & 1) << 2) | ((ry & 1) << 1) | (rz & 1)) * R2F_CLS + (rx >> 1) * R2F_XS + (ry >> 1) * R2F_RS +
           (rz >> 1);
}
constexpr bool r2f_conflict_free() {
    bool seen[32] = {};
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 4; ++j)
            for (int k = 0; k < 4; ++k) {
                const int b = (i * R2F_XS + j * R2F_RS + k) % 32;
                if (seen[b]) return false;
                seen[b] = true;
            }
    return true;
}
static_assert(r2f_conflict_free(), "a warp's 32 cells fall in 32 distinct banks");
static_assert(8 * R2F_XS + 8 * R2F_RS + 8 < R2F_CLS, "sub-lattice planes hold 9 x 9 x 9 cells");
static_assert(8 * R2F_CLS < (1 << 21) && FULL <= 2048, "halo offset and stencil index pack into one int");
// Dynamic shared memory of the split reach-2 P2P: the halo, then the 8 parity
// classes' packed partner lists.
inline int r2f_smem_bytes(const int counts[8]) {
    int n = 0;
    for (int p = 0; p < 8; ++p) n += counts[p];
    return R2F_SMEM_BYTES + 4 * n;
}

__global__ void __launch_bounds__(256) p2p_r2_split_kernel(BatchArgs a) {
    extern __shared__ float pmf[];
    __shared__ ItemInfo it;
    const int p = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = lane >> 4, j = (lane >> 2) & 3, k = lane & 3;
    const int cy = ((p >> 1) & 1) + 2 * j, cz = (p & 1) + 2 * k;
    const int cxa = ((p >> 2) & 1) + 2 * i, cxb = cxa + 4;
    const int own_a = i * R2F_XS + j * R2F_RS + k;   // plus the entry's delta: the partner of cell cxa
    constexpr int OFF_B = 2 * R2F_XS;                // cell cxb = cxa + 4
    const int n = a.t.count[p];
    // the 8 classes' packed partner lists (halo offset << 11 | stencil index),
    // resident for the whole launch: an entry costs one broadcast shared load
    // and one uniform constant-cache read
    int* s_pk = reinterpret_cast<int*>(pmf + 8 * R2F_CLS);
    int first = 0, total = 0;
    for (int q = 0; q < 8; ++q) {
        if (q == p) first = total;
        total += a.t.count[q];
    }
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int q = 0, b = 0;
        while (t >= b + a.t.count[q]) b += a.t.count[q++];
        s_pk[t] = __ldg(a.t.r2_p2p_delta + q * MAX_ENTRIES_R2 + (t - b));
    }
    const int* pk = s_pk + first;
    const int nleaf = a.wl.counts[WL_LEAF];
    for (int kk = blockIdx.x; kk < nleaf; kk += gridDim.x) {
        __syncthreads();   // `it` and the halo are reused
        load_item(a, a.wl.leaf[kk], it);
        const double dc0 = 1.0 / it.dx;
        for (int r = threadIdx.x; r < R2_REG * R2_REG * R2_REG; r += blockDim.x) {
            const int ax = r / (R2_REG * R2_REG) - R2_PAD, ay = (r / R2_REG) % R2_REG - R2_PAD,
                      az = r % R2_REG - R2_PAD;
            const int raw = raw_dir(ax, ay, az);
            const int src = (raw == 13) ? it.subgrid : it.nb[raw < 13 ? raw : raw - 1];
            double m = 0.0;
            if (raw == 13 || ((it.leafmask >> raw) & 1u))
                m = a.mon[(size_t)src * NCELL + (ax & 7) * 64 + (ay & 7) * 8 + (az & 7)];
            pmf[r2f_index(ax + R2_PAD, ay + R2_PAD, az + R2_PAD)] = (float)(m * dc0);
        }
        __syncthreads();
        double ga[4] = {0.0, 0.0, 0.0, 0.0}, gb[4] = {0.0, 0.0, 0.0, 0.0};
        float2 a01 = make_float2(0.f, 0.f), a23 = a01, b01 = a01, b23 = a01;
        for (int e0 = 0; e0 < n; e0 += R2_SPLIT_CHUNK) {
            const int e1 = min(e0 + R2_SPLIT_CHUNK, n);
#pragma unroll 4
            for (int e = e0; e < e1; ++e) {
                const int w = pk[e];
                const float4 f = c_four_f[w & 2047];
                const int d = own_a + (w >> 11);
                const float ma = pmf[d], mb = pmf[d + OFF_B];
                a01 = __ffma2_rn(make_float2(f.x, f.y), make_float2(ma, ma), a01);
                a23 = __ffma2_rn(make_float2(f.z, f.w), make_float2(ma, ma), a23);
                b01 = __ffma2_rn(make_float2(f.x, f.y), make_float2(mb, mb), b01);
                b23 = __ffma2_rn(make_float2(f.z, f.w), make_float2(mb, mb), b23);
            }
            ga[0] += (double)a01.x;
            ga[1] += (double)a01.y;
            ga[2] += (double)a23.x;
            ga[3] += (double)a23.y;
            gb[0] += (double)b01.x;
            gb[1] += (double)b01.y;
            gb[2] += (double)b23.x;
            gb[3] += (double)b23.y;
            a01 = a23 = b01 = b23 = make_float2(0.f, 0.f);
        }
        const double dc1 = -dc0;
        double* L = a.L + (size_t)it.subgrid * 20 * NCELL;
        const int cfa = cxa * 64 + cy * 8 + cz, cfb = cxb * 64 + cy * 8 + cz;
        L[cfa] = ga[0];
        L[cfb] = gb[0];
#pragma unroll
        for (int c = 1; c < 4; ++c) {
            L[c * NCELL + cfa] = ga[c] * dc1;
            L[c * NCELL + cfb] = gb[c] * dc1;
        }
    }
}

// Per-subgrid multipole sweep on the reference's SoA buffers (two tiles of
// 4 x 8 x 8 cells): phase-one partners take mon + M0 and the higher moments,
// monopole-only partners the mass alone (kokkos_kernel.hpp:241-283).
template <int PREC, bool RHO>
__global__ void __launch_bounds__(THREADS) soa_m2l_r2_kernel(SoaArgs a) {
    const int x0 = TILE_X * blockIdx.x;
    const CellMap c = cell_map(x0);
    auto padded = [](int x, int y, int z) {
        return (x + INX - PAD_OFF) * PSTRIDE * PSTRIDE + (y + INX - PAD_OFF) * PSTRIDE + (z + INX - PAD_OFF);
    };
    const int fc = padded(c.cx, c.cy, c.cz);
    double X[3], mc[20], acc[20], corr[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int q = 0; q < 3; ++q) X[q] = a.com[q * CL + fc];
#pragma unroll
    for (int q = 0; q < 20; ++q) {
        mc[q] = a.M[q * CL + fc] * stage_scale<PREC>(q);
        acc[q] = 0.0;
    }
    const double inv_m0 = 1.0 / mc[0];
    const int n = a.t.count[c.p];
    const int2* ent = a.t.entries_r2 + c.p * MAX_ENTRIES_R2;
#pragma unroll 1
    for (int e = 0; e < n; ++e) {
        const int y = __ldg(&ent[e].y);
        const bool far = (entry_flags(y) & F_FAR) != 0;
        const int f = padded(c.cx + entry_sx(y), c.cy + entry_sy(y), c.cz + entry_sz(y));
        double Y[3], mp[20];
        if (far) {
            mp[0] = __dadd_rn(__ldg(a.mon + f), __ldg(a.M + f)) * stage_scale<PREC>(0);
#pragma unroll
            for (int q = 1; q < 20; ++q) mp[q] = __ldg(a.M + q * CL + f) * stage_scale<PREC>(q);
        } else {
            mp[0] = __ldg(a.mon + f);
            if (mp[0] == 0.0) continue;   // no mass: contributes exactly zero
#pragma unroll
            for (int q = 1; q < 20; ++q) mp[q] = 0.0;
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) Y[q] = __ldg(a.com + q * CL + f);
        if (PREC == PREC_EXACT)
            exact_m2l_pair<RHO>(X, Y, mp, mc, acc, corr);
        else
            fast_m2l_pair<RHO>(X, Y, mp, mc + 10, inv_m0, acc, corr);
    }
    OutPtr out{a.L, a.Lc, CLU, false};
    const int cf = c.cx * 64 + c.cy * 8 + c.cz;
#pragma unroll
    for (int q = 0; q < 20; ++q) out.L[q * out.stride + cf] = acc[q];
    write_lc<RHO>(out, cf, corr);
}

}   // namespace otfmm
