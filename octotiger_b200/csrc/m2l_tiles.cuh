// Multipole (M2L) tiles of refined subgrids: halo staging into shared memory,
// the FP64 exact / fast tile sweeps, the FP32-split forms (single-role and
// warp-specialised), the root tile, and the persistent batched kernels.
// Part of libotfmm.so; included once, in order, by otfmm.cu (one translation unit).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/otfmm.h"
#include "pair_math.cuh"
#include "layout.cuh"

namespace otfmm {

// ---------------------------------------------------------------- staging
// Gathers the tile region from the subgrid pool
// (restates multipole update_input, octotiger/multipole_interactions/legacy/
// multipole_interaction_interface.hpp:88-281, for full-size neighbour payloads;
// leaf tiles follow monopole update_input + update_neighbor_input,
// octotiger/monopole_interactions/legacy/monopole_interaction_interface.hpp:64-143,
// p2m_interaction_interface.hpp:102-160).
template <int PREC>
__device__ void stage_region_pool(double* sm, const ItemInfo& it, int x0, bool leaf_tile, const double* __restrict__ M,
                                  const double* __restrict__ com, const double* __restrict__ mon) {
    for (int r = threadIdx.x; r < REG_CELLS; r += blockDim.x) {
        const int rx = r / (REG_YZ * REG_YZ), ry = (r / REG_YZ) % REG_YZ, rz = r % REG_YZ;
        const int ax = x0 - 2 + rx, ay = ry - 2, az = rz - 2;
        const int raw = raw_dir(ax, ay, az);
        const bool centre = (raw == 13);
        const int src = centre ? it.subgrid : it.nb[raw < 13 ? raw : raw - 1];
        const int lx = ax & 7, ly = ay & 7, lz = az & 7;
        const int u = lx * 64 + ly * 8 + lz;
        const int base = region_addr(ax, ay, az, x0);
        double v[NCOMP];
        if (src < 0) {
#pragma unroll
            for (int q = 0; q < NCOMP; ++q) v[q] = 0.0;
        } else {
            const bool use_mon = centre ? leaf_tile : ((it.leafmask >> raw) & 1u) != 0;
            if (use_mon) {
                v[0] = mon[(size_t)src * NCELL + u];
#pragma unroll
                for (int q = 1; q < 20; ++q) v[q] = 0.0;
                if (centre) {
#pragma unroll
                    for (int a = 0; a < 3; ++a) v[20 + a] = com[((size_t)src * 3 + a) * NCELL + u];
                } else {
                    // cell centre: i*dx + xbase - INX*dx with i the padded index (:221-234)
                    const int ip[3] = {ax + INX, ay + INX, az + INX};
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                        v[20 + a] = __dsub_rn(__dadd_rn(__dmul_rn((double)ip[a], it.dx), it.xbase[a]),
                                              __dmul_rn((double)INX, it.dx));
                }
            } else {
#pragma unroll
                for (int q = 0; q < 20; ++q) v[q] = M[((size_t)src * 20 + q) * NCELL + u] * stage_scale<PREC>(q);
#pragma unroll
                for (int a = 0; a < 3; ++a) v[20 + a] = com[((size_t)src * 3 + a) * NCELL + u];
            }
        }
#pragma unroll
        for (int q = 0; q < NCOMP; ++q) sm[base + q * SUB_YZ] = v[q];
    }
}

// Same region from the reference's 18^3 SoA buffers. m0 holds mon + M0, the
// value phase-one offsets use (:270-283 of kokkos_kernel.hpp).
template <int PREC>
__device__ void stage_region_soa(double* sm, int x0, const double* __restrict__ mon, const double* __restrict__ M,
                                 const double* __restrict__ com) {
    for (int r = threadIdx.x; r < REG_CELLS; r += blockDim.x) {
        const int rx = r / (REG_YZ * REG_YZ), ry = (r / REG_YZ) % REG_YZ, rz = r % REG_YZ;
        const int ax = x0 - 2 + rx, ay = ry - 2, az = rz - 2;
        const int f = (ax + INX - PAD_OFF) * PSTRIDE * PSTRIDE + (ay + INX - PAD_OFF) * PSTRIDE + (az + INX - PAD_OFF);
        const int base = region_addr(ax, ay, az, x0);
        sm[base] = __dadd_rn(mon[f], M[f]) * stage_scale<PREC>(0);
#pragma unroll
        for (int q = 1; q < 20; ++q) sm[base + q * SUB_YZ] = M[q * CL + f] * stage_scale<PREC>(q);
#pragma unroll
        for (int a = 0; a < 3; ++a) sm[base + (20 + a) * SUB_YZ] = com[a * CL + f];
    }
}

// ---------------------------------------------------------------- compute
struct CellMap {
    int p, i, j, k, cx, cy, cz, lane_off, own;
};
__device__ __forceinline__ CellMap cell_map(int x0) {
    CellMap c;
    const int lane = threadIdx.x & 31;
    c.p = threadIdx.x >> 5;
    c.i = lane >> 4;
    c.j = (lane >> 2) & 3;
    c.k = lane & 3;
    c.cx = x0 + ((c.p >> 2) & 1) + 2 * c.i;
    c.cy = ((c.p >> 1) & 1) + 2 * c.j;
    c.cz = (c.p & 1) + 2 * c.k;
    c.lane_off = c.i * XS + c.j * RB + c.k;
    c.own = c.p * CLS + (c.i + 1) * XS + (c.j + 1) * RB + (c.k + 1);
    return c;
}

struct OutPtr {
    double* L;
    double* Lc;
    int stride;   // component stride
    bool pool;    // pool outputs: L_c is written (zeros) for DRHODT too
};

template <bool RHO>
__device__ __forceinline__ void write_lc(const OutPtr& out, int cf, const double corr[3]) {
    if (RHO || out.pool) {
#pragma unroll
        for (int a = 0; a < 3; ++a) out.Lc[a * out.stride + cf] = RHO ? corr[a] : 0.0;
    }
}

// M2L over the staged region. near_mon != nullptr: monopole-only offsets read
// the partner mass from that 18^3 buffer (SoA path); else from the region for
// leaf-neighbour partners (bit set in monomask, indexed by raw direction).
template <int PREC, bool RHO>
__device__ void m2l_tile(const double* sm, int x0, const Tables& t, uint32_t monomask, const double* near_mon,
                         OutPtr out) {
    const CellMap c = cell_map(x0);
    double X[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) X[a] = sm[c.own + (20 + a) * SUB_YZ];
    double acc[20], corr[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int q = 0; q < 20; ++q) acc[q] = 0.0;
    const int n = t.count[c.p];
    const int2* ent = t.entries + c.p * MAX_ENTRIES;
    if (PREC == PREC_EXACT) {
        double mc[20];
#pragma unroll
        for (int q = 0; q < 20; ++q) mc[q] = sm[c.own + q * SUB_YZ];
        for (int e = 0; e < n; ++e) {
            const int2 en = __ldg(ent + e);
            const int pb = en.x + c.lane_off;
            double Y[3], mp[20];
#pragma unroll
            for (int a = 0; a < 3; ++a) Y[a] = sm[pb + (20 + a) * SUB_YZ];
            if (entry_flags(en.y) & F_FAR) {
#pragma unroll
                for (int q = 0; q < 20; ++q) mp[q] = sm[pb + q * SUB_YZ];
            } else {
                const int ax = c.cx + entry_sx(en.y), ay = c.cy + entry_sy(en.y), az = c.cz + entry_sz(en.y);
                double m0;
                if (near_mon) {
                    m0 = near_mon[(ax + INX - PAD_OFF) * PSTRIDE * PSTRIDE + (ay + INX - PAD_OFF) * PSTRIDE +
                                  (az + INX - PAD_OFF)];
                } else {
                    if (!((monomask >> raw_dir(ax, ay, az)) & 1u)) continue;   // contributes exactly zero
                    m0 = sm[pb];
                }
                mp[0] = m0;
#pragma unroll
                for (int q = 1; q < 20; ++q) mp[q] = 0.0;
            }
            exact_m2l_pair<RHO>(X, Y, mp, mc, acc, corr);
        }
    } else {
        const double inv_m0 = 1.0 / sm[c.own];
        double mc_oct[10];
#pragma unroll
        for (int o = 0; o < 10; ++o) mc_oct[o] = sm[c.own + (10 + o) * SUB_YZ];
        const int nfar = t.count_far[c.p];
        const int2* entf = t.entries_fast + c.p * MAX_ENTRIES;
        // full-multipole partners: branch-free, two pairs in flight
#pragma unroll 2
        for (int e = 0; e < nfar; ++e) {
            const int pb = __ldg(&entf[e].x) + c.lane_off;
            double Y[3], mp[20];
#pragma unroll
            for (int a = 0; a < 3; ++a) Y[a] = sm[pb + (20 + a) * SUB_YZ];
#pragma unroll
            for (int q = 0; q < 20; ++q) mp[q] = sm[pb + q * SUB_YZ];
            fast_m2l_pair<RHO>(X, Y, mp, mc_oct, inv_m0, acc, corr);
        }
        // monopole-only offsets: only leaf-neighbour partners contribute
#pragma unroll 1
        for (int e = nfar; e < n; ++e) {
            const int2 en = __ldg(entf + e);
            const int pb = en.x + c.lane_off;
            const int ax = c.cx + entry_sx(en.y), ay = c.cy + entry_sy(en.y), az = c.cz + entry_sz(en.y);
            double m0;
            if (near_mon) {
                m0 = near_mon[(ax + INX - PAD_OFF) * PSTRIDE * PSTRIDE + (ay + INX - PAD_OFF) * PSTRIDE +
                              (az + INX - PAD_OFF)];
            } else {
                if (!((monomask >> raw_dir(ax, ay, az)) & 1u)) continue;
                m0 = sm[pb];
            }
            double Y[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) Y[a] = sm[pb + (20 + a) * SUB_YZ];
            fast_m2l_mass_pair<RHO>(X, Y, m0, mc_oct, inv_m0, acc, corr);
        }
    }
    const int cf = c.cx * 64 + c.cy * 8 + c.cz;
#pragma unroll
    for (int q = 0; q < 20; ++q) out.L[q * out.stride + cf] = acc[q];
    write_lc<RHO>(out, cf, corr);
}

// Split staging from the pool: same sources as stage_region_pool, values in
// units of dx (inv_dx = 1/dx), multinomial factors folded in.
__device__ void stage_region_split(double* sm, const ItemInfo& it, int x0, double inv_dx, const double* __restrict__ M,
                                   const double* __restrict__ com, const double* __restrict__ mon) {
    float* smf = reinterpret_cast<float*>(sm);
    const double inv2 = inv_dx * inv_dx, inv3 = inv2 * inv_dx;
    for (int r = threadIdx.x; r < REG_CELLS; r += blockDim.x) {
        const int rx = r / (REG_YZ * REG_YZ), ry = (r / REG_YZ) % REG_YZ, rz = r % REG_YZ;
        const int ax = x0 - 2 + rx, ay = ry - 2, az = rz - 2;
        const int raw = raw_dir(ax, ay, az);
        const bool centre = (raw == 13);
        const int src = centre ? it.subgrid : it.nb[raw < 13 ? raw : raw - 1];
        const int u = (ax & 7) * 64 + (ay & 7) * 8 + (az & 7);
        const int cls = ((ax & 1) << 2) | ((ay & 1) << 1) | (az & 1);
        const int row = cls * S_CLS + (rx >> 1) * S_XS + (ry >> 1) * S_RB;
        const int zp = rz >> 1;
        double m[20], c[3];
        if (src < 0) {
#pragma unroll
            for (int q = 0; q < 20; ++q) m[q] = 0.0;
#pragma unroll
            for (int a = 0; a < 3; ++a) c[a] = 0.0;
        } else if (!centre && ((it.leafmask >> raw) & 1u)) {
            m[0] = mon[(size_t)src * NCELL + u];
#pragma unroll
            for (int q = 1; q < 20; ++q) m[q] = 0.0;
            const int ip[3] = {ax + INX, ay + INX, az + INX};
#pragma unroll
            for (int a = 0; a < 3; ++a)
                c[a] = __dsub_rn(__dadd_rn(__dmul_rn((double)ip[a], it.dx), it.xbase[a]), __dmul_rn((double)INX, it.dx));
        } else {
#pragma unroll
            for (int q = 0; q < 20; ++q) m[q] = M[((size_t)src * 20 + q) * NCELL + u];
#pragma unroll
            for (int a = 0; a < 3; ++a) c[a] = com[((size_t)src * 3 + a) * NCELL + u];
        }
#pragma unroll
        for (int q = 1; q < 4; ++q) m[q] *= inv_dx;
#pragma unroll
        for (int q = 4; q < 10; ++q) m[q] *= (factor_of(q) / 2.0) * inv2;
#pragma unroll
        for (int q = 10; q < 20; ++q) m[q] *= (factor_of(q) / 6.0) * inv3;
#pragma unroll
        for (int a = 0; a < 3; ++a) sm[row + a * SUB_YZ + zp] = c[a] * inv_dx;
        sm[row + 3 * SUB_YZ + zp] = m[0];
#pragma unroll
        for (int o = 0; o < 10; ++o) sm[row + (4 + o) * SUB_YZ + zp] = m[10 + o];
#pragma unroll
        for (int q = 0; q < 20; ++q) smf[2 * row + S_FOFF + q * SUB_YZ + zp] = (float)m[q];
    }
}

// M2L over the split-staged region: FP32 tensor and contraction with FP64
// chunk sums, FP64 centre-of-mass differences, derivative factors and L_c.
template <bool RHO>
__device__ void m2l_tile_split(const double* sm, int x0, const Tables& t, uint32_t monomask, double inv_dx,
                               OutPtr out) {
    const float* smf = reinterpret_cast<const float*>(sm);
    const CellMap c = cell_map(x0);
    const int lane_d = c.i * S_XS + c.j * S_RB + c.k;
    const int lane_f = 2 * (c.i * S_XS + c.j * S_RB) + c.k;
    const int own = c.p * S_CLS + (c.i + 1) * S_XS + (c.j + 1) * S_RB + (c.k + 1);
    double X[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) X[a] = sm[own + a * SUB_YZ];
    const double inv_m0 = 1.0 / sm[own + 3 * SUB_YZ];
    double mc_oct[10];
#pragma unroll
    for (int o = 0; o < 10; ++o) mc_oct[o] = sm[own + (4 + o) * SUB_YZ];
    double acc[20], corr[3] = {0.0, 0.0, 0.0};
    float accf[20];
#pragma unroll
    for (int q = 0; q < 20; ++q) {
        acc[q] = 0.0;
        accf[q] = 0.0f;
    }
    const int n = t.count[c.p];
    const int nfar = t.count_far[c.p];
    const int4* ent = t.entries_split + c.p * MAX_ENTRIES;
#pragma unroll 1
    for (int e0 = 0; e0 < nfar; e0 += SPLIT_CHUNK) {
        const int e1 = min(e0 + SPLIT_CHUNK, nfar);
#pragma unroll 2
        for (int e = e0; e < e1; ++e) {
            const int4 en = __ldg(ent + e);
            const int pd = en.x + lane_d, pf = en.z + lane_f;
            double Y[3], mp_oct[10];
            float mpf[20];
#pragma unroll
            for (int a = 0; a < 3; ++a) Y[a] = sm[pd + a * SUB_YZ];
            const double m0 = sm[pd + 3 * SUB_YZ];
            if (RHO) {
#pragma unroll
                for (int o = 0; o < 10; ++o) mp_oct[o] = sm[pd + (4 + o) * SUB_YZ];
            }
#pragma unroll
            for (int q = 0; q < 20; ++q) mpf[q] = smf[pf + q * SUB_YZ];
            split_m2l_pair<RHO>(X, Y, mpf, m0, mp_oct, mc_oct, inv_m0, accf, corr);
        }
#pragma unroll
        for (int q = 0; q < 20; ++q) {
            acc[q] += (double)accf[q];
            accf[q] = 0.0f;
        }
    }
    // monopole-only offsets (leaf-neighbour partners), FP64 in dx units
#pragma unroll 1
    for (int e = nfar; e < n; ++e) {
        const int4 en = __ldg(ent + e);
        const int ax = c.cx + entry_sx(en.y), ay = c.cy + entry_sy(en.y), az = c.cz + entry_sz(en.y);
        if (!((monomask >> raw_dir(ax, ay, az)) & 1u)) continue;
        const int pd = en.x + lane_d;
        double Y[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) Y[a] = sm[pd + a * SUB_YZ];
        fast_m2l_mass_pair<RHO>(X, Y, sm[pd + 3 * SUB_YZ], mc_oct, inv_m0, acc, corr);
    }
    // back to physical units: L_(n) = L'_(n) dx^-(n+1), L_c = L_c' dx^-2
    const double s1 = inv_dx, s2 = s1 * inv_dx, s3 = s2 * inv_dx, s4 = s3 * inv_dx;
    const int cf = c.cx * 64 + c.cy * 8 + c.cz;
#pragma unroll
    for (int q = 0; q < 20; ++q) out.L[q * out.stride + cf] = acc[q] * (q == 0 ? s1 : q < 4 ? s2 : q < 10 ? s3 : s4);
#pragma unroll
    for (int a = 0; a < 3; ++a) corr[a] *= s2;
    write_lc<RHO>(out, cf, corr);
}

// ------------------------------------------------ FP32 split, warp-specialised
// RHO multipole tiles with 16 warps on one staged region. Warps 0-7
// ("contraction warps") build each pair's derivative tensor in FP32 from the
// FP64 centre-of-mass difference and contract it with the FP32 partner
// moments, promoting FP32 partial sums to FP64 every CHUNK partners; warps
// 8-15 ("correction warps") compute the angular-momentum correction L_c of
// the same pairs entirely in FP64. Warp w serves the 32 target cells of
// parity class w & 7 in either role, so the FP64 pipe (correction warps) and
// the FP32 pipe (contraction warps) work side by side on every SM.
// Shared memory per parity class (4 x 6 x 6 sub-lattice), rows of 6 z-cells:
//   FP32 part: pairs (M0,M1) .. (M18,M19) as float2, [10 pairs][6 z] = 60 float2 per row;
//   FP64 part: (Px,Py) (Pz,m0) (O0,O1) .. (O8,O9) as double2, [7][6 z] = 42 per row.
// P = (centre of mass - xbase) / dx, moments in units of dx with the multinomial
// factors folded in (exact rescaling for dx = 2^-k). Lane l of a warp serves
// sub-lattice cell (i, j, k) = ((l >> 2) & 1, l >> 3, l & 3): a half-warp
// (16 lanes: k, i, two j) reads float2 at offsets k + {0, 8, 12, 4} mod 16
// (x stride 360, row stride 60), a quarter-warp (8 lanes: k, i) reads double2
// at k + {0, 4} mod 8 (x stride 252): both without bank conflicts. The stencil
// table follows the two parts: per parity class and entry, the float2 and
// double2 partner deltas packed as 16 + 16 bits.
constexpr int WS_THREADS = 512;
constexpr int WA_ROW = 10 * SUB_YZ;            // 60 float2
constexpr int WA_XS = SUB_YZ * WA_ROW;
constexpr int WA_CLS = (REG_X / 2) * WA_XS;
constexpr int WB_ROW = 7 * SUB_YZ;             // 42 double2
constexpr int WB_XS = SUB_YZ * WB_ROW;
constexpr int WB_CLS = (REG_X / 2) * WB_XS;
constexpr int WS_A_BYTES = 8 * WA_CLS * 8;
constexpr int WS_B_BYTES = 8 * WB_CLS * 16;
constexpr int WS_TABLE_BYTES = 8 * MAX_ENTRIES * 4;
constexpr int WS_SMEM_BYTES = WS_A_BYTES + WS_B_BYTES + WS_TABLE_BYTES;   // 92160 + 129024 + 6912 = 228096
static_assert(WA_ROW % 16 == 12 && WA_XS % 16 == 8, "float2 half-warps (k, i, j pair) conflict-free");
static_assert(WB_XS % 8 == 4, "double2 quarter-warps (k, i) conflict-free");
static_assert(8 * WA_CLS < 65536 && 8 * WB_CLS < 65536, "deltas fit 16 bits");
static_assert(WS_SMEM_BYTES + 256 <= 232448, "warp-specialised layout fits the 227 KB shared-memory limit");
static_assert(ROOT_SMEM_DOUBLES * 8 <= WS_A_BYTES + WS_B_BYTES, "root staging leaves the stencil table intact");
// Smallest squared distance (in dx^2) the FP32 derivative tensor accepts; it
// keeps d3 ~ r^-7 finite in FP32. Cells of one grid have distinct centres of
// mass at least ~0.2 dx apart; the FP64 forms clamp at 1e-20 like the reference.
constexpr float WS_R2_MIN = 1.0e-6f;

// Sign of moment k in the FP32 staging of the warp-specialised tiles: the
// contraction subtracts the dipole (k = 1..3) and octupole (k = 10..19) terms,
// so their staged copies are negated and every term becomes a plain FMA.
__host__ __device__ constexpr double ws_moment_sign(int k) { return ((k >= 1 && k <= 3) || k >= 10) ? -1.0 : 1.0; }

__device__ void stage_region_ws(float2* sa, double2* sb, const ItemInfo& it, int x0, double inv_dx,
                                const double* __restrict__ M, const double* __restrict__ com,
                                const double* __restrict__ mon) {
    const double inv2 = inv_dx * inv_dx, inv3 = inv2 * inv_dx;
    for (int r = threadIdx.x; r < REG_CELLS; r += blockDim.x) {
        const int rx = r / (REG_YZ * REG_YZ), ry = (r / REG_YZ) % REG_YZ, rz = r % REG_YZ;
        const int ax = x0 - 2 + rx, ay = ry - 2, az = rz - 2;
        const int raw = raw_dir(ax, ay, az);
        const bool centre = (raw == 13);
        const int src = centre ? it.subgrid : it.nb[raw < 13 ? raw : raw - 1];
        const int u = (ax & 7) * 64 + (ay & 7) * 8 + (az & 7);
        double m[20], P[3];
        if (src < 0) {
            // empty direction: zero moments at the cell's own centre (never at a
            // target's centre of mass, so the pair stays finite)
#pragma unroll
            for (int q = 0; q < 20; ++q) m[q] = 0.0;
            P[0] = ax;
            P[1] = ay;
            P[2] = az;
        } else if (!centre && ((it.leafmask >> raw) & 1u)) {
            m[0] = mon[(size_t)src * NCELL + u];
#pragma unroll
            for (int q = 1; q < 20; ++q) m[q] = 0.0;
            // leaf cell centre i*dx + xbase - INX*dx (monopole_interaction_interface.hpp:221-234)
            const int ip[3] = {ax + INX, ay + INX, az + INX};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const double c = __dsub_rn(__dadd_rn(__dmul_rn((double)ip[a], it.dx), it.xbase[a]),
                                           __dmul_rn((double)INX, it.dx));
                P[a] = (c - it.xbase[a]) * inv_dx;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 20; ++q) m[q] = M[((size_t)src * 20 + q) * NCELL + u];
#pragma unroll
            for (int a = 0; a < 3; ++a) P[a] = (com[((size_t)src * 3 + a) * NCELL + u] - it.xbase[a]) * inv_dx;
        }
#pragma unroll
        for (int q = 1; q < 4; ++q) m[q] *= inv_dx;
#pragma unroll
        for (int q = 4; q < 10; ++q) m[q] *= (factor_of(q) / 2.0) * inv2;
#pragma unroll
        for (int q = 10; q < 20; ++q) m[q] *= (factor_of(q) / 6.0) * inv3;
        const int cls = ((ax & 1) << 2) | ((ay & 1) << 1) | (az & 1);
        const int ua = cls * WA_CLS + (rx >> 1) * WA_XS + (ry >> 1) * WA_ROW + (rz >> 1);
        const int ub = cls * WB_CLS + (rx >> 1) * WB_XS + (ry >> 1) * WB_ROW + (rz >> 1);
        // the FP32 copy carries the sign of the terms: dipoles and octupoles negated
#pragma unroll
        for (int q = 0; q < 10; ++q)
            sa[ua + q * SUB_YZ] = make_float2((float)(ws_moment_sign(2 * q) * m[2 * q]),
                                              (float)(ws_moment_sign(2 * q + 1) * m[2 * q + 1]));
        sb[ub] = make_double2(P[0], P[1]);
        sb[ub + SUB_YZ] = make_double2(P[2], m[0]);
#pragma unroll
        for (int o = 0; o < 5; ++o) sb[ub + (2 + o) * SUB_YZ] = make_double2(m[10 + 2 * o], m[11 + 2 * o]);
    }
}

// FP32 derivative tensor and contraction of one pair (dX in units of dx).
// 1/r: hardware estimate plus one Newton step with an FMA residual
// (within about one FP32 ulp). m holds the staged moments, dipoles and
// octupoles negated (ws_moment_sign), so every term is an FMA. The terms of
// fast_low_terms / fast_high_terms in another order: L0 is the dot product of
// all moments with the tensor, 10 packed FMAs (__ffma2_rn) on the pairs
// (m_2k, m_2k+1) and (D_2k, D_2k+1) that sit side by side in registers anyway,
// with its second partial sum in *ext; the monopole part of L2..L19 likewise
// on the pairs (acc_2k, acc_2k+1); the rest are scalar FMAs.
template <bool DIPOLE>
__device__ __forceinline__ void ws_contract_pair(const float dX[3], const float m[20], float acc[20], float* ext) {
    const float r2 = fmaxf(fmaf(dX[0], dX[0], fmaf(dX[1], dX[1], dX[2] * dX[2])), WS_R2_MIN);
    const float y0 = rsqrtf(r2);
    const float h = fmaf(-r2 * y0, y0, 1.0f);
    const float rs = fmaf(0.5f * y0, h, y0);
    const float r2inv = rs * rs;
    const float d1 = rs * r2inv;
    const float d2 = -3.0f * d1 * r2inv;
    const float d3 = -5.0f * d2 * r2inv;
    float D[20];
    d_tensor<float>(dX, -rs, d1, d2, d3, D);
    float2 a0 = make_float2(acc[0], *ext);
    if (DIPOLE) {
        a0 = __ffma2_rn(make_float2(m[0], m[1]), make_float2(D[0], D[1]), a0);
        a0 = __ffma2_rn(make_float2(m[2], m[3]), make_float2(D[2], D[3]), a0);
    } else {
        a0.x = fmaf(m[0], D[0], a0.x);
    }
#pragma unroll
    for (int k = 2; k < 10; ++k) a0 = __ffma2_rn(make_float2(m[2 * k], m[2 * k + 1]), make_float2(D[2 * k], D[2 * k + 1]), a0);
    acc[0] = a0.x;
    *ext = a0.y;
    acc[1] = fmaf(m[0], D[1], acc[1]);
    const float2 m00 = make_float2(m[0], m[0]);
#pragma unroll
    for (int k = 1; k < 10; ++k) {
        const float2 r = __ffma2_rn(make_float2(D[2 * k], D[2 * k + 1]), m00, make_float2(acc[2 * k], acc[2 * k + 1]));
        acc[2 * k] = r.x;
        acc[2 * k + 1] = r.y;
    }
    if (DIPOLE) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) acc[1 + a] = fmaf(m[1 + a], D[quad_row(a, b)], acc[1 + a]);
    }
#pragma unroll
    for (int q = 0; q < 6; ++q)
#pragma unroll
        for (int a = 0; a < 3; ++a) acc[1 + a] = fmaf(m[4 + q], D[quad_axis(q, a)], acc[1 + a]);
#pragma unroll
    for (int q = 0; q < 6; ++q)
#pragma unroll
        for (int a = 0; a < 3; ++a) acc[4 + q] = fmaf(m[1 + a], D[quad_axis(q, a)], acc[4 + q]);
}

// Same contraction with packed FP32 FMAs (two products per instruction; on
// sm_100 these co-issue with the FP64 pipe far better than scalar FMAs).
// Accumulator pairs: A[k] = (L_2k, L_2k+1) for k = 0..9; A[10] = L0 quadrupole
// part, A[11] = L0 octupole part, A[12..14] = L1..L3 quadrupole
// parts, each as two partial sums. The derivative tensor is used as its
// natural pairs (D_2k, D_2k+1) plus the five pairs the quadrupole/dipole terms
// of L2, L3 and L4..L9 need: (D11,D13) (D14,D16) (D17,D18) (D12,D14) (D15,D17).
constexpr int WS_PACKED_ACC = 15;
__device__ __forceinline__ void ws_contract_pair_packed(const float dX[3], const float2 mm[10],
                                                        float2 A[WS_PACKED_ACC]) {
    const float r2 = fmaxf(fmaf(dX[0], dX[0], fmaf(dX[1], dX[1], dX[2] * dX[2])), WS_R2_MIN);
    const float y0 = rsqrtf(r2);
    const float h = fmaf(-r2 * y0, y0, 1.0f);
    const float rs = fmaf(0.5f * y0, h, y0);
    const float r2inv = rs * rs;
    const float d1 = rs * r2inv;
    const float d2 = -3.0f * d1 * r2inv;
    const float d3 = -5.0f * d2 * r2inv;
    float D[20];
    d_tensor<float>(dX, -rs, d1, d2, d3, D);
    float2 P[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) P[k] = make_float2(D[2 * k], D[2 * k + 1]);
    const float2 Q1 = make_float2(D[11], D[13]), Q2 = make_float2(D[14], D[16]), Q3 = make_float2(D[17], D[18]);
    const float2 R1 = make_float2(D[12], D[14]), R2 = make_float2(D[15], D[17]);
    const float2 b0 = make_float2(mm[0].x, mm[0].x);
    // staged dipoles carry their minus sign (ws_moment_sign)
    const float2 n1 = make_float2(mm[0].y, mm[0].y), n2 = make_float2(mm[1].x, mm[1].x),
                 n3 = make_float2(mm[1].y, mm[1].y);
    // monopole: L0..L19 += M0 D0..D19
#pragma unroll
    for (int k = 0; k < 10; ++k) A[k] = __ffma2_rn(b0, P[k], A[k]);
    // dipole part of L4..L9: -= M_(1+a) D[quad_axis(q, a)]
    A[2] = __ffma2_rn(n1, P[5], A[2]);
    A[3] = __ffma2_rn(n1, P[6], A[3]);
    A[4] = __ffma2_rn(n1, P[7], A[4]);
    A[2] = __ffma2_rn(n2, Q1, A[2]);
    A[3] = __ffma2_rn(n2, Q2, A[3]);
    A[4] = __ffma2_rn(n2, Q3, A[4]);
    A[2] = __ffma2_rn(n3, R1, A[2]);
    A[3] = __ffma2_rn(n3, R2, A[3]);
    A[4] = __ffma2_rn(n3, P[9], A[4]);
    // quadrupole part of L0 and L1..L3
#pragma unroll
    for (int q = 0; q < 3; ++q) A[10] = __ffma2_rn(mm[2 + q], P[2 + q], A[10]);
    A[12] = __ffma2_rn(mm[2], P[5], A[12]);
    A[12] = __ffma2_rn(mm[3], P[6], A[12]);
    A[12] = __ffma2_rn(mm[4], P[7], A[12]);
    A[13] = __ffma2_rn(mm[2], Q1, A[13]);
    A[13] = __ffma2_rn(mm[3], Q2, A[13]);
    A[13] = __ffma2_rn(mm[4], Q3, A[13]);
    A[14] = __ffma2_rn(mm[2], R1, A[14]);
    A[14] = __ffma2_rn(mm[3], R2, A[14]);
    A[14] = __ffma2_rn(mm[4], P[9], A[14]);
    // octupole part of L0 (staged octupoles carry their minus sign)
#pragma unroll
    for (int o = 0; o < 5; ++o) A[11] = __ffma2_rn(mm[5 + o], P[5 + o], A[11]);
}

// Folds the packed accumulators into the FP64 sums of L0..L19 and clears them.
__device__ __forceinline__ void ws_fold_packed(float2 A[WS_PACKED_ACC], double acc[20]) {
    acc[0] += (double)((A[0].x + (A[10].x + A[10].y)) + (A[11].x + A[11].y));
    acc[1] += (double)(A[0].y + (A[12].x + A[12].y));
    acc[2] += (double)(A[1].x + (A[13].x + A[13].y));
    acc[3] += (double)(A[1].y + (A[14].x + A[14].y));
#pragma unroll
    for (int k = 2; k < 10; ++k) {
        acc[2 * k] += (double)A[k].x;
        acc[2 * k + 1] += (double)A[k].y;
    }
#pragma unroll
    for (int k = 0; k < WS_PACKED_ACC; ++k) A[k] = make_float2(0.0f, 0.0f);
}

// Partner with mass only (monopole-only entries, leaf-neighbour partners).
__device__ __forceinline__ void ws_contract_mass(const float dX[3], float m0, float acc[20]) {
    const float r2 = fmaxf(fmaf(dX[0], dX[0], fmaf(dX[1], dX[1], dX[2] * dX[2])), WS_R2_MIN);
    const float y0 = rsqrtf(r2);
    const float h = fmaf(-r2 * y0, y0, 1.0f);
    const float rs = fmaf(0.5f * y0, h, y0);
    const float r2inv = rs * rs;
    const float d1 = rs * r2inv;
    const float d2 = -3.0f * d1 * r2inv;
    const float d3 = -5.0f * d2 * r2inv;
    float D[20];
    d_tensor<float>(dX, -rs, d1, d2, d3, D);
#pragma unroll
    for (int q = 0; q < 20; ++q) acc[q] = fmaf(m0, D[q], acc[q]);
}

// FP64 angular-momentum correction of one pair: g = O_p - O_c m_p / m_c
// against the fourth-order slice (compute_kernel_templates.hpp:232-334).
__device__ __forceinline__ void ws_correction_pair(const double dX[3], double m0p, const double op[10],
                                                   const double mc_oct[10], double inv_m0, double Lc[3]) {
    FastDerivs f;
    f.X00 = dX[0] * dX[0];
    f.X11 = dX[1] * dX[1];
    f.X22 = dX[2] * dX[2];
    f.X01 = dX[0] * dX[1];
    f.X02 = dX[0] * dX[2];
    f.X12 = dX[1] * dX[2];
    const double r2 = fmax(f.X00 + f.X11 + f.X22, 1.0e-20);
    const double y = (double)rsqrtf((float)r2);
    const double rs = y * fma(-0.5 * r2 * y, y, 1.5);   // one Newton step: ~1e-14 relative
    const double r2inv = rs * rs;
    const double d1 = rs * r2inv;
    f.d2 = -3.0 * d1 * r2inv;
    f.d3 = -5.0 * f.d2 * r2inv;
    const double n0 = m0p * inv_m0;
    double g[10];
#pragma unroll
    for (int o = 0; o < 10; ++o) g[o] = fma(-mc_oct[o], n0, op[o]);
    fast_upper_correction(f, g, Lc);
}

// Lane -> sub-lattice cell of the warp's parity class (see the layout above).
struct WsLane {
    int i, j, k;
};
__device__ __forceinline__ WsLane ws_lane() {
    const int lane = threadIdx.x & 31;
    return WsLane{(lane >> 2) & 1, lane >> 3, lane & 3};
}

// The contraction of one parity class over far entries [e_beg, e_end) of its
// list, plus the monopole-only entries when `mono`, into acc (FP64 sums of the
// FP32 chunk sums, in units of dx). DIPOLE: the partner dipole terms of L0..L3
// (the d(rho)/dt solve).
template <int CHUNK, bool PACKED, bool DIPOLE>
__device__ void ws_contraction_acc(const float2* sa, const double2* sb, const unsigned* s_ent, int x0, int p,
                                   const Tables& t, uint32_t monomask, int e_beg, int e_end, bool mono,
                                   double acc[20]) {
    const WsLane l = ws_lane();
    const int lane_a = l.i * WA_XS + l.j * WA_ROW + l.k;
    const int lane_b = l.i * WB_XS + l.j * WB_ROW + l.k;
    const int own_b = p * WB_CLS + WB_XS + WB_ROW + 1 + lane_b;
    const double2 o0 = sb[own_b], o1 = sb[own_b + SUB_YZ];
    const double Pc0 = o0.x, Pc1 = o0.y, Pc2 = o1.x;
    float accf[20], ext = 0.0f;
#pragma unroll
    for (int q = 0; q < 20; ++q) {
        acc[q] = 0.0;
        accf[q] = 0.0f;
    }
    const int n = t.count[p], nfar = t.count_far[p];
    const unsigned* ent = s_ent + p * MAX_ENTRIES;
    if (PACKED) {
        float2 A[WS_PACKED_ACC];
#pragma unroll
        for (int k = 0; k < WS_PACKED_ACC; ++k) A[k] = make_float2(0.0f, 0.0f);
#pragma unroll 1
        for (int e0 = e_beg; e0 < e_end; e0 += CHUNK) {
            const int e1 = min(e0 + CHUNK, e_end);
#pragma unroll 2
            for (int e = e0; e < e1; ++e) {
                const unsigned en = ent[e];
                const double2* pb = sb + (en >> 16) + lane_b;
                const double2 q0 = pb[0], q1 = pb[SUB_YZ];
                const float dX[3] = {(float)(Pc0 - q0.x), (float)(Pc1 - q0.y), (float)(Pc2 - q1.x)};
                const float2* pa = sa + (en & 0xffffu) + lane_a;
                float2 mm[10];
#pragma unroll
                for (int q = 0; q < 10; ++q) mm[q] = pa[q * SUB_YZ];
                ws_contract_pair_packed(dX, mm, A);
            }
            ws_fold_packed(A, acc);
        }
    } else {
#pragma unroll 1
        for (int e0 = e_beg; e0 < e_end; e0 += CHUNK) {
            const int e1 = min(e0 + CHUNK, e_end);
#pragma unroll 2
            for (int e = e0; e < e1; ++e) {
                const unsigned en = ent[e];
                const double2* pb = sb + (en >> 16) + lane_b;
                const double2 q0 = pb[0], q1 = pb[SUB_YZ];
                const float dX[3] = {(float)(Pc0 - q0.x), (float)(Pc1 - q0.y), (float)(Pc2 - q1.x)};
                const float2* pa = sa + (en & 0xffffu) + lane_a;
                float m[20];
#pragma unroll
                for (int q = 0; q < 10; ++q) {
                    const float2 v = pa[q * SUB_YZ];
                    m[2 * q] = v.x;
                    m[2 * q + 1] = v.y;
                }
                ws_contract_pair<DIPOLE>(dX, m, accf, &ext);
            }
            accf[0] += ext;
            ext = 0.0f;
#pragma unroll
            for (int q = 0; q < 20; ++q) {
                acc[q] += (double)accf[q];
                accf[q] = 0.0f;
            }
        }
    }
    const int cx = x0 + ((p >> 2) & 1) + 2 * l.i, cy = ((p >> 1) & 1) + 2 * l.j, cz = (p & 1) + 2 * l.k;
    if (mono && monomask) {
        // monopole-only offsets: only leaf-neighbour partners contribute
        const int4* gent = t.entries_ws + p * MAX_ENTRIES;
#pragma unroll 1
        for (int e = nfar; e < n; ++e) {
            const int4 en = __ldg(gent + e);
            const int ax = cx + entry_sx(en.z), ay = cy + entry_sy(en.z), az = cz + entry_sz(en.z);
            if (!((monomask >> raw_dir(ax, ay, az)) & 1u)) continue;
            const double2 q0 = sb[en.y + lane_b], q1 = sb[en.y + lane_b + SUB_YZ];
            const float dX[3] = {(float)(Pc0 - q0.x), (float)(Pc1 - q0.y), (float)(Pc2 - q1.x)};
            ws_contract_mass(dX, sa[en.x + lane_a].x, accf);
        }
#pragma unroll
        for (int q = 0; q < 20; ++q) acc[q] += (double)accf[q];
    }
}

// L of the warp's cells from the contraction sums: back to physical units,
// L_(n) = L'_(n) dx^-(n+1).
__device__ __forceinline__ void ws_write_l(const double acc[20], int x0, int p, double inv_dx, const OutPtr& out) {
    const WsLane l = ws_lane();
    const int cx = x0 + ((p >> 2) & 1) + 2 * l.i, cy = ((p >> 1) & 1) + 2 * l.j, cz = (p & 1) + 2 * l.k;
    const double s1 = inv_dx, s2 = s1 * inv_dx, s3 = s2 * inv_dx, s4 = s3 * inv_dx;
    const int cf = cx * 64 + cy * 8 + cz;
#pragma unroll
    for (int q = 0; q < 20; ++q) out.L[q * out.stride + cf] = acc[q] * (q == 0 ? s1 : q < 4 ? s2 : q < 10 ? s3 : s4);
}

__device__ void ws_correction_warp(const double2* sb, const unsigned* s_ent, int x0, int p, const Tables& t,
                                   uint32_t monomask, double inv_dx, const OutPtr& out) {
    const WsLane l = ws_lane();
    const int lane_b = l.i * WB_XS + l.j * WB_ROW + l.k;
    const int own_b = p * WB_CLS + WB_XS + WB_ROW + 1 + lane_b;
    const double2 o0 = sb[own_b], o1 = sb[own_b + SUB_YZ];
    const double Pc0 = o0.x, Pc1 = o0.y, Pc2 = o1.x;
    const double inv_m0 = 1.0 / o1.y;
    double mc_oct[10];
#pragma unroll
    for (int o = 0; o < 5; ++o) {
        const double2 v = sb[own_b + (2 + o) * SUB_YZ];
        mc_oct[2 * o] = v.x;
        mc_oct[2 * o + 1] = v.y;
    }
    double corr[3] = {0.0, 0.0, 0.0};
    const int n = t.count[p], nfar = t.count_far[p];
    const unsigned* ent = s_ent + p * MAX_ENTRIES;
#pragma unroll 2
    for (int e = 0; e < nfar; ++e) {
        const double2* pb = sb + (ent[e] >> 16) + lane_b;
        const double2 q0 = pb[0], q1 = pb[SUB_YZ];
        const double dX[3] = {Pc0 - q0.x, Pc1 - q0.y, Pc2 - q1.x};
        double op[10];
#pragma unroll
        for (int o = 0; o < 5; ++o) {
            const double2 v = pb[(2 + o) * SUB_YZ];
            op[2 * o] = v.x;
            op[2 * o + 1] = v.y;
        }
        ws_correction_pair(dX, q1.y, op, mc_oct, inv_m0, corr);
    }
    const int cx = x0 + ((p >> 2) & 1) + 2 * l.i, cy = ((p >> 1) & 1) + 2 * l.j, cz = (p & 1) + 2 * l.k;
    if (monomask) {
        const int4* gent = t.entries_ws + p * MAX_ENTRIES;
#pragma unroll 1
        for (int e = nfar; e < n; ++e) {
            const int4 en = __ldg(gent + e);
            const int ax = cx + entry_sx(en.z), ay = cy + entry_sy(en.z), az = cz + entry_sz(en.z);
            if (!((monomask >> raw_dir(ax, ay, az)) & 1u)) continue;
            const int pb = en.y + lane_b;
            const double2 q0 = sb[pb], q1 = sb[pb + SUB_YZ];
            const double dX[3] = {Pc0 - q0.x, Pc1 - q0.y, Pc2 - q1.x};
            double op[10];
#pragma unroll
            for (int o = 0; o < 10; ++o) op[o] = 0.0;   // leaf partners carry no octupole
            ws_correction_pair(dX, q1.y, op, mc_oct, inv_m0, corr);
        }
    }
    const double s2 = inv_dx * inv_dx;
    const int cf = cx * 64 + cy * 8 + cz;
#pragma unroll
    for (int a = 0; a < 3; ++a) out.Lc[a * out.stride + cf] = corr[a] * s2;
}

// Root node: partners are all own cells except the monopole-only stencil
// offsets and the cell itself (multipole_kernel_root_*_impl).
// Staged layout: sm[q * 512 + cell].
template <int PREC, bool RHO>
__device__ void root_tile(const double* sm, int x0, const Tables& t, OutPtr out) {
    const CellMap c = cell_map(x0);
    const int cu = c.cx * 64 + c.cy * 8 + c.cz;
    double X[3], acc[20], corr[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int a = 0; a < 3; ++a) X[a] = sm[(20 + a) * NCELL + cu];
#pragma unroll
    for (int q = 0; q < 20; ++q) acc[q] = 0.0;
    double mc[20];
#pragma unroll
    for (int q = 0; q < 20; ++q) mc[q] = sm[q * NCELL + cu];
    const double inv_m0 = 1.0 / mc[0];
    for (int pu = 0; pu < NCELL; ++pu) {
        const int sx = (pu >> 6) - c.cx, sy = ((pu >> 3) & 7) - c.cy, sz = (pu & 7) - c.cz;
        if (abs(sx) <= SMAX && abs(sy) <= SMAX && abs(sz) <= SMAX) {
            const int sidx = (sx + SMAX) * SINX * SINX + (sy + SMAX) * SINX + (sz + SMAX);
            if (!__ldg(t.phase + sidx) || (sx == 0 && sy == 0 && sz == 0)) continue;
        }
        double Y[3], mp[20];
#pragma unroll
        for (int a = 0; a < 3; ++a) Y[a] = sm[(20 + a) * NCELL + pu];
#pragma unroll
        for (int q = 0; q < 20; ++q) mp[q] = sm[q * NCELL + pu];
        if (PREC == PREC_EXACT)
            exact_m2l_pair<RHO>(X, Y, mp, mc, acc, corr);
        else
            fast_m2l_pair<RHO>(X, Y, mp, mc + 10, inv_m0, acc, corr);
    }
#pragma unroll
    for (int q = 0; q < 20; ++q) out.L[q * out.stride + cu] = acc[q];
    write_lc<RHO>(out, cu, corr);
}

// Root items in the fast forms: ROOT_UNITS_FAST units of 32 target cells, the
// partners of a cell spread over F = blockDim.x / 32 lanes (every F-th partner
// in cell order) and the F partial sums added in a fixed butterfly order, so a
// root solve spreads over 16 CTAs instead of two. The exact form keeps two
// tiles with one lane per cell (the reference's partner order).
constexpr int ROOT_UNITS_FAST = 16;
template <int PREC>
constexpr int root_units() {
    return PREC == PREC_EXACT ? 2 : ROOT_UNITS_FAST;
}

template <bool RHO, int F>
__device__ void root_unit_fast(const double* sm, int unit, const Tables& t, OutPtr out) {
    static_assert(32 % F == 0 && NCELL / ROOT_UNITS_FAST == 32, "F lanes per cell, 32 cells per unit");
    const int f = threadIdx.x % F, cu = unit * 32 + threadIdx.x / F;
    const int cx = cu >> 6, cy = (cu >> 3) & 7, cz = cu & 7;
    double X[3], acc[20], corr[3] = {0.0, 0.0, 0.0}, mc[20];
#pragma unroll
    for (int a = 0; a < 3; ++a) X[a] = sm[(20 + a) * NCELL + cu];
#pragma unroll
    for (int q = 0; q < 20; ++q) {
        acc[q] = 0.0;
        mc[q] = sm[q * NCELL + cu];
    }
    const double inv_m0 = 1.0 / mc[0];
    for (int pu = f; pu < NCELL; pu += F) {
        const int sx = (pu >> 6) - cx, sy = ((pu >> 3) & 7) - cy, sz = (pu & 7) - cz;
        if (abs(sx) <= SMAX && abs(sy) <= SMAX && abs(sz) <= SMAX) {
            const int sidx = (sx + SMAX) * SINX * SINX + (sy + SMAX) * SINX + (sz + SMAX);
            if (!__ldg(t.phase + sidx) || (sx == 0 && sy == 0 && sz == 0)) continue;
        }
        double Y[3], mp[20];
#pragma unroll
        for (int a = 0; a < 3; ++a) Y[a] = sm[(20 + a) * NCELL + pu];
#pragma unroll
        for (int q = 0; q < 20; ++q) mp[q] = sm[q * NCELL + pu];
        fast_m2l_pair<RHO>(X, Y, mp, mc + 10, inv_m0, acc, corr);
    }
#pragma unroll
    for (int o = F / 2; o > 0; o >>= 1) {
#pragma unroll
        for (int q = 0; q < 20; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
#pragma unroll
        for (int a = 0; a < 3; ++a) corr[a] += __shfl_xor_sync(0xffffffffu, corr[a], o);
    }
    if (f == 0) {
#pragma unroll
        for (int q = 0; q < 20; ++q) out.L[q * out.stride + cu] = acc[q];
        write_lc<RHO>(out, cu, corr);
    }
}

// Multipole tiles (two per refined item), persistent: one CTA per SM takes
// tiles from an atomic counter, root units (longest) first.
template <int PREC, bool RHO>
__global__ void __launch_bounds__(THREADS, 1) m2l_batch_kernel(BatchArgs a) {
    extern __shared__ double sm[];
    __shared__ ItemInfo it;
    __shared__ int tile;
    // the split form covers the multipole tiles; the root uses fast FP64
    constexpr int P64 = (PREC == PREC_SPLIT) ? PREC_FAST : PREC;
    constexpr int RU = root_units<P64>();
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
                    sm[q * NCELL + r] = (q < 20) ? a.M[(sub * 20 + q) * NCELL + r] * stage_scale<P64>(q)
                                                 : a.com[(sub * 3 + (q - 20)) * NCELL + r];
            __syncthreads();
            if (P64 == PREC_EXACT)
                root_tile<P64, RHO>(sm, x0, a.t, out);
            else
                root_unit_fast<RHO, THREADS / 32>(sm, t % RU, a.t, out);
        } else {
            // leaf neighbours, indexed by raw direction (monopole-only offsets)
            const uint32_t monomask = it.leafmask;
            if (PREC == PREC_SPLIT) {
                const double inv_dx = 1.0 / it.dx;
                stage_region_split(sm, it, x0, inv_dx, a.M, a.com, a.mon);
                __syncthreads();
                m2l_tile_split<RHO>(sm, x0, a.t, monomask, inv_dx, out);
            } else {
                stage_region_pool<P64>(sm, it, x0, false, a.M, a.com, a.mon);
                __syncthreads();
                m2l_tile<P64, RHO>(sm, x0, a.t, monomask, nullptr, out);
            }
        }
        __syncthreads();   // shared memory and `it` are reused by the next tile
    }
}

// Multipole tiles in the FP32 split precision, warp-specialised (see
// stage_region_ws); the d(rho)/dt solve, which has no L_c, gives all 16 warps
// to the contraction: persistent over the same tile counter as m2l_batch_kernel,
// 512 threads, one CTA per SM. Root items run the fast FP64 form in 16 units
// of 32 cells (16 lanes per cell).
template <int CHUNK, bool PACKED, bool RHO>
__global__ void __launch_bounds__(WS_THREADS, 1) m2l_split_ws_kernel(BatchArgs a) {
    extern __shared__ __align__(16) unsigned char ws_dyn[];
    float2* sa = reinterpret_cast<float2*>(ws_dyn);
    double2* sb = reinterpret_cast<double2*>(ws_dyn + WS_A_BYTES);
    unsigned* s_ent = reinterpret_cast<unsigned*>(ws_dyn + WS_A_BYTES + WS_B_BYTES);
    __shared__ ItemInfo it;
    __shared__ int tile;
    const int nroot = a.wl.counts[WL_ROOT], nm2l = a.wl.counts[WL_M2L];
    const int total = ROOT_UNITS_FAST * nroot + 2 * nm2l;
    const int warp = threadIdx.x >> 5;
    // far-first partner deltas of the 8 parity classes, resident for the whole launch
    for (int e = threadIdx.x; e < 8 * MAX_ENTRIES; e += blockDim.x) {
        const int4 en = a.t.entries_ws[e];
        s_ent[e] = (unsigned)en.x | ((unsigned)en.y << 16);
    }
    for (;;) {
        if (threadIdx.x == 0) tile = atomicAdd(a.wl.counts + WL_M2L_NEXT, 1);
        __syncthreads();
        const int t = tile;
        if (t >= total) break;
        const int item_idx = (t < ROOT_UNITS_FAST * nroot) ? a.wl.root[t / ROOT_UNITS_FAST]
                                                            : a.wl.m2l[(t - ROOT_UNITS_FAST * nroot) >> 1];
        load_item(a, item_idx, it);
        const int x0 = TILE_X * (t & 1);
        const size_t sub = (size_t)it.subgrid;
        OutPtr out{a.L + sub * 20 * NCELL, a.Lc + sub * 3 * NCELL, NCELL, true};
        if (it.kind == OTFMM_KIND_M2L_ROOT) {
            double* sm = reinterpret_cast<double*>(ws_dyn);
            for (int r = threadIdx.x; r < NCELL; r += blockDim.x)
                for (int q = 0; q < NCOMP; ++q)
                    sm[q * NCELL + r] = (q < 20) ? a.M[(sub * 20 + q) * NCELL + r] * stage_scale<PREC_FAST>(q)
                                                 : a.com[(sub * 3 + (q - 20)) * NCELL + r];
            __syncthreads();
            root_unit_fast<RHO, WS_THREADS / 32>(sm, t % ROOT_UNITS_FAST, a.t, out);
        } else {
            const uint32_t monomask = it.leafmask;
            const double inv_dx = 1.0 / it.dx;
            stage_region_ws(sa, sb, it, x0, inv_dx, a.M, a.com, a.mon);
            __syncthreads();
            if (RHO) {
                if (warp < 8) {
                    double acc[20];
                    ws_contraction_acc<CHUNK, PACKED, false>(sa, sb, s_ent, x0, warp, a.t, monomask, 0,
                                                             a.t.count_far[warp], true, acc);
                    ws_write_l(acc, x0, warp, inv_dx, out);
                } else {
                    ws_correction_warp(sb, s_ent, x0, warp & 7, a.t, monomask, inv_dx, out);
                }
            } else {
                // d(rho)/dt: no L_c, so all 16 warps contract, the far entries of a
                // parity class in two halves (the second with the monopole-only
                // entries), added in a fixed order through shared memory
                const int p = warp & 7, half = warp >> 3, nfar = a.t.count_far[p], mid = nfar / 2;
                double acc[20];
                ws_contraction_acc<CHUNK, false, true>(sa, sb, s_ent, x0, p, a.t, monomask, half ? mid : 0,
                                                       half ? nfar : mid, half == 1, acc);
                __syncthreads();   // the region is read; its first 40 KB take the second halves' sums
                double* part = reinterpret_cast<double*>(ws_dyn);
                const int slot = p * 32 + (threadIdx.x & 31);
                if (half) {
#pragma unroll
                    for (int q = 0; q < 20; ++q) part[q * THREADS + slot] = acc[q];
                }
                __syncthreads();
                if (!half) {
#pragma unroll
                    for (int q = 0; q < 20; ++q) acc[q] += part[q * THREADS + slot];
                    ws_write_l(acc, x0, p, inv_dx, out);
                    const WsLane l = ws_lane();
                    const int cf = (x0 + ((p >> 2) & 1) + 2 * l.i) * 64 + (((p >> 1) & 1) + 2 * l.j) * 8 +
                                   ((p & 1) + 2 * l.k);
#pragma unroll
                    for (int c = 0; c < 3; ++c) out.Lc[c * out.stride + cf] = 0.0;
                }
            }
        }
        __syncthreads();   // shared memory and `it` are reused by the next tile
    }
}


// ------------------------------------------------ FP32 split, fused (RHO)
// Every thread serves one target cell and computes, for each of its pairs,
// the FP64 geometry and angular-momentum correction L_c and the FP32
// derivative tensor and D.M contraction in one instruction stream. On sm_100
// an FP64 FMA and FP32 work issued from the same warp run side by side (the
// FP32 instructions fill the issue slots the FP64 pipe leaves), whereas warps
// that hold only FP64 work are starved by warps that hold only FP32 work; so
// both precisions share every warp here.
// Shared memory per parity class (4 x 6 x 6 sub-lattice):
//   FP32 part: float4 (Q0,Q1,Q2,Q3) (Q4,Q5,-O0,-O1) (-O2,-O3,-O4,-O5)
//     (-O6,-O7,-O8,-O9) (quadrupoles Q, octupoles O in units of dx with the
//     multinomial factors folded in, octupoles negated so that L0 is a plain
//     dot product), rows [4][6 z] = 24 float4, x stride 148 float4;
//   FP64 part: the double2 rows of the warp-specialised layout:
//     (Px,Py) (Pz,m0) (O0,O1) .. (O8,O9), P = (centre of mass - xbase) / dx.
// Lane l serves sub-lattice cell (i, j, k) = ((l >> 2) & 1, l >> 3, l & 3): a
// quarter-warp (8 lanes: k, i) reads float4 at k + 4 i and double2 at k + 4 i
// modulo 8 sixteen-byte slots (x strides 148 and 252): no bank conflicts.
constexpr int FZ_THREADS = 256;
constexpr int FZ_ROW = 4 * SUB_YZ;            // 24 float4
constexpr int FZ_XS = SUB_YZ * FZ_ROW + 4;    // 148 float4
constexpr int FZ_CLS = (REG_X / 2) * FZ_XS;   // 592 float4
constexpr int FZ_A_BYTES = 8 * FZ_CLS * 16;
constexpr int FZ_SMEM_BYTES = FZ_A_BYTES + WS_B_BYTES + WS_TABLE_BYTES;   // 75776 + 129024 + 6912 = 211712
static_assert(FZ_XS % 8 == 4 && WB_XS % 8 == 4, "quarter-warps (k, i) read distinct 16-byte slots");
static_assert(8 * FZ_CLS < 65536, "float4 deltas fit 16 bits");
static_assert(FZ_SMEM_BYTES + 256 <= 232448, "fused layout fits the 227 KB shared-memory limit");
static_assert(ROOT_SMEM_DOUBLES * 8 <= FZ_A_BYTES + WS_B_BYTES, "root staging leaves the stencil table intact");

__device__ void stage_region_fz(float4* sf, double2* sb, const ItemInfo& it, int x0, double inv_dx,
                                const double* __restrict__ M, const double* __restrict__ com,
                                const double* __restrict__ mon) {
    const double inv2 = inv_dx * inv_dx, inv3 = inv2 * inv_dx;
    for (int r = threadIdx.x; r < REG_CELLS; r += blockDim.x) {
        const int rx = r / (REG_YZ * REG_YZ), ry = (r / REG_YZ) % REG_YZ, rz = r % REG_YZ;
        const int ax = x0 - 2 + rx, ay = ry - 2, az = rz - 2;
        const int raw = raw_dir(ax, ay, az);
        const bool centre = (raw == 13);
        const int src = centre ? it.subgrid : it.nb[raw < 13 ? raw : raw - 1];
        const int u = (ax & 7) * 64 + (ay & 7) * 8 + (az & 7);
        double m0, q[6], o[10], P[3];
        if (src < 0) {
            // empty direction: zero moments at the cell's own centre (never at a
            // target's centre of mass, so the pair stays finite)
            m0 = 0.0;
#pragma unroll
            for (int k = 0; k < 6; ++k) q[k] = 0.0;
#pragma unroll
            for (int k = 0; k < 10; ++k) o[k] = 0.0;
            P[0] = ax;
            P[1] = ay;
            P[2] = az;
        } else if (!centre && ((it.leafmask >> raw) & 1u)) {
            m0 = mon[(size_t)src * NCELL + u];
#pragma unroll
            for (int k = 0; k < 6; ++k) q[k] = 0.0;
#pragma unroll
            for (int k = 0; k < 10; ++k) o[k] = 0.0;
            // leaf cell centre i*dx + xbase - INX*dx (monopole_interaction_interface.hpp:221-234)
            const int ip[3] = {ax + INX, ay + INX, az + INX};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const double c = __dsub_rn(__dadd_rn(__dmul_rn((double)ip[a], it.dx), it.xbase[a]),
                                           __dmul_rn((double)INX, it.dx));
                P[a] = (c - it.xbase[a]) * inv_dx;
            }
        } else {
            const double* Ms = M + (size_t)src * 20 * NCELL + u;
            m0 = Ms[0];
#pragma unroll
            for (int k = 0; k < 6; ++k) q[k] = Ms[(4 + k) * NCELL] * ((factor_of(4 + k) / 2.0) * inv2);
#pragma unroll
            for (int k = 0; k < 10; ++k) o[k] = Ms[(10 + k) * NCELL] * ((factor_of(10 + k) / 6.0) * inv3);
#pragma unroll
            for (int a = 0; a < 3; ++a) P[a] = (com[((size_t)src * 3 + a) * NCELL + u] - it.xbase[a]) * inv_dx;
        }
        const int cls = ((ax & 1) << 2) | ((ay & 1) << 1) | (az & 1);
        const int ua = cls * FZ_CLS + (rx >> 1) * FZ_XS + (ry >> 1) * FZ_ROW + (rz >> 1);
        const int ub = cls * WB_CLS + (rx >> 1) * WB_XS + (ry >> 1) * WB_ROW + (rz >> 1);
        sf[ua] = make_float4((float)q[0], (float)q[1], (float)q[2], (float)q[3]);
        sf[ua + SUB_YZ] = make_float4((float)q[4], (float)q[5], (float)-o[0], (float)-o[1]);
        sf[ua + 2 * SUB_YZ] = make_float4((float)-o[2], (float)-o[3], (float)-o[4], (float)-o[5]);
        sf[ua + 3 * SUB_YZ] = make_float4((float)-o[6], (float)-o[7], (float)-o[8], (float)-o[9]);
        sb[ub] = make_double2(P[0], P[1]);
        sb[ub + SUB_YZ] = make_double2(P[2], m0);
#pragma unroll
        for (int k = 0; k < 5; ++k) sb[ub + (2 + k) * SUB_YZ] = make_double2(o[2 * k], o[2 * k + 1]);
    }
}

// The FP32 half of a fused pair: derivative tensor and contraction with the
// partner's FP32 moments (RHO terms: monopole, quadrupole and octupole parts;
// the partner dipole does not enter), into the FP32 chunk sums acc (L0's
// second partial sum in *ext). 1/r comes in as rsf.
__device__ __forceinline__ void fz_contract(const float dXf[3], float rsf, float m0, const float4 f0, const float4 f1,
                                            const float4 f2, const float4 f3, float acc[20], float* ext) {
    const float r2invf = rsf * rsf;
    const float d1 = rsf * r2invf;
    const float d2 = -3.0f * d1 * r2invf;
    const float d3 = -5.0f * d2 * r2invf;
    float D[20];
    d_tensor<float>(dXf, -rsf, d1, d2, d3, D);
    // L0 = m0 D0 + sum Q_q D_(4+q) - sum O_o D_(10+o): a packed dot product
    float2 a0 = make_float2(fmaf(m0, D[0], acc[0]), *ext);
    a0 = __ffma2_rn(make_float2(f0.x, f0.y), make_float2(D[4], D[5]), a0);
    a0 = __ffma2_rn(make_float2(f0.z, f0.w), make_float2(D[6], D[7]), a0);
    a0 = __ffma2_rn(make_float2(f1.x, f1.y), make_float2(D[8], D[9]), a0);
    a0 = __ffma2_rn(make_float2(f1.z, f1.w), make_float2(D[10], D[11]), a0);
    a0 = __ffma2_rn(make_float2(f2.x, f2.y), make_float2(D[12], D[13]), a0);
    a0 = __ffma2_rn(make_float2(f2.z, f2.w), make_float2(D[14], D[15]), a0);
    a0 = __ffma2_rn(make_float2(f3.x, f3.y), make_float2(D[16], D[17]), a0);
    a0 = __ffma2_rn(make_float2(f3.z, f3.w), make_float2(D[18], D[19]), a0);
    acc[0] = a0.x;
    *ext = a0.y;
    // monopole part of L1..L19
    acc[1] = fmaf(m0, D[1], acc[1]);
    const float2 mm = make_float2(m0, m0);
#pragma unroll
    for (int k = 1; k < 10; ++k) {
        const float2 r = __ffma2_rn(make_float2(D[2 * k], D[2 * k + 1]), mm, make_float2(acc[2 * k], acc[2 * k + 1]));
        acc[2 * k] = r.x;
        acc[2 * k + 1] = r.y;
    }
    // quadrupole part of L1..L3
    const float Q[6] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y};
#pragma unroll
    for (int q = 0; q < 6; ++q)
#pragma unroll
        for (int a = 0; a < 3; ++a) acc[1 + a] = fmaf(Q[q], D[quad_axis(q, a)], acc[1 + a]);
}

// Geometry of a pair for both precisions from dX (units of dx, FP64): the FP32
// copy dXf, 1/r as an FP32 estimate refined by one FP32 Newton step (rsf,
// r^2 floored at 1e-6 dx^2 for the FP32 tensor, which no pair of distinct
// cells reaches) and by one FP64 Newton step from it (~1e-14 relative), the
// products X_ab, d2 = -3 r^-5 and d3 = 15 r^-7 in FP64. The FP32 side does not
// wait for the FP64 refinement.
__device__ __forceinline__ void fz_geometry(const double dX[3], float dXf[3], FastDerivs& f, float* rsf) {
    dXf[0] = (float)dX[0];
    dXf[1] = (float)dX[1];
    dXf[2] = (float)dX[2];
    const float r2f = fmaxf(fmaf(dXf[0], dXf[0], fmaf(dXf[1], dXf[1], dXf[2] * dXf[2])), WS_R2_MIN);
    const float y0 = rsqrtf(r2f);
    const float h = fmaf(-r2f * y0, y0, 1.0f);
    *rsf = fmaf(0.5f * y0, h, y0);
    f.X00 = dX[0] * dX[0];
    f.X11 = dX[1] * dX[1];
    f.X22 = dX[2] * dX[2];
    f.X01 = dX[0] * dX[1];
    f.X02 = dX[0] * dX[2];
    f.X12 = dX[1] * dX[2];
    // no FP64 clamp: the seed comes from the clamped FP32 r2, so the Newton
    // step stays finite at r2 = 0, and below r2 = 1e-20 a clamp would move rs
    // by less than 1e-14 of its value
    const double r2 = f.X00 + f.X11 + f.X22;
    const double y = (double)*rsf;
    const double rs = y * fma(-0.5 * r2 * y, y, 1.5);
    const double r2inv = rs * rs;
    const double m3 = -3.0 * r2inv, m5 = -5.0 * r2inv;
    const double d1 = rs * r2inv;
    f.d2 = d1 * m3;
    f.d3 = f.d2 * m5;
}

// L_c -= sum_o h_o U_o. (fourth-order slice, compute_kernel_templates.hpp:232-334)
// with each output's ten terms in two interleaved partial sums.
__device__ __forceinline__ void fz_upper(const FastDerivs& f, const double h[10], double Lc[3]) {
    const double d2 = f.d2, d3 = f.d3;
    const double e01 = d3 * f.X01, e02 = d3 * f.X02, e12 = d3 * f.X12;
    const double d3_6 = 6.0 * d3, d2_3 = 3.0 * d2;
    double U[15];
    U[0] = fma(d3_6, f.X00, d2_3);
    U[1] = 3.0 * e01;
    U[2] = 3.0 * e02;
    U[3] = fma(d3, f.X00 + f.X11, d2);
    U[4] = e12;
    U[5] = fma(d3, f.X00 + f.X22, d2);
    U[6] = U[1];
    U[7] = e02;
    U[8] = e01;
    U[9] = U[2];
    U[10] = fma(d3_6, f.X11, d2_3);
    U[11] = 3.0 * e12;
    U[12] = fma(d3, f.X11 + f.X22, d2);
    U[13] = U[11];
    U[14] = fma(d3_6, f.X22, d2_3);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        double t = Lc[j], t1 = -h[1] * U[upper_idx(1, j)];
#pragma unroll
        for (int o = 0; o < 10; o += 2) t = fma(-h[o], U[upper_idx(o, j)], t);
#pragma unroll
        for (int o = 3; o < 10; o += 2) t1 = fma(-h[o], U[upper_idx(o, j)], t1);
        Lc[j] = t + t1;
    }
}

// L_c of a cell, split as L_c = -sum_p O_p . U(d_p) + (O_c / m_c) . sum_p m_p U(d_p)
// (compute_kernel_templates.hpp:228-334 with g = O_p - O_c m_p / m_c expanded):
// per pair the partner part goes into La (even pairs) / Lb (odd pairs), and
// the mass-weighted geometry into V = sum m_p d2, W_ab = sum m_p d3 X_ab; the
// target part is formed once per cell from V, W (fz_finish_lc). Both parts are
// FP64 sums, so their difference keeps ~1e-16 of their size.
struct FzLc {
    double La[3], Lb[3], V, W[6];
};
__device__ __forceinline__ void fz_mass_geometry(const FastDerivs& f, double m0p, FzLc& z) {
    z.V = fma(m0p, f.d2, z.V);
    const double md3 = m0p * f.d3;
    z.W[0] = fma(md3, f.X00, z.W[0]);
    z.W[1] = fma(md3, f.X11, z.W[1]);
    z.W[2] = fma(md3, f.X22, z.W[2]);
    z.W[3] = fma(md3, f.X01, z.W[3]);
    z.W[4] = fma(md3, f.X02, z.W[4]);
    z.W[5] = fma(md3, f.X12, z.W[5]);
}
__device__ __forceinline__ void fz_finish_lc(const FzLc& z, const double c_oct[10], double Lc[3]) {
    // sum_p m_p U_k(d_p) is U_k with d2 -> V, d3 -> 1, X_ab -> W_ab
    FastDerivs w;
    w.d2 = z.V;
    w.d3 = 1.0;
    w.X00 = z.W[0];
    w.X11 = z.W[1];
    w.X22 = z.W[2];
    w.X01 = z.W[3];
    w.X02 = z.W[4];
    w.X12 = z.W[5];
    double neg_c[10];
#pragma unroll
    for (int o = 0; o < 10; ++o) neg_c[o] = -c_oct[o];
#pragma unroll
    for (int a = 0; a < 3; ++a) Lc[a] = z.La[a] + z.Lb[a];
    fast_upper_correction(w, neg_c, Lc);
}

// One far pair of the fused form into the FP32 sums and the L_c parts; CS is
// the component stride of the staged layout (float4 / double2 units).
template <int CS = SUB_YZ>
__device__ __forceinline__ void fz_far_pair(const double2* pb, const float4* pa, double Pc0, double Pc1, double Pc2,
                                            float accf[20], float* ext, double L[3], FzLc& z) {
    const double2 q0 = pb[0], q1 = pb[CS];
    double op[10];
#pragma unroll
    for (int o = 0; o < 5; ++o) {
        const double2 v = pb[(2 + o) * CS];
        op[2 * o] = v.x;
        op[2 * o + 1] = v.y;
    }
    const float4 f0 = pa[0], f1 = pa[CS], f2 = pa[2 * CS], f3 = pa[3 * CS];
    const double dX[3] = {Pc0 - q0.x, Pc1 - q0.y, Pc2 - q1.x};
    FastDerivs f;
    float dXf[3], rsf;
    fz_geometry(dX, dXf, f, &rsf);
    fz_upper(f, op, L);
    fz_mass_geometry(f, q1.y, z);
    fz_contract(dXf, rsf, (float)q1.y, f0, f1, f2, f3, accf, ext);
}

// A partner with mass only (a leaf neighbour's cell on a monopole-only
// offset): FP32 mass contraction and the mass-weighted L_c geometry (a leaf
// partner carries no octupole). cs = component stride of the double2 rows.
__device__ __forceinline__ void fz_mass_pair(const double2* pb, int cs, double Pc0, double Pc1, double Pc2,
                                             float accf[20], FzLc& z) {
    const double2 q0 = pb[0], q1 = pb[cs];
    const double dX[3] = {Pc0 - q0.x, Pc1 - q0.y, Pc2 - q1.x};
    FastDerivs f;
    float dXf[3], rsf;
    fz_geometry(dX, dXf, f, &rsf);
    fz_mass_geometry(f, q1.y, z);
    const float r2invf = rsf * rsf;
    const float d1 = rsf * r2invf;
    const float d2 = -3.0f * d1 * r2invf;
    const float d3 = -5.0f * d2 * r2invf;
    float D[20];
    d_tensor<float>(dXf, -rsf, d1, d2, d3, D);
    const float m0 = (float)q1.y;
#pragma unroll
    for (int q = 0; q < 20; ++q) accf[q] = fmaf(m0, D[q], accf[q]);
}

template <int CHUNK>
__device__ void fz_tile(const float4* sf, const double2* sb, const unsigned* s_ent, int x0, int p, const Tables& t,
                        uint32_t monomask, double inv_dx, const OutPtr& out) {
    const WsLane l = ws_lane();
    const int lane_b = l.i * WB_XS + l.j * WB_ROW + l.k;
    const int lane_f = l.i * FZ_XS + l.j * FZ_ROW + l.k;
    const int own_b = p * WB_CLS + WB_XS + WB_ROW + 1 + lane_b;
    const double2 o0 = sb[own_b], o1 = sb[own_b + SUB_YZ];
    const double Pc0 = o0.x, Pc1 = o0.y, Pc2 = o1.x;
    FzLc z;
#pragma unroll
    for (int a = 0; a < 3; ++a) z.La[a] = z.Lb[a] = 0.0;
    z.V = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) z.W[k] = 0.0;
    double acc[20];
    float accf[20], ext = 0.0f;
#pragma unroll
    for (int q = 0; q < 20; ++q) {
        acc[q] = 0.0;
        accf[q] = 0.0f;
    }
    const int n = t.count[p], nfar = t.count_far[p];
    const unsigned* ent = s_ent + p * MAX_ENTRIES;
#pragma unroll 1
    for (int e0 = 0; e0 < nfar; e0 += CHUNK) {
        const int e1 = min(e0 + CHUNK, nfar);
        int e = e0;
        // three pairs in flight (La, Lb, La: the L_c chains of consecutive pairs interleave)
#pragma unroll 1
        for (; e + 2 < e1; e += 3) {
            const unsigned ea = ent[e], eb = ent[e + 1], ec = ent[e + 2];
            fz_far_pair(sb + (ea & 0xffffu) + lane_b, sf + (ea >> 16) + lane_f, Pc0, Pc1, Pc2, accf, &ext, z.La, z);
            fz_far_pair(sb + (eb & 0xffffu) + lane_b, sf + (eb >> 16) + lane_f, Pc0, Pc1, Pc2, accf, &ext, z.Lb, z);
            fz_far_pair(sb + (ec & 0xffffu) + lane_b, sf + (ec >> 16) + lane_f, Pc0, Pc1, Pc2, accf, &ext, z.La, z);
        }
#pragma unroll 1
        for (; e + 1 < e1; e += 2) {
            const unsigned ea = ent[e], eb = ent[e + 1];
            fz_far_pair(sb + (ea & 0xffffu) + lane_b, sf + (ea >> 16) + lane_f, Pc0, Pc1, Pc2, accf, &ext, z.La, z);
            fz_far_pair(sb + (eb & 0xffffu) + lane_b, sf + (eb >> 16) + lane_f, Pc0, Pc1, Pc2, accf, &ext, z.Lb, z);
        }
        if (e < e1) {
            const unsigned ea = ent[e];
            fz_far_pair(sb + (ea & 0xffffu) + lane_b, sf + (ea >> 16) + lane_f, Pc0, Pc1, Pc2, accf, &ext, z.La, z);
        }
        accf[0] += ext;
        ext = 0.0f;
#pragma unroll
        for (int q = 0; q < 20; ++q) {
            acc[q] += (double)accf[q];
            accf[q] = 0.0f;
        }
    }
    const int cx = x0 + ((p >> 2) & 1) + 2 * l.i, cy = ((p >> 1) & 1) + 2 * l.j, cz = (p & 1) + 2 * l.k;
    if (monomask) {
        // monopole-only offsets: only leaf-neighbour partners contribute (as masses)
        const int4* gent = t.entries_ws + p * MAX_ENTRIES;
#pragma unroll 1
        for (int e = nfar; e < n; ++e) {
            const int4 en = __ldg(gent + e);
            const int ax = cx + entry_sx(en.z), ay = cy + entry_sy(en.z), az = cz + entry_sz(en.z);
            if (!((monomask >> raw_dir(ax, ay, az)) & 1u)) continue;
            fz_mass_pair(sb + en.y + lane_b, SUB_YZ, Pc0, Pc1, Pc2, accf, z);
        }
#pragma unroll
        for (int q = 0; q < 20; ++q) acc[q] += (double)accf[q];
    }
    // the target's part of L_c: O_c / m_c against the mass-weighted geometry
    const double inv_m0 = 1.0 / o1.y;
    double c_oct[10];
#pragma unroll
    for (int o = 0; o < 5; ++o) {
        const double2 v = sb[own_b + (2 + o) * SUB_YZ];
        c_oct[2 * o] = v.x * inv_m0;
        c_oct[2 * o + 1] = v.y * inv_m0;
    }
    double corr[3];
    fz_finish_lc(z, c_oct, corr);
    // back to physical units: L_(n) = L'_(n) dx^-(n+1), L_c = L_c' dx^-2
    const double s1 = inv_dx, s2 = s1 * inv_dx, s3 = s2 * inv_dx, s4 = s3 * inv_dx;
    const int cf = cx * 64 + cy * 8 + cz;
#pragma unroll
    for (int q = 0; q < 20; ++q) out.L[q * out.stride + cf] = acc[q] * (q == 0 ? s1 : q < 4 ? s2 : q < 10 ? s3 : s4);
#pragma unroll
    for (int a = 0; a < 3; ++a) out.Lc[a * out.stride + cf] = corr[a] * s2;
}

// RHO multipole tiles in the fused FP32-split form: persistent over the same
// tile counter as m2l_batch_kernel, 256 threads (one target cell each), one
// CTA per SM. Root items run the fast FP64 form in 16 units of 32 cells
// (8 lanes per cell).
template <int CHUNK>
__global__ void __launch_bounds__(FZ_THREADS, 1) m2l_split_fz_kernel(BatchArgs a) {
    extern __shared__ __align__(16) unsigned char fz_dyn[];
    float4* sf = reinterpret_cast<float4*>(fz_dyn);
    double2* sb = reinterpret_cast<double2*>(fz_dyn + FZ_A_BYTES);
    unsigned* s_ent = reinterpret_cast<unsigned*>(fz_dyn + FZ_A_BYTES + WS_B_BYTES);
    __shared__ ItemInfo it;
    __shared__ int tile;
    const int nroot = a.wl.counts[WL_ROOT], nm2l = a.wl.counts[WL_M2L];
    const int total = ROOT_UNITS_FAST * nroot + 2 * nm2l;
    const int warp = threadIdx.x >> 5;
    // far-first partner deltas of the 8 parity classes (double2 delta in the low
    // 16 bits, float4 delta in the high 16), resident for the whole launch
    for (int e = threadIdx.x; e < 8 * MAX_ENTRIES; e += blockDim.x) {
        const int4 en = a.t.entries_ws[e];
        s_ent[e] = (unsigned)en.y | ((unsigned)en.w << 16);
    }
    for (;;) {
        if (threadIdx.x == 0) tile = atomicAdd(a.wl.counts + WL_M2L_NEXT, 1);
        __syncthreads();
        const int t = tile;
        if (t >= total) break;
        const int item_idx = (t < ROOT_UNITS_FAST * nroot) ? a.wl.root[t / ROOT_UNITS_FAST]
                                                            : a.wl.m2l[(t - ROOT_UNITS_FAST * nroot) >> 1];
        load_item(a, item_idx, it);
        const int x0 = TILE_X * (t & 1);
        const size_t sub = (size_t)it.subgrid;
        OutPtr out{a.L + sub * 20 * NCELL, a.Lc + sub * 3 * NCELL, NCELL, true};
        if (it.kind == OTFMM_KIND_M2L_ROOT) {
            double* sm = reinterpret_cast<double*>(fz_dyn);
            for (int r = threadIdx.x; r < NCELL; r += blockDim.x)
                for (int q = 0; q < NCOMP; ++q)
                    sm[q * NCELL + r] = (q < 20) ? a.M[(sub * 20 + q) * NCELL + r] * stage_scale<PREC_FAST>(q)
                                                 : a.com[(sub * 3 + (q - 20)) * NCELL + r];
            __syncthreads();
            root_unit_fast<true, FZ_THREADS / 32>(sm, t % ROOT_UNITS_FAST, a.t, out);
        } else {
            const double inv_dx = 1.0 / it.dx;
            stage_region_fz(sf, sb, it, x0, inv_dx, a.M, a.com, a.mon);
            __syncthreads();
            fz_tile<CHUNK>(sf, sb, s_ent, x0, warp, a.t, it.leafmask, inv_dx, out);
        }
        __syncthreads();   // shared memory and `it` are reused by the next tile
    }
}

}   // namespace otfmm
