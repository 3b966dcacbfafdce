// B200-native FMM cell-interaction kernels for Octo-Tiger (sm_100a).
//
// Hot path: the multipole (M2L) stencil sweep of refined subgrids and the
// monopole (P2P + P2M) sweep of leaf subgrids, the work that
// node_server::compute_fmm hands to multipole_kernel_interface /
// monopole_kernel_interface (src/node_server.cpp:711-723).
//
// Design (one GPU):
//  * A work unit ("tile") is half a subgrid: 4 x 8 x 8 target cells, one
//    thread per cell, 256 threads per CTA, one CTA per SM.
//  * For theta >= 0.5 a cell's partners lie in the 6^3 fine block of its
//    parent's 3^3 coarse neighbourhood, so a tile needs the 8 x 12 x 12 cell
//    region around it. The CTA gathers that region straight from the subgrid
//    pool in HBM (own cells + 26 neighbours, on the device — no host staging)
//    into shared memory: 23 doubles per cell (mass, 19 higher moments,
//    centre of mass), 215 KB.
//  * Shared memory is split by cell parity: the 8 parity classes of the
//    region each form a 4 x 6 x 6 sub-lattice, stored as rows of
//    [23 components x 6 z] padded to 140 doubles. A warp owns the 32 target
//    cells of one parity class (2 x 4 x 4), so for every stencil offset the
//    warp reads 32 partners of one class: per half-warp 4 rows x 4 z whose
//    addresses are distinct modulo 16 double-words (140 = 12 mod 16) — no
//    bank conflicts — and every lane walks the same offset list (warp-uniform
//    control flow, offsets from a per-parity table).
//  * Offsets are visited in the reference's stencil order (x, y, z
//    lexicographic), so per-cell accumulation order equals the reference's
//    and the exact form is bit-identical to it.
//  * Leaf tiles gather the same region (masses of leaf cells, multipoles of
//    refined neighbours) and run P2P then P2M; the level-0 node runs the
//    root stencil over its 512 cells.
//  * One launch runs a whole work list (ragged mix of kinds); the hardware
//    block scheduler balances CTAs over the 148 SMs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/otfmm.h"
#include "pair_math.cuh"

namespace otfmm {

constexpr int INX = 8;
constexpr int NCELL = 512;
constexpr int SMAX = 5;
constexpr int SINX = 11;
constexpr int FULL = SINX * SINX * SINX;
constexpr int PSTRIDE = 18;
constexpr int ENTRIES = PSTRIDE * PSTRIDE * PSTRIDE;
constexpr int CL = ENTRIES + 19;   // reference input component stride
constexpr int CLU = NCELL + 19;    // reference output component stride
constexpr int PAD_OFF = 3;
constexpr double THETA_MIN = 0.34;

// Tile geometry for coarse reach 1 (theta >= 0.5).
constexpr int THREADS = 256;
constexpr int TILE_X = 4;
constexpr int REG_X = TILE_X + 4;          // region x extent, origin x0 - 2
constexpr int REG_YZ = INX + 4;            // region y, z extent, origin -2
constexpr int REG_CELLS = REG_X * REG_YZ * REG_YZ;   // 1152
constexpr int SUB_YZ = REG_YZ / 2;         // 6
constexpr int NCOMP = 23;                  // m0, M1..M19, com x/y/z
constexpr int RB = NCOMP * SUB_YZ + 2;     // 140 doubles per (x', y') row
constexpr int XS = SUB_YZ * RB;            // 840
constexpr int CLS = (REG_X / 2) * XS;      // 3360 doubles per parity class
constexpr int SMEM_DOUBLES = 8 * CLS;      // 26880 doubles = 215040 bytes
constexpr int MAX_ENTRIES = 216;           // 6^3 - 1 partners per cell at most
constexpr int ROOT_SMEM_DOUBLES = NCOMP * NCELL;
static_assert(ROOT_SMEM_DOUBLES <= SMEM_DOUBLES, "root staging fits");
static_assert(RB % 16 == 12 || RB % 16 == 4, "row stride must keep 4x4 lane blocks conflict-free");

// FP32-split layout: per cell 14 FP64 components (centre of mass / dx, mass,
// scaled octupoles for L_c) and 20 FP32 components (scaled moments). Rows of
// 6 cells: 84 doubles then 120 floats, padded to 148 doubles (= 4 mod 16:
// conflict-free 8-byte loads per half-warp); the x stride of 890 doubles
// makes the 32 lanes' 4-byte loads hit 32 distinct banks.
constexpr int S_DCOMP = 14;
constexpr int S_FCOMP = 20;
constexpr int S_RB = 148;
constexpr int S_FOFF = 2 * S_DCOMP * SUB_YZ;   // float offset of the FP32 part within a row
constexpr int S_XS = 890;
constexpr int S_CLS = (REG_X / 2) * S_XS;
constexpr int S_SMEM_DOUBLES = 8 * S_CLS;      // 28480 doubles = 227840 bytes
constexpr int SPLIT_CHUNK = 16;                // FP32 partial sums promoted to FP64 every 16 partners
static_assert(S_RB >= S_DCOMP * SUB_YZ + S_FCOMP * SUB_YZ / 2, "split row fits");
static_assert(S_RB % 16 == 4 || S_RB % 16 == 12, "split rows conflict-free for 8-byte loads");
static_assert(S_XS >= SUB_YZ * S_RB && (S_XS % 16 == 2 || S_XS % 16 == 6 || S_XS % 16 == 10 || S_XS % 16 == 14),
              "split x stride");
static_assert(S_SMEM_DOUBLES * 8 <= 232448, "split layout fits the 227 KB shared-memory limit");

// P2P layout: one leaf subgrid per CTA (512 threads, one cell each); the
// mass region -2..9 per axis split by parity into 6^3 sub-lattices with rows
// padded to 12 doubles (4x4 lane blocks conflict-free).
constexpr int P_THREADS = 512;
constexpr int P_REG = INX + 4;
constexpr int P_SUB = 6;
constexpr int P_RS = 12;
constexpr int P_XS = 80;                    // >= 6 rows of 12; = 16 mod 32 for the FP32 copy
constexpr int P_CLS = P_SUB * P_XS;
constexpr int P_SMEM_DOUBLES = 8 * P_CLS;   // 3840 elements
// Lane (i, j, k) = (l >> 4, (l >> 2) & 3, l & 3) reads element k + 12 j + 80 i:
// distinct 8-byte slots per half-warp and distinct 4-byte banks per warp.
static_assert(P_XS >= P_SUB * P_RS && P_RS % 16 == 12 && P_XS % 32 == 16, "P2P region strides");

// Monopole constants {-1/r, x/r^3, y/r^3, z/r^3} per stencil offset (they do
// not depend on theta), read warp-uniformly through the constant cache.
__constant__ double c_four[FULL][4];

// Entry flags
constexpr int F_FAR = 1;    // phase-one offset: full multipole partner
constexpr int F_NEAR = 2;   // monopole-only offset

struct Tables {
    const int2* entries;     // [8][MAX_ENTRIES]: x = smem delta, y = packed offset/flags/stencil index
    const int* count;        // [8]
    const int2* entries_fast;   // same entries, full-multipole (far) offsets first
    const int* count_far;       // [8] number of far offsets
    const int4* entries_split;  // far-first entries for the split layout: x = double delta, y = packed, z = float delta
    const int2* entries_p2p;    // stencil-order entries for the P2P layout: x = smem delta, y = stencil index
    const int4* entries_ws;     // far-first entries for the warp-specialised split layout: x = float2 delta,
                                // y = double2 delta, z = packed
    const double* four;      // [FULL][4] monopole constants
    const uint8_t* phase;    // [FULL] inner_stencil_masks (true outside the stencil)
    const int* p2m_start;    // [512][28]: per cell, start of the entries of raw direction r in p2m_list
    const uint16_t* p2m_list;   // partner cell index (in its neighbour) of every entry, grouped by direction
    const int* p2m_perm_start;  // [28]: start of raw direction r in p2m_perm
    const uint16_t* p2m_perm;   // per direction, the cells with partners there, most partners first
    const int16_t* p2m_slot;    // [27][512]: position of a cell in its direction's p2m_perm list, -1 if absent
    const double4* p2p_four;    // [8][MAX_ENTRIES]: monopole constants of entries_p2p (zeros past the count)
};

__device__ __forceinline__ int entry_sx(int y) { return (y & 15) - 8; }
__device__ __forceinline__ int entry_sy(int y) { return ((y >> 4) & 15) - 8; }
__device__ __forceinline__ int entry_sz(int y) { return ((y >> 8) & 15) - 8; }
__device__ __forceinline__ int entry_flags(int y) { return (y >> 12) & 3; }
__device__ __forceinline__ int entry_sidx(int y) { return (y >> 16) & 2047; }

// Raw direction (0..26, 13 = centre) of absolute cell coordinates a in [-8, 15].
__device__ __forceinline__ int raw_dir(int ax, int ay, int az) {
    return ((ax >> 3) + 1) + 3 * ((ay >> 3) + 1) + 9 * ((az >> 3) + 1);
}

enum : int { PREC_EXACT = OTFMM_FP64_EXACT, PREC_FAST = OTFMM_FP64, PREC_SPLIT = OTFMM_FP32_SPLIT };

// Scaling folded into staged moments by the fast form.
template <int PREC>
__device__ __forceinline__ double stage_scale(int q) {
    if (PREC == PREC_FAST) {
        if (q >= 4 && q < 10) return factor_of(q) / 2.0;
        if (q >= 10 && q < 20) return factor_of(q) / 6.0;
    }
    return 1.0;
}

__device__ __forceinline__ int region_addr(int ax, int ay, int az, int x0) {
    const int rx = ax - x0 + 2, ry = ay + 2, rz = az + 2;
    const int cls = ((ax & 1) << 2) | ((ay & 1) << 1) | (az & 1);
    return cls * CLS + (rx >> 1) * XS + (ry >> 1) * RB + (rz >> 1);
}

struct ItemInfo {
    int subgrid, kind;
    int nb[26];
    double dx, xbase[3];
};

// ---------------------------------------------------------------- staging
// Gathers the tile region from the subgrid pool
// (restates multipole update_input, octotiger/multipole_interactions/legacy/
// multipole_interaction_interface.hpp:88-281, for full-size neighbour payloads;
// leaf tiles follow monopole update_input + update_neighbor_input,
// octotiger/monopole_interactions/legacy/monopole_interaction_interface.hpp:64-143,
// p2m_interaction_interface.hpp:102-160).
template <int PREC>
__device__ void stage_region_pool(double* sm, const ItemInfo& it, int x0, bool leaf_tile, const double* __restrict__ M,
                                  const double* __restrict__ com, const double* __restrict__ mon,
                                  const uint8_t* __restrict__ is_leaf) {
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
            const bool use_mon = centre ? leaf_tile : (is_leaf[src] != 0);
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
                                   const double* __restrict__ com, const double* __restrict__ mon,
                                   const uint8_t* __restrict__ is_leaf) {
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
        } else if (!centre && is_leaf[src]) {
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

__device__ void stage_region_ws(float2* sa, double2* sb, const ItemInfo& it, int x0, double inv_dx,
                                const double* __restrict__ M, const double* __restrict__ com,
                                const double* __restrict__ mon, const uint8_t* __restrict__ is_leaf) {
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
        } else if (!centre && is_leaf[src]) {
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
#pragma unroll
        for (int q = 0; q < 10; ++q) sa[ua + q * SUB_YZ] = make_float2((float)m[2 * q], (float)m[2 * q + 1]);
        sb[ub] = make_double2(P[0], P[1]);
        sb[ub + SUB_YZ] = make_double2(P[2], m[0]);
#pragma unroll
        for (int o = 0; o < 5; ++o) sb[ub + (2 + o) * SUB_YZ] = make_double2(m[10 + 2 * o], m[11 + 2 * o]);
    }
}

// FP32 derivative tensor and contraction of one pair (dX in units of dx).
// 1/r: hardware estimate plus one Newton step with an FMA residual
// (within about one FP32 ulp).
__device__ __forceinline__ void ws_contract_pair(const float dX[3], const float m[20], float acc[20]) {
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
    fast_low_terms<float>(m, D, acc, false);
    fast_high_terms<float>(m, D, acc);
}

// Same contraction with packed FP32 FMAs (two products per instruction; on
// sm_100 these co-issue with the FP64 pipe far better than scalar FMAs).
// Accumulator pairs: A[k] = (L_2k, L_2k+1) for k = 0..9; A[10] = L0 quadrupole
// part, A[11] = L0 octupole part (subtracted), A[12..14] = L1..L3 quadrupole
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
    const float2 n1 = make_float2(-mm[0].y, -mm[0].y), n2 = make_float2(-mm[1].x, -mm[1].x),
                 n3 = make_float2(-mm[1].y, -mm[1].y);
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
    // octupole part of L0 (subtracted when the pairs are folded)
#pragma unroll
    for (int o = 0; o < 5; ++o) A[11] = __ffma2_rn(mm[5 + o], P[5 + o], A[11]);
}

// Folds the packed accumulators into the FP64 sums of L0..L19 and clears them.
__device__ __forceinline__ void ws_fold_packed(float2 A[WS_PACKED_ACC], double acc[20]) {
    acc[0] += (double)((A[0].x + (A[10].x + A[10].y)) - (A[11].x + A[11].y));
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

template <int CHUNK, bool PACKED>
__device__ void ws_contraction_warp(const float2* sa, const double2* sb, const unsigned* s_ent, int x0, int p,
                                    const Tables& t, uint32_t monomask, double inv_dx, const OutPtr& out) {
    const WsLane l = ws_lane();
    const int lane_a = l.i * WA_XS + l.j * WA_ROW + l.k;
    const int lane_b = l.i * WB_XS + l.j * WB_ROW + l.k;
    const int own_b = p * WB_CLS + WB_XS + WB_ROW + 1 + lane_b;
    const double2 o0 = sb[own_b], o1 = sb[own_b + SUB_YZ];
    const double Pc0 = o0.x, Pc1 = o0.y, Pc2 = o1.x;
    double acc[20];
    float accf[20];
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
        for (int e0 = 0; e0 < nfar; e0 += CHUNK) {
            const int e1 = min(e0 + CHUNK, nfar);
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
        for (int e0 = 0; e0 < nfar; e0 += CHUNK) {
            const int e1 = min(e0 + CHUNK, nfar);
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
                ws_contract_pair(dX, m, accf);
            }
#pragma unroll
            for (int q = 0; q < 20; ++q) {
                acc[q] += (double)accf[q];
                accf[q] = 0.0f;
            }
        }
    }
    const int cx = x0 + ((p >> 2) & 1) + 2 * l.i, cy = ((p >> 1) & 1) + 2 * l.j, cz = (p & 1) + 2 * l.k;
    if (monomask) {
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
    // back to physical units: L_(n) = L'_(n) dx^-(n+1)
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

// ---------------------------------------------------------------- kernels
// Device-side work lists, filled by classify_kernel: item indices per kind
// and the counters the persistent launches take their tiles from.
enum : int { WL_M2L = 0, WL_LEAF = 1, WL_P2M = 2, WL_M2L_NEXT = 3, WL_P2M_NEXT = 4, WL_ROOT = 5, WL_COUNTERS = 8 };
struct WorkLists {
    int* m2l;      // refined, non-root items
    int* root;     // level-0 items
    int* leaf;     // leaf items
    int* p2m;      // leaf items with a refined neighbour
    int* counts;   // WL_* counters
};

struct BatchArgs {
    const double* M;
    const double* com;
    const double* mon;
    const uint8_t* is_leaf;
    int n_sub;
    const otfmm_work_item* items;
    int n_items;
    double* L;
    double* Lc;
    Tables t;
    int* err;
    WorkLists wl;
    int p2m_lanes;   // fast-form P2M: at most this many lanes share one cell's entries (1..16, power of two)
};

__device__ __forceinline__ bool item_valid(const BatchArgs& a, const otfmm_work_item& w) {
    bool b = (w.subgrid < 0 || w.subgrid >= a.n_sub || w.kind < 0 || w.kind > 2 || !(w.dx > 0.0));
    for (int d = 0; d < 26; ++d) b |= (w.neighbors[d] < -1 || w.neighbors[d] >= a.n_sub);
    if (!b && w.kind != OTFMM_KIND_M2L_ROOT) b |= (a.is_leaf[w.subgrid] != 0) != (w.kind == OTFMM_KIND_LEAF);
    return !b;
}

// One thread per work item: validates it (a malformed item raises the error
// flag and is dropped before anything reads with its fields) and appends it
// to the list of its kind.
__global__ void classify_kernel(BatchArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_items) return;
    const otfmm_work_item& w = a.items[i];
    if (!item_valid(a, w)) {
        atomicOr(a.err, 1);
        return;
    }
    if (w.kind == OTFMM_KIND_M2L) {
        a.wl.m2l[atomicAdd(a.wl.counts + WL_M2L, 1)] = i;
    } else if (w.kind == OTFMM_KIND_M2L_ROOT) {
        a.wl.root[atomicAdd(a.wl.counts + WL_ROOT, 1)] = i;
    } else {
        a.wl.leaf[atomicAdd(a.wl.counts + WL_LEAF, 1)] = i;
        bool refined_nb = false;
        for (int d = 0; d < 26; ++d) refined_nb |= (w.neighbors[d] >= 0 && !a.is_leaf[w.neighbors[d]]);
        if (refined_nb) a.wl.p2m[atomicAdd(a.wl.counts + WL_P2M, 1)] = i;
    }
}

// Copies an item (already validated by classify_kernel) into shared memory.
__device__ __forceinline__ void load_item(const BatchArgs& a, int item_idx, ItemInfo& it) {
    if (threadIdx.x == 0) {
        const otfmm_work_item& w = a.items[item_idx];
        it.subgrid = w.subgrid;
        it.kind = w.kind;
        it.dx = w.dx;
        for (int q = 0; q < 3; ++q) it.xbase[q] = w.xbase[q];
        for (int d = 0; d < 26; ++d) it.nb[d] = w.neighbors[d];
    }
    __syncthreads();
}

// Multipole tiles (two per refined item), persistent: one CTA per SM takes
// tiles from an atomic counter, root tiles (longest) first.
template <int PREC, bool RHO>
__global__ void __launch_bounds__(THREADS, 1) m2l_batch_kernel(BatchArgs a) {
    extern __shared__ double sm[];
    __shared__ ItemInfo it;
    __shared__ int tile;
    const int nroot = a.wl.counts[WL_ROOT], nm2l = a.wl.counts[WL_M2L];
    const int total = 2 * (nroot + nm2l);
    // the split form covers the multipole tiles; the root tile uses fast FP64
    constexpr int P64 = (PREC == PREC_SPLIT) ? PREC_FAST : PREC;
    for (;;) {
        if (threadIdx.x == 0) tile = atomicAdd(a.wl.counts + WL_M2L_NEXT, 1);
        __syncthreads();
        const int t = tile;
        if (t >= total) break;
        const int item_idx = (t < 2 * nroot) ? a.wl.root[t >> 1] : a.wl.m2l[(t - 2 * nroot) >> 1];
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
            root_tile<P64, RHO>(sm, x0, a.t, out);
        } else {
            // leaf neighbours, indexed by raw direction (monopole-only offsets)
            uint32_t monomask = 0;
            for (int d = 0; d < 26; ++d) {
                const int nb = it.nb[d];
                if (nb >= 0 && a.is_leaf[nb]) monomask |= 1u << (d < 13 ? d : d + 1);
            }
            if (PREC == PREC_SPLIT) {
                const double inv_dx = 1.0 / it.dx;
                stage_region_split(sm, it, x0, inv_dx, a.M, a.com, a.mon, a.is_leaf);
                __syncthreads();
                m2l_tile_split<RHO>(sm, x0, a.t, monomask, inv_dx, out);
            } else {
                stage_region_pool<P64>(sm, it, x0, false, a.M, a.com, a.mon, a.is_leaf);
                __syncthreads();
                m2l_tile<P64, RHO>(sm, x0, a.t, monomask, nullptr, out);
            }
        }
        __syncthreads();   // shared memory and `it` are reused by the next tile
    }
}

// RHO multipole tiles in the FP32 split precision, warp-specialised (see
// stage_region_ws): persistent over the same tile counter as m2l_batch_kernel,
// 512 threads, one CTA per SM. The root tile runs the fast FP64 form on the
// first 256 threads.
template <int CHUNK, bool PACKED>
__global__ void __launch_bounds__(WS_THREADS, 1) m2l_split_ws_kernel(BatchArgs a) {
    extern __shared__ __align__(16) unsigned char ws_dyn[];
    float2* sa = reinterpret_cast<float2*>(ws_dyn);
    double2* sb = reinterpret_cast<double2*>(ws_dyn + WS_A_BYTES);
    unsigned* s_ent = reinterpret_cast<unsigned*>(ws_dyn + WS_A_BYTES + WS_B_BYTES);
    __shared__ ItemInfo it;
    __shared__ int tile;
    const int nroot = a.wl.counts[WL_ROOT], nm2l = a.wl.counts[WL_M2L];
    const int total = 2 * (nroot + nm2l);
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
        const int item_idx = (t < 2 * nroot) ? a.wl.root[t >> 1] : a.wl.m2l[(t - 2 * nroot) >> 1];
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
            if (threadIdx.x < THREADS) root_tile<PREC_FAST, true>(sm, x0, a.t, out);
        } else {
            uint32_t monomask = 0;
            for (int d = 0; d < 26; ++d) {
                const int nb = it.nb[d];
                if (nb >= 0 && a.is_leaf[nb]) monomask |= 1u << (d < 13 ? d : d + 1);
            }
            const double inv_dx = 1.0 / it.dx;
            stage_region_ws(sa, sb, it, x0, inv_dx, a.M, a.com, a.mon, a.is_leaf);
            __syncthreads();
            if (warp < 8)
                ws_contraction_warp<CHUNK, PACKED>(sa, sb, s_ent, x0, warp, a.t, monomask, inv_dx, out);
            else
                ws_correction_warp(sb, s_ent, x0, warp & 7, a.t, monomask, inv_dx, out);
        }
        __syncthreads();   // shared memory and `it` are reused by the next tile
    }
}

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

// ---------------------------------------------------------------- tree passes
// taylor<4> shift operators (octotiger/taylor.hpp:222-318) in the reference's
// operation order with explicitly rounded IEEE operations; component order of
// src/taylor.cpp:10-56 (0 monopole, 1..3 dipole, 4..9 quadrupole, 10..19 octupole).
__device__ __forceinline__ int t2(int a, int b) { return quad_row(a, b); }
__device__ __forceinline__ int t3(int a, int b, int c) {
    // sorted indices (a <= b <= c) of the symmetric octupole
    const int lo = min(a, min(b, c)), hi = max(a, max(b, c)), mid = a + b + c - lo - hi;
    return quad_axis(quad_row(lo, mid) - 4, hi);
}
// B = A >> X (operator>>=, :222-255)
__device__ void shift_up_exact(const double A[20], const double X[3], double B[20]) {
#pragma unroll
    for (int j = 0; j < 20; ++j) B[j] = A[j];
#pragma unroll
    for (int a = 0; a < 3; ++a) B[1 + a] = OT_ADD(B[1 + a], OT_MUL(A[0], X[a]));
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = a; b < 3; ++b) {
            const int k = t2(a, b);
            B[k] = OT_ADD(B[k], OT_ADD(OT_MUL(A[1 + a], X[b]), OT_MUL(X[a], A[1 + b])));
            B[k] = OT_ADD(B[k], OT_MUL(OT_MUL(A[0], X[a]), X[b]));
        }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = a; b < 3; ++b)
#pragma unroll
            for (int c = b; c < 3; ++c) {
                const int k = t3(a, b, c);
                B[k] = OT_ADD(B[k], OT_ADD(OT_ADD(OT_MUL(A[t2(a, b)], X[c]), OT_MUL(A[t2(b, c)], X[a])),
                                           OT_MUL(A[t2(c, a)], X[b])));
                B[k] = OT_ADD(B[k], OT_ADD(OT_ADD(OT_MUL(OT_MUL(A[1 + a], X[b]), X[c]),
                                                  OT_MUL(OT_MUL(A[1 + b], X[c]), X[a])),
                                           OT_MUL(OT_MUL(A[1 + c], X[a]), X[b])));
                B[k] = OT_ADD(B[k], OT_MUL(OT_MUL(OT_MUL(A[0], X[a]), X[b]), X[c]));
            }
}
// B = A << X (operator<<=, :263-318)
__device__ void shift_down_exact(const double A[20], const double X[3], double B[20]) {
    const double half = 1.0 / 2.0, sixth = 1.0 / 6.0;
#pragma unroll
    for (int j = 0; j < 20; ++j) B[j] = A[j];
#pragma unroll
    for (int a = 0; a < 3; ++a) B[0] = OT_ADD(B[0], OT_MUL(A[1 + a], X[a]));
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) B[0] = OT_ADD(B[0], OT_MUL(OT_MUL(OT_MUL(A[t2(a, b)], X[a]), X[b]), half));
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) B[1 + a] = OT_ADD(B[1 + a], OT_MUL(A[t2(a, b)], X[b]));
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                B[0] = OT_ADD(B[0], OT_MUL(OT_MUL(OT_MUL(OT_MUL(A[t3(a, b, c)], X[a]), X[b]), X[c]), sixth));
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                B[1 + a] = OT_ADD(B[1 + a], OT_MUL(OT_MUL(OT_MUL(A[t3(a, b, c)], X[b]), X[c]), half));
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = a; c < 3; ++c) B[t2(a, c)] = OT_ADD(B[t2(a, c)], OT_MUL(A[t3(a, b, c)], X[b]));
}

struct TreeArgs {
    double* M;
    double* com;
    const double* mon;
    const uint8_t* is_leaf;
    double* com1;
    int n_sub;
    const otfmm_tree_node* nodes;
    int first;   // first record of the level
    double* L;
    double* Lc;
    double* G;
    double gconst;
    int correct_am;
    int* err;
};

__device__ __forceinline__ bool tree_node_valid(const TreeArgs& a, const otfmm_tree_node& nd) {
    return nd.subgrid >= 0 && nd.subgrid < a.n_sub && nd.parent >= -1 && nd.parent < a.n_sub && nd.octant >= 0 &&
           nd.octant < 8 && nd.dx > 0.0 && (nd.parent < 0 || a.is_leaf[nd.parent] == 0);
}

// One CTA (64 threads, one per coarse cell) per node of the level.
template <bool RHO>
__global__ void __launch_bounds__(64) upward_level_kernel(TreeArgs a) {
    const otfmm_tree_node nd = a.nodes[a.first + blockIdx.x];
    if (!tree_node_valid(a, nd)) {
        if (threadIdx.x == 0) atomicOr(a.err, 2);
        return;
    }
    const size_t s = (size_t)nd.subgrid;
    const bool leaf = a.is_leaf[s] != 0;
    double* M = a.M + s * 20 * NCELL;
    double* com = a.com + s * 3 * NCELL;
    const double* mon = a.mon + s * NCELL;
    double* com1 = a.com1 + s * 3 * 64;
    if (RHO && leaf) {
        // leaf centres of mass: the cell centres x0 + i dx (grid_fmm.cpp:1659-1673)
        for (int u = threadIdx.x; u < NCELL; u += blockDim.x) {
            const int i[3] = {u >> 6, (u >> 3) & 7, u & 7};
#pragma unroll
            for (int d = 0; d < 3; ++d) com[d * NCELL + u] = OT_ADD(nd.xbase[d], OT_MUL((double)i[d], nd.dx));
        }
        __syncthreads();
    }
    const int p = threadIdx.x, ip = p >> 4, jp = (p >> 2) & 3, kp = p & 3;
    int cell[8];
#pragma unroll
    for (int ci = 0; ci < 8; ++ci)
        cell[ci] = 64 * (2 * ip + (ci & 1)) + 8 * (2 * jp + ((ci >> 1) & 1)) + (2 * kp + ((ci >> 2) & 1));
    double Y[3];
    if (RHO) {
        double mc[8];
#pragma unroll
        for (int ci = 0; ci < 8; ++ci) mc[ci] = leaf ? mon[cell[ci]] : M[cell[ci]];
        double mtot = mc[0];
#pragma unroll
        for (int ci = 1; ci < 8; ++ci) mtot = OT_ADD(mtot, mc[ci]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double sx = OT_MUL(com[d * NCELL + cell[0]], mc[0]);
#pragma unroll
            for (int ci = 1; ci < 8; ++ci) sx = OT_ADD(sx, OT_MUL(com[d * NCELL + cell[ci]], mc[ci]));
            Y[d] = __ddiv_rn(sx, mtot);
            com1[d * 64 + p] = Y[d];
        }
    } else {
#pragma unroll
        for (int d = 0; d < 3; ++d) Y[d] = com1[d * 64 + p];
    }
    double MM[20];
#pragma unroll 1
    for (int ci = 0; ci < 8; ++ci) {
        const int c = cell[ci];
        double A[20], B[20], X[3];
        if (leaf) {
            A[0] = mon[c];
#pragma unroll
            for (int j = 1; j < 20; ++j) A[j] = 0.0;
        } else {
#pragma unroll
            for (int j = 0; j < 20; ++j) A[j] = M[j * NCELL + c];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) X[d] = OT_SUB(com[d * NCELL + c], Y[d]);
        shift_up_exact(A, X, B);
#pragma unroll
        for (int j = 0; j < 20; ++j) MM[j] = (ci == 0) ? B[j] : OT_ADD(MM[j], B[j]);
    }
    if (nd.parent >= 0) {
        const size_t ps = (size_t)nd.parent;
        const int o = nd.octant;
        const int io = (ip + 4 * (o & 1)) * 64 + (jp + 4 * ((o >> 1) & 1)) * 8 + (kp + 4 * ((o >> 2) & 1));
#pragma unroll
        for (int j = 0; j < 20; ++j) a.M[(ps * 20 + j) * NCELL + io] = MM[j];
        if (RHO)
#pragma unroll
            for (int d = 0; d < 3; ++d) a.com[(ps * 3 + d) * NCELL + io] = Y[d];
    }
}

// One CTA (512 threads, one per fine cell) per node of the level.
template <bool RHO>
__global__ void __launch_bounds__(NCELL) downward_level_kernel(TreeArgs a) {
    const otfmm_tree_node nd = a.nodes[a.first + blockIdx.x];
    if (!tree_node_valid(a, nd)) {
        if (threadIdx.x == 0) atomicOr(a.err, 2);
        return;
    }
    const size_t s = (size_t)nd.subgrid;
    const int c = threadIdx.x, ic = c >> 6, jc = (c >> 3) & 7, kc = c & 7;
    const int p = 16 * (ic >> 1) + 4 * (jc >> 1) + (kc >> 1);
    double l[20], lc[3] = {0.0, 0.0, 0.0};
    if (nd.parent >= 0) {
        const size_t ps = (size_t)nd.parent;
        const int o = nd.octant;
        const int io = ((ic >> 1) + 4 * (o & 1)) * 64 + ((jc >> 1) + 4 * ((o >> 1) & 1)) * 8 + ((kc >> 1) + 4 * ((o >> 2) & 1));
#pragma unroll
        for (int j = 0; j < 20; ++j) l[j] = a.L[(ps * 20 + j) * NCELL + io];
        if (RHO)
#pragma unroll
            for (int d = 0; d < 3; ++d) lc[d] = a.Lc[(ps * 3 + d) * NCELL + io];
    } else {
#pragma unroll
        for (int j = 0; j < 20; ++j) l[j] = 0.0;
    }
    double X[3], B[20];
#pragma unroll
    for (int d = 0; d < 3; ++d) X[d] = OT_SUB(a.com[(s * 3 + d) * NCELL + c], a.com1[(s * 3 + d) * 64 + p]);
    shift_down_exact(l, X, B);
    double* L = a.L + s * 20 * NCELL;
    double* Lc = a.Lc + s * 3 * NCELL;
#pragma unroll
    for (int j = 0; j < 20; ++j) L[j * NCELL + c] = OT_ADD(L[j * NCELL + c], B[j]);
    if (RHO)
#pragma unroll
        for (int d = 0; d < 3; ++d) Lc[d * NCELL + c] = OT_ADD(Lc[d * NCELL + c], lc[d]);
    if (a.is_leaf[s]) {
        double* G = a.G + s * 4 * NCELL;
        G[c] = OT_MUL(a.gconst, L[c]);
        if (RHO) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                double g = OT_MUL(-a.gconst, L[(1 + d) * NCELL + c]);
                if (a.correct_am) g = OT_SUB(g, OT_MUL(a.gconst, Lc[d * NCELL + c]));
                G[(1 + d) * NCELL + c] = g;
            }
        }
    }
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

__global__ void zero_kernel(double* p, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = 0.0;
}

// FMA issue-rate probes: 8 independent chains per thread.
template <class T>
__global__ void fma_probe_kernel(T* out, int iters, T x, T y) {
    T a0 = threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fma(a0, x, y); a1 = fma(a1, x, y); a2 = fma(a2, x, y); a3 = fma(a3, x, y);
            a4 = fma(a4, x, y); a5 = fma(a5, x, y); a6 = fma(a6, x, y); a7 = fma(a7, x, y);
        }
    }
    const T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == (T)-12345.0) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Staging for otfmm_m2l_soa_host_noalloc: up to NOALLOC_MAX_SUBGRIDS
// subgrids' SoA inputs and outputs (1.22 MB each), resident in every device
// that loads the library until the process exits.
constexpr int NOALLOC_MAX_SUBGRIDS = 4;
constexpr size_t NOALLOC_SLOT = ENTRIES + 23 * (size_t)CL + 23 * (size_t)CLU;   // doubles per subgrid
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_MAX_SUBGRIDS * NOALLOC_SLOT];

}   // namespace otfmm

// ======================================================================== host
using namespace otfmm;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}
int cuda_fail(cudaError_t e, const char* what) {
    return fail(OTFMM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define OT_CUDA(call)                                     \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

// Stencil generators, restating multipole_interactions::calculate_stencil +
// calculate_stencil_masks (src/multipole_interactions/util/calculate_stencil.cpp:23-160)
// and the monopole ones (src/monopole_interactions/util/calculate_stencil.cpp:19-178):
// offsets j - i, over the 8 parity classes i, whose parents are not well
// separated (theta_c > theta); phase one when the cells themselves are
// (theta_f <= theta).
double recip_dist(long a0, long a1, long a2, long b0, long b1, long b2) {
    const double t = double((a0 - b0) * (a0 - b0) + (a1 - b1) * (a1 - b1) + (a2 - b2) * (a2 - b2));
    return t > 0.0 ? 1.0 / std::sqrt(t) : 1.0e10;
}

struct HostStencil {
    uint8_t mask[FULL];
    uint8_t phase[FULL];
    double four[FULL][4];
    int n_mpole = 0, n_phase_one = 0;
    int maxabs = 0;
};

void build_host_stencil(double theta, HostStencil& st) {
    std::memset(st.mask, 0, sizeof st.mask);
    std::memset(st.phase, 1, sizeof st.phase);
    std::memset(st.four, 0, sizeof st.four);
    struct E { int x, y, z; bool ph; };
    std::vector<E> sup;
    for (long i0 = 0; i0 < 2; ++i0)
        for (long i1 = 0; i1 < 2; ++i1)
            for (long i2 = 0; i2 < 2; ++i2)
                for (long j0 = i0 - INX; j0 < i0 + INX; ++j0)
                    for (long j1 = i1 - INX; j1 < i1 + INX; ++j1)
                        for (long j2 = i2 - INX; j2 < i2 + INX; ++j2) {
                            if (i0 == j0 && i1 == j1 && i2 == j2) continue;
                            const double tf = recip_dist(i0, i1, i2, j0, j1, j2);
                            const double tc = recip_dist((i0 + INX) / 2 - INX / 2, (i1 + INX) / 2 - INX / 2,
                                                         (i2 + INX) / 2 - INX / 2, (j0 + INX) / 2 - INX / 2,
                                                         (j1 + INX) / 2 - INX / 2, (j2 + INX) / 2 - INX / 2);
                            if (!(tc > theta)) continue;
                            const E e{int(j0 - i0), int(j1 - i1), int(j2 - i2), tf <= theta};
                            bool found = false;
                            for (const E& s : sup)
                                if (s.x == e.x && s.y == e.y && s.z == e.z) { found = true; break; }
                            if (!found) sup.push_back(e);
                        }
    for (const E& e : sup) st.maxabs = std::max({st.maxabs, std::abs(e.x), std::abs(e.y), std::abs(e.z)});
    if (st.maxabs > SMAX) return;
    for (const E& e : sup) {
        const int idx = (e.x + SMAX) * SINX * SINX + (e.y + SMAX) * SINX + (e.z + SMAX);
        st.mask[idx] = 1;
        if (!e.ph) st.phase[idx] = 0;
        ++st.n_mpole;
        if (e.ph) ++st.n_phase_one;
        const double x = e.x, y = e.y, z = e.z;
        const double r = std::sqrt(x * x + y * y + z * z);
        const double r3 = r * r * r;
        st.four[idx][0] = -1.0 / r;
        st.four[idx][1] = x / r3;
        st.four[idx][2] = y / r3;
        st.four[idx][3] = z / r3;
    }
}

int coarse_of(int i) { return ((i + INX) >> 1) - INX / 2; }

// Per parity class: the partner offsets in stencil (x, y, z) order that pass
// the per-cell coarse criterion dist^2 < 1/theta^2
// (kokkos_kernel.hpp:241-256), packed with their shared-memory delta. False
// when the stencil reaches further than one coarse cell (theta < 0.5).
bool build_entries(const HostStencil& st, double theta, std::vector<int2>& entries, int counts[8], int& reach) {
    const double trs = (1.0 / theta) * (1.0 / theta);
    entries.assign(8 * MAX_ENTRIES, int2{0, 0});
    reach = 0;
    for (int p = 0; p < 8; ++p) {
        const int px = (p >> 2) & 1, py = (p >> 1) & 1, pz = p & 1;
        int n = 0;
        for (int sx = -SMAX; sx <= SMAX; ++sx)
            for (int sy = -SMAX; sy <= SMAX; ++sy)
                for (int sz = -SMAX; sz <= SMAX; ++sz) {
                    const int idx = (sx + SMAX) * SINX * SINX + (sy + SMAX) * SINX + (sz + SMAX);
                    if (!st.mask[idx]) continue;
                    const int a = coarse_of(px + INX) - coarse_of(px + INX + sx);
                    const int b = coarse_of(py + INX) - coarse_of(py + INX + sy);
                    const int c = coarse_of(pz + INX) - coarse_of(pz + INX + sz);
                    if (!(double(a * a + b * b + c * c) < trs)) continue;
                    reach = std::max({reach, std::abs(a), std::abs(b), std::abs(c)});
                    if (reach > 1 || n >= MAX_ENTRIES) return false;
                    const int qx = px + 2 + sx, qy = py + 2 + sy, qz = pz + 2 + sz;   // >= 0 for reach 1
                    const int cls = (((px + sx) & 1) << 2) | (((py + sy) & 1) << 1) | ((pz + sz) & 1);
                    const int delta = cls * CLS + (qx >> 1) * XS + (qy >> 1) * RB + (qz >> 1);
                    const int flags = st.phase[idx] ? F_FAR : F_NEAR;
                    const int packed = (sx + 8) | ((sy + 8) << 4) | ((sz + 8) << 8) | (flags << 12) | (idx << 16);
                    entries[p * MAX_ENTRIES + n] = int2{delta, packed};
                    ++n;
                }
        counts[p] = n;
    }
    return true;
}

}   // namespace

struct otfmm_context {
    int device = 0;
    double theta = 0.5;
    int reach = 1;     // coarse reach of the stencil (1 for theta >= 0.5)
    HostStencil st;
    int counts[8] = {};
    int2* d_entries = nullptr;
    int* d_count = nullptr;
    int2* d_entries_fast = nullptr;
    int* d_count_far = nullptr;
    int4* d_entries_split = nullptr;
    int2* d_entries_p2p = nullptr;
    int4* d_entries_ws = nullptr;
    int* d_p2m_start = nullptr;
    uint16_t* d_p2m_list = nullptr;
    int* d_p2m_perm_start = nullptr;
    uint16_t* d_p2m_perm = nullptr;
    int16_t* d_p2m_slot = nullptr;
    int p2m_groups_max = 0;   // cells with partners summed over the 26 directions
    double4* d_p2p_four = nullptr;
    int counts_far[8] = {};
    double* d_four = nullptr;
    uint8_t* d_phase = nullptr;
    int* d_err = nullptr;
    double* d_soa_scratch = nullptr;   // host-buffer path staging
    int* d_lists = nullptr;            // batched work lists (grown on demand)
    int list_capacity = 0;
    otfmm_tuning tuning = {OTFMM_SPLIT_WARP_SPECIALISED, 16, 32, 16};
    // otfmm_batch_host: device copies of the pool, work list and outputs, a
    // pinned host copy of the reordered work list, two copy streams and events
    struct HostPath {
        int n_sub = 0, n_items = 0;
        double *M = nullptr, *com = nullptr, *mon = nullptr, *L = nullptr, *Lc = nullptr;
        uint8_t* is_leaf = nullptr;
        otfmm_work_item* items = nullptr;
        otfmm_work_item* items_pinned = nullptr;
        cudaStream_t h2d = nullptr, d2h = nullptr;
        cudaEvent_t ev[3 * 16 + 4] = {};
        bool ready = false;
        std::mutex mu;   // one host-path call at a time per context
    } hp;
    std::mutex mu;
    Tables tables() const { return Tables{d_entries,    d_count, d_entries_fast, d_count_far, d_entries_split, d_entries_p2p,
                      d_entries_ws, d_four,  d_phase,        d_p2m_start,     d_p2m_list,    d_p2m_perm_start,
                      d_p2m_perm,   d_p2m_slot,     d_p2p_four}; }
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

bool g_attr_set[8] = {};
std::mutex g_attr_mu;

template <class K>
int set_smem(K kernel, int bytes) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    return OTFMM_OK;
}

int ensure_attributes(int device) {
    std::lock_guard<std::mutex> lock(g_attr_mu);
    if (device < 0 || device >= 8) return OTFMM_OK;
    if (g_attr_set[device]) return OTFMM_OK;
    const int bytes = SMEM_DOUBLES * (int)sizeof(double);
    int rc = OTFMM_OK;
    rc = rc ? rc : set_smem(m2l_batch_kernel<PREC_EXACT, true>, bytes);
    rc = rc ? rc : set_smem(m2l_batch_kernel<PREC_EXACT, false>, bytes);
    rc = rc ? rc : set_smem(m2l_batch_kernel<PREC_FAST, true>, bytes);
    rc = rc ? rc : set_smem(m2l_batch_kernel<PREC_FAST, false>, bytes);
    rc = rc ? rc : set_smem(m2l_batch_kernel<PREC_SPLIT, true>, S_SMEM_DOUBLES * (int)sizeof(double));
    rc = rc ? rc : set_smem(m2l_batch_kernel<PREC_SPLIT, false>, S_SMEM_DOUBLES * (int)sizeof(double));
    rc = rc ? rc : set_smem(m2l_split_ws_kernel<16, false>, WS_SMEM_BYTES);
    rc = rc ? rc : set_smem(m2l_split_ws_kernel<8, false>, WS_SMEM_BYTES);
    rc = rc ? rc : set_smem(m2l_split_ws_kernel<16, true>, WS_SMEM_BYTES);
    rc = rc ? rc : set_smem(m2l_split_ws_kernel<8, true>, WS_SMEM_BYTES);
    rc = rc ? rc : set_smem(p2p_batch_kernel<PREC_EXACT>, P2P_SMEM_BYTES);
    rc = rc ? rc : set_smem(p2p_batch_kernel<PREC_FAST>, P2P_SMEM_BYTES);
    rc = rc ? rc : set_smem(p2p_leaf_kernel<double, 0>, p2_smem_bytes<double>());
    rc = rc ? rc : set_smem(p2p_leaf_kernel<float, 32>, p2_smem_bytes<float>());
    rc = rc ? rc : set_smem(p2p_leaf_kernel<float, 16>, p2_smem_bytes<float>());
    rc = rc ? rc : set_smem(p2m_fast_kernel<true>, 7 * 8 * 6 * NCELL);
    rc = rc ? rc : set_smem(p2m_fast_kernel<false>, 7 * 8 * 6 * NCELL);
    rc = rc ? rc : set_smem(soa_m2l_kernel<PREC_EXACT, true, false>, bytes);
    rc = rc ? rc : set_smem(soa_m2l_kernel<PREC_EXACT, false, false>, bytes);
    rc = rc ? rc : set_smem(soa_m2l_kernel<PREC_FAST, true, false>, bytes);
    rc = rc ? rc : set_smem(soa_m2l_kernel<PREC_FAST, false, false>, bytes);
    rc = rc ? rc : set_smem(soa_m2l_kernel<PREC_EXACT, true, true>, bytes);
    rc = rc ? rc : set_smem(soa_m2l_kernel<PREC_EXACT, false, true>, bytes);
    rc = rc ? rc : set_smem(soa_m2l_kernel<PREC_FAST, true, true>, bytes);
    rc = rc ? rc : set_smem(soa_m2l_kernel<PREC_FAST, false, true>, bytes);
    if (rc == OTFMM_OK) g_attr_set[device] = true;
    return rc;
}

int check_precision(int precision, bool batched = false) {
    if (precision == OTFMM_FP64_EXACT || precision == OTFMM_FP64) return OTFMM_OK;
    if (precision == OTFMM_FP32_SPLIT && batched) return OTFMM_OK;
    return fail(OTFMM_ERR_UNSUPPORTED, "precision not available for this entry point (FP32 split is batched only)");
}

}   // namespace

extern "C" {

const char* otfmm_last_error(void) { return g_last_error.c_str(); }

const char* otfmm_build_info(void) {
    return "otfmm sm_100a; tiles of 4x8x8 cells, 256 threads, 215040 B (FP64) / 227840 B (FP32 split) shared memory; theta >= 0.5";
}

int otfmm_create(int device, double theta, otfmm_context** out) {
    if (!out) return fail(OTFMM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!(theta >= THETA_MIN)) return fail(OTFMM_ERR_THETA, "theta below the compiled minimum 0.34");
    int ndev = 0;
    OT_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(OTFMM_ERR_INVALID, "device index out of range");
    auto* ctx = new otfmm_context();
    ctx->device = device;
    ctx->theta = theta;
    build_host_stencil(theta, ctx->st);
    if (ctx->st.maxabs > SMAX) {
        delete ctx;
        return fail(OTFMM_ERR_THETA, "stencil exceeds the compiled maximum width");
    }
    // Per-parity offset lists in stencil order, filtered by the coarse criterion.
    std::vector<int2> entries;
    int reach = 0;
    if (!build_entries(ctx->st, theta, entries, ctx->counts, reach)) {
        delete ctx;
        return fail(OTFMM_ERR_UNSUPPORTED, "theta < 0.5 (coarse reach 2) is not built into this library");
    }
    ctx->reach = reach;
    // P2P-layout table (stencil order)
    std::vector<int2> entries_p2p(8 * MAX_ENTRIES, int2{0, 0});
    std::vector<double4> p2p_four(8 * MAX_ENTRIES, double4{0.0, 0.0, 0.0, 0.0});
    for (int p = 0; p < 8; ++p)
        for (int e = 0; e < ctx->counts[p]; ++e) {
            const int2 en = entries[p * MAX_ENTRIES + e];
            const int sx = (en.y & 15) - 8, sy = ((en.y >> 4) & 15) - 8, sz = ((en.y >> 8) & 15) - 8;
            const int px = (p >> 2) & 1, py = (p >> 1) & 1, pz = p & 1;
            const int cls = (((px + sx) & 1) << 2) | (((py + sy) & 1) << 1) | ((pz + sz) & 1);
            const int delta = cls * P_CLS + ((px + sx + 2) >> 1) * P_XS + ((py + sy + 2) >> 1) * P_RS + ((pz + sz + 2) >> 1);
            entries_p2p[p * MAX_ENTRIES + e] = int2{delta, (en.y >> 16) & 2047};
            const double* f = ctx->st.four[(en.y >> 16) & 2047];
            p2p_four[p * MAX_ENTRIES + e] = double4{f[0], f[1], f[2], f[3]};
        }
    // split-layout table (far first, like the fast one)
    std::vector<int4> entries_split(8 * MAX_ENTRIES, int4{0, 0, 0, 0});
    std::vector<int4> entries_ws(8 * MAX_ENTRIES, int4{0, 0, 0, 0});
    // fast-form table: far offsets first (accumulation order is free there)
    std::vector<int2> entries_fast(entries.size(), int2{0, 0});
    for (int p = 0; p < 8; ++p) {
        int k = 0;
        for (int pass = 0; pass < 2; ++pass)
            for (int e = 0; e < ctx->counts[p]; ++e) {
                const int2 en = entries[p * MAX_ENTRIES + e];
                const bool far = ((en.y >> 12) & 3) == F_FAR;
                if (far == (pass == 0)) {
                    const int sx = (en.y & 15) - 8, sy = ((en.y >> 4) & 15) - 8, sz = ((en.y >> 8) & 15) - 8;
                    const int px = (p >> 2) & 1, py = (p >> 1) & 1, pz = p & 1;
                    const int qx = px + 2 + sx, qy = py + 2 + sy, qz = pz + 2 + sz;
                    const int cls = (((px + sx) & 1) << 2) | (((py + sy) & 1) << 1) | ((pz + sz) & 1);
                    const int row = cls * S_CLS + (qx >> 1) * S_XS + (qy >> 1) * S_RB;
                    entries_split[p * MAX_ENTRIES + k] = int4{row + (qz >> 1), en.y, 2 * row + S_FOFF + (qz >> 1), 0};
                    entries_ws[p * MAX_ENTRIES + k] =
                        int4{cls * WA_CLS + (qx >> 1) * WA_XS + (qy >> 1) * WA_ROW + (qz >> 1),
                             cls * WB_CLS + (qx >> 1) * WB_XS + (qy >> 1) * WB_ROW + (qz >> 1), en.y, 0};
                    entries_fast[p * MAX_ENTRIES + k++] = en;
                }
                if (pass == 0 && far) ++ctx->counts_far[p];
            }
    }
    // P2M: per target cell, its stencil entries grouped by the raw direction of
    // the partner (stencil order inside a group), as partner cell indices
    std::vector<int> p2m_start(NCELL * 28, 0);
    std::vector<uint16_t> p2m_list;
    p2m_list.reserve((size_t)NCELL * MAX_ENTRIES);
    for (int cu = 0; cu < NCELL; ++cu) {
        const int cx = cu >> 6, cy = (cu >> 3) & 7, cz = cu & 7;
        const int p = ((cx & 1) << 2) | ((cy & 1) << 1) | (cz & 1);
        for (int r = 0; r < 27; ++r) {
            p2m_start[cu * 28 + r] = (int)p2m_list.size();
            if (r == 13) continue;
            for (int e2 = 0; e2 < ctx->counts[p]; ++e2) {
                const int y = entries[p * MAX_ENTRIES + e2].y;
                const int ax = cx + (y & 15) - 8, ay = cy + ((y >> 4) & 15) - 8, az = cz + ((y >> 8) & 15) - 8;
                const int raw = ((ax >> 3) + 1) + 3 * ((ay >> 3) + 1) + 9 * ((az >> 3) + 1);
                if (raw == r) p2m_list.push_back((uint16_t)((ax & 7) * 64 + (ay & 7) * 8 + (az & 7)));
            }
        }
        p2m_start[cu * 28 + 27] = (int)p2m_list.size();
    }
    // per direction: the cells with partners there, most partners first
    std::vector<int> p2m_perm_start(28, 0);
    std::vector<uint16_t> p2m_perm;
    for (int r = 0; r < 27; ++r) {
        p2m_perm_start[r] = (int)p2m_perm.size();
        std::vector<std::pair<int, int>> cells;
        for (int cu = 0; cu < NCELL; ++cu) {
            const int cnt = p2m_start[cu * 28 + r + 1] - p2m_start[cu * 28 + r];
            if (cnt > 0) cells.push_back({-cnt, cu});
        }
        std::sort(cells.begin(), cells.end());
        for (const auto& c : cells) p2m_perm.push_back((uint16_t)c.second);
    }
    p2m_perm_start[27] = (int)p2m_perm.size();
    std::vector<int16_t> p2m_slot(27 * NCELL, -1);
    for (int r = 0; r < 27; ++r)
        for (int t = p2m_perm_start[r]; t < p2m_perm_start[r + 1]; ++t)
            p2m_slot[r * NCELL + p2m_perm[t]] = (int16_t)(t - p2m_perm_start[r]);
    ctx->p2m_groups_max = (int)p2m_perm.size();
    DeviceGuard g(device);
    cudaError_t e;
    if ((e = cudaMalloc(&ctx->d_p2m_slot, sizeof(int16_t) * p2m_slot.size())) != cudaSuccess ||
        (e = cudaMemcpy(ctx->d_p2m_slot, p2m_slot.data(), sizeof(int16_t) * p2m_slot.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_p2p_four, sizeof(double4) * p2p_four.size())) != cudaSuccess ||
        (e = cudaMemcpy(ctx->d_p2p_four, p2p_four.data(), sizeof(double4) * p2p_four.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_p2m_perm_start, sizeof(int) * p2m_perm_start.size())) != cudaSuccess ||
        (e = cudaMemcpy(ctx->d_p2m_perm_start, p2m_perm_start.data(), sizeof(int) * p2m_perm_start.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_p2m_perm, sizeof(uint16_t) * std::max<size_t>(1, p2m_perm.size()))) != cudaSuccess ||
        (e = cudaMemcpy(ctx->d_p2m_perm, p2m_perm.data(), sizeof(uint16_t) * p2m_perm.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_p2m_start, sizeof(int) * p2m_start.size())) != cudaSuccess ||
        (e = cudaMemcpy(ctx->d_p2m_start, p2m_start.data(), sizeof(int) * p2m_start.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_p2m_list, sizeof(uint16_t) * p2m_list.size())) != cudaSuccess ||
        (e = cudaMemcpy(ctx->d_p2m_list, p2m_list.data(), sizeof(uint16_t) * p2m_list.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_entries, sizeof(int2) * entries.size())) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_count, sizeof(int) * 8)) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_four, sizeof(double) * 4 * FULL)) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_phase, FULL)) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_err, sizeof(int))) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_entries_fast, sizeof(int2) * entries_fast.size())) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_count_far, sizeof(int) * 8)) != cudaSuccess ||
        (e = cudaMemcpy(ctx->d_entries_fast, entries_fast.data(), sizeof(int2) * entries_fast.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(ctx->d_count_far, ctx->counts_far, sizeof(int) * 8, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_entries_split, sizeof(int4) * entries_split.size())) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_entries_p2p, sizeof(int2) * entries_p2p.size())) != cudaSuccess ||
        (e = cudaMalloc(&ctx->d_entries_ws, sizeof(int4) * entries_ws.size())) != cudaSuccess ||
        (e = cudaMemcpy(ctx->d_entries_ws, entries_ws.data(), sizeof(int4) * entries_ws.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(ctx->d_entries_p2p, entries_p2p.data(), sizeof(int2) * entries_p2p.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpyToSymbol(c_four, ctx->st.four, sizeof(double) * 4 * FULL)) != cudaSuccess ||
        (e = cudaMemcpy(ctx->d_entries_split, entries_split.data(), sizeof(int4) * entries_split.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(ctx->d_entries, entries.data(), sizeof(int2) * entries.size(), cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMemcpy(ctx->d_count, ctx->counts, sizeof(int) * 8, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(ctx->d_four, ctx->st.four, sizeof(double) * 4 * FULL, cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMemcpy(ctx->d_phase, ctx->st.phase, FULL, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(ctx->d_err, 0, sizeof(int))) != cudaSuccess) {
        otfmm_destroy(ctx);
        return cuda_fail(e, "otfmm_create");
    }
    const int rc = ensure_attributes(device);
    if (rc != OTFMM_OK) {
        otfmm_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return OTFMM_OK;
}

int otfmm_destroy(otfmm_context* ctx) {
    if (!ctx) return OTFMM_OK;
    DeviceGuard g(ctx->device);
    cudaFree(ctx->d_entries);
    cudaFree(ctx->d_count);
    cudaFree(ctx->d_entries_fast);
    cudaFree(ctx->d_entries_split);
    cudaFree(ctx->d_entries_p2p);
    cudaFree(ctx->d_entries_ws);
    cudaFree(ctx->d_p2m_start);
    cudaFree(ctx->d_p2m_list);
    cudaFree(ctx->d_p2m_perm_start);
    cudaFree(ctx->d_p2m_perm);
    cudaFree(ctx->d_p2p_four);
    cudaFree(ctx->d_p2m_slot);
    {
        auto& hp = ctx->hp;
        if (hp.ready) {
            cudaStreamSynchronize(hp.h2d);
            cudaStreamSynchronize(hp.d2h);
            for (auto& e : hp.ev) cudaEventDestroy(e);
            cudaStreamDestroy(hp.h2d);
            cudaStreamDestroy(hp.d2h);
        }
        cudaFree(hp.M);
        cudaFree(hp.com);
        cudaFree(hp.mon);
        cudaFree(hp.L);
        cudaFree(hp.Lc);
        cudaFree(hp.is_leaf);
        cudaFree(hp.items);
        cudaFreeHost(hp.items_pinned);
    }
    cudaFree(ctx->d_count_far);
    cudaFree(ctx->d_four);
    cudaFree(ctx->d_phase);
    cudaFree(ctx->d_err);
    cudaFree(ctx->d_soa_scratch);
    cudaFree(ctx->d_lists);
    delete ctx;
    return OTFMM_OK;
}

int otfmm_stencil_info(const otfmm_context* ctx, int32_t counts[3], uint8_t* mpole_mask, uint8_t* mpole_phase,
                       uint8_t* p2p_mask) {
    if (!ctx || !counts) return fail(OTFMM_ERR_INVALID, "NULL argument");
    counts[0] = ctx->st.n_mpole;
    counts[1] = ctx->st.n_phase_one;
    counts[2] = ctx->st.n_mpole;   // the monopole stencil is the same offset set
    if (mpole_mask) std::memcpy(mpole_mask, ctx->st.mask, FULL);
    if (mpole_phase) std::memcpy(mpole_phase, ctx->st.phase, FULL);
    if (p2p_mask) std::memcpy(p2p_mask, ctx->st.mask, FULL);
    return OTFMM_OK;
}

int otfmm_m2l_soa(otfmm_context* ctx, const double* mon, const double* M, const double* com, double* L, double* L_c,
                  int gsolve_type, int use_root_stencil, int precision, void* stream) {
    if (!ctx || !M || !com || !L) return fail(OTFMM_ERR_INVALID, "NULL argument");
    const bool rho = (gsolve_type == OTFMM_RHO);
    if (gsolve_type != OTFMM_RHO && gsolve_type != OTFMM_DRHODT) return fail(OTFMM_ERR_INVALID, "bad gsolve_type");
    if (rho && !L_c) return fail(OTFMM_ERR_INVALID, "L_c is NULL for RHO");
    if (!use_root_stencil && !mon) return fail(OTFMM_ERR_INVALID, "mon is NULL");
    int rc = check_precision(precision);
    if (rc) return rc;
    DeviceGuard g(ctx->device);
    SoaArgs a{mon, M, com, L, L_c, ctx->tables()};
    const size_t bytes = SMEM_DOUBLES * sizeof(double);
    cudaStream_t s = (cudaStream_t)stream;
#define OT_SOA(P, R, T) soa_m2l_kernel<P, R, T><<<2, THREADS, bytes, s>>>(a)
    if (precision == OTFMM_FP64_EXACT) {
        if (use_root_stencil) { if (rho) OT_SOA(PREC_EXACT, true, true); else OT_SOA(PREC_EXACT, false, true); }
        else { if (rho) OT_SOA(PREC_EXACT, true, false); else OT_SOA(PREC_EXACT, false, false); }
    } else {
        if (use_root_stencil) { if (rho) OT_SOA(PREC_FAST, true, true); else OT_SOA(PREC_FAST, false, true); }
        else { if (rho) OT_SOA(PREC_FAST, true, false); else OT_SOA(PREC_FAST, false, false); }
    }
#undef OT_SOA
    OT_CUDA(cudaGetLastError());
    return OTFMM_OK;
}

int otfmm_m2l_soa_host(otfmm_context* ctx, const double* mon, const double* M, const double* com, double* L,
                       double* L_c, int gsolve_type, int use_root_stencil, int precision) {
    if (!ctx || !M || !com || !L) return fail(OTFMM_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceGuard g(ctx->device);
    const size_t n_in = ENTRIES + 20 * (size_t)CL + 3 * (size_t)CL, n_out = 23 * (size_t)CLU;
    if (!ctx->d_soa_scratch) OT_CUDA(cudaMalloc(&ctx->d_soa_scratch, sizeof(double) * (n_in + n_out)));
    double* d_mon = ctx->d_soa_scratch;
    double* d_M = d_mon + ENTRIES;
    double* d_com = d_M + 20 * CL;
    double* d_L = d_com + 3 * CL;
    double* d_Lc = d_L + 20 * CLU;
    if (mon) OT_CUDA(cudaMemcpy(d_mon, mon, sizeof(double) * ENTRIES, cudaMemcpyHostToDevice));
    OT_CUDA(cudaMemcpy(d_M, M, sizeof(double) * 20 * CL, cudaMemcpyHostToDevice));
    OT_CUDA(cudaMemcpy(d_com, com, sizeof(double) * 3 * CL, cudaMemcpyHostToDevice));
    int rc = otfmm_m2l_soa(ctx, mon ? d_mon : nullptr, d_M, d_com, d_L, d_Lc, gsolve_type, use_root_stencil,
                           precision, nullptr);
    if (rc) return rc;
    OT_CUDA(cudaMemcpy(L, d_L, sizeof(double) * 20 * CLU, cudaMemcpyDeviceToHost));
    if (gsolve_type == OTFMM_RHO && L_c) OT_CUDA(cudaMemcpy(L_c, d_Lc, sizeof(double) * 3 * CLU, cudaMemcpyDeviceToHost));
    return OTFMM_OK;
}

// Host-buffer multipole call that allocates nothing: device staging comes
// from the static g_noalloc_scratch array. Its device address is looked up
// once per device (cudaGetSymbolAddress, on the first call on that device,
// which should therefore come before any stream capture); later calls reuse
// it. The array is shared by every call: calls are serialised here, and each
// call clears the output staging it reads back.
int otfmm_m2l_soa_host_noalloc(otfmm_context* ctx, int32_t n_subgrids, const double* mon, const double* M,
                               const double* com, double* L, double* L_c, int gsolve_type, int use_root_stencil,
                               int precision, void* stream) {
    static std::mutex mu;
    static double* scratch_ptr[64] = {};
    if (!ctx || !M || !com || !L) return fail(OTFMM_ERR_INVALID, "NULL argument");
    if (n_subgrids < 1 || n_subgrids > NOALLOC_MAX_SUBGRIDS)
        return fail(OTFMM_ERR_INVALID, "n_subgrids must be 1.." + std::to_string(NOALLOC_MAX_SUBGRIDS) +
                                           ": the static staging array holds at most that many subgrids");
    const bool rho = (gsolve_type == OTFMM_RHO);
    if (gsolve_type != OTFMM_RHO && gsolve_type != OTFMM_DRHODT) return fail(OTFMM_ERR_INVALID, "bad gsolve_type");
    if (rho && !L_c) return fail(OTFMM_ERR_INVALID, "L_c is NULL for RHO");
    if (!use_root_stencil && !mon) return fail(OTFMM_ERR_INVALID, "mon is NULL");
    if (ctx->device < 0 || ctx->device >= 64) return fail(OTFMM_ERR_INVALID, "device index out of range");
    int rc = check_precision(precision);
    if (rc) return rc;
    std::lock_guard<std::mutex> lock(mu);
    DeviceGuard g(ctx->device);
    if (!scratch_ptr[ctx->device]) {
        double* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        scratch_ptr[ctx->device] = ptr;
    }
    cudaStream_t s = (cudaStream_t)stream;
    for (int i = 0; i < n_subgrids; ++i) {
        double* d_mon = scratch_ptr[ctx->device] + i * NOALLOC_SLOT;
        double* d_M = d_mon + ENTRIES;
        double* d_com = d_M + 20 * (size_t)CL;
        double* d_L = d_com + 3 * (size_t)CL;
        double* d_Lc = d_L + 20 * (size_t)CLU;
        if (!use_root_stencil)
            OT_CUDA(cudaMemcpyAsync(d_mon, mon + (size_t)i * ENTRIES, sizeof(double) * ENTRIES, cudaMemcpyHostToDevice, s));
        OT_CUDA(cudaMemcpyAsync(d_M, M + (size_t)i * 20 * CL, sizeof(double) * 20 * CL, cudaMemcpyHostToDevice, s));
        OT_CUDA(cudaMemcpyAsync(d_com, com + (size_t)i * 3 * CL, sizeof(double) * 3 * CL, cudaMemcpyHostToDevice, s));
        OT_CUDA(cudaMemsetAsync(d_L, 0, sizeof(double) * 23 * CLU, s));
        rc = otfmm_m2l_soa(ctx, use_root_stencil ? nullptr : d_mon, d_M, d_com, d_L, d_Lc, gsolve_type,
                           use_root_stencil, precision, stream);
        if (rc) return rc;
        OT_CUDA(cudaMemcpyAsync(L + (size_t)i * 20 * CLU, d_L, sizeof(double) * 20 * CLU, cudaMemcpyDeviceToHost, s));
        if (rho)
            OT_CUDA(cudaMemcpyAsync(L_c + (size_t)i * 3 * CLU, d_Lc, sizeof(double) * 3 * CLU, cudaMemcpyDeviceToHost, s));
    }
    OT_CUDA(cudaStreamSynchronize(s));
    return OTFMM_OK;
}

int otfmm_p2p_soa(otfmm_context* ctx, const double* mon, double dx, double* L4, int precision, void* stream) {
    if (!ctx || !mon || !L4) return fail(OTFMM_ERR_INVALID, "NULL argument");
    if (!(dx > 0.0)) return fail(OTFMM_ERR_INVALID, "dx must be positive");
    int rc = check_precision(precision);
    if (rc) return rc;
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (precision == OTFMM_FP64_EXACT)
        soa_p2p_kernel<PREC_EXACT><<<4, 128, 0, s>>>(mon, dx, L4, ctx->tables());
    else
        soa_p2p_kernel<PREC_FAST><<<4, 128, 0, s>>>(mon, dx, L4, ctx->tables());
    OT_CUDA(cudaGetLastError());
    return OTFMM_OK;
}

int otfmm_p2m_soa(otfmm_context* ctx, int d, const double* neighbor_M, const double* neighbor_com,
                  const double* inner_com, double* L4, double* L_c, int gsolve_type, int reset_lc, int precision,
                  void* stream) {
    if (!ctx || !neighbor_M || !neighbor_com || !inner_com || !L4) return fail(OTFMM_ERR_INVALID, "NULL argument");
    if (d < 0 || d >= 26) return fail(OTFMM_ERR_INVALID, "direction out of range");
    const bool rho = (gsolve_type == OTFMM_RHO);
    if (rho && !L_c) return fail(OTFMM_ERR_INVALID, "L_c is NULL for RHO");
    int rc = check_precision(precision);
    if (rc) return rc;
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (rho && reset_lc) {
        zero_kernel<<<(3 * CLU + 255) / 256, 256, 0, s>>>(L_c, 3 * CLU);
    }
    const Tables t = ctx->tables();
    if (precision == OTFMM_FP64_EXACT) {
        if (rho) soa_p2m_kernel<PREC_EXACT, true><<<4, 128, 0, s>>>(d, neighbor_M, neighbor_com, inner_com, L4, L_c, t);
        else soa_p2m_kernel<PREC_EXACT, false><<<4, 128, 0, s>>>(d, neighbor_M, neighbor_com, inner_com, L4, L_c, t);
    } else {
        if (rho) soa_p2m_kernel<PREC_FAST, true><<<4, 128, 0, s>>>(d, neighbor_M, neighbor_com, inner_com, L4, L_c, t);
        else soa_p2m_kernel<PREC_FAST, false><<<4, 128, 0, s>>>(d, neighbor_M, neighbor_com, inner_com, L4, L_c, t);
    }
    OT_CUDA(cudaGetLastError());
    return OTFMM_OK;
}

int otfmm_stage_soa(otfmm_context* ctx, const double* pool_M, const double* pool_com, const double* pool_mon,
                    const uint8_t* pool_is_leaf, int32_t n_subgrids, const otfmm_work_item* item, double* mon,
                    double* M, double* com, void* stream) {
    if (!ctx || !pool_M || !pool_com || !pool_mon || !pool_is_leaf || !item || !mon)
        return fail(OTFMM_ERR_INVALID, "NULL argument");
    const otfmm_work_item& w = *item;
    if (w.kind < 0 || w.kind > 2 || w.subgrid < 0 || w.subgrid >= n_subgrids)
        return fail(OTFMM_ERR_INVALID, "work item out of range");
    for (int d = 0; d < 26; ++d)
        if (w.neighbors[d] < -1 || w.neighbors[d] >= n_subgrids) return fail(OTFMM_ERR_INVALID, "neighbour out of range");
    if (w.kind != OTFMM_KIND_LEAF && (!M || !com)) return fail(OTFMM_ERR_INVALID, "M / com NULL for a multipole item");
    DeviceGuard g(ctx->device);
    stage_soa_kernel<<<(CL + 255) / 256, 256, 0, (cudaStream_t)stream>>>(pool_M, pool_com, pool_mon, pool_is_leaf, w,
                                                                         mon, M, com);
    OT_CUDA(cudaGetLastError());
    return OTFMM_OK;
}

int otfmm_stage_p2m_soa(otfmm_context* ctx, const double* pool_M, const double* pool_com, int32_t n_subgrids,
                        int32_t neighbor, int d, double* neighbor_M, double* neighbor_com, int32_t* stride,
                        void* stream) {
    if (!ctx || !pool_M || !pool_com || !neighbor_M || !neighbor_com) return fail(OTFMM_ERR_INVALID, "NULL argument");
    if (d < 0 || d >= 26) return fail(OTFMM_ERR_INVALID, "direction out of range");
    if (neighbor < 0 || neighbor >= n_subgrids) return fail(OTFMM_ERR_INVALID, "neighbour out of range");
    const int r = d < 13 ? d : d + 1;
    int size = 1;
    for (int a = 0; a < 3; ++a) size *= ((r / (a == 0 ? 1 : a == 1 ? 3 : 9)) % 3 == 1) ? INX : SMAX;
    if (stride) *stride = size + 19;
    DeviceGuard g(ctx->device);
    stage_p2m_kernel<<<(size + 19 + 127) / 128, 128, 0, (cudaStream_t)stream>>>(pool_M, pool_com, neighbor, d,
                                                                                 neighbor_M, neighbor_com);
    OT_CUDA(cudaGetLastError());
    return OTFMM_OK;
}

}   // extern "C"

namespace {

int check_tuning(const otfmm_tuning& t) {
    if (t.split_m2l_form != OTFMM_SPLIT_WARP_SPECIALISED && t.split_m2l_form != OTFMM_SPLIT_SINGLE_ROLE &&
        t.split_m2l_form != OTFMM_SPLIT_WARP_SPECIALISED_PACKED)
        return fail(OTFMM_ERR_INVALID, "unknown split M2L form");
    if (t.split_m2l_chunk != 8 && t.split_m2l_chunk != 16) return fail(OTFMM_ERR_INVALID, "split M2L chunk must be 8 or 16");
    if (t.split_p2p_chunk != 16 && t.split_p2p_chunk != 32) return fail(OTFMM_ERR_INVALID, "split P2P chunk must be 16 or 32");
    if (t.p2m_lanes != 4 && t.p2m_lanes != 8 && t.p2m_lanes != 16) return fail(OTFMM_ERR_INVALID, "P2M lanes must be 4, 8 or 16");
    return OTFMM_OK;
}

int check_batch_args(otfmm_context* ctx, const double* pool_M, const double* pool_com, const double* pool_mon,
                     const uint8_t* pool_is_leaf, int32_t n_subgrids, const otfmm_work_item* items, int32_t n_items,
                     double* L, double* L_c, int gsolve_type, int precision) {
    if (!ctx || !pool_M || !pool_com || !pool_mon || !pool_is_leaf || !items || !L || !L_c)
        return fail(OTFMM_ERR_INVALID, "NULL argument");
    if (n_subgrids <= 0 || n_items < 0 || n_items > (1 << 29)) return fail(OTFMM_ERR_INVALID, "bad sizes");
    if (gsolve_type != OTFMM_RHO && gsolve_type != OTFMM_DRHODT) return fail(OTFMM_ERR_INVALID, "bad gsolve_type");
    return check_precision(precision, true);
}

// Enqueues one batched solve on `s`: counter resets, classification into the
// device work lists `lists` (capacity `cap` items), then the persistent
// multipole, P2P and P2M launches with the variants of `tu`. Only stream
// operations: safe inside a stream capture.
int enqueue_batch(otfmm_context* ctx, const double* pool_M, const double* pool_com, const double* pool_mon,
                  const uint8_t* pool_is_leaf, int32_t n_subgrids, const otfmm_work_item* items, int32_t n_items,
                  double* L, double* L_c, int gsolve_type, int precision, int* lists, int cap, int* err,
                  const otfmm_tuning& tu, cudaStream_t s, cudaEvent_t* marks = nullptr, bool reset_err = true) {
    // marks (optional): 5 events recorded around the 4 kernel launches
    auto mark = [&](int i) {
        if (marks) cudaEventRecord(marks[i], s);
    };
    WorkLists wl{lists, lists + cap, lists + 2 * (size_t)cap, lists + 3 * (size_t)cap, lists + 4 * (size_t)cap};
    if (reset_err) OT_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    OT_CUDA(cudaMemsetAsync(wl.counts, 0, sizeof(int) * WL_COUNTERS, s));
    BatchArgs a{pool_M, pool_com, pool_mon, pool_is_leaf, n_subgrids, items, n_items, L, L_c, ctx->tables(),
                err, wl, tu.p2m_lanes};
    const size_t bytes = SMEM_DOUBLES * sizeof(double);
    const bool rho = (gsolve_type == OTFMM_RHO);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    // classify, then multipole tiles, P2P of the leaves and P2M (stream
    // order keeps the reference's P2P-then-P2M accumulation order)
    mark(0);
    classify_kernel<<<(n_items + 255) / 256, 256, 0, s>>>(a);
    mark(1);
    const dim3 tiles_grid(sms), p2p_grid(P2P_CTAS_PER_SM * sms), p2m_grid(std::min(n_items, 8 * sms));
    if (precision == OTFMM_FP64_EXACT) {
        if (rho) m2l_batch_kernel<PREC_EXACT, true><<<tiles_grid, THREADS, bytes, s>>>(a);
        else m2l_batch_kernel<PREC_EXACT, false><<<tiles_grid, THREADS, bytes, s>>>(a);
        mark(2);
        p2p_batch_kernel<PREC_EXACT><<<p2p_grid, P2P_THREADS, P2P_SMEM_BYTES, s>>>(a);
        mark(3);
        if (rho) p2m_batch_kernel<PREC_EXACT, true><<<p2m_grid, P_THREADS, 0, s>>>(a);
        else p2m_batch_kernel<PREC_EXACT, false><<<p2m_grid, P_THREADS, 0, s>>>(a);
    } else {
        if (precision == OTFMM_FP32_SPLIT) {
            const size_t sbytes = S_SMEM_DOUBLES * sizeof(double);
            if (rho && tu.split_m2l_form != OTFMM_SPLIT_SINGLE_ROLE) {
                const bool packed = (tu.split_m2l_form == OTFMM_SPLIT_WARP_SPECIALISED_PACKED);
                if (tu.split_m2l_chunk == 8) {
                    if (packed) m2l_split_ws_kernel<8, true><<<tiles_grid, WS_THREADS, WS_SMEM_BYTES, s>>>(a);
                    else m2l_split_ws_kernel<8, false><<<tiles_grid, WS_THREADS, WS_SMEM_BYTES, s>>>(a);
                } else {
                    if (packed) m2l_split_ws_kernel<16, true><<<tiles_grid, WS_THREADS, WS_SMEM_BYTES, s>>>(a);
                    else m2l_split_ws_kernel<16, false><<<tiles_grid, WS_THREADS, WS_SMEM_BYTES, s>>>(a);
                }
            } else if (rho) {
                m2l_batch_kernel<PREC_SPLIT, true><<<tiles_grid, THREADS, sbytes, s>>>(a);
            } else {
                m2l_batch_kernel<PREC_SPLIT, false><<<tiles_grid, THREADS, sbytes, s>>>(a);
            }
            mark(2);
            if (tu.split_p2p_chunk == 16) p2p_leaf_kernel<float, 16><<<sms, P2_THREADS, p2_smem_bytes<float>(), s>>>(a);
            else p2p_leaf_kernel<float, 32><<<sms, P2_THREADS, p2_smem_bytes<float>(), s>>>(a);
        } else {
            if (rho) m2l_batch_kernel<PREC_FAST, true><<<tiles_grid, THREADS, bytes, s>>>(a);
            else m2l_batch_kernel<PREC_FAST, false><<<tiles_grid, THREADS, bytes, s>>>(a);
            mark(2);
            p2p_leaf_kernel<double, 0><<<sms, P2_THREADS, p2_smem_bytes<double>(), s>>>(a);
        }
        mark(3);
        const size_t part_bytes = sizeof(double) * 7 * (size_t)ctx->p2m_groups_max;
        if (rho) p2m_fast_kernel<true><<<p2m_grid, P_THREADS, part_bytes, s>>>(a);
        else p2m_fast_kernel<false><<<p2m_grid, P_THREADS, part_bytes, s>>>(a);
    }
    mark(4);
    OT_CUDA(cudaGetLastError());
    return OTFMM_OK;
}

// Grows the context's work-list storage to hold n_items (a device allocation,
// after the stream's earlier work is done).
int ensure_list_capacity(otfmm_context* ctx, int32_t n_items, cudaStream_t s) {
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (n_items <= ctx->list_capacity) return OTFMM_OK;
    OT_CUDA(cudaStreamSynchronize(s));
    cudaFree(ctx->d_lists);
    ctx->d_lists = nullptr;
    const int cap = std::max(n_items, 2 * ctx->list_capacity);
    OT_CUDA(cudaMalloc(&ctx->d_lists, sizeof(int) * (4 * (size_t)cap + WL_COUNTERS)));
    ctx->list_capacity = cap;
    return OTFMM_OK;
}

}   // namespace

struct otfmm_plan {
    otfmm_context* ctx = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int* lists = nullptr;
    int* err = nullptr;
};

extern "C" {

int otfmm_batch(otfmm_context* ctx, const double* pool_M, const double* pool_com, const double* pool_mon,
                const uint8_t* pool_is_leaf, int32_t n_subgrids, const otfmm_work_item* items, int32_t n_items,
                double* L, double* L_c, int gsolve_type, int precision, void* stream) {
    int rc = check_batch_args(ctx, pool_M, pool_com, pool_mon, pool_is_leaf, n_subgrids, items, n_items, L, L_c,
                              gsolve_type, precision);
    if (rc) return rc;
    if (n_items == 0) return OTFMM_OK;
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    rc = ensure_list_capacity(ctx, n_items, s);
    if (rc) return rc;
    return enqueue_batch(ctx, pool_M, pool_com, pool_mon, pool_is_leaf, n_subgrids, items, n_items, L, L_c,
                         gsolve_type, precision, ctx->d_lists, ctx->list_capacity, ctx->d_err, ctx->tuning, s);
}

int otfmm_upward(otfmm_context* ctx, double* pool_M, double* pool_com, const double* pool_mon,
                 const uint8_t* pool_is_leaf, double* com1, int32_t n_subgrids, const otfmm_tree_node* nodes,
                 const int32_t* level_start, int32_t n_levels, int gsolve_type, void* stream) {
    if (!ctx || !pool_M || !pool_com || !pool_mon || !pool_is_leaf || !com1 || !nodes || !level_start)
        return fail(OTFMM_ERR_INVALID, "NULL argument");
    if (n_subgrids <= 0 || n_levels <= 0) return fail(OTFMM_ERR_INVALID, "bad sizes");
    if (gsolve_type != OTFMM_RHO && gsolve_type != OTFMM_DRHODT) return fail(OTFMM_ERR_INVALID, "bad gsolve_type");
    for (int l = 0; l < n_levels; ++l)
        if (level_start[l] < 0 || level_start[l + 1] < level_start[l])
            return fail(OTFMM_ERR_INVALID, "level_start must be non-decreasing");
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    OT_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), s));
    TreeArgs a{pool_M, pool_com, pool_mon, pool_is_leaf, com1, n_subgrids, nodes, 0, nullptr, nullptr, nullptr,
               0.0, 0, ctx->d_err};
    for (int l = n_levels - 1; l >= 0; --l) {
        const int n = level_start[l + 1] - level_start[l];
        if (n == 0) continue;
        a.first = level_start[l];
        if (gsolve_type == OTFMM_RHO) upward_level_kernel<true><<<n, 64, 0, s>>>(a);
        else upward_level_kernel<false><<<n, 64, 0, s>>>(a);
    }
    OT_CUDA(cudaGetLastError());
    return OTFMM_OK;
}

int otfmm_downward(otfmm_context* ctx, const double* pool_com, const uint8_t* pool_is_leaf, const double* com1,
                   int32_t n_subgrids, const otfmm_tree_node* nodes, const int32_t* level_start, int32_t n_levels,
                   double* L, double* L_c, double* G, double gconst, int correct_am_grav, int gsolve_type,
                   void* stream) {
    if (!ctx || !pool_com || !pool_is_leaf || !com1 || !nodes || !level_start || !L || !L_c || !G)
        return fail(OTFMM_ERR_INVALID, "NULL argument");
    if (n_subgrids <= 0 || n_levels <= 0) return fail(OTFMM_ERR_INVALID, "bad sizes");
    if (gsolve_type != OTFMM_RHO && gsolve_type != OTFMM_DRHODT) return fail(OTFMM_ERR_INVALID, "bad gsolve_type");
    for (int l = 0; l < n_levels; ++l)
        if (level_start[l] < 0 || level_start[l + 1] < level_start[l])
            return fail(OTFMM_ERR_INVALID, "level_start must be non-decreasing");
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    OT_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), s));
    TreeArgs a{nullptr, const_cast<double*>(pool_com), nullptr, pool_is_leaf, const_cast<double*>(com1), n_subgrids,
               nodes, 0, L, L_c, G, gconst, correct_am_grav, ctx->d_err};
    for (int l = 0; l < n_levels; ++l) {
        const int n = level_start[l + 1] - level_start[l];
        if (n == 0) continue;
        a.first = level_start[l];
        if (gsolve_type == OTFMM_RHO) downward_level_kernel<true><<<n, NCELL, 0, s>>>(a);
        else downward_level_kernel<false><<<n, NCELL, 0, s>>>(a);
    }
    OT_CUDA(cudaGetLastError());
    return OTFMM_OK;
}

int otfmm_batch_profile(otfmm_context* ctx, const double* pool_M, const double* pool_com, const double* pool_mon,
                        const uint8_t* pool_is_leaf, int32_t n_subgrids, const otfmm_work_item* items,
                        int32_t n_items, double* L, double* L_c, int gsolve_type, int precision, float kernel_ms[4],
                        void* stream) {
    if (!kernel_ms) return fail(OTFMM_ERR_INVALID, "kernel_ms is NULL");
    int rc = check_batch_args(ctx, pool_M, pool_com, pool_mon, pool_is_leaf, n_subgrids, items, n_items, L, L_c,
                              gsolve_type, precision);
    if (rc) return rc;
    if (n_items == 0) return fail(OTFMM_ERR_INVALID, "empty work list");
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    rc = ensure_list_capacity(ctx, n_items, s);
    if (rc) return rc;
    cudaEvent_t ev[5] = {};
    for (auto& e : ev) OT_CUDA(cudaEventCreate(&e));
    rc = enqueue_batch(ctx, pool_M, pool_com, pool_mon, pool_is_leaf, n_subgrids, items, n_items, L, L_c,
                       gsolve_type, precision, ctx->d_lists, ctx->list_capacity, ctx->d_err, ctx->tuning, s, ev);
    cudaError_t e = cudaEventSynchronize(ev[4]);
    for (int k = 0; k < 4 && rc == OTFMM_OK && e == cudaSuccess; ++k) e = cudaEventElapsedTime(&kernel_ms[k], ev[k], ev[k + 1]);
    for (auto& x : ev) cudaEventDestroy(x);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "otfmm_batch_profile");
    return OTFMM_OK;
}

int otfmm_batch_host(otfmm_context* ctx, const double* pool_M, const double* pool_com, const double* pool_mon,
                     const uint8_t* pool_is_leaf, int32_t n_subgrids, const otfmm_work_item* items, int32_t n_items,
                     double* L, double* L_c, int gsolve_type, int precision, void* stream) {
    int rc = check_batch_args(ctx, pool_M, pool_com, pool_mon, pool_is_leaf, n_subgrids, items, n_items, L, L_c,
                              gsolve_type, precision);
    if (rc) return rc;
    // host-side checks of the fields used to order the work (the device re-validates everything)
    for (int i = 0; i < n_items; ++i) {
        const otfmm_work_item& w = items[i];
        if (w.subgrid < 0 || w.subgrid >= n_subgrids) return fail(OTFMM_ERR_INVALID, "work item out of range");
        for (int d = 0; d < 26; ++d)
            if (w.neighbors[d] < -1 || w.neighbors[d] >= n_subgrids)
                return fail(OTFMM_ERR_INVALID, "neighbour out of range");
    }
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    auto& hp = ctx->hp;
    std::lock_guard<std::mutex> lock(hp.mu);
    if (!hp.ready) {
        OT_CUDA(cudaStreamCreateWithFlags(&hp.h2d, cudaStreamNonBlocking));
        OT_CUDA(cudaStreamCreateWithFlags(&hp.d2h, cudaStreamNonBlocking));
        for (auto& e : hp.ev) OT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        hp.ready = true;
    }
    cudaEvent_t* ev_h2d = hp.ev;          // [16] pool chunk k arrived
    cudaEvent_t* ev_comp = hp.ev + 16;    // [16] item chunk c computed
    cudaEvent_t* ev_d2h = hp.ev + 32;     // [16] outputs of pool chunk k copied
    cudaEvent_t ev_start = hp.ev[48], ev_items = hp.ev[49], ev_done = hp.ev[50];
    // the previous call's copies out of the pinned work list and into the host outputs are done
    OT_CUDA(cudaEventSynchronize(ev_items));
    // device buffers and the work-list storage, grown on demand
    if (n_subgrids > hp.n_sub) {
        OT_CUDA(cudaStreamSynchronize(s));
        OT_CUDA(cudaDeviceSynchronize());
        cudaFree(hp.M);
        cudaFree(hp.com);
        cudaFree(hp.mon);
        cudaFree(hp.L);
        cudaFree(hp.Lc);
        cudaFree(hp.is_leaf);
        hp.M = hp.com = hp.mon = hp.L = hp.Lc = nullptr;
        hp.is_leaf = nullptr;
        hp.n_sub = 0;
        const size_t n = (size_t)n_subgrids;
        OT_CUDA(cudaMalloc(&hp.M, sizeof(double) * 20 * NCELL * n));
        OT_CUDA(cudaMalloc(&hp.com, sizeof(double) * 3 * NCELL * n));
        OT_CUDA(cudaMalloc(&hp.mon, sizeof(double) * NCELL * n));
        OT_CUDA(cudaMalloc(&hp.L, sizeof(double) * 20 * NCELL * n));
        OT_CUDA(cudaMalloc(&hp.Lc, sizeof(double) * 3 * NCELL * n));
        OT_CUDA(cudaMalloc(&hp.is_leaf, n));
        hp.n_sub = n_subgrids;
    }
    if (n_items > hp.n_items) {
        OT_CUDA(cudaDeviceSynchronize());
        cudaFree(hp.items);
        cudaFreeHost(hp.items_pinned);
        hp.items = nullptr;
        hp.items_pinned = nullptr;
        hp.n_items = 0;
        OT_CUDA(cudaMalloc(&hp.items, sizeof(otfmm_work_item) * (size_t)n_items));
        OT_CUDA(cudaMallocHost(&hp.items_pinned, sizeof(otfmm_work_item) * (size_t)n_items));
        hp.n_items = n_items;
    }
    if (n_items == 0) return OTFMM_OK;
    rc = ensure_list_capacity(ctx, n_items, s);
    if (rc) return rc;
    // Pool chunks [bnd[k], bnd[k+1]); an item runs once every pool record it reads
    // has arrived, i.e. in the chunk of the largest index it reads; the outputs
    // of pool chunk k are final after the last item chunk writing them.
    const int K = std::max(1, std::min(16, n_subgrids / 64));
    std::vector<int> bnd(K + 1);
    for (int k = 0; k <= K; ++k) bnd[k] = (int)((long long)n_subgrids * k / K);
    auto chunk_of = [&](int idx) { return (int)((long long)idx * K / n_subgrids); };
    std::vector<int> cidx(n_items), need(K, 0);
    for (int i = 0; i < n_items; ++i) {
        const otfmm_work_item& w = items[i];
        int mx = w.subgrid;
        for (int d = 0; d < 26; ++d) mx = std::max(mx, w.neighbors[d]);
        int c = chunk_of(mx);
        while (c + 1 <= K - 1 && bnd[c + 1] <= mx) ++c;   // exact chunk of mx
        while (c > 0 && bnd[c] > mx) --c;
        cidx[i] = c;
        int ks = chunk_of(w.subgrid);
        while (ks + 1 <= K - 1 && bnd[ks + 1] <= w.subgrid) ++ks;
        while (ks > 0 && bnd[ks] > w.subgrid) --ks;
        need[ks] = std::max(need[ks], c);
    }
    std::vector<int> first(K + 1, 0);
    for (int i = 0; i < n_items; ++i) ++first[cidx[i] + 1];
    for (int c = 0; c < K; ++c) first[c + 1] += first[c];
    {
        std::vector<int> fill(first.begin(), first.end() - 1);
        for (int i = 0; i < n_items; ++i) hp.items_pinned[fill[cidx[i]]++] = items[i];
    }
    for (int k = 1; k < K; ++k) need[k] = std::max(need[k], need[k - 1]);   // copy out in pool order
    const size_t cell = NCELL * sizeof(double);
    OT_CUDA(cudaEventRecord(ev_start, s));
    OT_CUDA(cudaStreamWaitEvent(hp.h2d, ev_start, 0));
    OT_CUDA(cudaStreamWaitEvent(hp.d2h, ev_start, 0));
    OT_CUDA(cudaMemcpyAsync(hp.is_leaf, pool_is_leaf, (size_t)n_subgrids, cudaMemcpyHostToDevice, hp.h2d));
    OT_CUDA(cudaMemcpyAsync(hp.items, hp.items_pinned, sizeof(otfmm_work_item) * (size_t)n_items,
                            cudaMemcpyHostToDevice, hp.h2d));
    for (int k = 0; k < K; ++k) {
        const size_t a = bnd[k], n = bnd[k + 1] - bnd[k];
        OT_CUDA(cudaMemcpyAsync(hp.M + a * 20 * NCELL, pool_M + a * 20 * NCELL, n * 20 * cell, cudaMemcpyHostToDevice,
                                hp.h2d));
        OT_CUDA(cudaMemcpyAsync(hp.com + a * 3 * NCELL, pool_com + a * 3 * NCELL, n * 3 * cell,
                                cudaMemcpyHostToDevice, hp.h2d));
        OT_CUDA(cudaMemcpyAsync(hp.mon + a * NCELL, pool_mon + a * NCELL, n * cell, cudaMemcpyHostToDevice, hp.h2d));
        OT_CUDA(cudaEventRecord(ev_h2d[k], hp.h2d));
    }
    OT_CUDA(cudaEventRecord(ev_items, hp.h2d));
    // outputs start from zero, as compute_fmm zeroes L / L_c (src/node_server.cpp:701-705)
    OT_CUDA(cudaMemsetAsync(hp.L, 0, sizeof(double) * 20 * NCELL * (size_t)n_subgrids, s));
    OT_CUDA(cudaMemsetAsync(hp.Lc, 0, sizeof(double) * 3 * NCELL * (size_t)n_subgrids, s));
    OT_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), s));
    for (int c = 0; c < K; ++c) {
        OT_CUDA(cudaStreamWaitEvent(s, ev_h2d[c], 0));
        const int n = first[c + 1] - first[c];
        if (n > 0) {
            rc = enqueue_batch(ctx, hp.M, hp.com, hp.mon, hp.is_leaf, n_subgrids, hp.items + first[c], n, hp.L,
                               hp.Lc, gsolve_type, precision, ctx->d_lists, ctx->list_capacity, ctx->d_err,
                               ctx->tuning, s, nullptr, false);
            if (rc) return rc;
        }
        OT_CUDA(cudaEventRecord(ev_comp[c], s));
    }
    for (int k = 0; k < K; ++k) {
        OT_CUDA(cudaStreamWaitEvent(hp.d2h, ev_comp[need[k]], 0));
        const size_t a = bnd[k], n = bnd[k + 1] - bnd[k];
        OT_CUDA(cudaMemcpyAsync(L + a * 20 * NCELL, hp.L + a * 20 * NCELL, n * 20 * cell, cudaMemcpyDeviceToHost,
                                hp.d2h));
        OT_CUDA(cudaMemcpyAsync(L_c + a * 3 * NCELL, hp.Lc + a * 3 * NCELL, n * 3 * cell, cudaMemcpyDeviceToHost,
                                hp.d2h));
        OT_CUDA(cudaEventRecord(ev_d2h[k], hp.d2h));
    }
    OT_CUDA(cudaEventRecord(ev_done, hp.d2h));
    OT_CUDA(cudaStreamWaitEvent(s, ev_done, 0));
    return OTFMM_OK;
}

int otfmm_get_tuning(const otfmm_context* ctx, otfmm_tuning* out) {
    if (!ctx || !out) return fail(OTFMM_ERR_INVALID, "NULL argument");
    *out = ctx->tuning;
    return OTFMM_OK;
}

int otfmm_set_tuning(otfmm_context* ctx, const otfmm_tuning* t) {
    if (!ctx || !t) return fail(OTFMM_ERR_INVALID, "NULL argument");
    const int rc = check_tuning(*t);
    if (rc) return rc;
    ctx->tuning = *t;
    return OTFMM_OK;
}

int otfmm_plan_create(otfmm_context* ctx, const double* pool_M, const double* pool_com, const double* pool_mon,
                      const uint8_t* pool_is_leaf, int32_t n_subgrids, const otfmm_work_item* items, int32_t n_items,
                      double* L, double* L_c, int gsolve_type, int precision, otfmm_plan** out) {
    if (!out) return fail(OTFMM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int rc = check_batch_args(ctx, pool_M, pool_com, pool_mon, pool_is_leaf, n_subgrids, items, n_items, L, L_c,
                              gsolve_type, precision);
    if (rc) return rc;
    if (n_items == 0) return fail(OTFMM_ERR_INVALID, "empty work list");
    DeviceGuard g(ctx->device);
    auto* plan = new otfmm_plan();
    plan->ctx = ctx;
    cudaStream_t cs = nullptr;
    cudaError_t e;
    if ((e = cudaMalloc(&plan->lists, sizeof(int) * (4 * (size_t)n_items + WL_COUNTERS))) != cudaSuccess ||
        (e = cudaMalloc(&plan->err, sizeof(int))) != cudaSuccess ||
        (e = cudaMemset(plan->err, 0, sizeof(int))) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
        if (cs) cudaStreamDestroy(cs);
        otfmm_plan_destroy(plan);
        return cuda_fail(e, "otfmm_plan_create");
    }
    rc = enqueue_batch(ctx, pool_M, pool_com, pool_mon, pool_is_leaf, n_subgrids, items, n_items, L, L_c,
                       gsolve_type, precision, plan->lists, n_items, plan->err, ctx->tuning, cs);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(cs, &graph);
    cudaStreamDestroy(cs);
    plan->graph = graph;
    if (rc == OTFMM_OK && e != cudaSuccess) rc = cuda_fail(e, "cudaStreamEndCapture");
    if (rc == OTFMM_OK && (e = cudaGraphInstantiate(&plan->exec, plan->graph, 0)) != cudaSuccess)
        rc = cuda_fail(e, "cudaGraphInstantiate");
    if (rc != OTFMM_OK) {
        const std::string msg = g_last_error;
        otfmm_plan_destroy(plan);
        return fail(rc, msg);
    }
    *out = plan;
    return OTFMM_OK;
}

int otfmm_plan_launch(otfmm_plan* plan, void* stream) {
    if (!plan || !plan->exec) return fail(OTFMM_ERR_INVALID, "NULL plan");
    DeviceGuard g(plan->ctx->device);
    OT_CUDA(cudaGraphLaunch(plan->exec, (cudaStream_t)stream));
    return OTFMM_OK;
}

int otfmm_plan_status(otfmm_plan* plan, void* stream) {
    if (!plan) return fail(OTFMM_ERR_INVALID, "NULL plan");
    DeviceGuard g(plan->ctx->device);
    int h = 0;
    OT_CUDA(cudaMemcpyAsync(&h, plan->err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    OT_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if (h) return fail(OTFMM_ERR_DEVICE, "a work item failed validation on the device");
    return OTFMM_OK;
}

int otfmm_plan_destroy(otfmm_plan* plan) {
    if (!plan) return OTFMM_OK;
    DeviceGuard g(plan->ctx->device);
    if (plan->exec) cudaGraphExecDestroy(plan->exec);
    if (plan->graph) cudaGraphDestroy(plan->graph);
    cudaFree(plan->lists);
    cudaFree(plan->err);
    delete plan;
    return OTFMM_OK;
}

int otfmm_autotune(otfmm_context* ctx, const double* pool_M, const double* pool_com, const double* pool_mon,
                   const uint8_t* pool_is_leaf, int32_t n_subgrids, const otfmm_work_item* items, int32_t n_items,
                   double* L, double* L_c, int gsolve_type, int precision, int repeats, otfmm_tuning* chosen,
                   void* stream) {
    int rc = check_batch_args(ctx, pool_M, pool_com, pool_mon, pool_is_leaf, n_subgrids, items, n_items, L, L_c,
                              gsolve_type, precision);
    if (rc) return rc;
    if (n_items == 0 || repeats < 1) return fail(OTFMM_ERR_INVALID, "empty work list or repeats < 1");
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    rc = ensure_list_capacity(ctx, n_items, s);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    OT_CUDA(cudaEventCreate(&e0));
    OT_CUDA(cudaEventCreate(&e1));
    // median of `repeats` timed solves after one warm-up
    auto time_of = [&](const otfmm_tuning& tu, float& med) -> int {
        std::vector<float> ts;
        for (int r = 0; r <= repeats; ++r) {
            OT_CUDA(cudaEventRecord(e0, s));
            int rc2 = enqueue_batch(ctx, pool_M, pool_com, pool_mon, pool_is_leaf, n_subgrids, items, n_items, L,
                                    L_c, gsolve_type, precision, ctx->d_lists, ctx->list_capacity, ctx->d_err, tu, s);
            if (rc2) return rc2;
            OT_CUDA(cudaEventRecord(e1, s));
            OT_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            OT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (r > 0) ts.push_back(ms);
        }
        std::sort(ts.begin(), ts.end());
        med = ts[ts.size() / 2];
        return OTFMM_OK;
    };
    // coordinate descent over the variant dimensions, starting from the current choice
    otfmm_tuning best = ctx->tuning;
    float tbest = 0.f;
    rc = time_of(best, tbest);
    const int forms[3] = {OTFMM_SPLIT_WARP_SPECIALISED_PACKED, OTFMM_SPLIT_WARP_SPECIALISED, OTFMM_SPLIT_SINGLE_ROLE};
    const int m2l_chunks[2] = {8, 16}, p2p_chunks[2] = {16, 32}, lanes[3] = {4, 8, 16};
    const bool split = (precision == OTFMM_FP32_SPLIT), fast = (precision != OTFMM_FP64_EXACT);
    for (int dim = 0; dim < 4 && rc == OTFMM_OK; ++dim) {
        const int nvar = (dim == 3 || dim == 0) ? 3 : 2;
        if ((dim < 3 && !split) || (dim == 3 && !fast)) continue;
        for (int v = 0; v < nvar && rc == OTFMM_OK; ++v) {
            otfmm_tuning tu = best;
            if (dim == 0) tu.split_m2l_form = forms[v];
            if (dim == 1) tu.split_m2l_chunk = m2l_chunks[v];
            if (dim == 2) tu.split_p2p_chunk = p2p_chunks[v];
            if (dim == 3) tu.p2m_lanes = lanes[v];
            if (std::memcmp(&tu, &best, sizeof tu) == 0) continue;
            float t = 0.f;
            rc = time_of(tu, t);
            if (rc == OTFMM_OK && t < tbest) {
                tbest = t;
                best = tu;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    ctx->tuning = best;
    if (chosen) *chosen = best;
    return OTFMM_OK;
}

long long otfmm_count_pairs(const otfmm_context* ctx, const uint8_t* is_leaf, int32_t n_subgrids,
                            const otfmm_work_item* items, int32_t n_items, long long per_class[4]) {
    if (!ctx || !is_leaf || (!items && n_items > 0) || n_items < 0) return fail(OTFMM_ERR_INVALID, "bad arguments");
    long long cls[4] = {0, 0, 0, 0};
    // partners per cell of each parity, and per cell the offsets by direction
    for (int i = 0; i < n_items; ++i) {
        const otfmm_work_item& w = items[i];
        if (w.subgrid < 0 || w.subgrid >= n_subgrids || w.kind < 0 || w.kind > 2)
            return fail(OTFMM_ERR_INVALID, "work item out of range");
        if (w.kind == OTFMM_KIND_M2L_ROOT) {
            long long n = 0;
            for (int c = 0; c < NCELL; ++c)
                for (int q = 0; q < NCELL; ++q) {
                    const int sx = (q >> 6) - (c >> 6), sy = ((q >> 3) & 7) - ((c >> 3) & 7), sz = (q & 7) - (c & 7);
                    if (std::abs(sx) <= SMAX && std::abs(sy) <= SMAX && std::abs(sz) <= SMAX) {
                        const int idx = (sx + SMAX) * SINX * SINX + (sy + SMAX) * SINX + (sz + SMAX);
                        if (!ctx->st.phase[idx] || (sx == 0 && sy == 0 && sz == 0)) continue;
                    }
                    ++n;
                }
            cls[1] += n;
            continue;
        }
        long long per_cell = 0;
        for (int p = 0; p < 8; ++p) per_cell += ctx->counts[p];
        const long long stencil_pairs = per_cell * (NCELL / 8);
        if (w.kind == OTFMM_KIND_M2L) {
            cls[0] += stencil_pairs;
            continue;
        }
        cls[2] += stencil_pairs;
        // P2M: stencil partners that fall into a refined neighbour
        uint32_t refmask = 0;
        for (int d = 0; d < 26; ++d) {
            const int nb = w.neighbors[d];
            if (nb < -1 || nb >= n_subgrids) return fail(OTFMM_ERR_INVALID, "neighbour out of range");
            if (nb >= 0 && !is_leaf[nb]) refmask |= 1u << (d < 13 ? d : d + 1);
        }
        if (!refmask) continue;
        for (int c = 0; c < NCELL; ++c) {
            const int cx = c >> 6, cy = (c >> 3) & 7, cz = c & 7;
            const int p = ((cx & 1) << 2) | ((cy & 1) << 1) | (cz & 1);
            // host copy of the entry offsets (same order and filter as the device table)
            for (int sx = -SMAX; sx <= SMAX; ++sx)
                for (int sy = -SMAX; sy <= SMAX; ++sy)
                    for (int sz = -SMAX; sz <= SMAX; ++sz) {
                        const int idx = (sx + SMAX) * SINX * SINX + (sy + SMAX) * SINX + (sz + SMAX);
                        if (!ctx->st.mask[idx]) continue;
                        const int a = coarse_of(cx + INX) - coarse_of(cx + INX + sx);
                        const int b = coarse_of(cy + INX) - coarse_of(cy + INX + sy);
                        const int cc = coarse_of(cz + INX) - coarse_of(cz + INX + sz);
                        if (!(double(a * a + b * b + cc * cc) < (1.0 / ctx->theta) * (1.0 / ctx->theta))) continue;
                        const int ax = cx + sx, ay = cy + sy, az = cz + sz;
                        const int raw = ((ax >> 3) + 1) + 3 * ((ay >> 3) + 1) + 9 * ((az >> 3) + 1);
                        if ((refmask >> raw) & 1u) ++cls[3];
                    }
            (void)p;
        }
    }
    if (per_class)
        for (int c = 0; c < 4; ++c) per_class[c] = cls[c];
    return cls[0] + cls[1] + cls[2] + cls[3];
}

int otfmm_batch_status(otfmm_context* ctx, void* stream) {
    if (!ctx) return fail(OTFMM_ERR_INVALID, "NULL context");
    DeviceGuard g(ctx->device);
    int h = 0;
    OT_CUDA(cudaMemcpyAsync(&h, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    OT_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if (h) return fail(OTFMM_ERR_DEVICE, "a work item failed validation on the device");
    return OTFMM_OK;
}

int otfmm_device_alloc(otfmm_context* ctx, size_t bytes, void** ptr) {
    if (!ctx || !ptr) return fail(OTFMM_ERR_INVALID, "NULL argument");
    DeviceGuard g(ctx->device);
    OT_CUDA(cudaMalloc(ptr, bytes));
    return OTFMM_OK;
}

int otfmm_device_free(void* ptr) {
    OT_CUDA(cudaFree(ptr));
    return OTFMM_OK;
}

int otfmm_copy_to_device(otfmm_context* ctx, void* dst, const void* src, size_t bytes) {
    if (!ctx || !dst || !src) return fail(OTFMM_ERR_INVALID, "NULL argument");
    DeviceGuard g(ctx->device);
    OT_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    return OTFMM_OK;
}

int otfmm_copy_to_host(otfmm_context* ctx, void* dst, const void* src, size_t bytes) {
    if (!ctx || !dst || !src) return fail(OTFMM_ERR_INVALID, "NULL argument");
    DeviceGuard g(ctx->device);
    OT_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
    return OTFMM_OK;
}

int otfmm_measure_fma_peaks(int device, double* fp64_tflops, double* fp32_tflops) {
    if (!fp64_tflops || !fp32_tflops) return fail(OTFMM_ERR_INVALID, "NULL argument");
    DeviceGuard g(device);
    int sms = 0;
    OT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int blocks = sms * 8, threads = 256, iters = 4096;
    void* out = nullptr;
    OT_CUDA(cudaMalloc(&out, sizeof(double) * blocks * threads));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const double fmas = double(blocks) * threads * iters * 16 * 8;
    float best64 = 1e30f, best32 = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        float ms = 0;
        cudaEventRecord(e0);
        fma_probe_kernel<double><<<blocks, threads>>>((double*)out, iters, 0.999999, 1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) best64 = std::min(best64, ms);
        cudaEventRecord(e0);
        fma_probe_kernel<float><<<blocks, threads>>>((float*)out, iters, 0.999999f, 1e-7f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) best32 = std::min(best32, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    OT_CUDA(cudaGetLastError());
    *fp64_tflops = 2.0 * fmas / (best64 * 1e-3) / 1e12;
    *fp32_tflops = 2.0 * fmas / (best32 * 1e-3) / 1e12;
    return OTFMM_OK;
}

}   // extern "C"
