// Layout of the FMM interaction kernels: reference constants (GRIDDIM 8), the
// tile geometry and shared-memory layouts, the per-context stencil tables, and
// the batched-solve arguments with the device-side work lists and the work-item
// classification kernel.
// Part of libotfmm.so; included once, in order, by otfmm.cu (one translation unit).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

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
constexpr int MAX_ENTRIES = 216;           // 6^3 - 1 partners per cell at most (coarse reach 1)
constexpr int MAX_ENTRIES_R2 = 1000;       // partners per cell at most for theta >= 0.34 (coarse reach 2)
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
// The same constants rounded to FP32 (the split P2P of theta < 0.5 reads them by
// stencil index, warp-uniformly).
__constant__ float4 c_four_f[FULL];

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
    const int2* entries_r2;     // [8][MAX_ENTRIES_R2]: stencil-order entries of any reach (x = plane delta,
                                // y = packed)
    const int* r2_sx_start;     // [8][12]: first entry of each sx = -5 .. 5 in entries_r2 (and the end)
    const double4* r2_four;     // [8][MAX_ENTRIES_R2]: monopole constants of the entries_r2 offsets
    const double4* p2p_box;     // [8][216]: per parity, monopole constants over the 6^3 partner box (box
                                // position (i, j, k) = offset + 2 + parity), zero off the stencil and at the cell
    const double4* p2p_cube;    // [343]: monopole constants of the offsets -3..3 per axis, zero at the centre
    // P2M by coarse cell (reach 1): the 8 cells of a coarse cell share their partners in a direction
    const int* pc_unit_start;   // [28]: first unit (4 coarse cells) of raw direction r
    const int16_t* pc_coarse;   // [units][4]: coarse cell (x 16 + y 4 + z) of each unit slot, -1 past the end
    const int2* pc_range;       // [27][64]: partner range in pc_list of coarse cell C in direction r
    const uint16_t* pc_list;    // partner cells as indices into the direction's slab (see pc_slab_shape),
                                // stencil order of the coarse cell's first cell
    const int16_t* pc_slot;     // [27][64]: slot of coarse cell C among direction r's units, -1 if none
    const int* pc_parts;        // [27]: parts each unit's partner lists of direction r are cut in
    const int* r2_p2p_delta;    // [8][MAX_ENTRIES_R2]: each entries_r2 partner's offset in the split reach-2 P2P
                                // halo << 11 | its stencil index
    // P2M by octant (reach 1)
    const int4* po_box;         // [27][8][2]: sub-slab of direction r for octant o: (low x, y, z, cells), (extents)
    const int2* po_range;       // [27][64]: partner range in po_list of coarse cell C in direction r
    const uint16_t* po_list;    // partner cells as indices into the sub-slab of (r, octant of C)
    const int2* entries_r2s;    // entries_r2 with each sx group's full-multipole entries first
    const int* r2s_far_end;     // [8][11]: end of each sx group's full-multipole entries in entries_r2s
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
    uint32_t leafmask;   // raw directions (13 = centre, never set) whose neighbour is a leaf
    uint32_t nbmask;     // raw directions with a neighbour
};


// ---------------------------------------------------------------- kernels
// Device-side work lists, filled by classify_kernel: item indices per kind
// and the counters the persistent launches take their tiles from.
enum : int {
    WL_M2L = 0,
    WL_LEAF = 1,
    WL_P2M = 2,
    WL_M2L_NEXT = 3,
    WL_P2M_NEXT = 4,
    WL_ROOT = 5,
    WL_LEAF_NEXT = 6,
    WL_P2M_UNITS = 7,        // P2M octant units listed from the front of p2m_units
    WL_P2M_UNITS_BACK = 8,   // ... and from its back
    WL_COUNTERS = 10
};
struct WorkLists {
    int* m2l;        // refined, non-root items
    int* root;       // level-0 items
    int* leaf;       // leaf items
    int* p2m;        // leaf items with a refined neighbour
    int* counts;     // WL_* counters
    int* p2m_units;  // P2M octant units (item << 3 | octant), unit_cap entries
    int unit_cap;
};
// Work-list storage (ints) for a capacity of cap items: four item lists, the
// counters, 8 P2M octant units per item.
constexpr size_t work_list_ints(size_t cap) { return 12 * cap + WL_COUNTERS; }
__host__ __device__ inline WorkLists work_lists(int* base, size_t cap) {
    return WorkLists{base, base + cap, base + 2 * cap, base + 3 * cap, base + 4 * cap, base + 4 * cap + WL_COUNTERS,
                     (int)(8 * cap)};
}

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

// Raw-direction bit mask (bit 13, the centre, left out) of 26 per-direction flags.
__device__ __forceinline__ uint32_t raw_bits(uint32_t dirbits) {
    return (dirbits & 0x1fffu) | ((dirbits >> 13) << 14);
}

// Raw directions (bit r, centre excluded) facing octant o = sx + 2 sy + 4 sz
// of a subgrid (4x4x4 cells): every offset component is 0 or points out of
// the octant's side.
__host__ __device__ constexpr uint32_t octant_dirs(int o) {
    uint32_t m = 0;
    for (int r = 0; r < 27; ++r) {
        const int d[3] = {r % 3 - 1, (r / 3) % 3 - 1, r / 9 - 1};
        bool ok = (r != 13);
        for (int c = 0; c < 3; ++c) {
            const int s = (o >> c) & 1;
            ok = ok && (d[c] == 0 || d[c] == 2 * s - 1);
        }
        if (ok) m |= 1u << r;
    }
    return m;
}
__constant__ uint32_t c_octant_dirs[8] = {octant_dirs(0), octant_dirs(1), octant_dirs(2), octant_dirs(3),
                                          octant_dirs(4), octant_dirs(5), octant_dirs(6), octant_dirs(7)};
// Raw directions across a face (one non-zero offset component).
constexpr uint32_t FACE_DIRS = (1u << 4) | (1u << 10) | (1u << 12) | (1u << 14) | (1u << 16) | (1u << 22);

// Reserves n slots of a list for each lane of a full warp with one atomic
// (lanes in order): returns the lane's first slot.
__device__ __forceinline__ int warp_reserve(int* counter, int n) {
    const int lane = threadIdx.x & 31;
    int incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    int base = 0;
    if (lane == 31 && incl > 0) base = atomicAdd(counter, incl);
    return __shfl_sync(0xffffffffu, base, 31) + incl - n;
}

// One thread per work item (blocks of whole warps): validates it (a malformed
// item raises the error flag and is dropped before anything reads with its
// fields) and appends it to the list of its kind, one atomic per warp and
// list. A leaf with refined neighbours also goes to the P2M list, with its
// P2M octant units (unit = item << 3 | octant, item < 2^27): the octants
// facing a refined neighbour across a face from the front of p2m_units, the
// others from its back (the P2M kernel takes the front ones first).
__global__ void classify_kernel(BatchArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int kind = -1;
    uint32_t refmask = 0;
    if (i < a.n_items) {
        const otfmm_work_item& w = a.items[i];
        if (!item_valid(a, w)) {
            atomicOr(a.err, 1);
        } else {
            kind = w.kind;
            if (kind == OTFMM_KIND_LEAF) {
                uint32_t refined = 0;
                for (int d = 0; d < 26; ++d)
                    if (w.neighbors[d] >= 0 && !a.is_leaf[w.neighbors[d]]) refined |= 1u << d;
                refmask = raw_bits(refined);
            }
        }
    }
    const int s_m2l = warp_reserve(a.wl.counts + WL_M2L, kind == OTFMM_KIND_M2L);
    const int s_root = warp_reserve(a.wl.counts + WL_ROOT, kind == OTFMM_KIND_M2L_ROOT);
    const int s_leaf = warp_reserve(a.wl.counts + WL_LEAF, kind == OTFMM_KIND_LEAF);
    const int s_p2m = warp_reserve(a.wl.counts + WL_P2M, refmask != 0);
    if (kind == OTFMM_KIND_M2L) a.wl.m2l[s_m2l] = i;
    if (kind == OTFMM_KIND_M2L_ROOT) a.wl.root[s_root] = i;
    if (kind == OTFMM_KIND_LEAF) a.wl.leaf[s_leaf] = i;
    if (refmask) a.wl.p2m[s_p2m] = i;
    uint32_t front = 0, back = 0;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const uint32_t m = refmask & c_octant_dirs[o];
        if (m & FACE_DIRS) front |= 1u << o;
        else if (m) back |= 1u << o;
    }
    int sf = warp_reserve(a.wl.counts + WL_P2M_UNITS, __popc(front));
    int sb = warp_reserve(a.wl.counts + WL_P2M_UNITS_BACK, __popc(back));
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const int unit = (int)(((unsigned)i << 3) | (unsigned)o);
        if ((front >> o) & 1u) a.wl.p2m_units[sf++] = unit;
        if ((back >> o) & 1u) a.wl.p2m_units[a.wl.unit_cap - 1 - sb++] = unit;
    }
}


// Copies an item (already validated by classify_kernel) into shared memory:
// the first warp, one lane per direction, with the leaf / neighbour masks.
__device__ __forceinline__ void load_item(const BatchArgs& a, int item_idx, ItemInfo& it) {
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        const otfmm_work_item& w = a.items[item_idx];
        int nb = -1;
        if (lane < 26) {
            nb = w.neighbors[lane];
            it.nb[lane] = nb;
        }
        const bool leaf = nb >= 0 && a.is_leaf[nb] != 0;
        const uint32_t lb = __ballot_sync(0xffffffffu, leaf), eb = __ballot_sync(0xffffffffu, nb >= 0);
        if (lane == 0) {
            it.subgrid = w.subgrid;
            it.kind = w.kind;
            it.dx = w.dx;
            for (int q = 0; q < 3; ++q) it.xbase[q] = w.xbase[q];
            it.leafmask = raw_bits(lb);
            it.nbmask = raw_bits(eb);
        }
    }
    __syncthreads();
}

}   // namespace otfmm
