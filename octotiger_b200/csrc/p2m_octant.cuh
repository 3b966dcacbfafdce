// P2M (leaf targets, refined-neighbour multipole partners) by octant, reach 1:
// the fast FP64 form and the FP32-split form (derivative tensor and the
// contraction into L0..L3 in FP32; pair geometry and the angular correction
// L_c in FP64).
// Part of libotfmm.so; included once, in order, by otfmm.cu (one translation unit).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/otfmm.h"
#include "layout.cuh"
#include "leaf_kernels.cuh"
#include "m2l_tiles.cuh"
#include "pair_math.cuh"

namespace otfmm {

// Work unit: one octant (4x4x4 cells, 8 coarse cells) of a leaf with a
// refined neighbour in at least one of the 7 directions that face it
// (classify_kernel lists them; octants that face a refined neighbour across a
// face first). Every target cell belongs to exactly one unit, which forms its
// whole P2M sum, so no partial crosses units and the result does not depend
// on the schedule.
//   * the partner sub-slabs (Tables::po_box: the part of a refined
//     neighbour's 2-cell slab that the octant's cells reach) of the octant's
//     refined directions are staged once, in units of dx from the leaf's
//     origin, with the fast form's factors folded into the moments;
//   * the octant's coarse cells with partners go to the 4 warps in turn;
//     lane = 8 f + c: cell c of the coarse cell (whose 8 cells share one
//     partner list per direction) and partner stride f (partners f, f + 4, ...
//     of each list), so the 8 lanes of a cell read one partner together and a
//     warp has no divergence;
//   * directions in raw order, partners in list order; the four strides are
//     added by a fixed butterfly; the unit adds the sum to the P2P result in L
//     and writes L_c of its cells with partners.
// 128-thread CTAs, four per SM (shared memory and 124 registers allow four).
// Split form: FP32 sums promoted to FP64 after each direction (at most 18
// partners in FP32).
constexpr int PO_THREADS = 128;
constexpr int PO_CTAS_PER_SM = 4;
constexpr int PO_CELLS = 296;                    // sub-slabs of 3 faces (2x6x6), 3 edges (2x2x6), a corner
constexpr int PO_ROW_BYTES = 192;                // staged bytes of one slab cell
constexpr int PO_SMEM_BYTES = PO_CELLS * PO_ROW_BYTES;   // 56832
static_assert(PO_CTAS_PER_SM * (PO_SMEM_BYTES + 1024 + 256) <= 233472, "four CTAs per SM");

// FP32-split pair: target at X (units of dx, FP64), partner slab cell v.
// Rows: sf = (Q0..Q3), (Q4, Q5, -O0, -O1), (-O2..-O5), (-O6..-O9), (m, -D0, -D1, -D2)
// and sd = (P0, P1), (P2, 0), (O0, O1) .. (O8, O9), with row stride PO_CELLS.
template <bool RHO>
__device__ __forceinline__ void p2m_split_pair(const double X[3], const float4* __restrict__ sf,
                                               const double2* __restrict__ sd, int v, float2& a0, float acc[3],
                                               double Lc[3]) {
    const double2 pa = sd[v], pb = sd[PO_CELLS + v];
    const double dX[3] = {X[0] - pa.x, X[1] - pa.y, X[2] - pb.x};
    float dXf[3], rsf;
    if (RHO) {
        FastDerivs f;
        fz_geometry(dX, dXf, f, &rsf);
        double h[10];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const double2 o = sd[(2 + k) * PO_CELLS + v];
            h[2 * k] = o.x;
            h[2 * k + 1] = o.y;
        }
        fz_upper(f, h, Lc);
    } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) dXf[c] = (float)dX[c];
        const float r2f = fmaxf(fmaf(dXf[0], dXf[0], fmaf(dXf[1], dXf[1], dXf[2] * dXf[2])), WS_R2_MIN);
        const float y0 = rsqrtf(r2f);
        rsf = fmaf(0.5f * y0, fmaf(-r2f * y0, y0, 1.0f), y0);
    }
    const float r2invf = rsf * rsf;
    const float d1 = rsf * r2invf;
    const float d2 = -3.0f * d1 * r2invf;
    const float d3 = -5.0f * d2 * r2invf;
    float D[20];
    d_tensor<float>(dXf, -rsf, d1, d2, d3, D);
    const float4 f0 = sf[v], f1 = sf[PO_CELLS + v], f2 = sf[2 * PO_CELLS + v], f3 = sf[3 * PO_CELLS + v],
                 f4 = sf[4 * PO_CELLS + v];
    // L0 = m D0 + sum Q_q D_(4+q) - sum O_o D_(10+o) (- sum D_a D_(1+a)), two packed partial sums
    float2 s = __ffma2_rn(make_float2(f0.x, f0.y), make_float2(D[4], D[5]), a0);
    s = __ffma2_rn(make_float2(f0.z, f0.w), make_float2(D[6], D[7]), s);
    s = __ffma2_rn(make_float2(f1.x, f1.y), make_float2(D[8], D[9]), s);
    s = __ffma2_rn(make_float2(f1.z, f1.w), make_float2(D[10], D[11]), s);
    s = __ffma2_rn(make_float2(f2.x, f2.y), make_float2(D[12], D[13]), s);
    s = __ffma2_rn(make_float2(f2.z, f2.w), make_float2(D[14], D[15]), s);
    s = __ffma2_rn(make_float2(f3.x, f3.y), make_float2(D[16], D[17]), s);
    s = __ffma2_rn(make_float2(f3.z, f3.w), make_float2(D[18], D[19]), s);
    s.x = fmaf(f4.x, D[0], s.x);
    if (!RHO) {
        s.y = fmaf(f4.y, D[1], s.y);
        s.x = fmaf(f4.z, D[2], s.x);
        s.y = fmaf(f4.w, D[3], s.y);
    }
    a0 = s;
    // L_(1+a) = m D_(1+a) + sum Q_q D_(quad_axis(q, a)) (- D_a sum_b D_(quad_row(a, b)))
    const float Q[6] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float t = fmaf(f4.x, D[1 + a], acc[a]);
#pragma unroll
        for (int q = 0; q < 6; ++q) t = fmaf(Q[q], D[quad_axis(q, a)], t);
        if (!RHO) {
            const float md = a == 0 ? f4.y : a == 1 ? f4.z : f4.w;
#pragma unroll
            for (int b = 0; b < 3; ++b) t = fmaf(md, D[quad_row(a, b)], t);
        }
        acc[a] = t;
    }
}

// Fast FP64 pair on the same staging: rows (P0, P1), (P2, m), (Q0, Q1) ..
// (Q4, Q5), (O0, O1) .. (O8, O9), (D0, D1), (D2, 0).
template <bool RHO>
__device__ __forceinline__ void p2m_fast_pair(const double X[3], const double2* __restrict__ sd, int v,
                                              double L[4], double Lc[3]) {
    double mp[20], Y[3];
    const double2 pa = sd[v], pb = sd[PO_CELLS + v];
    Y[0] = pa.x;
    Y[1] = pa.y;
    Y[2] = pb.x;
    mp[0] = pb.y;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const double2 w = sd[(2 + k) * PO_CELLS + v];
        mp[4 + 2 * k] = w.x;
        mp[5 + 2 * k] = w.y;
    }
    if (!RHO) {
        const double2 w0 = sd[10 * PO_CELLS + v], w1 = sd[11 * PO_CELLS + v];
        mp[1] = w0.x;
        mp[2] = w0.y;
        mp[3] = w1.x;
    } else {
        mp[1] = mp[2] = mp[3] = 0.0;
    }
    fast_p2m_pair<RHO>(X, Y, mp, L, Lc);
}

// One staged sub-slab cell: scaled moments and the centre of mass in units
// of dx from the leaf's origin.
struct SlabCell {
    double m0, q[6], o[10], dp[3], P[3];
};

// Loads staged cell t of the unit (directions dirs, first cells cell0).
template <bool RHO>
__device__ __forceinline__ SlabCell load_slab_cell(const BatchArgs& a, const ItemInfo& it, int oct,
                                                   const int8_t* dirs, const int* cell0, int t, double inv_dx,
                                                   double inv2, double inv3) {
    int k = 0;
    while (cell0[k + 1] <= t) ++k;
    const int r = dirs[k], idx = t - cell0[k];
    const int4 lo = __ldg(a.t.po_box + (r * 8 + oct) * 2), n = __ldg(a.t.po_box + (r * 8 + oct) * 2 + 1);
    const int x = lo.x + idx / (n.y * n.z), y = lo.y + (idx / n.z) % n.y, z = lo.z + idx % n.z;
    const int uc = x * 64 + y * 8 + z;
    const size_t nb = (size_t)it.nb[r < 13 ? r : r - 1];
    const double* Ms = a.M + nb * 20 * NCELL + uc;
    SlabCell c;
    c.m0 = __ldg(Ms);
#pragma unroll
    for (int k2 = 0; k2 < 6; ++k2) c.q[k2] = __ldg(Ms + (4 + k2) * NCELL) * ((factor_of(4 + k2) / 2.0) * inv2);
#pragma unroll
    for (int k2 = 0; k2 < 10; ++k2) c.o[k2] = __ldg(Ms + (10 + k2) * NCELL) * ((factor_of(10 + k2) / 6.0) * inv3);
#pragma unroll
    for (int d = 0; d < 3; ++d) c.dp[d] = RHO ? 0.0 : __ldg(Ms + (1 + d) * NCELL) * inv_dx;
#pragma unroll
    for (int d = 0; d < 3; ++d) c.P[d] = (__ldg(a.com + (nb * 3 + d) * NCELL + uc) - it.xbase[d]) * inv_dx;
    return c;
}

// Writes staged cell t in the split rows (sf, sd) or the fast rows (sd).
template <bool SPLIT, bool RHO>
__device__ __forceinline__ void store_slab_cell(float4* sf, double2* sd, int t, const SlabCell& c) {
    if (SPLIT) {
        sf[t] = make_float4((float)c.q[0], (float)c.q[1], (float)c.q[2], (float)c.q[3]);
        sf[PO_CELLS + t] = make_float4((float)c.q[4], (float)c.q[5], (float)-c.o[0], (float)-c.o[1]);
        sf[2 * PO_CELLS + t] = make_float4((float)-c.o[2], (float)-c.o[3], (float)-c.o[4], (float)-c.o[5]);
        sf[3 * PO_CELLS + t] = make_float4((float)-c.o[6], (float)-c.o[7], (float)-c.o[8], (float)-c.o[9]);
        sf[4 * PO_CELLS + t] = make_float4((float)c.m0, (float)-c.dp[0], (float)-c.dp[1], (float)-c.dp[2]);
        sd[t] = make_double2(c.P[0], c.P[1]);
        sd[PO_CELLS + t] = make_double2(c.P[2], 0.0);
        if (RHO) {
#pragma unroll
            for (int k = 0; k < 5; ++k) sd[(2 + k) * PO_CELLS + t] = make_double2(c.o[2 * k], c.o[2 * k + 1]);
        }
    } else {
        sd[t] = make_double2(c.P[0], c.P[1]);
        sd[PO_CELLS + t] = make_double2(c.P[2], c.m0);
#pragma unroll
        for (int k = 0; k < 3; ++k) sd[(2 + k) * PO_CELLS + t] = make_double2(c.q[2 * k], c.q[2 * k + 1]);
#pragma unroll
        for (int k = 0; k < 5; ++k) sd[(5 + k) * PO_CELLS + t] = make_double2(c.o[2 * k], c.o[2 * k + 1]);
        if (!RHO) {
            sd[10 * PO_CELLS + t] = make_double2(c.dp[0], c.dp[1]);
            sd[11 * PO_CELLS + t] = make_double2(c.dp[2], 0.0);
        }
    }
}

template <int PREC, bool RHO>
__global__ void __launch_bounds__(PO_THREADS, PO_CTAS_PER_SM) p2m_octant_kernel(BatchArgs a) {
    extern __shared__ __align__(16) unsigned char po_dyn[];
    constexpr bool SPLIT = (PREC == PREC_SPLIT);
    // split: 5 float4 rows, then 7 double2 rows; fast: 12 double2 rows
    float4* sf = reinterpret_cast<float4*>(po_dyn);
    double2* sd = reinterpret_cast<double2*>(po_dyn + (SPLIT ? 5 * PO_CELLS * 16 : 0));
    __shared__ ItemInfo it;
    __shared__ int s_unit, s_nr, s_ncc;
    __shared__ int8_t s_rdir[8];          // the octant's refined directions, in raw order
    __shared__ int s_rcell[9];            // their first staged cell
    __shared__ int8_t s_cc[8];            // the octant's coarse cells with partners there
    const int n_front = a.wl.counts[WL_P2M_UNITS], total = n_front + a.wl.counts[WL_P2M_UNITS_BACK];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int f = lane >> 3, ci = lane & 7;
    for (;;) {
        __syncthreads();   // `it`, the direction tables and the slabs are reused
        if (threadIdx.x == 0) s_unit = atomicAdd(a.wl.counts + WL_P2M_NEXT, 1);
        __syncthreads();
        const int u = s_unit;
        if (u >= total) break;
        const int unit = (u < n_front) ? a.wl.p2m_units[u] : a.wl.p2m_units[a.wl.unit_cap - 1 - (u - n_front)];
        const int oct = unit & 7;
        load_item(a, (int)((unsigned)unit >> 3), it);
        if (warp == 0) {
            // lane l < n: the l-th refined direction facing the octant (raw
            // order) and where its sub-slab starts
            const uint32_t m = it.nbmask & ~it.leafmask & c_octant_dirs[oct];
            const int n = __popc(m);
            int r = 0, incl = 0;
            if (lane < n) {
                r = (int)__fns(m, 0, lane + 1);
                incl = __ldg(a.t.po_box + (r * 8 + oct) * 2).w;
            }
#pragma unroll
            for (int o = 1; o < 8; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane < n) {
                s_rdir[lane] = (int8_t)r;
                s_rcell[lane + 1] = incl;
            }
            // lane w < 8: coarse cell w of the octant, if it has partners there
            const int C = (2 * (oct & 1) + (lane & 1)) * 16 + (2 * ((oct >> 1) & 1) + ((lane >> 1) & 1)) * 4 +
                          2 * ((oct >> 2) & 1) + ((lane >> 2) & 1);
            bool any = false;
            for (int k = 0; k < n; ++k) {
                const int rk = __shfl_sync(0xffffffffu, r, k);
                if (lane < 8) {
                    const int2 be = __ldg(a.t.po_range + rk * 64 + C);
                    any |= be.y > be.x;
                }
            }
            const unsigned act = __ballot_sync(0xffffffffu, lane < 8 && any);
            if (lane < 8 && any) s_cc[__popc(act & ((1u << lane) - 1u))] = (int8_t)C;
            if (lane == 0) {
                s_rcell[0] = 0;
                s_nr = n;
                s_ncc = __popc(act);
            }
        }
        __syncthreads();
        const int nr = s_nr;
        const size_t sub = (size_t)it.subgrid;
        const double inv_dx = 1.0 / it.dx, inv2 = inv_dx * inv_dx, inv3 = inv2 * inv_dx;
        // stage the sub-slabs (scaled, in units of dx from the leaf's origin)
        for (int t = threadIdx.x; t < s_rcell[nr]; t += PO_THREADS)
            store_slab_cell<SPLIT, RHO>(sf, sd, t, load_slab_cell<RHO>(a, it, oct, s_rdir, s_rcell, t, inv_dx, inv2, inv3));
        __syncthreads();
        for (int j = warp; j < s_ncc; j += PO_THREADS / 32) {
            const int C = s_cc[j];
            const int cu = (2 * (C >> 4) + (ci & 1)) * 64 + (2 * ((C >> 2) & 3) + ((ci >> 1) & 1)) * 8 +
                           (2 * (C & 3) + (ci >> 2));
            double X[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) X[c] = (__ldg(a.com + (sub * 3 + c) * NCELL + cu) - it.xbase[c]) * inv_dx;
            double acc[4] = {0.0, 0.0, 0.0, 0.0}, corr[3] = {0.0, 0.0, 0.0};
            for (int k = 0; k < nr; ++k) {
                const int2 be = __ldg(a.t.po_range + s_rdir[k] * 64 + C);
                if (SPLIT) {
                    const float4* sfk = sf + s_rcell[k];
                    const double2* sdk = sd + s_rcell[k];
                    float2 a0 = make_float2(0.0f, 0.0f);
                    float a13[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll 2
                    for (int q = be.x + f; q < be.y; q += 4)
                        p2m_split_pair<RHO>(X, sfk, sdk, __ldg(a.t.po_list + q), a0, a13, corr);
                    acc[0] += (double)a0.x + (double)a0.y;
#pragma unroll
                    for (int c = 0; c < 3; ++c) acc[1 + c] += (double)a13[c];
                } else {
                    const double2* sdk = sd + s_rcell[k];
#pragma unroll 2
                    for (int q = be.x + f; q < be.y; q += 4)
                        p2m_fast_pair<RHO>(X, sdk, __ldg(a.t.po_list + q), acc, corr);
                }
            }
            // the four partner strides of a cell, in a fixed order
#pragma unroll
            for (int o = 8; o <= 16; o <<= 1) {
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
#pragma unroll
                for (int q = 0; q < 3; ++q) corr[q] += __shfl_xor_sync(0xffffffffu, corr[q], o);
            }
            if (f == 0) {
                // back to physical units: L0 dx^-1, L1..L3 dx^-2, L_c dx^-2
                double* L = a.L + sub * 20 * NCELL + cu;
                double* Lc = a.Lc + sub * 3 * NCELL + cu;
                L[0] += acc[0] * inv_dx;
#pragma unroll
                for (int q = 1; q < 4; ++q) L[q * NCELL] += acc[q] * inv2;
#pragma unroll
                for (int q = 0; q < 3; ++q) Lc[q * NCELL] = RHO ? corr[q] * inv2 : 0.0;
            }
        }
    }
}

}   // namespace otfmm
