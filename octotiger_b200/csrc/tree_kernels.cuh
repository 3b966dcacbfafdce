// Tree passes of a gravity solve: upward M2M and downward L2L with the
// leaves' gravity output, one launch per octree level.
// Part of libotfmm.so; included once, in order, by otfmm.cu (one translation unit).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/otfmm.h"
#include "pair_math.cuh"
#include "layout.cuh"

namespace otfmm {

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

}   // namespace otfmm
