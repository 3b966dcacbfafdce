// TEST INFRASTRUCTURE ONLY — not part of the product path.
//
// CPU restatement of the two tree passes around Octo-Tiger's interaction
// kernels (the oracle for the device upward / downward passes):
//   * upward (M2M), grid::compute_multipoles (src/grid_fmm.cpp:1639-1803) with
//     the octant gather of node_server::compute_fmm (src/node_server.cpp:613-636):
//     per node, the centres of mass of the 64 coarse cells (RHO) and the child
//     multipoles shifted to them (taylor::operator>>=, octotiger/taylor.hpp:222-255)
//     and summed, written into the parent's cells of this node's octant;
//   * downward (L2L), grid::compute_expansions (src/grid_fmm.cpp:1525-1637) with
//     the octant scatter of node_server (src/node_server.cpp:760-786): every
//     fine cell adds its parent cell's expansion shifted to the cell's centre of
//     mass (taylor::operator<<=, octotiger/taylor.hpp:263-318) and the parent's
//     L_c; leaves turn L, L_c into the gravity output.
// The shift operators are a template policy, so the same loops run with the
// scalar restatement (otfmm_oracle.cpp) and with the reference's own taylor<4>
// (ref_driver.cpp). Sums over the 8 children of a coarse cell run child 0..7 in
// order (the reference sums SIMD lanes; its lane order is the library's).
#pragma once

#include <cstdint>

namespace ora {

// One node of the octree for the tree passes (48 bytes).
struct TreeNode {
    int32_t subgrid;   // pool index of this node
    int32_t parent;    // pool index of the parent, -1 for the root
    int32_t octant;    // this node's octant in its parent: x + 2 y + 4 z (geo::octant)
    int32_t reserved;
    double dx;         // cell size
    double xbase[3];   // centre of inner cell (0,0,0)
};
static_assert(sizeof(TreeNode) == 48, "tree node layout");

struct TreePool {
    double* M;          // [n][20][512]
    double* com;        // [n][3][512]
    const double* mon;  // [n][512]
    const uint8_t* is_leaf;
    double* com1;       // [n][3][64]: centres of mass of each node's 4^3 coarse cells
    int32_t n;
};

constexpr int TP_NCELL = 512;
constexpr int TP_NCOARSE = 64;

// Fine cell of coarse cell (ip, jp, kp) and child ci (grid_fmm.cpp:1690-1695).
inline int tp_child(int ip, int jp, int kp, int ci) {
    return 64 * (2 * ip + (ci & 1)) + 8 * (2 * jp + ((ci >> 1) & 1)) + (2 * kp + ((ci >> 2) & 1));
}
// Cell of the parent's 8^3 grid that coarse cell (ip, jp, kp) of a child in octant o maps to.
inline int tp_parent_cell(int ip, int jp, int kp, int o) {
    return (ip + 4 * (o & 1)) * 64 + (jp + 4 * ((o >> 1) & 1)) * 8 + (kp + 4 * ((o >> 2) & 1));
}

// Upward pass of one node. Its own cells (M / com for refined nodes, mon for
// leaves) are complete: the children ran before.
template <class Shift>
void upward_node(const Shift& S, TreePool& P, const TreeNode& nd, bool rho) {
    const size_t s = (size_t)nd.subgrid;
    const bool leaf = P.is_leaf[s] != 0;
    double* M = P.M + s * 20 * TP_NCELL;
    double* com = P.com + s * 3 * TP_NCELL;
    const double* mon = P.mon + s * TP_NCELL;
    double* com1 = P.com1 + s * 3 * TP_NCOARSE;
    if (rho && leaf) {
        // leaf centres of mass: the cell centres x0 + i dx (grid_fmm.cpp:1659-1673)
        for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 8; ++j)
                for (int k = 0; k < 8; ++k) {
                    const int u = 64 * i + 8 * j + k;
                    com[0 * TP_NCELL + u] = nd.xbase[0] + i * nd.dx;
                    com[1 * TP_NCELL + u] = nd.xbase[1] + j * nd.dx;
                    com[2 * TP_NCELL + u] = nd.xbase[2] + k * nd.dx;
                }
    }
    for (int ip = 0; ip < 4; ++ip)
        for (int jp = 0; jp < 4; ++jp)
            for (int kp = 0; kp < 4; ++kp) {
                const int p = 16 * ip + 4 * jp + kp;
                if (rho) {
                    double mc[8], X[3][8];
                    for (int ci = 0; ci < 8; ++ci) {
                        const int c = tp_child(ip, jp, kp, ci);
                        mc[ci] = leaf ? mon[c] : M[c];
                        for (int d = 0; d < 3; ++d) X[d][ci] = com[d * TP_NCELL + c];
                    }
                    double mtot = mc[0];
                    for (int ci = 1; ci < 8; ++ci) mtot = mtot + mc[ci];
                    for (int d = 0; d < 3; ++d) {
                        double sx = X[d][0] * mc[0];
                        for (int ci = 1; ci < 8; ++ci) sx = sx + X[d][ci] * mc[ci];
                        com1[d * TP_NCOARSE + p] = sx / mtot;
                    }
                }
                double MM[20];
                for (int ci = 0; ci < 8; ++ci) {
                    const int c = tp_child(ip, jp, kp, ci);
                    double A[20], B[20], dx[3];
                    if (leaf) {
                        A[0] = mon[c];
                        for (int j = 1; j < 20; ++j) A[j] = 0.0;
                    } else {
                        for (int j = 0; j < 20; ++j) A[j] = M[j * TP_NCELL + c];
                    }
                    for (int d = 0; d < 3; ++d) dx[d] = com[d * TP_NCELL + c] - com1[d * TP_NCOARSE + p];
                    S.up(A, dx, B);
                    for (int j = 0; j < 20; ++j) MM[j] = (ci == 0) ? B[j] : MM[j] + B[j];
                }
                if (nd.parent >= 0) {
                    const size_t ps = (size_t)nd.parent;
                    const int io = tp_parent_cell(ip, jp, kp, nd.octant);
                    for (int j = 0; j < 20; ++j) P.M[(ps * 20 + j) * TP_NCELL + io] = MM[j];
                    if (rho)
                        for (int d = 0; d < 3; ++d) P.com[(ps * 3 + d) * TP_NCELL + io] = com1[d * TP_NCOARSE + p];
                }
            }
}

// Downward pass of one node: its parent's L / L_c are final (the parent ran
// before). L, L_c are [n][20][512] / [n][3][512]; G is [n][4][512]: for leaves
// (RHO) phi, g_x, g_y, g_z; (DRHODT) d phi / dt in slot 0.
template <class Shift>
void downward_node(const Shift& S, const TreePool& P, const TreeNode& nd, double* L, double* Lc, double* G,
                   double gconst, bool correct_am, bool rho) {
    const size_t s = (size_t)nd.subgrid;
    const bool leaf = P.is_leaf[s] != 0;
    const double* com = P.com + s * 3 * TP_NCELL;
    const double* com1 = P.com1 + s * 3 * TP_NCOARSE;
    double* Ls = L + s * 20 * TP_NCELL;
    double* Lcs = Lc + s * 3 * TP_NCELL;
    for (int ip = 0; ip < 4; ++ip)
        for (int jp = 0; jp < 4; ++jp)
            for (int kp = 0; kp < 4; ++kp) {
                const int p = 16 * ip + 4 * jp + kp;
                double l[20], lc[3] = {0.0, 0.0, 0.0};
                if (nd.parent >= 0) {
                    const size_t ps = (size_t)nd.parent;
                    const int io = tp_parent_cell(ip, jp, kp, nd.octant);
                    for (int j = 0; j < 20; ++j) l[j] = L[(ps * 20 + j) * TP_NCELL + io];
                    if (rho)
                        for (int d = 0; d < 3; ++d) lc[d] = Lc[(ps * 3 + d) * TP_NCELL + io];
                } else {
                    for (int j = 0; j < 20; ++j) l[j] = 0.0;
                }
                for (int ci = 0; ci < 8; ++ci) {
                    const int c = tp_child(ip, jp, kp, ci);
                    double dX[3], B[20];
                    for (int d = 0; d < 3; ++d) dX[d] = com[d * TP_NCELL + c] - com1[d * TP_NCOARSE + p];
                    S.down(l, dX, B);
                    for (int j = 0; j < 20; ++j) Ls[j * TP_NCELL + c] = Ls[j * TP_NCELL + c] + B[j];
                    if (rho)
                        for (int d = 0; d < 3; ++d) Lcs[d * TP_NCELL + c] = Lcs[d * TP_NCELL + c] + lc[d];
                }
            }
    if (leaf) {
        double* Gs = G + s * 4 * TP_NCELL;
        for (int u = 0; u < TP_NCELL; ++u) {
            if (rho) {
                Gs[u] = gconst * Ls[u];
                for (int d = 0; d < 3; ++d) {
                    double g = -gconst * Ls[(1 + d) * TP_NCELL + u];
                    if (correct_am) g = g - gconst * Lcs[d * TP_NCELL + u];
                    Gs[(1 + d) * TP_NCELL + u] = g;
                }
            } else {
                Gs[u] = gconst * Ls[u];
            }
        }
    }
}

// Whole passes: nodes sorted by level (root first), level l in
// [level_start[l], level_start[l + 1]).
template <class Shift>
void upward_pass(const Shift& S, TreePool& P, const TreeNode* nodes, const int32_t* level_start, int n_levels,
                 bool rho) {
    for (int l = n_levels - 1; l >= 0; --l)
        for (int i = level_start[l]; i < level_start[l + 1]; ++i) upward_node(S, P, nodes[i], rho);
}

template <class Shift>
void downward_pass(const Shift& S, const TreePool& P, const TreeNode* nodes, const int32_t* level_start, int n_levels,
                   double* L, double* Lc, double* G, double gconst, bool correct_am, bool rho) {
    for (int l = 0; l < n_levels; ++l)
        for (int i = level_start[l]; i < level_start[l + 1]; ++i)
            downward_node(S, P, nodes[i], L, Lc, G, gconst, correct_am, rho);
}

}   // namespace ora
