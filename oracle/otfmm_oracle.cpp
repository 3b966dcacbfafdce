// TEST INFRASTRUCTURE ONLY — the oracle. Never linked into the product path.
//
// Scalar FP64 restatement of Octo-Tiger's FMM cell-interaction kernels:
//   * pair arithmetic of octotiger/multipole_interactions/kernel/compute_kernel_templates.hpp:67-391
//     and octotiger/monopole_interactions/kernel/monopole_kernel_templates.hpp:16-239,
//     with the same operation order (built with -ffp-contract=off, so every
//     product and sum is rounded exactly where the reference rounds it);
//   * the sweeps of the Kokkos host kernels
//     (octotiger/multipole_interactions/kernel/kokkos_kernel.hpp:137-321 rho,
//     :324-471 root rho, :474-633 non-rho, :637-764 root non-rho;
//     octotiger/monopole_interactions/kernel/kokkos_kernel.hpp:143-320 P2P,
//     :517-709 P2M non-rho, :711-942 P2M rho), one cell at a time, partners
//     in the same (x, y, z) stencil order, so the accumulation order matches;
//   * staging and the work-list driver from oracle_core.hpp.
// Parity is pinned against the reference's own templates compiled by
// oracle/build_ref.sh (bit-for-bit) and against the committed golden vectors.
#include "oracle_core.hpp"
#include "tree_passes.hpp"

namespace ora {
namespace {

constexpr double kFactor[20] = {1, 1, 1, 1, 1, 2, 2, 1, 2, 1, 1, 3, 3, 3, 6, 3, 1, 3, 3, 1};
// Octupole index reached from quadrupole q (0..5 for 4..9) along axis a.
constexpr int kQuadAxis[6][3] = {{10, 11, 12}, {11, 13, 14}, {12, 14, 15},
                                 {13, 16, 17}, {14, 17, 18}, {15, 18, 19}};
// Quadrupole index of (axis a, axis b): row a of the symmetric 3x3 map.
constexpr int kQuadRow[3][3] = {{4, 5, 6}, {5, 7, 8}, {6, 8, 9}};
// Angular-correction operand of D_upper per (octupole k-10, output j).
constexpr int kUpperIdx[10][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}, {3, 6, 7}, {4, 7, 8},
                                  {5, 8, 9}, {6, 10, 11}, {7, 11, 12}, {8, 12, 13}, {9, 13, 14}};

struct Derivs {
    double d2, d3, X00, X11, X22;
    double D[20];
};

// compute_d_factors (compute_kernel_templates.hpp:67-139)
inline void d_factors(const double dX[3], Derivs& f) {
    f.X00 = dX[0] * dX[0];
    f.X11 = dX[1] * dX[1];
    f.X22 = dX[2] * dX[2];
    const double r2 = f.X00 + f.X11 + f.X22;
    const double r2inv = 1.0 / std::max(r2, 1.0e-20);
    const double d0 = -std::sqrt(r2inv);
    const double d1 = -d0 * r2inv;
    const double d2 = -3.0 * d1 * r2inv;
    const double d3 = -5.0 * d2 * r2inv;
    f.d2 = d2;
    f.d3 = d3;
    double* D = f.D;
    D[0] = d0;
    for (int a = 0; a < 3; ++a) D[1 + a] = dX[a] * d1;
    const double X12 = dX[1] * dX[2], X01 = dX[0] * dX[1], X02 = dX[0] * dX[2];
    D[4] = d2 * f.X00 + d1;
    D[5] = d2 * X01;
    D[6] = d2 * X02;
    D[7] = d2 * f.X11 + d1;
    D[8] = d2 * X12;
    D[9] = d2 * f.X22 + d1;
    const double d2x0 = d2 * dX[0], d2x1 = d2 * dX[1], d2x2 = d2 * dX[2];
    D[10] = d3 * f.X00 * dX[0] + 3.0 * d2x0;
    D[11] = d3 * f.X00 * dX[1] + d2x1;
    D[12] = d3 * f.X00 * dX[2] + d2x2;
    D[13] = d3 * dX[0] * f.X11 + d2x0;
    D[14] = d3 * dX[0] * X12;
    D[15] = d3 * dX[0] * f.X22 + d2x0;
    D[16] = d3 * f.X11 * dX[1] + 3.0 * d2x1;
    D[17] = d3 * f.X11 * dX[2] + d2x2;
    D[18] = d3 * dX[1] * f.X22 + d2x1;
    D[19] = d3 * f.X22 * dX[2] + 3.0 * d2x2;
}

// Fourth-order slice used by the angular correction
// (compute_kernel_templates.hpp:232-325; monopole_kernel_templates.hpp:75-179).
inline void d_upper(const Derivs& f, const double dX[3], double U[15]) {
    const double d2 = f.d2, d3 = f.d3;
    const double d3x00 = d3 * f.X00, d3x11 = d3 * f.X11, d3x22 = d3 * f.X22;
    const double d3x01 = d3 * dX[0] * dX[1], d3x02 = d3 * dX[0] * dX[2], d3x12 = d3 * dX[1] * dX[2];
    U[0] = dX[0] * dX[0] * d3 + 2.0 * d2;
    U[0] += d2;
    U[0] += 5.0 * d3x00;
    U[1] = 3.0 * d3x01;
    U[2] = 3.0 * d3x02;
    U[3] = d2;
    U[3] += d3x11;
    U[3] += d3x00;
    U[4] = d3x12;
    U[5] = d2;
    U[5] += d3x22;
    U[5] += d3x00;
    U[6] = 3.0 * d3x01;
    U[7] = d3x02;
    U[8] = d3x01;
    U[9] = 3.0 * d3x02;
    U[10] = dX[1] * dX[1] * d3 + 2.0 * d2;
    U[10] += d2;
    U[10] += 5.0 * d3x11;
    U[11] = 3.0 * d3x12;
    U[12] = d2;
    U[12] += d3x22;
    U[12] += d3x11;
    U[13] = 3.0 * d3x12;
    U[14] = dX[2] * dX[2] * d3 + 2.0 * d2;
    U[14] += d2;
    U[14] += 5.0 * d3x22;
}

inline void add_monopole_terms(const double m[20], const double D[20], double* L) {
    for (int a = 0; a < 4; ++a) L[a] += m[0] * D[a];
}

// Partner dipole block of compute_kernel_non_rho (:378-389) and
// compute_kernel_p2m_non_rho (monopole_kernel_templates.hpp:205-216).
inline void add_dipole_terms(const double m[20], const double D[20], double* L) {
    for (int a = 0; a < 3; ++a) {
        L[0] -= m[1 + a] * D[1 + a];
        for (int b = 0; b < 3; ++b) L[1 + a] -= m[1 + a] * D[kQuadRow[a][b]];
    }
}

// Quadrupole and octupole partner moments acting on L0..L3
// (compute_interaction_multipole_non_rho :144-183 / compute_interaction_p2m_non_rho).
inline void add_quad_oct_terms(const double m[20], const double D[20], double* L) {
    for (int q = 0; q < 6; ++q) {
        const int k = 4 + q;
        const double fh = kFactor[k] / 2.0;
        L[0] += m[k] * (D[k] * fh);
        for (int a = 0; a < 3; ++a) L[1 + a] += m[k] * (D[kQuadAxis[q][a]] * fh);
    }
    for (int k = 10; k < 20; ++k) L[0] -= m[k] * (D[k] * (kFactor[k] / 6.0));
}

// Higher local-expansion terms L4..L19 (:185-221).
inline void add_higher_terms(const double m[20], const double D[20], double* L) {
    for (int q = 0; q < 6; ++q) L[4 + q] += m[0] * D[4 + q];
    for (int a = 0; a < 3; ++a)
        for (int q = 0; q < 6; ++q) L[4 + q] -= m[1 + a] * D[kQuadAxis[q][a]];
    for (int o = 0; o < 10; ++o) L[10 + o] += m[0] * D[10 + o];
}

// compute_kernel_rho (:336-359) and compute_kernel_non_rho (:361-391)
inline void m2l_pair(const double X[3], const double Y[3], const double mp[20], const double mc[20],
                     double L[20], double Lc[3], bool rho) {
    const double dX[3] = {X[0] - Y[0], X[1] - Y[1], X[2] - Y[2]};
    Derivs f;
    d_factors(dX, f);
    add_monopole_terms(mp, f.D, L);
    if (!rho) add_dipole_terms(mp, f.D, L);
    add_quad_oct_terms(mp, f.D, L);
    add_higher_terms(mp, f.D, L);
    if (rho) {
        // compute_interaction_multipole_rho (:224-334)
        double U[15];
        d_upper(f, dX, U);
        const double n0 = mp[0] / mc[0];
        for (int k = 10; k < 20; ++k) {
            const double n0t = mp[k] - mc[k] * n0;
            const double f6 = kFactor[k] / 6.0;
            for (int j = 0; j < 3; ++j) Lc[j] -= n0t * (U[kUpperIdx[k - 10][j]] * f6);
        }
    }
}

// compute_kernel_p2m_rho / _non_rho (monopole_kernel_templates.hpp:188-239)
inline void p2m_pair(const double X[3], const double Y[3], const double mp[20], double L[4], double Lc[3],
                     bool rho) {
    const double dX[3] = {X[0] - Y[0], X[1] - Y[1], X[2] - Y[2]};
    Derivs f;
    d_factors(dX, f);
    add_monopole_terms(mp, f.D, L);
    if (!rho) add_dipole_terms(mp, f.D, L);
    add_quad_oct_terms(mp, f.D, L);
    if (rho) {
        double U[15];
        d_upper(f, dX, U);
        for (int k = 10; k < 20; ++k) {
            const double f6 = kFactor[k] / 6.0;
            for (int j = 0; j < 3; ++j) Lc[j] -= mp[k] * (U[kUpperIdx[k - 10][j]] * f6);
        }
    }
}

// ---------------------------------------------------------------- sweeps
void m2l_soa(const Stencil& st, const double* mon, const double* M, const double* com, double* L,
             double* Lc, bool rho, bool root) {
    const double trs = (1.0 / st.theta) * (1.0 / st.theta);
    for (int x = 0; x < INX; ++x)
        for (int y = 0; y < INX; ++y)
            for (int z = 0; z < INX; ++z) {
                const int cx = x + INX, cy = y + INX, cz = z + INX;
                const int cf = flat_padded(cx, cy, cz), cu = flat_inner(x, y, z);
                double mc[20], X[3], acc[20] = {0}, corr[3] = {0}, mp[20], Y[3];
                for (int c = 0; c < 20; ++c) mc[c] = M[c * CL + cf];
                for (int c = 0; c < 3; ++c) X[c] = com[c * CL + cf];
                if (root) {
                    // multipole_kernel_root_*_impl: every inner partner except
                    // the monopole-only stencil entries and the cell itself.
                    for (int px = 0; px < INX; ++px)
                        for (int py = 0; py < INX; ++py)
                            for (int pz = 0; pz < INX; ++pz) {
                                const int sx = px - x, sy = py - y, sz = pz - z;
                                if (std::abs(sx) <= SMAX && std::abs(sy) <= SMAX && std::abs(sz) <= SMAX &&
                                    (!st.mpole_phase[stencil_index(sx, sy, sz)] || (sx == 0 && sy == 0 && sz == 0)))
                                    continue;
                                const int pf = flat_padded(px + INX, py + INX, pz + INX);
                                for (int c = 0; c < 3; ++c) Y[c] = com[c * CL + pf];
                                for (int c = 0; c < 20; ++c) mp[c] = M[c * CL + pf];
                                m2l_pair(X, Y, mp, mc, acc, corr, rho);
                            }
                } else {
                    const int ccx = coarse(cx), ccy = coarse(cy), ccz = coarse(cz);
                    for (int sx = -SMAX; sx <= SMAX; ++sx) {
                        const int dxc = ccx - coarse(cx + sx);
                        for (int sy = -SMAX; sy <= SMAX; ++sy) {
                            const int dyc = ccy - coarse(cy + sy);
                            for (int sz = -SMAX; sz <= SMAX; ++sz) {
                                const int idx = stencil_index(sx, sy, sz);
                                if (!st.mpole_mask[idx]) continue;
                                const int dzc = ccz - coarse(cz + sz);
                                if (!(double(dxc * dxc + dyc * dyc + dzc * dzc) < trs)) continue;
                                const int pf = flat_padded(cx + sx, cy + sy, cz + sz);
                                const bool phase = st.mpole_phase[idx] != 0;
                                for (int c = 0; c < 3; ++c) Y[c] = com[c * CL + pf];
                                mp[0] = mon[pf];
                                mp[0] += phase ? M[pf] : 0.0;
                                for (int c = 1; c < 20; ++c) mp[c] = phase ? M[c * CL + pf] : 0.0;
                                m2l_pair(X, Y, mp, mc, acc, corr, rho);
                            }
                        }
                    }
                }
                for (int c = 0; c < 20; ++c) L[c * CLU + cu] = acc[c];
                if (rho)
                    for (int c = 0; c < 3; ++c) Lc[c * CLU + cu] = corr[c];
            }
}

// p2p_kernel_impl (monopole kokkos_kernel.hpp:143-320)
void p2p_soa(const Stencil& st, const double* mon, double dx, double* L4) {
    const double trs = (1.0 / st.theta) * (1.0 / st.theta);
    const double dc0 = 1.0 / dx, dc1 = -1.0 / dx;
    for (int x = 0; x < INX; ++x)
        for (int y = 0; y < INX; ++y)
            for (int z = 0; z < INX; ++z) {
                const int cx = x + INX, cy = y + INX, cz = z + INX;
                const int ccx = coarse(cx), ccy = coarse(cy), ccz = coarse(cz);
                double acc[4] = {0, 0, 0, 0};
                for (int sx = -SMAX; sx <= SMAX; ++sx) {
                    const int dxc = ccx - coarse(cx + sx);
                    for (int sy = -SMAX; sy <= SMAX; ++sy) {
                        const int dyc = ccy - coarse(cy + sy);
                        for (int sz = -SMAX; sz <= SMAX; ++sz) {
                            const int idx = stencil_index(sx, sy, sz);
                            if (!st.p2p_mask[idx]) continue;
                            const int dzc = ccz - coarse(cz + sz);
                            if (!(double(dxc * dxc + dyc * dyc + dzc * dzc) < trs)) continue;
                            const double m = mon[flat_padded(cx + sx, cy + sy, cz + sz)] * dc0;
                            const double* four = st.four[idx];
                            acc[0] += four[0] * m;
                            for (int a = 1; a < 4; ++a) acc[a] += four[a] * m * dc1;
                        }
                    }
                }
                for (int c = 0; c < 4; ++c) L4[c * CLU + flat_inner(x, y, z)] = acc[c];
            }
}

// p2m_kernel_impl_rho / _non_rho for one refined neighbour direction d.
void p2m_dir(const Stencil& st, int d, const double* nM, const double* ncom, int stride, const double* icom,
             double* L4, double* Lc, bool rho, bool reset) {
    const double trs = (1.0 / st.theta) * (1.0 / st.theta);
    int o[3], s[3], e[3], sz[3], cs[3], ce[3];
    dir_offsets(d, o);
    padding_box(o, s, e, sz);
    p2m_cells(o, cs, ce);
    if (rho && reset)
        for (int c = 0; c < 3; ++c)
            for (int u = 0; u < NCELL; ++u) Lc[c * CLU + u] = 0.0;
    for (int cx = cs[0]; cx < ce[0]; ++cx)
        for (int cy = cs[1]; cy < ce[1]; ++cy)
            for (int cz = cs[2]; cz < ce[2]; ++cz) {
                const int cu = flat_inner(cx, cy, cz);
                const int ccx = coarse(cx + INX), ccy = coarse(cy + INX), ccz = coarse(cz + INX);
                double X[3], acc[4], corr[3] = {0, 0, 0}, mp[20], Y[3];
                for (int c = 0; c < 3; ++c) X[c] = icom[c * CLU + cu];
                for (int c = 0; c < 4; ++c) acc[c] = L4[c * CLU + cu];
                if (rho)
                    for (int c = 0; c < 3; ++c) corr[c] = Lc[c * CLU + cu];
                for (int x = s[0]; x < e[0]; ++x)
                    for (int y = s[1]; y < e[1]; ++y)
                        for (int z = s[2]; z < e[2]; ++z) {
                            const int px = INX + o[0] * INX + x, py = INX + o[1] * INX + y, pz = INX + o[2] * INX + z;
                            const int sx = px - (cx + INX), sy = py - (cy + INX), szz = pz - (cz + INX);
                            if (std::abs(sx) > SMAX || std::abs(sy) > SMAX || std::abs(szz) > SMAX) continue;
                            if (!st.p2p_mask[stencil_index(sx, sy, szz)]) continue;
                            const int a = ccx - coarse(px), b = ccy - coarse(py), c = ccz - coarse(pz);
                            if (!(double(a * a + b * b + c * c) < trs)) continue;
                            const int f = (x - s[0]) * (sz[1] * sz[2]) + (y - s[1]) * sz[2] + (z - s[2]);
                            for (int q = 0; q < 3; ++q) Y[q] = ncom[size_t(q) * stride + f];
                            for (int q = 0; q < 20; ++q) mp[q] = nM[size_t(q) * stride + f];
                            p2m_pair(X, Y, mp, acc, corr, rho);
                        }
                for (int c = 0; c < 4; ++c) L4[c * CLU + cu] = acc[c];
                if (rho)
                    for (int c = 0; c < 3; ++c) Lc[c * CLU + cu] = corr[c];
            }
}

struct OracleKernels {
    void m2l(const Stencil& st, const M2LInput& in, double* L, double* Lc, int rho, bool root) const {
        m2l_soa(st, in.mon.data(), in.M.data(), in.com.data(), L, Lc, rho != 0, root);
    }
    void p2p(const Stencil& st, const double* mon, double dx, double* L4) const { p2p_soa(st, mon, dx, L4); }
    void p2m(const Stencil& st, int d, const double* nM, const double* ncom, int stride, const double* icom,
             double* L4, double* Lc, int rho, bool reset) const {
        p2m_dir(st, d, nM, ncom, stride, icom, L4, Lc, rho != 0, reset);
    }
};

}   // namespace
}   // namespace ora

// ---------------------------------------------------------------- C ABI (ctypes)
// Shift operators of taylor<4> (octotiger/taylor.hpp:222-318) restated with
// the reference's operation order; component order of src/taylor.cpp:10-56.
struct ScalarShift {
    static int i2(int a, int b) { return ora::kQuadRow[a][b]; }
    static int i3(int a, int b, int c) {
        static constexpr int m3[3][3][3] = {{{10, 11, 12}, {11, 13, 14}, {12, 14, 15}},
                                            {{11, 13, 14}, {13, 16, 17}, {14, 17, 18}},
                                            {{12, 14, 15}, {14, 17, 18}, {15, 18, 19}}};
        return m3[a][b][c];
    }
    // B = A >> X (operator>>=, :222-255)
    void up(const double A[20], const double X[3], double B[20]) const {
        for (int j = 0; j < 20; ++j) B[j] = A[j];
        for (int a = 0; a < 3; ++a) B[1 + a] += A[0] * X[a];
        for (int a = 0; a < 3; ++a)
            for (int b = a; b < 3; ++b) {
                B[i2(a, b)] += A[1 + a] * X[b] + X[a] * A[1 + b];
                B[i2(a, b)] += A[0] * X[a] * X[b];
            }
        for (int a = 0; a < 3; ++a)
            for (int b = a; b < 3; ++b)
                for (int c = b; c < 3; ++c) {
                    B[i3(a, b, c)] += A[i2(a, b)] * X[c] + A[i2(b, c)] * X[a] + A[i2(c, a)] * X[b];
                    B[i3(a, b, c)] += A[1 + a] * X[b] * X[c] + A[1 + b] * X[c] * X[a] + A[1 + c] * X[a] * X[b];
                    B[i3(a, b, c)] += A[0] * X[a] * X[b] * X[c];
                }
    }
    // B = A << X (operator<<=, :263-318)
    void down(const double A[20], const double X[3], double B[20]) const {
        constexpr double half = 1.0 / 2.0, sixth = 1.0 / 6.0;
        for (int j = 0; j < 20; ++j) B[j] = A[j];
        for (int a = 0; a < 3; ++a) B[0] += A[1 + a] * X[a];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) B[0] += A[i2(a, b)] * X[a] * X[b] * half;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) B[1 + a] += A[i2(a, b)] * X[b];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 3; ++c) B[0] += A[i3(a, b, c)] * X[a] * X[b] * X[c] * sixth;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 3; ++c) B[1 + a] += A[i3(a, b, c)] * X[b] * X[c] * half;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                for (int c = a; c < 3; ++c) B[i2(a, c)] += A[i3(a, b, c)] * X[b];
    }
};

extern "C" {

int oracle_shift(const double* A, const double* X, double* B, int down) {
    ScalarShift S;
    if (down) S.down(A, X, B);
    else S.up(A, X, B);
    return 0;
}

int oracle_upward(double* M, double* com, const double* mon, const uint8_t* is_leaf, double* com1, int n,
                  const ora::TreeNode* nodes, const int32_t* level_start, int n_levels, int rho) {
    ora::TreePool P{M, com, mon, is_leaf, com1, n};
    ora::upward_pass(ScalarShift{}, P, nodes, level_start, n_levels, rho != 0);
    return 0;
}

int oracle_downward(const double* com, const uint8_t* is_leaf, const double* com1, int n, const ora::TreeNode* nodes,
                    const int32_t* level_start, int n_levels, double* L, double* Lc, double* G, double gconst,
                    int correct_am, int rho) {
    ora::TreePool P{nullptr, const_cast<double*>(com), nullptr, is_leaf, const_cast<double*>(com1), n};
    ora::downward_pass(ScalarShift{}, P, nodes, level_start, n_levels, L, Lc, G, gconst, correct_am != 0, rho != 0);
    return 0;
}

int oracle_build_stencil(double theta, uint8_t* mpole_mask, uint8_t* mpole_phase, uint8_t* p2p_mask,
                         double* four, int* counts) {
    ora::Stencil st;
    ora::build_stencil(theta, st);
    if (!st.ok) return -1;
    std::memcpy(mpole_mask, st.mpole_mask, ora::FULL);
    std::memcpy(mpole_phase, st.mpole_phase, ora::FULL);
    std::memcpy(p2p_mask, st.p2p_mask, ora::FULL);
    std::memcpy(four, st.four, sizeof(st.four));
    counts[0] = st.n_mpole;
    counts[1] = st.n_phase_one;
    counts[2] = st.n_p2p;
    return 0;
}

int oracle_m2l_soa(double theta, const double* mon, const double* M, const double* com, double* L, double* Lc,
                   int rho, int root) {
    const ora::Stencil& st = ora::stencil_for(theta);
    if (!st.ok) return -1;
    ora::m2l_soa(st, mon, M, com, L, Lc, rho != 0, root != 0);
    return 0;
}

int oracle_p2p_soa(double theta, const double* mon, double dx, double* L4) {
    const ora::Stencil& st = ora::stencil_for(theta);
    if (!st.ok) return -1;
    ora::p2p_soa(st, mon, dx, L4);
    return 0;
}

int oracle_p2m_dir(double theta, int d, const double* nM, const double* ncom, int stride, const double* icom,
                   double* L4, double* Lc, int rho, int reset) {
    const ora::Stencil& st = ora::stencil_for(theta);
    if (!st.ok) return -1;
    ora::p2m_dir(st, d, nM, ncom, stride, icom, L4, Lc, rho != 0, reset != 0);
    return 0;
}

int oracle_stage_m2l(const double* M, const double* com, const double* mon, const uint8_t* is_leaf, int n_sub,
                     const ora::WorkItem* item, double* mon_soa, double* M_soa, double* com_soa) {
    ora::Pool pool{M, com, mon, is_leaf, n_sub};
    ora::M2LInput in;
    ora::stage_m2l(pool, *item, in);
    std::memcpy(mon_soa, in.mon.data(), sizeof(double) * ora::ENTRIES);
    std::memcpy(M_soa, in.M.data(), sizeof(double) * 20 * ora::CL);
    std::memcpy(com_soa, in.com.data(), sizeof(double) * 3 * ora::CL);
    return 0;
}

int oracle_stage_p2p(const double* M, const double* com, const double* mon, const uint8_t* is_leaf, int n_sub,
                     const ora::WorkItem* item, double* mon_soa) {
    ora::Pool pool{M, com, mon, is_leaf, n_sub};
    ora::stage_p2p(pool, *item, mon_soa);
    return 0;
}

// Returns the slab stride (size + SOA_PADDING); nM / ncom must hold 20 / 3 x 419 doubles.
int oracle_stage_p2m(const double* M, const double* com, const double* mon, const uint8_t* is_leaf, int n_sub,
                     int nb, int d, double* nM, double* ncom) {
    ora::Pool pool{M, com, mon, is_leaf, n_sub};
    std::vector<double> a, b;
    const int stride = ora::stage_p2m(pool, nb, d, a, b);
    std::memcpy(nM, a.data(), sizeof(double) * a.size());
    std::memcpy(ncom, b.data(), sizeof(double) * b.size());
    return stride;
}

int oracle_batch(double theta, const double* M, const double* com, const double* mon, const uint8_t* is_leaf,
                 int n_sub, const ora::WorkItem* items, int n_items, int rho, double* L_out, double* Lc_out,
                 int nthreads) {
    if (!ora::stencil_for(theta).ok) return -1;
    ora::Pool pool{M, com, mon, is_leaf, n_sub};
    ora::run_batch(ora::OracleKernels{}, theta, pool, items, n_items, rho, L_out, Lc_out, nthreads);
    return 0;
}

long long oracle_count_pairs(double theta, const uint8_t* is_leaf, int n_sub, const ora::WorkItem* items,
                             int n_items, long long* per_class /*4: m2l, root, p2p, p2m*/) {
    const ora::Stencil& st = ora::stencil_for(theta);
    if (!st.ok) return -1;
    ora::Pool pool{nullptr, nullptr, nullptr, is_leaf, n_sub};
    long long total = 0;
    if (per_class) per_class[0] = per_class[1] = per_class[2] = per_class[3] = 0;
    for (int i = 0; i < n_items; ++i) {
        long long n4[4];
        ora::count_pairs(st, pool, items[i], n4);
        for (int c = 0; c < 4; ++c) {
            total += n4[c];
            if (per_class) per_class[c] += n4[c];
        }
    }
    return total;
}

}   // extern "C"
