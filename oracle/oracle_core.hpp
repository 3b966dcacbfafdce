// TEST INFRASTRUCTURE ONLY — not part of the product path.
//
// CPU restatement of Octo-Tiger's FMM cell-interaction kernels (the oracle).
// This header holds the pieces shared by the scalar oracle (otfmm_oracle.cpp)
// and by the build of the reference's own kernel arithmetic (ref_driver.cpp):
//   * the interaction constants for GRIDDIM 8 / theta_min 0.34,
//   * the stencil generators,
//   * the AoS -> SoA halo staging of one work item from a subgrid pool,
//   * the work-list driver that runs a batch of work items on host threads.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
// it, and only as the checker. Reference citations are path:line within the
// Octo-Tiger source tree.
#pragma once

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace ora {

// octotiger/common_kernel/interaction_constants.hpp:173-214 with
// OCTOTIGER_GRIDDIM=8, OCTOTIGER_THETA_MINIMUM=0.34.
constexpr int INX = 8;
constexpr int NCELL = INX * INX * INX;             // 512 inner cells
constexpr int SMAX = 5;                            // STENCIL_MAX (= STENCIL_WIDTH)
constexpr int SINX = 2 * SMAX + 1;                 // STENCIL_INX = 11
constexpr int FULL = SINX * SINX * SINX;           // FULL_STENCIL_SIZE = 1331
constexpr int PSTRIDE = INX + 2 * SMAX;            // PADDED_STRIDE = 18
constexpr int ENTRIES = PSTRIDE * PSTRIDE * PSTRIDE; // 5832
constexpr int SOA_PAD = 19;                        // SOA_PADDING
constexpr int CL = ENTRIES + SOA_PAD;              // input component stride 5851
constexpr int CLU = NCELL + SOA_PAD;               // output component stride 531
constexpr int PAD_OFF = INX - SMAX;                // PADDING_OFFSET = 3
constexpr double THETA_MIN = 0.34;

// Work-item kinds (what node_server::compute_fmm dispatches, src/node_server.cpp:711-723).
enum Kind : int32_t { KIND_M2L = 0, KIND_M2L_ROOT = 1, KIND_LEAF = 2 };

// One work item: a subgrid, how it is solved and its 26 same-level neighbours
// (pool index or -1 for an empty direction), in geo::direction flat order
// (octotiger/geometry.hpp:91-197).
struct WorkItem {
    int32_t subgrid;
    int32_t kind;
    int32_t neighbors[26];
    double dx;
    double xbase[3];   // centre of inner cell (0,0,0), src/node_server.cpp:712-715
};
static_assert(sizeof(WorkItem) == 144, "work item layout");

// Resident subgrid pool: per subgrid M[20][512], com[3][512], mon[512].
struct Pool {
    const double* M;
    const double* com;
    const double* mon;
    const uint8_t* is_leaf;   // leaf subgrids are seen as monopole neighbours
    int32_t n;
};

// multiindex.hpp:103-116, 72-79
inline int flat_padded(int x, int y, int z) {
    return (x - PAD_OFF) * PSTRIDE * PSTRIDE + (y - PAD_OFF) * PSTRIDE + (z - PAD_OFF);
}
inline int flat_inner(int x, int y, int z) { return x * INX * INX + y * INX + z; }
inline int coarse(int i) { return ((i + INX) >> 1) - INX / 2; }
inline int stencil_index(int sx, int sy, int sz) {
    return (sx + SMAX) * SINX * SINX + (sy + SMAX) * SINX + (sz + SMAX);
}

// Flat neighbour index d (0..25) -> raw direction 0..26 without the centre,
// and the per-axis offsets (geometry.hpp:111-122, 181-186).
inline int dir_raw(int d) { return d < 13 ? d : d + 1; }
inline void dir_offsets(int d, int o[3]) {
    const int r = dir_raw(d);
    o[0] = r % 3 - 1;
    o[1] = (r / 3) % 3 - 1;
    o[2] = r / 9 - 1;
}

// ---------------------------------------------------------------- stencils
// helper.hpp:20-30
inline double reciprocal_distance(int64_t i0, int64_t i1, int64_t i2, int64_t j0, int64_t j1,
                                  int64_t j2) {
    const double tmp = double((i0 - j0) * (i0 - j0) + (i1 - j1) * (i1 - j1) + (i2 - j2) * (i2 - j2));
    if (tmp > 0.0) return 1.0 / std::sqrt(tmp);
    return 1.0e+10;
}

struct Stencil {
    double theta = -1.0;
    uint8_t mpole_mask[FULL];   // stencil_masks: superimposed two-phase stencil
    uint8_t mpole_phase[FULL];  // inner_stencil_masks / "indicators" (true outside the stencil)
    uint8_t p2p_mask[FULL];     // monopole stencil mask
    double four[FULL][4];       // monopole constants {-1/r, x/r^3, y/r^3, z/r^3}
    int n_mpole = 0, n_phase_one = 0, n_p2p = 0;
    bool ok = false;
};

// Restates multipole_interactions::calculate_stencil + calculate_stencil_masks
// (src/multipole_interactions/util/calculate_stencil.cpp:23-160) and
// monopole_interactions::calculate_stencil + calculate_stencil_masks
// (src/monopole_interactions/util/calculate_stencil.cpp:19-178).
inline void build_stencil(double theta, Stencil& st) {
    st.theta = theta;
    std::memset(st.mpole_mask, 0, sizeof(st.mpole_mask));
    std::memset(st.mpole_phase, 1, sizeof(st.mpole_phase));
    std::memset(st.p2p_mask, 0, sizeof(st.p2p_mask));
    for (int i = 0; i < FULL; ++i)
        for (int c = 0; c < 4; ++c) st.four[i][c] = 0.0;
    struct E { int x, y, z; bool phase; };
    std::vector<E> mp_super, p2p_super;
    int maxabs = 0;
    for (int64_t i0 = 0; i0 < 2; ++i0)
        for (int64_t i1 = 0; i1 < 2; ++i1)
            for (int64_t i2 = 0; i2 < 2; ++i2) {
                std::vector<E> mp, pp;
                for (int64_t j0 = i0 - INX; j0 < i0 + INX; ++j0)
                    for (int64_t j1 = i1 - INX; j1 < i1 + INX; ++j1)
                        for (int64_t j2 = i2 - INX; j2 < i2 + INX; ++j2) {
                            if (i0 == j0 && i1 == j1 && i2 == j2) continue;
                            const int64_t i0c = (i0 + INX) / 2 - INX / 2, i1c = (i1 + INX) / 2 - INX / 2,
                                          i2c = (i2 + INX) / 2 - INX / 2;
                            const int64_t j0c = (j0 + INX) / 2 - INX / 2, j1c = (j1 + INX) / 2 - INX / 2,
                                          j2c = (j2 + INX) / 2 - INX / 2;
                            const double tf = reciprocal_distance(i0, i1, i2, j0, j1, j2);
                            const double tc = reciprocal_distance(i0c, i1c, i2c, j0c, j1c, j2c);
                            const E e{int(j0 - i0), int(j1 - i1), int(j2 - i2), false};
                            if (tc > theta) {
                                E m = e;
                                m.phase = (tf <= theta);
                                mp.push_back(m);
                                pp.push_back(e);
                            }
                        }
                auto merge = [](std::vector<E>& sup, const std::vector<E>& part) {
                    for (const E& e : part) {
                        bool found = false;
                        for (const E& s : sup)
                            if (s.x == e.x && s.y == e.y && s.z == e.z) { found = true; break; }
                        if (!found) sup.push_back(e);
                    }
                };
                merge(mp_super, mp);
                merge(p2p_super, pp);
            }
    for (const E& e : mp_super) maxabs = std::max({maxabs, std::abs(e.x), std::abs(e.y), std::abs(e.z)});
    for (const E& e : p2p_super) maxabs = std::max({maxabs, std::abs(e.x), std::abs(e.y), std::abs(e.z)});
    st.ok = (maxabs <= SMAX);
    if (!st.ok) return;
    for (const E& e : mp_super) {
        const int idx = stencil_index(e.x, e.y, e.z);
        st.mpole_mask[idx] = 1;
        if (!e.phase) st.mpole_phase[idx] = 0;
        ++st.n_mpole;
        if (e.phase) ++st.n_phase_one;
    }
    for (const E& e : p2p_super) {
        const int idx = stencil_index(e.x, e.y, e.z);
        st.p2p_mask[idx] = 1;
        ++st.n_p2p;
        const double x = e.x, y = e.y, z = e.z;
        const double tmp = x * x + y * y + z * z;
        const double r = std::sqrt(tmp);
        const double r3 = r * r * r;
        st.four[idx][0] = -1.0 / r;
        st.four[idx][1] = x / r3;
        st.four[idx][2] = y / r3;
        st.four[idx][3] = z / r3;
    }
}

// Thread-local cache, like the reference's static thread_local stencils
// (src/multipole_interactions/legacy/multipole_interaction_interface.cpp:46-76).
inline const Stencil& stencil_for(double theta) {
    thread_local Stencil st;
    if (st.theta != theta) build_stencil(theta, st);
    return st;
}

// ---------------------------------------------------------------- staging
// Reference layouts of one work item's kernel input / output.
struct M2LInput {
    std::vector<double> mon, M, com;
    M2LInput() : mon(ENTRIES, 0.0), M(20 * CL, 0.0), com(3 * CL, 0.0) {}
};

// iterate_inner_cells_padding (octotiger/common_kernel/interactions_iterators.hpp:65-128):
// neighbour direction o -> range of neighbour-local cells and the logical
// padded index of local cell 0.
inline void padding_range(const int o[3], int start[3], int end[3], int pstart[3]) {
    for (int a = 0; a < 3; ++a) {
        start[a] = (o[a] == -1) ? INX - SMAX : 0;
        end[a] = (o[a] == 1) ? SMAX : INX;
        pstart[a] = (o[a] == 1) ? 2 * INX : (o[a] == 0 ? INX : 0);
    }
}

// multipole_interactions::update_input
// (octotiger/multipole_interactions/legacy/multipole_interaction_interface.hpp:88-281),
// with every neighbour payload full-size (512 cells).
inline void stage_m2l(const Pool& pool, const WorkItem& it, M2LInput& in) {
    std::fill(in.mon.begin(), in.mon.end(), 0.0);
    std::fill(in.M.begin(), in.M.end(), 0.0);
    std::fill(in.com.begin(), in.com.end(), 0.0);
    const double* Ms = pool.M + size_t(it.subgrid) * 20 * NCELL;
    const double* Cs = pool.com + size_t(it.subgrid) * 3 * NCELL;
    for (int x = 0; x < INX; ++x)
        for (int y = 0; y < INX; ++y)
            for (int z = 0; z < INX; ++z) {
                const int f = flat_padded(x + INX, y + INX, z + INX), u = flat_inner(x, y, z);
                for (int c = 0; c < 20; ++c) in.M[c * CL + f] = Ms[c * NCELL + u];
                for (int c = 0; c < 3; ++c) in.com[c * CL + f] = Cs[c * NCELL + u];
                in.mon[f] = 0.0;
            }
    if (it.kind == KIND_M2L_ROOT) return;
    for (int d = 0; d < 26; ++d) {
        const int nb = it.neighbors[d];
        if (nb < 0) continue;   // empty direction: zeros
        int o[3], s[3], e[3], p[3];
        dir_offsets(d, o);
        padding_range(o, s, e, p);
        const bool mono = pool.is_leaf[nb] != 0;
        const double* Mn = pool.M + size_t(nb) * 20 * NCELL;
        const double* Cn = pool.com + size_t(nb) * 3 * NCELL;
        const double* mn = pool.mon + size_t(nb) * NCELL;
        for (int x = s[0]; x < e[0]; ++x)
            for (int y = s[1]; y < e[1]; ++y)
                for (int z = s[2]; z < e[2]; ++z) {
                    const int ix = x + p[0], iy = y + p[1], iz = z + p[2];
                    const int f = flat_padded(ix, iy, iz), u = flat_inner(x, y, z);
                    if (!mono) {
                        for (int c = 0; c < 20; ++c) in.M[c * CL + f] = Mn[c * NCELL + u];
                        for (int c = 0; c < 3; ++c) in.com[c * CL + f] = Cn[c * NCELL + u];
                        in.mon[f] = 0.0;
                    } else {
                        // monopole neighbour: cell centre as centre of mass (:221-234)
                        in.com[0 * CL + f] = ix * it.dx + it.xbase[0] - INX * it.dx;
                        in.com[1 * CL + f] = iy * it.dx + it.xbase[1] - INX * it.dx;
                        in.com[2 * CL + f] = iz * it.dx + it.xbase[2] - INX * it.dx;
                        for (int c = 0; c < 20; ++c) in.M[c * CL + f] = 0.0;
                        in.mon[f] = mn[u];
                    }
                }
    }
}

// monopole_interactions::update_input
// (octotiger/monopole_interactions/legacy/monopole_interaction_interface.hpp:64-143).
inline void stage_p2p(const Pool& pool, const WorkItem& it, double* mon_soa /*ENTRIES*/) {
    std::fill(mon_soa, mon_soa + ENTRIES, 0.0);
    const double* ms = pool.mon + size_t(it.subgrid) * NCELL;
    for (int x = 0; x < INX; ++x)
        for (int y = 0; y < INX; ++y)
            for (int z = 0; z < INX; ++z)
                mon_soa[flat_padded(x + INX, y + INX, z + INX)] = ms[flat_inner(x, y, z)];
    for (int d = 0; d < 26; ++d) {
        const int nb = it.neighbors[d];
        if (nb < 0 || !pool.is_leaf[nb]) continue;   // refined or empty: zeros
        int o[3], s[3], e[3], p[3];
        dir_offsets(d, o);
        padding_range(o, s, e, p);
        const double* mn = pool.mon + size_t(nb) * NCELL;
        for (int x = s[0]; x < e[0]; ++x)
            for (int y = s[1]; y < e[1]; ++y)
                for (int z = s[2]; z < e[2]; ++z)
                    mon_soa[flat_padded(x + p[0], y + p[1], z + p[2])] = mn[flat_inner(x, y, z)];
    }
}

// get_padding_real_size / start / end (src/common_kernel/interactions_iterators.cpp:14-62)
inline void padding_box(const int o[3], int start[3], int end[3], int size[3]) {
    for (int a = 0; a < 3; ++a) {
        start[a] = (o[a] == -1) ? INX - SMAX : 0;
        end[a] = (o[a] == 1) ? SMAX : INX;
        size[a] = end[a] - start[a];
    }
}

// monopole_interactions::update_neighbor_input
// (octotiger/monopole_interactions/legacy/p2m_interaction_interface.hpp:102-160):
// the refined neighbour's slab in its own SoA layout (stride size+SOA_PAD).
inline int stage_p2m(const Pool& pool, int nb, int d, std::vector<double>& nM, std::vector<double>& ncom) {
    int o[3], s[3], e[3], sz[3];
    dir_offsets(d, o);
    padding_box(o, s, e, sz);
    const int size = sz[0] * sz[1] * sz[2];
    const int stride = size + SOA_PAD;
    nM.assign(size_t(20) * stride, 0.0);
    ncom.assign(size_t(3) * stride, 0.0);
    const double* Mn = pool.M + size_t(nb) * 20 * NCELL;
    const double* Cn = pool.com + size_t(nb) * 3 * NCELL;
    for (int x = s[0]; x < e[0]; ++x)
        for (int y = s[1]; y < e[1]; ++y)
            for (int z = s[2]; z < e[2]; ++z) {
                const int f = (x - s[0]) * (sz[1] * sz[2]) + (y - s[1]) * sz[2] + (z - s[2]);
                const int u = flat_inner(x, y, z);
                for (int c = 0; c < 20; ++c) nM[size_t(c) * stride + f] = Mn[c * NCELL + u];
                for (int c = 0; c < 3; ++c) ncom[size_t(c) * stride + f] = Cn[c * NCELL + u];
            }
    return stride;
}

// P2M cell range per direction
// (octotiger/monopole_interactions/kernel/kokkos_kernel.hpp:1116-1129).
inline void p2m_cells(const int o[3], int cs[3], int ce[3]) {
    for (int a = 0; a < 3; ++a) {
        cs[a] = (o[a] == 1) ? INX - (SMAX + 1) : 0;
        ce[a] = (o[a] == -1) ? SMAX + 1 : INX;
    }
}

// ---------------------------------------------------------------- counting
// Cell-interactions the reference evaluates for one work item: (cell,
// partner) pairs that pass the stencil and coarse-distance masks.
// n[0] M2L, n[1] root M2L, n[2] P2P, n[3] P2M pairs.
inline void count_pairs(const Stencil& st, const Pool& pool, const WorkItem& it, long long n4[4]) {
    const double trs = (1.0 / st.theta) * (1.0 / st.theta);
    long long n = 0;
    n4[0] = n4[1] = n4[2] = n4[3] = 0;
    if (it.kind == KIND_M2L_ROOT) {
        for (int c = 0; c < NCELL; ++c)
            for (int p = 0; p < NCELL; ++p) {
                const int sx = p / 64 - c / 64, sy = (p / 8) % 8 - (c / 8) % 8, sz = p % 8 - c % 8;
                const bool inbox = std::abs(sx) <= SMAX && std::abs(sy) <= SMAX && std::abs(sz) <= SMAX;
                if (inbox && (!st.mpole_phase[stencil_index(sx, sy, sz)] || (sx == 0 && sy == 0 && sz == 0)))
                    continue;
                ++n;
            }
        n4[1] = n;
        return;
    }
    const uint8_t* mask = (it.kind == KIND_M2L) ? st.mpole_mask : st.p2p_mask;
    for (int x = 0; x < INX; ++x)
        for (int y = 0; y < INX; ++y)
            for (int z = 0; z < INX; ++z)
                for (int sx = -SMAX; sx <= SMAX; ++sx)
                    for (int sy = -SMAX; sy <= SMAX; ++sy)
                        for (int sz = -SMAX; sz <= SMAX; ++sz) {
                            if (!mask[stencil_index(sx, sy, sz)]) continue;
                            const int dxc = coarse(x + INX) - coarse(x + INX + sx);
                            const int dyc = coarse(y + INX) - coarse(y + INX + sy);
                            const int dzc = coarse(z + INX) - coarse(z + INX + sz);
                            if (double(dxc * dxc + dyc * dyc + dzc * dzc) < trs) ++n;
                        }
    n4[it.kind == KIND_LEAF ? 2 : 0] = n;
    n = 0;
    if (it.kind == KIND_LEAF) {
        // P2M pairs with refined neighbours
        for (int d = 0; d < 26; ++d) {
            const int nb = it.neighbors[d];
            if (nb < 0 || pool.is_leaf[nb]) continue;
            int o[3], s[3], e[3], sz[3], cs[3], ce[3];
            dir_offsets(d, o);
            padding_box(o, s, e, sz);
            p2m_cells(o, cs, ce);
            for (int cx = cs[0]; cx < ce[0]; ++cx)
                for (int cy = cs[1]; cy < ce[1]; ++cy)
                    for (int cz = cs[2]; cz < ce[2]; ++cz)
                        for (int x = s[0]; x < e[0]; ++x)
                            for (int y = s[1]; y < e[1]; ++y)
                                for (int z = s[2]; z < e[2]; ++z) {
                                    const int px = INX + o[0] * INX + x, py = INX + o[1] * INX + y,
                                              pz = INX + o[2] * INX + z;
                                    const int sx = px - (cx + INX), sy = py - (cy + INX), sz2 = pz - (cz + INX);
                                    if (std::abs(sx) > SMAX || std::abs(sy) > SMAX || std::abs(sz2) > SMAX) continue;
                                    if (!st.p2p_mask[stencil_index(sx, sy, sz2)]) continue;
                                    const int a = coarse(cx + INX) - coarse(px), b = coarse(cy + INX) - coarse(py),
                                              c = coarse(cz + INX) - coarse(pz);
                                    if (double(a * a + b * b + c * c) < trs) ++n;
                                }
        }
        n4[3] = n;
    }
}

// ---------------------------------------------------------------- batch driver
// Runs a work list on `nthreads` host threads. `Kernels` supplies the per-item
// SoA compute: m2l(st, in, L, Lc, rho, root), p2p(st, mon, dx, L4),
// p2m(st, d, nM, ncom, stride, icom, L4, Lc, rho, reset).
// Output per subgrid: L[20][512] and Lc[3][512] (leaf items fill L[0..3]).
template <class Kernels>
void run_batch(const Kernels& K, double theta, const Pool& pool, const WorkItem* items, int n_items,
               int rho, double* L_out, double* Lc_out, int nthreads) {
    std::atomic<int> next{0};
    auto worker = [&]() {
        const Stencil& st = stencil_for(theta);
        M2LInput in;
        std::vector<double> L(20 * CLU), Lc(3 * CLU), icom(3 * CLU), nM, ncom, mon(ENTRIES);
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n_items) break;
            const WorkItem& it = items[i];
            std::fill(L.begin(), L.end(), 0.0);
            std::fill(Lc.begin(), Lc.end(), 0.0);
            if (it.kind == KIND_M2L || it.kind == KIND_M2L_ROOT) {
                stage_m2l(pool, it, in);
                K.m2l(st, in, L.data(), Lc.data(), rho, it.kind == KIND_M2L_ROOT);
            } else {
                stage_p2p(pool, it, mon.data());
                K.p2p(st, mon.data(), it.dx, L.data());
                const double* Cs = pool.com + size_t(it.subgrid) * 3 * NCELL;
                for (int c = 0; c < 3; ++c)
                    for (int u = 0; u < NCELL; ++u) icom[c * CLU + u] = Cs[c * NCELL + u];
                bool reset = true;
                for (int d = 0; d < 26; ++d) {
                    const int nb = it.neighbors[d];
                    if (nb < 0 || pool.is_leaf[nb]) continue;
                    const int stride = stage_p2m(pool, nb, d, nM, ncom);
                    K.p2m(st, d, nM.data(), ncom.data(), stride, icom.data(), L.data(), Lc.data(), rho, reset);
                    reset = false;
                }
            }
            double* Lo = L_out + size_t(it.subgrid) * 20 * NCELL;
            double* Lco = Lc_out + size_t(it.subgrid) * 3 * NCELL;
            const int ncomp = (it.kind == KIND_LEAF) ? 4 : 20;
            for (int c = 0; c < 20; ++c)
                for (int u = 0; u < NCELL; ++u) Lo[c * NCELL + u] = (c < ncomp) ? L[c * CLU + u] : 0.0;
            for (int c = 0; c < 3; ++c)
                for (int u = 0; u < NCELL; ++u) Lco[c * NCELL + u] = rho ? Lc[c * CLU + u] : 0.0;
        }
    };
    nthreads = std::max(1, nthreads);
    std::vector<std::thread> pool_threads;
    for (int t = 1; t < nthreads; ++t) pool_threads.emplace_back(worker);
    worker();
    for (auto& t : pool_threads) t.join();
}

}   // namespace ora
