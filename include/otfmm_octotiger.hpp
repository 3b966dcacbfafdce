// otfmm_octotiger.hpp — drop-in host adapter for Octo-Tiger (header only).
//
// The bodies of a new `interaction_device_kernel_type` branch in
//   octotiger::fmm::multipole_interactions::multipole_kernel_interface
//     (src/multipole_interactions/multipole_kernel_interface.cpp:73-169)
//   octotiger::fmm::monopole_interactions::monopole_kernel_interface
//     (src/monopole_interactions/monopole_kernel_interface.cpp:97-198)
// on top of the C ABI in otfmm.h. The functions take the same arguments with
// the same meaning as the reference's interfaces and leave the grid in the
// same state:
//   * multipole: L += M2L result (all 20 components), L_c = correction (RHO);
//   * monopole: L[0..3] += P2P + P2M, L_c = P2M correction when a neighbour is
//     refined (RHO), otherwise L_c untouched;
// and stage the 26-neighbour halo the way update_input does
// (octotiger/multipole_interactions/legacy/multipole_interaction_interface.hpp:88-281,
//  octotiger/monopole_interactions/legacy/monopole_interaction_interface.hpp:64-143,
//  octotiger/monopole_interactions/legacy/p2m_interaction_interface.hpp:102-160).
// Neighbour payloads are full size (512 cells) or compressed the way
// grid::get_gravity_boundary packs remote neighbours (src/grid_fmm.cpp:1805-1850):
// element k of the payload is the neighbour's cell grid->get_ilist_n_bnd(dir)[k].second.
// The overloads that take the grid (the reference's own argument lists) expand
// compressed payloads as update_input does: the direction's halo band is reset
// (zeros; leaf neighbours in the multipole staging keep their cell-centre
// COMs), then the listed cells are filled. Without a grid a compressed payload
// is an error (OTFMM_ERR_INVALID), as is a listed cell outside the halo band or
// a list longer than its payload.
//
// Template parameters are Octo-Tiger's own types (multipole = taylor<4>,
// expansion = taylor<4>, space_vector, neighbor_gravity_type with
// .data.M / .data.m / .data.x and .is_monopole), so the header compiles inside
// the reference tree; tests/cpp instantiates it with plain stand-ins.
//
// Errors: every function returns the otfmm status; the *_or_abort wrappers
// print to std::cerr and abort(), which is what the reference does on
// misconfiguration (multipole_kernel_interface.cpp:107-158).
#pragma once

#include <algorithm>
#include <array>
#include <cstddef>
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <iostream>
#include <memory>
#include <type_traits>
#include <utility>
#include <vector>

#include "otfmm.h"

namespace otfmm_octotiger {

constexpr int INX = 8;
constexpr int NCELL = 512;
constexpr int SMAX = 5;
constexpr int PSTRIDE = INX + 2 * SMAX;
constexpr int ENTRIES = PSTRIDE * PSTRIDE * PSTRIDE;
constexpr int CL = ENTRIES + 19;
constexpr int CLU = NCELL + 19;

inline int flat_padded(int x, int y, int z) { return (x - 3) * PSTRIDE * PSTRIDE + (y - 3) * PSTRIDE + (z - 3); }
inline int flat_inner(int x, int y, int z) { return x * INX * INX + y * INX + z; }
inline void dir_offsets(int d, int o[3]) {
    const int r = d < 13 ? d : d + 1;
    o[0] = r % 3 - 1;
    o[1] = (r / 3) % 3 - 1;
    o[2] = r / 9 - 1;
}
// neighbour-local cell range inside the 18^3 halo and the padded index of
// local cell 0 (iterate_inner_cells_padding, interactions_iterators.hpp:65-128)
inline void padding_range(const int o[3], int s[3], int e[3], int p[3]) {
    for (int a = 0; a < 3; ++a) {
        s[a] = (o[a] == -1) ? INX - SMAX : 0;
        e[a] = (o[a] == 1) ? SMAX : INX;
        p[a] = (o[a] == 1) ? 2 * INX : (o[a] == 0 ? INX : 0);
    }
}

inline bool in_band(const int o[3], int x, int y, int z) {
    int s[3], e[3], p[3];
    padding_range(o, s, e, p);
    return x >= s[0] && x < e[0] && y >= s[1] && y < e[1] && z >= s[2] && z < e[2];
}

// Walks the cells of direction d's compressed payload of `payload_size`
// elements: put(k, x, y, z) for payload element k and neighbour-local cell
// (x, y, z) (flat_index_to_multiindex_not_padded, multiindex.hpp:82-91).
// GridPtr is a pointer-like to Octo-Tiger's grid, or std::nullptr_t where the
// caller has none.
template <class GridPtr, class F>
int expand_compressed(const GridPtr& grid, int d, size_t payload_size, F&& put) {
    if constexpr (std::is_same_v<GridPtr, std::nullptr_t>) {
        (void)grid, (void)d, (void)payload_size, (void)put;
        return OTFMM_ERR_INVALID;
    } else {
        if (!grid) return OTFMM_ERR_INVALID;
        int o[3];
        dir_offsets(d, o);
        size_t k = 0;
        for (const auto& cell : grid->get_ilist_n_bnd(d)) {
            const int u = static_cast<int>(cell.second);
            if (k >= payload_size || u < 0 || u >= NCELL) return OTFMM_ERR_INVALID;
            const int x = u / (INX * INX), y = (u / INX) % INX, z = u % INX;
            if (!in_band(o, x, y, z)) return OTFMM_ERR_INVALID;
            put(k, x, y, z);
            ++k;
        }
        return OTFMM_OK;
    }
}

// Host and device staging of one subgrid, reused across calls of a thread
// (the reference recycles its buffers through CPPuddle).
struct Staging {
    std::vector<double> mon, M, com, L, Lc;
    Staging() : mon(ENTRIES), M(20 * CL), com(3 * CL), L(20 * CLU), Lc(3 * CLU) {}
};
inline Staging& thread_staging() {
    thread_local Staging s;
    return s;
}

template <class Multipole, class SpaceVector, class Neighbor, class GridPtr = std::nullptr_t>
int stage_multipole_input(const std::vector<Multipole>& M_ptr, const SpaceVector* com0,
                          const std::vector<Neighbor>& neighbors, double dx, const std::array<double, 3>& xbase,
                          bool is_root, Staging& st, const GridPtr& grid = nullptr) {
    std::fill(st.mon.begin(), st.mon.end(), 0.0);
    std::fill(st.M.begin(), st.M.end(), 0.0);
    std::fill(st.com.begin(), st.com.end(), 0.0);
    for (int x = 0; x < INX; ++x)
        for (int y = 0; y < INX; ++y)
            for (int z = 0; z < INX; ++z) {
                const int f = flat_padded(x + INX, y + INX, z + INX), u = flat_inner(x, y, z);
                for (int c = 0; c < 20; ++c) st.M[c * CL + f] = M_ptr[u][c];
                for (int c = 0; c < 3; ++c) st.com[c * CL + f] = com0[u][c];
            }
    if (is_root) return OTFMM_OK;
    for (int d = 0; d < 26; ++d) {
        const Neighbor& nb = neighbors[d];
        int o[3], s[3], e[3], p[3];
        dir_offsets(d, o);
        padding_range(o, s, e, p);
        const bool full = nb.is_monopole ? (nb.data.m && nb.data.m->size() == NCELL)
                                         : (nb.data.M && nb.data.M->size() == NCELL && nb.data.x &&
                                            nb.data.x->size() == NCELL);
        for (int x = s[0]; x < e[0]; ++x)
            for (int y = s[1]; y < e[1]; ++y)
                for (int z = s[2]; z < e[2]; ++z) {
                    const int ix = x + p[0], iy = y + p[1], iz = z + p[2];
                    const int f = flat_padded(ix, iy, iz), u = flat_inner(x, y, z);
                    if (!nb.is_monopole) {
                        if (!full) continue;   // empty direction or compressed payload: zeros first
                        for (int c = 0; c < 20; ++c) st.M[c * CL + f] = (*nb.data.M)[u][c];
                        for (int c = 0; c < 3; ++c) st.com[c * CL + f] = (*nb.data.x)[u][c];
                    } else {
                        if (!nb.data.m) continue;
                        st.com[0 * CL + f] = ix * dx + xbase[0] - INX * dx;
                        st.com[1 * CL + f] = iy * dx + xbase[1] - INX * dx;
                        st.com[2 * CL + f] = iz * dx + xbase[2] - INX * dx;
                        if (full) st.mon[f] = (*nb.data.m)[u];
                    }
                }
        if (full || (nb.is_monopole ? !nb.data.m : !nb.data.M)) continue;
        int rc;
        if (nb.is_monopole) {
            const auto& m = *nb.data.m;
            rc = expand_compressed(grid, d, m.size(), [&](size_t k, int x, int y, int z) {
                st.mon[flat_padded(x + p[0], y + p[1], z + p[2])] = m[k];
            });
        } else {
            const auto& nM = *nb.data.M;
            const size_t n = nb.data.x ? std::min(nM.size(), nb.data.x->size()) : 0;
            rc = expand_compressed(grid, d, n, [&](size_t k, int x, int y, int z) {
                const int f = flat_padded(x + p[0], y + p[1], z + p[2]);
                for (int c = 0; c < 20; ++c) st.M[c * CL + f] = nM[k][c];
                for (int c = 0; c < 3; ++c) st.com[c * CL + f] = (*nb.data.x)[k][c];
            });
        }
        if (rc != OTFMM_OK) return rc;
    }
    return OTFMM_OK;
}

// monopole update_input (monopole_interaction_interface.hpp:64-143): the 18^3
// mass buffer `mon` (ENTRIES) gets the own masses, leaf neighbours' masses and
// zeros elsewhere.
template <class Neighbor, class GridPtr = std::nullptr_t>
int stage_monopole_input(const std::vector<double>& monopoles, const std::vector<Neighbor>& neighbors, double* mon,
                         const GridPtr& grid = nullptr) {
    std::fill(mon, mon + ENTRIES, 0.0);
    for (int x = 0; x < INX; ++x)
        for (int y = 0; y < INX; ++y)
            for (int z = 0; z < INX; ++z) mon[flat_padded(x + INX, y + INX, z + INX)] = monopoles[flat_inner(x, y, z)];
    for (int d = 0; d < 26; ++d) {
        const Neighbor& nb = neighbors[d];
        if (!nb.is_monopole || !nb.data.m) continue;
        int o[3], s[3], e[3], p[3];
        dir_offsets(d, o);
        padding_range(o, s, e, p);
        const auto& m = *nb.data.m;
        if (m.size() == NCELL) {
            for (int x = s[0]; x < e[0]; ++x)
                for (int y = s[1]; y < e[1]; ++y)
                    for (int z = s[2]; z < e[2]; ++z)
                        mon[flat_padded(x + p[0], y + p[1], z + p[2])] = m[flat_inner(x, y, z)];
        } else {
            const int rc = expand_compressed(grid, d, m.size(), [&](size_t k, int x, int y, int z) {
                mon[flat_padded(x + p[0], y + p[1], z + p[2])] = m[k];
            });
            if (rc != OTFMM_OK) return rc;
        }
    }
    return OTFMM_OK;
}

// update_neighbor_input (p2m_interaction_interface.hpp:102-160): refined
// neighbour d's slab of 8x8x5, 8x5x5 or 5x5x5 cells in its own SoA layout,
// component stride *stride (cells + 19); nM / ncom hold 20 x 419 / 3 x 419.
template <class Neighbor, class GridPtr = std::nullptr_t>
int stage_p2m_slab(const Neighbor& nb, int d, double* nM, double* ncom, int* stride,
                   const GridPtr& grid = nullptr) {
    int o[3], s[3], e[3], sz[3];
    dir_offsets(d, o);
    for (int a = 0; a < 3; ++a) {
        s[a] = (o[a] == -1) ? INX - SMAX : 0;
        e[a] = (o[a] == 1) ? SMAX : INX;
        sz[a] = e[a] - s[a];
    }
    const int st = sz[0] * sz[1] * sz[2] + 19;
    *stride = st;
    const auto& M = *nb.data.M;
    const size_t n_x = nb.data.x ? nb.data.x->size() : 0;
    std::fill(nM, nM + 20 * st, 0.0);
    std::fill(ncom, ncom + 3 * st, 0.0);
    if (M.size() == NCELL && n_x == NCELL) {
        for (int x = s[0]; x < e[0]; ++x)
            for (int y = s[1]; y < e[1]; ++y)
                for (int z = s[2]; z < e[2]; ++z) {
                    const int f = (x - s[0]) * (sz[1] * sz[2]) + (y - s[1]) * sz[2] + (z - s[2]);
                    const int u = flat_inner(x, y, z);
                    for (int c = 0; c < 20; ++c) nM[c * st + f] = M[u][c];
                    for (int c = 0; c < 3; ++c) ncom[c * st + f] = (*nb.data.x)[u][c];
                }
        return OTFMM_OK;
    }
    // compressed payload: the listed cells over the zeros
    return expand_compressed(grid, d, std::min(M.size(), n_x), [&](size_t k, int x, int y, int z) {
        const int f = (x - s[0]) * (sz[1] * sz[2]) + (y - s[1]) * sz[2] + (z - s[2]);
        for (int c = 0; c < 20; ++c) nM[c * st + f] = M[k][c];
        for (int c = 0; c < 3; ++c) ncom[c * st + f] = (*nb.data.x)[k][c];
    });
}

// multipole_kernel_interface(monopoles, M_ptr, com_ptr, neighbors, type, dx,
// is_direction_empty, xbase, grid, use_root_stencil): L += result,
// L_c = correction (RHO). `monopoles` is not read: a refined node's own cells
// enter as multipoles (update_input sets their monopole slots to zero).
template <class Multipole, class SpaceVector, class Neighbor, class Expansion, class GridPtr>
int multipole_kernel_impl(otfmm_context* ctx, const std::vector<Multipole>& M_ptr,
                          const std::vector<std::shared_ptr<std::vector<SpaceVector>>>& com_ptr,
                          const std::vector<Neighbor>& neighbors, int type, double dx, std::array<double, 3> xbase,
                          std::vector<Expansion>& L, std::vector<SpaceVector>& L_c, bool use_root_stencil,
                          int precision, const GridPtr& grid) {
    Staging& st = thread_staging();
    int rc = stage_multipole_input(M_ptr, com_ptr[0]->data(), neighbors, dx, xbase, use_root_stencil, st, grid);
    if (rc != OTFMM_OK) return rc;
    rc = otfmm_m2l_soa_host(ctx, use_root_stencil ? nullptr : st.mon.data(), st.M.data(), st.com.data(),
                            st.L.data(), st.Lc.data(), type, use_root_stencil ? 1 : 0, precision);
    if (rc != OTFMM_OK) return rc;
    for (int c = 0; c < 20; ++c)
        for (int u = 0; u < NCELL; ++u) L[u][c] += st.L[c * CLU + u];
    if (type == OTFMM_RHO)
        for (int c = 0; c < 3; ++c)
            for (int u = 0; u < NCELL; ++u) L_c[u][c] = st.Lc[c * CLU + u];
    return OTFMM_OK;
}

// L and L_c passed explicitly; every neighbour payload full size.
template <class Multipole, class SpaceVector, class Neighbor, class Expansion>
int multipole_kernel_interface(otfmm_context* ctx, const std::vector<double>& /*monopoles*/,
                               const std::vector<Multipole>& M_ptr,
                               const std::vector<std::shared_ptr<std::vector<SpaceVector>>>& com_ptr,
                               const std::vector<Neighbor>& neighbors, int type, double dx,
                               const std::array<bool, 26>& /*is_direction_empty*/, std::array<double, 3> xbase,
                               std::vector<Expansion>& L, std::vector<SpaceVector>& L_c, bool use_root_stencil,
                               int precision = OTFMM_FP64) {
    return multipole_kernel_impl(ctx, M_ptr, com_ptr, neighbors, type, dx, xbase, L, L_c, use_root_stencil,
                                 precision, nullptr);
}

// The reference's argument list (multipole_kernel_interface.hpp:18-22): the
// result goes to grid->get_L() / grid->get_L_c(), compressed payloads are
// expanded with grid->get_ilist_n_bnd(dir).
template <class Multipole, class SpaceVector, class Neighbor, class GridPtr>
int multipole_kernel_interface(otfmm_context* ctx, const std::vector<double>& /*monopoles*/,
                               const std::vector<Multipole>& M_ptr,
                               const std::vector<std::shared_ptr<std::vector<SpaceVector>>>& com_ptr,
                               const std::vector<Neighbor>& neighbors, int type, double dx,
                               const std::array<bool, 26>& /*is_direction_empty*/, std::array<double, 3> xbase,
                               const GridPtr& grid, bool use_root_stencil, int precision = OTFMM_FP64) {
    if (!grid) return OTFMM_ERR_INVALID;
    return multipole_kernel_impl(ctx, M_ptr, com_ptr, neighbors, type, dx, xbase, grid->get_L(), grid->get_L_c(),
                                 use_root_stencil, precision, grid);
}

template <class Multipole, class SpaceVector, class Neighbor, class Expansion>
void multipole_kernel_interface_or_abort(otfmm_context* ctx, const std::vector<double>& monopoles,
                                         const std::vector<Multipole>& M_ptr,
                                         const std::vector<std::shared_ptr<std::vector<SpaceVector>>>& com_ptr,
                                         const std::vector<Neighbor>& neighbors, int type, double dx,
                                         const std::array<bool, 26>& empty, std::array<double, 3> xbase,
                                         std::vector<Expansion>& L, std::vector<SpaceVector>& L_c,
                                         bool use_root_stencil, int precision = OTFMM_FP64) {
    const int rc = multipole_kernel_interface(ctx, monopoles, M_ptr, com_ptr, neighbors, type, dx, empty, xbase, L,
                                              L_c, use_root_stencil, precision);
    if (rc != OTFMM_OK) {
        std::cerr << "otfmm multipole kernel failed (" << rc << "): " << otfmm_last_error() << std::endl;
        std::abort();
    }
}

// monopole_kernel_interface(monopoles, com_ptr, neighbors, type, dx,
// is_direction_empty, grid, contains_multipole_neighbor): L[0..3] += P2P (+ P2M),
// L_c = P2M correction when a neighbour is refined (RHO). Device staging is
// allocated once per thread.
template <class SpaceVector, class Neighbor, class Expansion, class GridPtr>
int monopole_kernel_impl(otfmm_context* ctx, const std::vector<double>& monopoles,
                         const std::vector<std::shared_ptr<std::vector<SpaceVector>>>& com_ptr,
                         const std::vector<Neighbor>& neighbors, int type, double dx, std::vector<Expansion>& L,
                         std::vector<SpaceVector>& L_c, bool contains_multipole_neighbor, int precision,
                         const GridPtr& grid) {
    struct Dev {
        double* buf = nullptr;
        ~Dev() { if (buf) otfmm_device_free(buf); }
    };
    thread_local Dev dev;
    constexpr size_t n_mon = ENTRIES, n_L4 = 4 * CLU, n_Lc = 3 * CLU, n_icom = 3 * CLU, n_nM = 20 * 419,
                     n_ncom = 3 * 419;
    constexpr size_t total = n_mon + n_L4 + n_Lc + n_icom + n_nM + n_ncom;
    if (!dev.buf) {
        const int rc = otfmm_device_alloc(ctx, total * sizeof(double), reinterpret_cast<void**>(&dev.buf));
        if (rc != OTFMM_OK) return rc;
    }
    double* d_mon = dev.buf;
    double* d_L4 = d_mon + n_mon;
    double* d_Lc = d_L4 + n_L4;
    double* d_icom = d_Lc + n_Lc;
    double* d_nM = d_icom + n_icom;
    double* d_ncom = d_nM + n_nM;
    std::vector<double> mon(ENTRIES);
    int rc = stage_monopole_input(monopoles, neighbors, mon.data(), grid);
    if (rc == OTFMM_OK) rc = otfmm_copy_to_device(ctx, d_mon, mon.data(), sizeof(double) * ENTRIES);
    if (rc == OTFMM_OK) rc = otfmm_p2p_soa(ctx, d_mon, dx, d_L4, precision == OTFMM_FP64_EXACT ? OTFMM_FP64_EXACT : OTFMM_FP64, nullptr);
    if (rc != OTFMM_OK) return rc;
    bool any_p2m = false;
    if (contains_multipole_neighbor) {
        std::vector<double> icom(3 * CLU, 0.0), nM(20 * 419, 0.0), ncom(3 * 419, 0.0);
        const SpaceVector* com0 = com_ptr[0]->data();
        for (int c = 0; c < 3; ++c)
            for (int u = 0; u < NCELL; ++u) icom[c * CLU + u] = com0[u][c];
        rc = otfmm_copy_to_device(ctx, d_icom, icom.data(), sizeof(double) * 3 * CLU);
        if (rc != OTFMM_OK) return rc;
        for (int d = 0; d < 26; ++d) {
            const Neighbor& nb = neighbors[d];
            if (nb.is_monopole || !nb.data.M) continue;
            int stride = 0;
            rc = stage_p2m_slab(nb, d, nM.data(), ncom.data(), &stride, grid);
            if (rc != OTFMM_OK) return rc;
            rc = otfmm_copy_to_device(ctx, d_nM, nM.data(), sizeof(double) * 20 * stride);
            if (rc == OTFMM_OK) rc = otfmm_copy_to_device(ctx, d_ncom, ncom.data(), sizeof(double) * 3 * stride);
            if (rc == OTFMM_OK)
                rc = otfmm_p2m_soa(ctx, d, d_nM, d_ncom, d_icom, d_L4, d_Lc, type, any_p2m ? 0 : 1,
                                   precision == OTFMM_FP64_EXACT ? OTFMM_FP64_EXACT : OTFMM_FP64, nullptr);
            if (rc != OTFMM_OK) return rc;
            any_p2m = true;
        }
    }
    Staging& st = thread_staging();
    rc = otfmm_copy_to_host(ctx, st.L.data(), d_L4, sizeof(double) * 4 * CLU);
    if (rc == OTFMM_OK && any_p2m && type == OTFMM_RHO) rc = otfmm_copy_to_host(ctx, st.Lc.data(), d_Lc, sizeof(double) * 3 * CLU);
    if (rc != OTFMM_OK) return rc;
    for (int c = 0; c < 4; ++c)
        for (int u = 0; u < NCELL; ++u) L[u][c] += st.L[c * CLU + u];
    if (any_p2m && type == OTFMM_RHO)
        for (int c = 0; c < 3; ++c)
            for (int u = 0; u < NCELL; ++u) L_c[u][c] = st.Lc[c * CLU + u];
    return OTFMM_OK;
}

// L and L_c passed explicitly; every neighbour payload full size.
template <class SpaceVector, class Neighbor, class Expansion>
int monopole_kernel_interface(otfmm_context* ctx, const std::vector<double>& monopoles,
                              const std::vector<std::shared_ptr<std::vector<SpaceVector>>>& com_ptr,
                              const std::vector<Neighbor>& neighbors, int type, double dx,
                              const std::array<bool, 26>& /*is_direction_empty*/, std::vector<Expansion>& L,
                              std::vector<SpaceVector>& L_c, bool contains_multipole_neighbor,
                              int precision = OTFMM_FP64) {
    return monopole_kernel_impl(ctx, monopoles, com_ptr, neighbors, type, dx, L, L_c, contains_multipole_neighbor,
                                precision, nullptr);
}

// The reference's argument list (monopole_kernel_interface.hpp:19-23): the
// result goes to grid->get_L() / grid->get_L_c(), compressed payloads are
// expanded with grid->get_ilist_n_bnd(dir).
template <class SpaceVector, class Neighbor, class GridPtr>
int monopole_kernel_interface(otfmm_context* ctx, const std::vector<double>& monopoles,
                              const std::vector<std::shared_ptr<std::vector<SpaceVector>>>& com_ptr,
                              const std::vector<Neighbor>& neighbors, int type, double dx,
                              const std::array<bool, 26>& /*is_direction_empty*/, const GridPtr& grid,
                              bool contains_multipole_neighbor, int precision = OTFMM_FP64) {
    if (!grid) return OTFMM_ERR_INVALID;
    return monopole_kernel_impl(ctx, monopoles, com_ptr, neighbors, type, dx, grid->get_L(), grid->get_L_c(),
                                contains_multipole_neighbor, precision, grid);
}

// ---------------------------------------------------------------- aggregated calls
// The same two interfaces on an otfmm_aggregator (otfmm.h): the call's records
// (its own subgrid, then its neighbours' payloads) go into the open batch's
// pinned pool slots - a payload that aliases data already in the batch (same
// address) is not copied again - and its work item joins the batched solve.
// Each interface comes as a pair: *_submit returns as soon as the call is in
// its batch (many calls of a thread may be in flight, as HPX tasks are), and
// finish() waits for the call's batch and updates the grid exactly as the
// per-call overloads do; the plain overloads do both. `type` must be the
// aggregator's solve type; the precision is the aggregator's.
template <class T>
inline uint64_t data_key(const T* p) {
    return static_cast<uint64_t>(reinterpret_cast<std::uintptr_t>(p));
}

// A submitted call: its ticket, its result buffers and where they go.
template <class GridPtr>
struct AggregatedCall {
    otfmm_aggregator* agg = nullptr;
    int64_t ticket = 0;
    int ncomp = 20;          // L components the call's kind writes (20 multipole, 4 monopole)
    bool write_lc = false;   // L_c = result (RHO multipole; RHO monopole with a refined neighbour)
    bool in_place = true;    // let the batch write a grid of flat cells itself (set before submitting)
    bool direct = false;     // the batch writes the grid's cells itself (otfmm_aggregator_submit_aos)
    GridPtr grid{};
    std::vector<double> L, Lc;   // SoA results otherwise, applied by finish()
};

// Cell u's component c of `v` (taylor<4> / space_vector cells) is the double
// at data() + u * K + c: K doubles per cell, reached through operator[] as
// plain members. Checked on the element type and on the addresses of cells 0
// and 1; such a grid gets its results written in place by the batch.
template <int K, class V>
inline double* flat_cells(V& v) {
    using E = typename V::value_type;
    if constexpr (sizeof(E) == K * sizeof(double) && std::is_standard_layout_v<E> &&
                  std::is_same_v<decltype(std::declval<E&>()[0]), double&>) {
        if (v.size() < (size_t)NCELL) return nullptr;
        double* base = reinterpret_cast<double*>(v.data());
        const bool flat = &v[0][0] == base && &v[0][K - 1] == base + K - 1 && &v[1][0] == base + K;
        return flat ? base : nullptr;
    } else {
        return nullptr;
    }
}

// Rows c = 0..K-1 (row stride NCELL) of a pool record from the cells' AoS
// values src[u][c], 8 cells at a time, so that every block writes whole cache
// lines of each row (about twice as fast as a cell-by-cell transpose).
template <int K, class AoS>
inline void aos_to_soa(double* dst, const AoS& src) {
    for (int u0 = 0; u0 < NCELL; u0 += 8)
        for (int c = 0; c < K; ++c)
            for (int u = u0; u < u0 + 8; ++u) dst[c * NCELL + u] = src[u][c];
}

// Reserves, fills and submits one call: own record (M + com for a refined node,
// masses + com for a leaf) and the 26 neighbour payloads.
template <class Multipole, class SpaceVector, class Neighbor, class GridPtr>
int aggregated_submit(otfmm_aggregator* agg, int kind, const std::vector<Multipole>* own_M,
                      const std::vector<double>* own_mon, const SpaceVector* own_com,
                      const std::vector<Neighbor>& neighbors, double dx, const std::array<double, 3>& xbase,
                      const GridPtr& grid, AggregatedCall<GridPtr>& call) {
    uint64_t keys[27];
    uint8_t leaf[27], need[27], fill[27];
    int32_t slots[27];
    int dir_of[27];
    const bool own_leaf = (kind == OTFMM_KIND_LEAF);
    keys[0] = own_leaf ? data_key(own_mon->data()) : data_key(own_M->data());
    leaf[0] = own_leaf ? 1 : 0;
    need[0] = own_leaf ? (OTFMM_AGG_MON | OTFMM_AGG_COM) : (OTFMM_AGG_M | OTFMM_AGG_COM);
    dir_of[0] = -1;
    int n = 1;
    if (kind != OTFMM_KIND_M2L_ROOT) {
        for (int d = 0; d < 26; ++d) {
            const Neighbor& nb = neighbors[d];
            if (nb.is_monopole) {
                if (!nb.data.m) continue;
                keys[n] = nb.data.m->size() == NCELL ? data_key(nb.data.m->data()) : 0;
                leaf[n] = 1;
                need[n] = OTFMM_AGG_MON;
            } else {
                if (!nb.data.M) continue;
                const bool full = nb.data.M->size() == NCELL && nb.data.x && nb.data.x->size() == NCELL;
                keys[n] = full ? data_key(nb.data.M->data()) : 0;
                leaf[n] = 0;
                need[n] = OTFMM_AGG_M | OTFMM_AGG_COM;
            }
            dir_of[n++] = d;
        }
    }
    int64_t ticket = 0;
    int rc = otfmm_aggregator_reserve(agg, n, keys, leaf, need, slots, fill, &ticket);
    if (rc != OTFMM_OK) return rc;
    otfmm_work_item item{};
    item.subgrid = slots[0];
    item.kind = kind;
    item.dx = dx;
    for (int a = 0; a < 3; ++a) item.xbase[a] = xbase[a];
    for (int d = 0; d < 26; ++d) item.neighbors[d] = -1;
    for (int i = 0; i < n && rc == OTFMM_OK; ++i) {
        if (i > 0) item.neighbors[dir_of[i]] = slots[i];
        if (!fill[i]) continue;
        double *M, *com, *mon;
        rc = otfmm_aggregator_record(agg, ticket, slots[i], &M, &com, &mon);
        if (rc != OTFMM_OK) break;
        if (i == 0) {
            if (fill[0] & OTFMM_AGG_M) aos_to_soa<20>(M, *own_M);
            if (fill[0] & OTFMM_AGG_COM) aos_to_soa<3>(com, own_com);
            if (fill[0] & OTFMM_AGG_MON) std::copy(own_mon->begin(), own_mon->begin() + NCELL, mon);
            continue;
        }
        const int d = dir_of[i];
        const Neighbor& nb = neighbors[d];
        if (keys[i] != 0) {   // full-size payload
            if (fill[i] & OTFMM_AGG_MON) std::copy(nb.data.m->begin(), nb.data.m->begin() + NCELL, mon);
            if (fill[i] & OTFMM_AGG_M) aos_to_soa<20>(M, *nb.data.M);
            if (fill[i] & OTFMM_AGG_COM) aos_to_soa<3>(com, *nb.data.x);
            continue;
        }
        // compressed payload (get_ilist_n_bnd order): zeros, then the listed cells
        std::fill(M, M + 20 * NCELL, 0.0);
        std::fill(com, com + 3 * NCELL, 0.0);
        std::fill(mon, mon + NCELL, 0.0);
        if (nb.is_monopole) {
            const auto& m = *nb.data.m;
            rc = expand_compressed(grid, d, m.size(), [&](size_t k, int x, int y, int z) {
                mon[flat_inner(x, y, z)] = m[k];
            });
        } else {
            const auto& nM = *nb.data.M;
            const size_t cnt = nb.data.x ? std::min(nM.size(), nb.data.x->size()) : 0;
            rc = expand_compressed(grid, d, cnt, [&](size_t k, int x, int y, int z) {
                const int u = flat_inner(x, y, z);
                for (int c = 0; c < 20; ++c) M[c * NCELL + u] = nM[k][c];
                for (int c = 0; c < 3; ++c) com[c * NCELL + u] = (*nb.data.x)[k][c];
            });
        }
    }
    call.agg = agg;
    call.ticket = ticket;
    call.grid = grid;
    if (rc != OTFMM_OK) {
        // withdraw the reservation so that the batch can run without this call
        item.subgrid = -1;
        otfmm_aggregator_submit(agg, ticket, &item, nullptr, nullptr);
        call.agg = nullptr;
        return rc;
    }
    double* gL = flat_cells<20>(grid->get_L());
    double* gLc = call.write_lc ? flat_cells<3>(grid->get_L_c()) : nullptr;
    call.direct = call.in_place && gL && (gLc || !call.write_lc);
    if (call.direct) {
        rc = otfmm_aggregator_submit_aos(agg, ticket, &item, gL, 20, gLc, 3);
    } else {
        call.L.assign((size_t)call.ncomp * NCELL, 0.0);
        call.Lc.assign(3 * NCELL, 0.0);
        rc = otfmm_aggregator_submit(agg, ticket, &item, call.L.data(), call.Lc.data());
    }
    if (rc != OTFMM_OK) call.agg = nullptr;
    return rc;
}

// 1 once a submitted call's batch has run (finish() then returns at once), 0
// before, < 0 on error. Does not wait for other callers; it may run a batch
// that is ready to run (the batch's solve time). An HPX task polls and yields
// in between instead of blocking its worker thread in finish().
template <class GridPtr>
int ready(const AggregatedCall<GridPtr>& call) {
    if (!call.agg) return OTFMM_ERR_INVALID;
    return otfmm_aggregator_poll(call.agg, call.ticket);
}

// Waits for a submitted call's batch, then updates the grid: L += result,
// L_c = result where the reference sets it (a grid of flat cells was updated
// by the batch already).
template <class GridPtr>
int finish(AggregatedCall<GridPtr>& call) {
    if (!call.agg) return OTFMM_ERR_INVALID;
    const int rc = otfmm_aggregator_wait(call.agg, call.ticket);
    call.agg = nullptr;
    if (rc != OTFMM_OK || call.direct) return rc;
    auto& gL = call.grid->get_L();
    for (int u0 = 0; u0 < NCELL; u0 += 8)
        for (int c = 0; c < call.ncomp; ++c)
            for (int u = u0; u < u0 + 8; ++u) gL[u][c] += call.L[c * NCELL + u];
    if (call.write_lc) {
        auto& gLc = call.grid->get_L_c();
        for (int u0 = 0; u0 < NCELL; u0 += 8)
            for (int c = 0; c < 3; ++c)
                for (int u = u0; u < u0 + 8; ++u) gLc[u][c] = call.Lc[c * NCELL + u];
    }
    return OTFMM_OK;
}

// multipole_kernel_interface on an aggregator, the reference's argument list
// (multipole_kernel_interface.hpp:18-22): submit now, finish() later.
template <class Multipole, class SpaceVector, class Neighbor, class GridPtr>
int multipole_kernel_interface_submit(otfmm_aggregator* agg, const std::vector<double>& /*monopoles*/,
                                      const std::vector<Multipole>& M_ptr,
                                      const std::vector<std::shared_ptr<std::vector<SpaceVector>>>& com_ptr,
                                      const std::vector<Neighbor>& neighbors, int type, double dx,
                                      const std::array<bool, 26>& /*is_direction_empty*/,
                                      std::array<double, 3> xbase, const GridPtr& grid, bool use_root_stencil,
                                      AggregatedCall<GridPtr>& call) {
    if (!agg || !grid || M_ptr.size() != NCELL || com_ptr.empty() || !com_ptr[0]) return OTFMM_ERR_INVALID;
    call.ncomp = 20;
    call.write_lc = (type == OTFMM_RHO);
    const int kind = use_root_stencil ? OTFMM_KIND_M2L_ROOT : OTFMM_KIND_M2L;
    return aggregated_submit(agg, kind, &M_ptr, static_cast<const std::vector<double>*>(nullptr),
                             com_ptr[0]->data(), neighbors, dx, xbase, grid, call);
}

template <class Multipole, class SpaceVector, class Neighbor, class GridPtr>
int multipole_kernel_interface(otfmm_aggregator* agg, const std::vector<double>& monopoles,
                               const std::vector<Multipole>& M_ptr,
                               const std::vector<std::shared_ptr<std::vector<SpaceVector>>>& com_ptr,
                               const std::vector<Neighbor>& neighbors, int type, double dx,
                               const std::array<bool, 26>& is_direction_empty, std::array<double, 3> xbase,
                               const GridPtr& grid, bool use_root_stencil) {
    AggregatedCall<GridPtr> call;
    const int rc = multipole_kernel_interface_submit(agg, monopoles, M_ptr, com_ptr, neighbors, type, dx,
                                                     is_direction_empty, xbase, grid, use_root_stencil, call);
    return rc != OTFMM_OK ? rc : finish(call);
}

// monopole_kernel_interface on an aggregator, the reference's argument list
// (monopole_kernel_interface.hpp:19-23): L[0..3] += P2P (+ P2M); L_c = the P2M
// correction when a neighbour is refined (RHO).
template <class SpaceVector, class Neighbor, class GridPtr>
int monopole_kernel_interface_submit(otfmm_aggregator* agg, const std::vector<double>& monopoles,
                                     const std::vector<std::shared_ptr<std::vector<SpaceVector>>>& com_ptr,
                                     const std::vector<Neighbor>& neighbors, int type, double dx,
                                     const std::array<bool, 26>& /*is_direction_empty*/, const GridPtr& grid,
                                     bool contains_multipole_neighbor, AggregatedCall<GridPtr>& call) {
    if (!agg || !grid || monopoles.size() != NCELL || com_ptr.empty() || !com_ptr[0]) return OTFMM_ERR_INVALID;
    call.ncomp = 4;
    call.write_lc = contains_multipole_neighbor && type == OTFMM_RHO;
    using Multipole = std::array<double, 20>;
    const std::array<double, 3> xbase{0.0, 0.0, 0.0};   // leaves use integer offsets only
    return aggregated_submit(agg, OTFMM_KIND_LEAF, static_cast<const std::vector<Multipole>*>(nullptr), &monopoles,
                             com_ptr[0]->data(), neighbors, dx, xbase, grid, call);
}

template <class SpaceVector, class Neighbor, class GridPtr>
int monopole_kernel_interface(otfmm_aggregator* agg, const std::vector<double>& monopoles,
                              const std::vector<std::shared_ptr<std::vector<SpaceVector>>>& com_ptr,
                              const std::vector<Neighbor>& neighbors, int type, double dx,
                              const std::array<bool, 26>& is_direction_empty, const GridPtr& grid,
                              bool contains_multipole_neighbor) {
    AggregatedCall<GridPtr> call;
    const int rc = monopole_kernel_interface_submit(agg, monopoles, com_ptr, neighbors, type, dx, is_direction_empty,
                                                    grid, contains_multipole_neighbor, call);
    return rc != OTFMM_OK ? rc : finish(call);
}

}   // namespace otfmm_octotiger
