// Drives include/otfmm_octotiger.hpp with stand-ins for Octo-Tiger's types.
// Reads one work item and its subgrid pool from a binary file (written by
// tests/test_gpu_adapter.py), builds the AoS inputs node_server::compute_fmm
// hands to the interaction interfaces, calls the adapter and writes the grid's
// L (512 x 20) and L_c (512 x 3) after the call.
//
// Payload modes (5th argument):
//   0  full-size payloads, L / L_c passed explicitly;
//   1  the grid overloads; every other neighbour with data sends a compressed
//      payload listing all cells of its halo band in a shuffled order;
//   2  as 1, but every third listed cell is left out of the list;
//   3  the grid overloads with full-size payloads whose cells left out in
//      mode 2 are zeroed (mode 2 must equal this bit for bit);
//   4  the compressed payloads of mode 1 through the overloads without a grid
//      (must fail with OTFMM_ERR_INVALID: exit code 7).
#include <array>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <vector>

#include "octotiger_standins.hpp"

int main(int argc, char** argv) {
    if (argc != 5 && argc != 6) {
        std::fprintf(stderr, "usage: adapter_test in.bin out.bin precision theta [mode]\n");
        return 2;
    }
    const int mode = argc == 6 ? std::atoi(argv[5]) : 0;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    auto rd = [&](void* p, size_t size, size_t count) {
        if (std::fread(p, size, count, f) != count) std::exit(6);
    };
    int32_t n, kind, type, subgrid, nb[26];
    double dx, xbase[3];
    rd(&n, 4, 1);
    rd(&kind, 4, 1);
    rd(&type, 4, 1);
    rd(&subgrid, 4, 1);
    rd(nb, 4, 26);
    rd(&dx, 8, 1);
    rd(xbase, 8, 3);
    std::vector<double> M(size_t(n) * 20 * 512), com(size_t(n) * 3 * 512), mon(size_t(n) * 512);
    std::vector<uint8_t> is_leaf(n);
    rd(M.data(), 8, M.size());
    rd(com.data(), 8, com.size());
    rd(mon.data(), 8, mon.size());
    rd(is_leaf.data(), 1, n);
    std::fclose(f);
    auto multipoles_of = [&](int s) {
        auto v = std::make_shared<std::vector<multipole>>(512);
        for (int u = 0; u < 512; ++u)
            for (int c = 0; c < 20; ++c) (*v)[u][c] = M[(size_t(s) * 20 + c) * 512 + u];
        return v;
    };
    auto coms_of = [&](int s) {
        auto v = std::make_shared<std::vector<space_vector>>(512);
        for (int u = 0; u < 512; ++u)
            for (int c = 0; c < 3; ++c) (*v)[u][c] = com[(size_t(s) * 3 + c) * 512 + u];
        return v;
    };
    auto masses_of = [&](int s) {
        return std::make_shared<std::vector<double>>(mon.begin() + size_t(s) * 512, mon.begin() + size_t(s + 1) * 512);
    };
    // what compute_fmm collects (src/node_server.cpp:667-690): one entry per direction
    std::vector<neighbor_gravity_type> neighbors(26);
    std::array<bool, 26> empty{};
    bool contains_multipole = false;
    for (int d = 0; d < 26; ++d) {
        empty[d] = nb[d] < 0;
        if (nb[d] < 0) continue;
        neighbors[d].is_monopole = is_leaf[nb[d]] != 0;
        if (neighbors[d].is_monopole) {
            neighbors[d].data.m = masses_of(nb[d]);
        } else {
            neighbors[d].data.M = multipoles_of(nb[d]);
            neighbors[d].data.x = coms_of(nb[d]);
            contains_multipole = true;
        }
    }
    auto g = std::make_shared<grid>();
    if (mode != 0) {
        for (int d = 1; d < 26; d += 2) {
            neighbor_gravity_type& n = neighbors[d];
            if (!n.data.M && !n.data.m) continue;
            std::vector<boundary_interaction_type> all = band_list(d, 97u + unsigned(d)), kept;
            for (size_t i = 0; i < all.size(); ++i)
                if (mode == 1 || mode == 4 || i % 3 != 2) kept.push_back(all[i]);
            if (mode == 3) {
                // full payload, the left-out cells zeroed
                for (size_t i = 2; i < all.size(); i += 3) {
                    const int u = all[i].second;
                    if (n.is_monopole) {
                        (*n.data.m)[u] = 0.0;
                    } else {
                        (*n.data.M)[u] = multipole{};
                        (*n.data.x)[u] = space_vector{};
                    }
                }
                continue;
            }
            g->ilist_n_bnd[d] = kept;
            if (n.is_monopole) {
                auto m = std::make_shared<std::vector<double>>();
                for (auto c : kept) m->push_back((*n.data.m)[c.second]);
                n.data.m = m;
            } else {
                auto Mc = std::make_shared<std::vector<multipole>>();
                auto xc = std::make_shared<std::vector<space_vector>>();
                for (auto c : kept) {
                    Mc->push_back((*n.data.M)[c.second]);
                    xc->push_back((*n.data.x)[c.second]);
                }
                n.data.M = Mc;
                n.data.x = xc;
            }
        }
    }
    std::vector<std::shared_ptr<std::vector<space_vector>>> com_ptr{coms_of(subgrid)};
    std::vector<double> monopoles(mon.begin() + size_t(subgrid) * 512, mon.begin() + size_t(subgrid + 1) * 512);
    std::vector<expansion> L(512);        // zeroed by compute_fmm before the call
    std::vector<space_vector> L_c(512);
    otfmm_context* ctx = nullptr;
    int rc = otfmm_create(0, std::atof(argv[4]), &ctx);
    if (rc != OTFMM_OK) {
        std::fprintf(stderr, "create: %s\n", otfmm_last_error());
        return 4;
    }
    const int precision = std::atoi(argv[3]);
    const std::array<double, 3> xb{xbase[0], xbase[1], xbase[2]};
    const bool with_grid = mode == 1 || mode == 2 || mode == 3;
    if (kind == OTFMM_KIND_LEAF) {
        if (with_grid)
            rc = otfmm_octotiger::monopole_kernel_interface(ctx, monopoles, com_ptr, neighbors, type, dx, empty, g,
                                                            contains_multipole, precision);
        else
            rc = otfmm_octotiger::monopole_kernel_interface(ctx, monopoles, com_ptr, neighbors, type, dx, empty, L,
                                                            L_c, contains_multipole, precision);
    } else {
        if (with_grid)
            rc = otfmm_octotiger::multipole_kernel_interface(ctx, monopoles, *multipoles_of(subgrid), com_ptr,
                                                             neighbors, type, dx, empty, xb, g,
                                                             kind == OTFMM_KIND_M2L_ROOT, precision);
        else
            rc = otfmm_octotiger::multipole_kernel_interface(ctx, monopoles, *multipoles_of(subgrid), com_ptr,
                                                             neighbors, type, dx, empty, xb, L, L_c,
                                                             kind == OTFMM_KIND_M2L_ROOT, precision);
    }
    otfmm_destroy(ctx);
    if (mode == 4) return rc == OTFMM_ERR_INVALID ? 7 : 8;
    if (rc != OTFMM_OK) {
        std::fprintf(stderr, "adapter: %d %s\n", rc, otfmm_last_error());
        return 5;
    }
    if (with_grid) {
        L = g->L;
        L_c = g->L_c;
    }
    FILE* o = std::fopen(argv[2], "wb");
    for (int u = 0; u < 512; ++u) std::fwrite(L[u].v.data(), 8, 20, o);
    for (int u = 0; u < 512; ++u) std::fwrite(L_c[u].data(), 8, 3, o);
    std::fclose(o);
    return 0;
}
