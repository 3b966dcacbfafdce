// Drives include/otfmm_octotiger.hpp with stand-ins for Octo-Tiger's types.
// Reads one work item and its subgrid pool from a binary file (written by
// tests/test_gpu_adapter.py), builds the AoS inputs node_server::compute_fmm
// hands to the interaction interfaces, calls the adapter and writes the grid's
// L (512 x 20) and L_c (512 x 3) after the call.
#include <array>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <vector>

#include "otfmm_octotiger.hpp"

struct multipole {
    std::array<double, 20> v{};
    double& operator[](int i) { return v[i]; }
    const double& operator[](int i) const { return v[i]; }
};
using expansion = multipole;
using space_vector = std::array<double, 3>;
struct gravity_boundary_type {
    std::shared_ptr<std::vector<multipole>> M;
    std::shared_ptr<std::vector<double>> m;
    std::shared_ptr<std::vector<space_vector>> x;
};
struct neighbor_gravity_type {
    gravity_boundary_type data;
    bool is_monopole = false;
};

int main(int argc, char** argv) {
    if (argc != 5) {
        std::fprintf(stderr, "usage: adapter_test in.bin out.bin precision theta\n");
        return 2;
    }
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
    if (kind == OTFMM_KIND_LEAF) {
        rc = otfmm_octotiger::monopole_kernel_interface(ctx, monopoles, com_ptr, neighbors, type, dx, empty, L, L_c,
                                                        contains_multipole, precision);
    } else {
        rc = otfmm_octotiger::multipole_kernel_interface(ctx, monopoles, *multipoles_of(subgrid), com_ptr, neighbors,
                                                         type, dx, empty, xb, L, L_c, kind == OTFMM_KIND_M2L_ROOT,
                                                         precision);
    }
    if (rc != OTFMM_OK) {
        std::fprintf(stderr, "adapter: %s\n", otfmm_last_error());
        return 5;
    }
    otfmm_destroy(ctx);
    FILE* o = std::fopen(argv[2], "wb");
    for (int u = 0; u < 512; ++u) std::fwrite(L[u].v.data(), 8, 20, o);
    for (int u = 0; u < 512; ++u) std::fwrite(L_c[u].data(), 8, 3, o);
    std::fclose(o);
    return 0;
}
