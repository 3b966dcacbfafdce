// Stand-ins for the Octo-Tiger types the adapter in include/otfmm_octotiger.hpp
// is written against (taylor<4>, space_vector, gravity_boundary_type,
// neighbor_gravity_type, boundary_interaction_type and the grid accessors
// get_L / get_L_c / get_ilist_n_bnd), plus a shuffled halo-band cell list
// standing in for grid::get_ilist_n_bnd.
#pragma once

#include <array>
#include <cstdint>
#include <memory>
#include <utility>
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
struct boundary_interaction_type {
    std::uint16_t second;
};
struct grid {
    std::vector<multipole> L = std::vector<multipole>(512);
    std::vector<space_vector> L_c = std::vector<space_vector>(512);
    std::array<std::vector<boundary_interaction_type>, 26> ilist_n_bnd;
    std::vector<multipole>& get_L() { return L; }
    std::vector<space_vector>& get_L_c() { return L_c; }
    const std::vector<boundary_interaction_type>& get_ilist_n_bnd(int d) const { return ilist_n_bnd[d]; }
};

// halo band of direction d in the neighbour's frame, shuffled (fixed LCG)
inline std::vector<boundary_interaction_type> band_list(int d, unsigned seed) {
    int o[3], s[3], e[3], p[3];
    otfmm_octotiger::dir_offsets(d, o);
    otfmm_octotiger::padding_range(o, s, e, p);
    std::vector<boundary_interaction_type> l;
    for (int x = s[0]; x < e[0]; ++x)
        for (int y = s[1]; y < e[1]; ++y)
            for (int z = s[2]; z < e[2]; ++z) l.push_back({std::uint16_t(64 * x + 8 * y + z)});
    unsigned r = seed * 2654435761u + 12345u;
    for (size_t i = l.size(); i > 1; --i) {
        r = r * 1664525u + 1013904223u;
        std::swap(l[i - 1], l[(r >> 8) % i]);
    }
    return l;
}
