// CPU check of the adapter's halo staging (include/otfmm_octotiger.hpp) for
// compressed neighbour payloads, no device needed: for seeded neighbours
// (refined, leaf and empty directions) it stages the multipole input, the
// monopole input and the P2M slabs three ways and compares the buffers bit
// for bit:
//   * compressed payloads listing the whole halo band (shuffled) == full size;
//   * compressed payloads with every third listed cell left out == full size
//     with those cells zeroed (update_input resets the band, then fills);
// and checks that a compressed payload without a grid, a listed cell outside
// the halo band and a list longer than its payload are rejected.
// Prints "staging ok" and exits 0 on success.
#include <cstdio>
#include <cstring>
#include <random>

#include "octotiger_standins.hpp"

namespace oo = otfmm_octotiger;

struct Staged {
    std::vector<double> mon, M, com, pmon;
    std::vector<std::vector<double>> slabM, slabX;
};

static void fail(const char* what) {
    std::fprintf(stderr, "staging test failed: %s\n", what);
    std::exit(1);
}

template <class GridPtr>
static int stage_all(const std::vector<multipole>& own, const std::vector<space_vector>& own_x,
                     const std::vector<double>& own_m, const std::vector<neighbor_gravity_type>& nbs, const GridPtr& g,
                     Staged& out) {
    oo::Staging st;
    const std::array<double, 3> xbase{0.25, -0.125, 0.5};
    int rc = oo::stage_multipole_input(own, own_x.data(), nbs, 1.0 / 64, xbase, false, st, g);
    if (rc != OTFMM_OK) return rc;
    out.mon = st.mon;
    out.M = st.M;
    out.com = st.com;
    out.pmon.assign(oo::ENTRIES, -1.0);
    rc = oo::stage_monopole_input(own_m, nbs, out.pmon.data(), g);
    if (rc != OTFMM_OK) return rc;
    out.slabM.clear();
    out.slabX.clear();
    for (int d = 0; d < 26; ++d) {
        if (nbs[d].is_monopole || !nbs[d].data.M) continue;
        std::vector<double> nM(20 * 419, -1.0), nX(3 * 419, -1.0);
        int stride = 0;
        rc = oo::stage_p2m_slab(nbs[d], d, nM.data(), nX.data(), &stride, g);
        if (rc != OTFMM_OK) return rc;
        nM.resize(20 * stride);
        nX.resize(3 * stride);
        out.slabM.push_back(nM);
        out.slabX.push_back(nX);
    }
    return OTFMM_OK;
}

static bool same(const Staged& a, const Staged& b) {
    auto eq = [](const std::vector<double>& x, const std::vector<double>& y) {
        return x.size() == y.size() && std::memcmp(x.data(), y.data(), x.size() * sizeof(double)) == 0;
    };
    if (!eq(a.mon, b.mon) || !eq(a.M, b.M) || !eq(a.com, b.com) || !eq(a.pmon, b.pmon)) return false;
    if (a.slabM.size() != b.slabM.size()) return false;
    for (size_t i = 0; i < a.slabM.size(); ++i)
        if (!eq(a.slabM[i], b.slabM[i]) || !eq(a.slabX[i], b.slabX[i])) return false;
    return true;
}

int main() {
    std::mt19937_64 rng(20261203);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    std::vector<multipole> own(512);
    std::vector<space_vector> own_x(512);
    std::vector<double> own_m(512);
    for (int u = 0; u < 512; ++u) {
        for (int c = 0; c < 20; ++c) own[u][c] = U(rng);
        for (int c = 0; c < 3; ++c) own_x[u][c] = U(rng);
        own_m[u] = 1.5 + U(rng);
    }
    // directions: every 5th empty, every 3rd a leaf, the rest refined
    std::vector<neighbor_gravity_type> full(26);
    for (int d = 0; d < 26; ++d) {
        if (d % 5 == 4) {
            full[d].is_monopole = (d % 2) == 0;
            continue;
        }
        if (d % 3 == 0) {
            full[d].is_monopole = true;
            full[d].data.m = std::make_shared<std::vector<double>>(512);
            for (auto& v : *full[d].data.m) v = 1.5 + U(rng);
        } else {
            full[d].data.M = std::make_shared<std::vector<multipole>>(512);
            full[d].data.x = std::make_shared<std::vector<space_vector>>(512);
            for (auto& v : *full[d].data.M)
                for (int c = 0; c < 20; ++c) v[c] = U(rng);
            for (auto& v : *full[d].data.x)
                for (int c = 0; c < 3; ++c) v[c] = U(rng);
        }
    }
    auto deep_copy = [](const std::vector<neighbor_gravity_type>& in) {
        std::vector<neighbor_gravity_type> out(in.size());
        for (size_t d = 0; d < in.size(); ++d) {
            out[d].is_monopole = in[d].is_monopole;
            if (in[d].data.m) out[d].data.m = std::make_shared<std::vector<double>>(*in[d].data.m);
            if (in[d].data.M) out[d].data.M = std::make_shared<std::vector<multipole>>(*in[d].data.M);
            if (in[d].data.x) out[d].data.x = std::make_shared<std::vector<space_vector>>(*in[d].data.x);
        }
        return out;
    };
    // compress the payloads of `dirs` to `lists` (grid::get_gravity_boundary's packing)
    auto compress = [](std::vector<neighbor_gravity_type>& nbs, grid& g, int d,
                       const std::vector<boundary_interaction_type>& list) {
        g.ilist_n_bnd[d] = list;
        neighbor_gravity_type& n = nbs[d];
        if (n.is_monopole) {
            auto m = std::make_shared<std::vector<double>>();
            for (auto c : list) m->push_back((*n.data.m)[c.second]);
            n.data.m = m;
        } else {
            auto M = std::make_shared<std::vector<multipole>>();
            auto x = std::make_shared<std::vector<space_vector>>();
            for (auto c : list) {
                M->push_back((*n.data.M)[c.second]);
                x->push_back((*n.data.x)[c.second]);
            }
            n.data.M = M;
            n.data.x = x;
        }
    };

    Staged ref, got;
    if (stage_all(own, own_x, own_m, full, nullptr, ref) != OTFMM_OK) fail("full-size staging");

    // 1. whole band, shuffled: equal to full size
    {
        auto nbs = deep_copy(full);
        auto g = std::make_shared<grid>();
        for (int d = 0; d < 26; ++d)
            if (nbs[d].data.m || nbs[d].data.M) compress(nbs, *g, d, band_list(d, 7u + unsigned(d)));
        if (stage_all(own, own_x, own_m, nbs, g, got) != OTFMM_OK) fail("compressed staging");
        if (!same(ref, got)) fail("compressed (whole band) differs from full size");
    }
    // 2. every third listed cell left out: equal to full size with those cells zeroed
    {
        auto nbs = deep_copy(full), zeroed = deep_copy(full);
        auto g = std::make_shared<grid>();
        for (int d = 0; d < 26; ++d) {
            if (!nbs[d].data.m && !nbs[d].data.M) continue;
            const auto all = band_list(d, 31u + unsigned(d));
            std::vector<boundary_interaction_type> kept;
            for (size_t i = 0; i < all.size(); ++i) {
                if (i % 3 != 2) {
                    kept.push_back(all[i]);
                    continue;
                }
                const int u = all[i].second;
                if (zeroed[d].is_monopole) {
                    (*zeroed[d].data.m)[u] = 0.0;
                } else {
                    (*zeroed[d].data.M)[u] = multipole{};
                    (*zeroed[d].data.x)[u] = space_vector{};
                }
            }
            compress(nbs, *g, d, kept);
        }
        Staged want;
        if (stage_all(own, own_x, own_m, zeroed, nullptr, want) != OTFMM_OK) fail("zeroed staging");
        if (stage_all(own, own_x, own_m, nbs, g, got) != OTFMM_OK) fail("subset staging");
        if (!same(want, got)) fail("compressed (subset) differs from zeroed full size");
        if (same(ref, got)) fail("leaving cells out changed nothing");
    }
    // 3. rejected: no grid; a cell outside the band; a list longer than its payload
    for (int d : {1, 3}) {   // a refined and a leaf direction
        auto nbs = deep_copy(full);
        auto g = std::make_shared<grid>();
        compress(nbs, *g, d, band_list(d, 5u));
        if (stage_all(own, own_x, own_m, nbs, nullptr, got) != OTFMM_ERR_INVALID) fail("no grid accepted");
        auto bad = g->ilist_n_bnd[d];
        bad.push_back(bad.front());   // one element more than the payload
        g->ilist_n_bnd[d] = bad;
        if (stage_all(own, own_x, own_m, nbs, g, got) != OTFMM_ERR_INVALID) fail("long list accepted");
        bad.pop_back();
        int o[3];
        oo::dir_offsets(d, o);
        // the cell diagonally opposite the band: never inside it
        const int x = o[0] == 1 ? 7 : 0, y = o[1] == 1 ? 7 : 0, z = o[2] == 1 ? 7 : 0;
        bad[0].second = std::uint16_t(64 * x + 8 * y + z);
        g->ilist_n_bnd[d] = bad;
        if (stage_all(own, own_x, own_m, nbs, g, got) != OTFMM_ERR_INVALID) fail("out-of-band cell accepted");
    }
    // flat_cells: the grid cells the aggregated calls write in place are K
    // contiguous doubles reached through operator[]; anything else is refused
    {
        std::vector<multipole> L(512);
        if (oo::flat_cells<20>(L) != &L[0][0]) fail("taylor<4>-like cells not flat");
        std::vector<space_vector> Lc(512);
        if (oo::flat_cells<3>(Lc) != &Lc[0][0]) fail("space_vector cells not flat");
        struct Tagged {
            double v[20];
            int tag;
            double& operator[](int i) { return v[i]; }
        };
        std::vector<Tagged> T(512);
        if (oo::flat_cells<20>(T) != nullptr) fail("cells with another member taken as flat");
        struct Proxy {
            std::array<double, 20> v;
            double operator[](int i) const { return v[i]; }
        };
        std::vector<Proxy> P(512);
        if (oo::flat_cells<20>(P) != nullptr) fail("cells read by value taken as flat");
        std::vector<multipole> few(100);
        if (oo::flat_cells<20>(few) != nullptr) fail("fewer than 512 cells taken as flat");
    }
    std::printf("staging ok\n");
    return 0;
}
