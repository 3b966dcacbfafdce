// TEST INFRASTRUCTURE ONLY — compiled by oracle/build_ref.sh into oracle/_ref/.
//
// Runs Octo-Tiger's own kernel arithmetic on the CPU. The per-pair math, the
// stencil generators and the multipole shift operators are the reference's,
// included from its source tree at build time (nothing of it is copied into
// this repository):
//   octotiger/multipole_interactions/kernel/compute_kernel_templates.hpp
//   octotiger/monopole_interactions/kernel/monopole_kernel_templates.hpp
//   src/multipole_interactions/util/calculate_stencil.cpp
//   src/monopole_interactions/util/calculate_stencil.cpp
//   octotiger/taylor.hpp, src/taylor.cpp (tree passes, oracle/tree_passes.hpp)
// The sweep loops of the reference live in its Kokkos kernels
// (octotiger/multipole_interactions/kernel/kokkos_kernel.hpp:137-764,
// octotiger/monopole_interactions/kernel/kokkos_kernel.hpp:143-943), which need
// Kokkos/HPX and cannot be built here; they are restated below with the same
// structure as the reference's host SIMD build: std::experimental::simd lanes
// along z, masked partner loads, the same stencil loop order. The reference
// instantiates those kernels with std::experimental::simd when built with
// OCTOTIGER_KOKKOS_SIMD_LIBRARY=STD (octotiger/common_kernel/std_simd.hpp).
// Staging and the batch driver come from oracle_core.hpp.
#include <experimental/simd>

#include "oracle_core.hpp"

#include "octotiger/options.hpp"   // shim: provides opts().theta (oracle/ref_shim)

#include "octotiger/common_kernel/interaction_constants.hpp"
#include "octotiger/common_kernel/multiindex.hpp"
#include "octotiger/multipole_interactions/kernel/compute_kernel_templates.hpp"
#include "octotiger/monopole_interactions/kernel/monopole_kernel_templates.hpp"

#include "src/monopole_interactions/util/calculate_stencil.cpp"
#include "src/multipole_interactions/util/calculate_stencil.cpp"

// The shift operators of the tree passes: the reference's taylor<4> class and
// its index maps (octotiger/taylor.hpp, src/taylor.cpp), included in place.
#include "octotiger/taylor.hpp"
#include "src/taylor.cpp"
#include "tree_passes.hpp"

namespace stdx = std::experimental;
namespace ofmm = octotiger::fmm;

static otfmm_ref_opts g_opts{0.5};
otfmm_ref_opts& opts() { return g_opts; }

namespace {

using scalar_simd = stdx::simd<double, stdx::simd_abi::scalar>;
using native_simd = stdx::native_simd<double>;

template <class S>
inline S choose(const typename S::mask_type& m, const S& a, const S& b) {
    S r = b;
    stdx::where(m, r) = a;
    return r;
}
template <class S>
inline S load(const double* p) {
    return S(p, stdx::element_aligned);
}
template <class S>
inline void store(const S& v, double* p) {
    v.copy_to(p, stdx::element_aligned);
}
template <class S>
struct max_fn {
    S operator()(const S& a, const S& b) const { return stdx::max(a, b); }
};

// Stencil masks exactly as get_host_masks builds them (kokkos_kernel.hpp:28-56;
// monopole kokkos_kernel.hpp:34-76), from the reference generators.
struct RefStencil {
    double theta = -1;
    std::vector<int> masks, indicators, p2p_masks;
    std::vector<double> four;   // 4 per stencil index
};

const RefStencil& ref_stencil(double theta) {
    static std::mutex mu;
    static RefStencil cache;
    std::lock_guard<std::mutex> lock(mu);
    if (cache.theta != theta) {
        g_opts.theta = theta;
        RefStencil s;
        s.theta = theta;
        auto sup = ofmm::multipole_interactions::calculate_stencil();
        auto mp = ofmm::multipole_interactions::calculate_stencil_masks(sup);
        s.masks.assign(ofmm::FULL_STENCIL_SIZE, 0);
        s.indicators.assign(ofmm::FULL_STENCIL_SIZE, 0);
        for (int i = 0; i < ofmm::FULL_STENCIL_SIZE; ++i) {
            s.masks[i] = mp.first[i] ? 1 : 0;
            s.indicators[i] = mp.second[i] ? 1 : 0;
        }
        auto p2p = ofmm::monopole_interactions::calculate_stencil();
        auto pm = ofmm::monopole_interactions::calculate_stencil_masks(p2p.first);
        s.p2p_masks.assign(ofmm::FULL_STENCIL_SIZE, 0);
        s.four.assign(4 * ofmm::FULL_STENCIL_SIZE, 0.0);
        for (int i = 0; i < ofmm::FULL_STENCIL_SIZE; ++i) {
            s.p2p_masks[i] = pm.first[i] ? 1 : 0;
            for (int c = 0; c < 4; ++c) s.four[4 * i + c] = pm.second[i][c];
        }
        cache = s;
    }
    return cache;
}

constexpr int INX = ora::INX;
constexpr int CL = ora::CL;
constexpr int CLU = ora::CLU;

// multipole_kernel_rho_impl / multipole_kernel_non_rho_impl with one block
// (the host launch, kokkos_kernel.hpp:884-939).
template <class S>
void sweep_m2l_nonroot(const RefStencil& st, const double* mon, const double* com, const double* M, double* L,
                 double* Lc, bool rho) {
    using mask_t = typename S::mask_type;
    constexpr int W = S::size();
    const S theta_rec_sq((1.0 / st.theta) * (1.0 / st.theta));
    for (int idx = 0; idx < INX; ++idx)
        for (int idy = 0; idy < INX; ++idy)
            for (int idz = 0; idz < INX / W; ++idz) {
                const ofmm::multiindex<> cell(idx + INX, idy + INX, idz * W + INX);
                const int cflat = ofmm::to_flat_index_padded(cell);
                const ofmm::multiindex<> cu(idx, idy, idz * W);
                const int cuflat = ofmm::to_inner_flat_index_not_padded(cu);
                const int ccx = ((cell.x + INX) >> 1) - INX / 2, ccy = ((cell.y + INX) >> 1) - INX / 2;
                int ccz[W];
                for (int i = 0; i < W; ++i) ccz[i] = ((cell.z + i + INX) >> 1) - INX / 2;
                S m_cell[20], X[3], tmp[20], corr[3], mp[20], Y[3];
                for (int c = 0; c < 20; ++c) m_cell[c] = load<S>(M + c * CL + cflat);
                for (int c = 0; c < 3; ++c) X[c] = load<S>(com + c * CL + cflat);
                for (int c = 0; c < 20; ++c) tmp[c] = S(0.0);
                for (int c = 0; c < 3; ++c) corr[c] = S(0.0);
                double tc[W];
                for (int x = 0; x < ofmm::NUMBER_MULTIPOLE_BLOCKS; ++x) {
                    const int sx = x + ofmm::STENCIL_MIN;
                    const int pcx = ((cell.x + sx + INX) >> 1) - INX / 2;
                    const int dxc = (ccx - pcx) * (ccx - pcx);
                    for (int y = 0; y < ofmm::NUMBER_MULTIPOLE_BLOCKS; ++y) {
                        const int sy = y + ofmm::STENCIL_MIN;
                        const int pcy = ((cell.y + sy + INX) >> 1) - INX / 2;
                        const int dyc = (ccy - pcy) * (ccy - pcy);
                        for (int sz = ofmm::STENCIL_MIN; sz <= ofmm::STENCIL_MAX; ++sz) {
                            const int index = x * ofmm::STENCIL_INX * ofmm::STENCIL_INX + y * ofmm::STENCIL_INX +
                                              (sz - ofmm::STENCIL_MIN);
                            if (!st.masks[index]) continue;
                            const ofmm::multiindex<> p(cell.x + sx, cell.y + sy, cell.z + sz);
                            for (int i = 0; i < W; ++i) {
                                const int pcz = ((p.z + i + INX) >> 1) - INX / 2;
                                tc[i] = double(dxc + dyc + (ccz[i] - pcz) * (ccz[i] - pcz));
                            }
                            const S tcs(tc, stdx::element_aligned);
                            mask_t mask = tcs < theta_rec_sq;
                            if (!stdx::any_of(mask)) continue;
                            const int pflat = ofmm::to_flat_index_padded(p);
                            for (int c = 0; c < 3; ++c) Y[c] = load<S>(com + c * CL + pflat);
                            mp[0] = choose(mask, load<S>(mon + pflat), S(0.0));
                            if (!st.indicators[index]) mask = mask_t(false);
                            mp[0] += choose(mask, load<S>(M + pflat), S(0.0));
                            for (int c = 1; c < 20; ++c) mp[c] = choose(mask, load<S>(M + c * CL + pflat), S(0.0));
                            if (rho)
                                ofmm::multipole_interactions::compute_kernel_rho(X, Y, mp, tmp, corr, m_cell,
                                                                                 max_fn<S>{});
                            else
                                ofmm::multipole_interactions::compute_kernel_non_rho(X, Y, mp, tmp, max_fn<S>{});
                        }
                    }
                }
                for (int c = 0; c < 20; ++c) store(tmp[c], L + c * CLU + cuflat);
                if (rho)
                    for (int c = 0; c < 3; ++c) store(corr[c], Lc + c * CLU + cuflat);
            }
}

// multipole_kernel_root_rho_impl / _root_non_rho_impl (kokkos_kernel.hpp:324-471, 637-764)
template <class S>
void sweep_m2l_root(const RefStencil& st, const double* com, const double* M, double* L, double* Lc, bool rho) {
    using mask_t = typename S::mask_type;
    constexpr int W = S::size();
    for (int idx = 0; idx < INX; ++idx)
        for (int idy = 0; idy < INX; ++idy)
            for (int idz = 0; idz < INX / W; ++idz) {
                const ofmm::multiindex<> cell(idx + INX, idy + INX, idz * W + INX);
                const int cflat = ofmm::to_flat_index_padded(cell);
                const ofmm::multiindex<> cu(idx, idy, idz * W);
                const int cuflat = ofmm::to_inner_flat_index_not_padded(cu);
                S m_cell[20], X[3], tmp[20], corr[3], mp[20], Y[3];
                for (int c = 0; c < 20; ++c) m_cell[c] = load<S>(M + c * CL + cflat);
                for (int c = 0; c < 3; ++c) X[c] = load<S>(com + c * CL + cflat);
                for (int c = 0; c < 20; ++c) tmp[c] = S(0.0);
                for (int c = 0; c < 3; ++c) corr[c] = S(0.0);
                double helper[W];
                for (int x = 0; x < INX; ++x) {
                    const int sx = x - cu.x;
                    for (int y = 0; y < INX; ++y) {
                        const int sy = y - cu.y;
                        for (int z = 0; z < INX; ++z) {
                            const int sz = z - cu.z;
                            for (int i = 0; i < W; ++i) helper[i] = 0.0;
                            if (sx >= ofmm::STENCIL_MIN && sx <= ofmm::STENCIL_MAX && sy >= ofmm::STENCIL_MIN &&
                                sy <= ofmm::STENCIL_MAX) {
                                for (int i = 0; i < W && sz - ofmm::STENCIL_MIN - i >= 0; ++i) {
                                    const int index = (sx - ofmm::STENCIL_MIN) * ofmm::STENCIL_INX * ofmm::STENCIL_INX +
                                                      (sy - ofmm::STENCIL_MIN) * ofmm::STENCIL_INX +
                                                      (sz - ofmm::STENCIL_MIN - i);
                                    if (sz - i <= ofmm::STENCIL_MAX)
                                        if (!st.indicators[index] || (sx == 0 && sy == 0 && sz - i == 0))
                                            helper[i] = 12.0;
                                }
                            }
                            const S h(helper, stdx::element_aligned);
                            const mask_t mask = h < S(1.0);
                            if (!stdx::any_of(mask)) continue;
                            const ofmm::multiindex<> p(x + INX, y + INX, z + INX);
                            const int pflat = ofmm::to_flat_index_padded(p);
                            for (int c = 0; c < 3; ++c) Y[c] = choose(mask, S(com[c * CL + pflat]), S(0.0));
                            for (int c = 0; c < 20; ++c) mp[c] = choose(mask, S(M[c * CL + pflat]), S(0.0));
                            if (rho)
                                ofmm::multipole_interactions::compute_kernel_rho(X, Y, mp, tmp, corr, m_cell,
                                                                                 max_fn<S>{});
                            else
                                ofmm::multipole_interactions::compute_kernel_non_rho(X, Y, mp, tmp, max_fn<S>{});
                        }
                    }
                }
                for (int c = 0; c < 20; ++c) store(tmp[c], L + c * CLU + cuflat);
                if (rho)
                    for (int c = 0; c < 3; ++c) store(corr[c], Lc + c * CLU + cuflat);
            }
}

// p2p_kernel_impl (monopole kokkos_kernel.hpp:143-320); one y row per pass.
template <class S>
void sweep_p2p(const RefStencil& st, const double* mon, double dx, double* L4) {
    using mask_t = typename S::mask_type;
    constexpr int W = S::size();
    const S theta_rec_sq((1.0 / st.theta) * (1.0 / st.theta));
    const double dcomp[2] = {1.0 / dx, -1.0 / dx};
    for (int idx = 0; idx < INX; ++idx)
        for (int idy = 0; idy < INX; ++idy)
            for (int idz = 0; idz < INX / W; ++idz) {
                const ofmm::multiindex<> cell(idx + INX, idy + INX, idz * W + INX);
                const ofmm::multiindex<> cu(idx, idy, idz * W);
                const int cuflat = ofmm::to_inner_flat_index_not_padded(cu);
                const int ccx = ((cell.x + INX) >> 1) - INX / 2, ccy = ((cell.y + INX) >> 1) - INX / 2;
                int ccz[W];
                for (int i = 0; i < W; ++i) ccz[i] = ((cell.z + i + INX) >> 1) - INX / 2;
                S tmp[4] = {S(0.0), S(0.0), S(0.0), S(0.0)};
                double tc[W];
                for (int x = 0; x < ofmm::NUMBER_P2P_BLOCKS; ++x) {
                    const int sx = x + ofmm::STENCIL_MIN;
                    const int pcx = ((cell.x + sx + INX) >> 1) - INX / 2;
                    const int dxc = (ccx - pcx) * (ccx - pcx);
                    for (int sy = ofmm::STENCIL_MIN; sy <= ofmm::STENCIL_MAX; ++sy) {
                        const int pcy = ((cell.y + sy + INX) >> 1) - INX / 2;
                        const int dyc = (ccy - pcy) * (ccy - pcy);
                        const int y = sy - ofmm::STENCIL_MIN;
                        for (int sz = ofmm::STENCIL_MIN; sz <= ofmm::STENCIL_MAX; ++sz) {
                            const int index = x * ofmm::STENCIL_INX * ofmm::STENCIL_INX + y * ofmm::STENCIL_INX +
                                              (sz - ofmm::STENCIL_MIN);
                            if (!st.p2p_masks[index]) continue;
                            const ofmm::multiindex<> p(cell.x + sx, cell.y + sy, cell.z + sz);
                            for (int i = 0; i < W; ++i) {
                                const int pcz = ((p.z + i + INX) >> 1) - INX / 2;
                                tc[i] = double(dxc + dyc + (ccz[i] - pcz) * (ccz[i] - pcz));
                            }
                            const S tcs(tc, stdx::element_aligned);
                            const mask_t mask = tcs < theta_rec_sq;
                            if (!stdx::any_of(mask)) continue;
                            const int pflat = ofmm::to_flat_index_padded(p);
                            S m = choose(mask, load<S>(mon + pflat), S(0.0));
                            m = m * dcomp[0];
                            const S four[4] = {S(st.four[index * 4 + 0]), S(st.four[index * 4 + 1]),
                                               S(st.four[index * 4 + 2]), S(st.four[index * 4 + 3])};
                            tmp[0] += four[0] * m;
                            tmp[1] += four[1] * m * dcomp[1];
                            tmp[2] += four[2] * m * dcomp[1];
                            tmp[3] += four[3] * m * dcomp[1];
                        }
                    }
                }
                for (int c = 0; c < 4; ++c) store(tmp[c], L4 + c * CLU + cuflat);
            }
}

// p2m_kernel_impl_rho / _non_rho (monopole kokkos_kernel.hpp:517-942)
template <class S>
void sweep_p2m(const RefStencil& st, int d, const double* nM, const double* ncom, int stride, const double* icom,
         double* L4, double* Lc, bool rho, bool reset) {
    using mask_t = typename S::mask_type;
    constexpr int W = S::size();
    int o[3], s[3], e[3], nsz[3], cs[3], ce[3];
    ora::dir_offsets(d, o);
    ora::padding_box(o, s, e, nsz);
    ora::p2m_cells(o, cs, ce);
    if (rho && reset)
        for (int c = 0; c < 3; ++c)
            for (int u = 0; u < ora::NCELL; ++u) Lc[c * CLU + u] = 0.0;
    const S theta_rec_sq((1.0 / st.theta) * (1.0 / st.theta));
    const int nz = ce[2] - cs[2];
    const int nidz = nz / W + (nz % W == 0 ? 0 : 1);
    for (int idx = 0; idx < ce[0] - cs[0]; ++idx)
        for (int idy = 0; idy < ce[1] - cs[1]; ++idy)
            for (int idz = 0; idz < nidz; ++idz) {
                const ofmm::multiindex<> cell(idx + INX + cs[0], idy + INX + cs[1], idz * W + INX + cs[2]);
                const ofmm::multiindex<> cu(idx + cs[0], idy + cs[1], idz * W + cs[2]);
                const int cuflat = ofmm::to_inner_flat_index_not_padded(cu);
                const int ccx = ((cell.x + INX) >> 1) - INX / 2, ccy = ((cell.y + INX) >> 1) - INX / 2;
                int ccz[W];
                for (int i = 0; i < W; ++i) ccz[i] = ((cell.z + i + INX) >> 1) - INX / 2;
                S X[3], tmp[4], corr[3], mp[20], Y[3];
                for (int c = 0; c < 3; ++c) X[c] = load<S>(icom + c * CLU + cuflat);
                for (int c = 0; c < 4; ++c) tmp[c] = load<S>(L4 + c * CLU + cuflat);
                if (rho)
                    for (int c = 0; c < 3; ++c) corr[c] = load<S>(Lc + c * CLU + cuflat);
                double mh[W], tc[W];
                for (int x = s[0]; x < e[0]; ++x)
                    for (int y = s[1]; y < e[1]; ++y)
                        for (int z = s[2]; z < e[2]; ++z) {
                            const ofmm::multiindex<> pi(INX + o[0] * INX + x, INX + o[1] * INX + y,
                                                        INX + o[2] * INX + z);
                            const ofmm::multiindex<> se(pi.x - cell.x - ofmm::STENCIL_MIN,
                                                        pi.y - cell.y - ofmm::STENCIL_MIN,
                                                        pi.z - cell.z - ofmm::STENCIL_MIN);
                            const long sflat = long(se.x) * ofmm::STENCIL_INX * ofmm::STENCIL_INX +
                                               long(se.y) * ofmm::STENCIL_INX + se.z;
                            for (int i = 0; i < W; ++i) {
                                if (sflat - i >= 0 && sflat - i < ofmm::FULL_STENCIL_SIZE)
                                    mh[i] = double(st.p2p_masks[sflat - i]);
                                else
                                    mh[i] = 0.0;
                                if (cu.z + i >= INX || idz * W + i >= nz) mh[i] = 0.0;
                            }
                            const S mhs(mh, stdx::element_aligned);
                            const mask_t mask1 = S(0.0) < mhs;
                            if (!stdx::any_of(mask1)) continue;
                            const int pcx = ((pi.x + INX) >> 1) - INX / 2, pcy = ((pi.y + INX) >> 1) - INX / 2,
                                      pcz = ((pi.z + INX) >> 1) - INX / 2;
                            for (int i = 0; i < W; ++i)
                                tc[i] = double((ccx - pcx) * (ccx - pcx) + (ccy - pcy) * (ccy - pcy) +
                                               (ccz[i] - pcz) * (ccz[i] - pcz));
                            const S tcs(tc, stdx::element_aligned);
                            const mask_t mask2 = tcs < theta_rec_sq;
                            if (!stdx::any_of(mask2)) continue;
                            const mask_t mask = mask1 && mask2;
                            const int f = (x - s[0]) * (nsz[1] * nsz[2]) + (y - s[1]) * nsz[2] + (z - s[2]);
                            for (int c = 0; c < 3; ++c) Y[c] = S(ncom[size_t(c) * stride + f]);
                            for (int c = 0; c < 20; ++c) mp[c] = choose(mask, S(nM[size_t(c) * stride + f]), S(0.0));
                            if (rho)
                                ofmm::monopole_interactions::compute_kernel_p2m_rho(X, Y, mp, tmp, corr, max_fn<S>{});
                            else
                                ofmm::monopole_interactions::compute_kernel_p2m_non_rho(X, Y, mp, tmp, max_fn<S>{});
                        }
                // Full-width stores like the reference (lanes past the z range
                // write back the values they loaded).
                for (int c = 0; c < 4; ++c) store(tmp[c], L4 + c * CLU + cuflat);
                if (rho)
                    for (int c = 0; c < 3; ++c) store(corr[c], Lc + c * CLU + cuflat);
            }
}

template <class S>
struct RefKernels {
    void m2l(const ora::Stencil& ost, const ora::M2LInput& in, double* L, double* Lc, int rho, bool root) const {
        const RefStencil& st = ref_stencil(ost.theta);
        if (root)
            sweep_m2l_root<S>(st, in.com.data(), in.M.data(), L, Lc, rho != 0);
        else
            sweep_m2l_nonroot<S>(st, in.mon.data(), in.com.data(), in.M.data(), L, Lc, rho != 0);
    }
    void p2p(const ora::Stencil& ost, const double* mon, double dx, double* L4) const {
        sweep_p2p<S>(ref_stencil(ost.theta), mon, dx, L4);
    }
    void p2m(const ora::Stencil& ost, int d, const double* nM, const double* ncom, int stride, const double* icom,
             double* L4, double* Lc, int rho, bool reset) const {
        sweep_p2m<S>(ref_stencil(ost.theta), d, nM, ncom, stride, icom, L4, Lc, rho != 0, reset);
    }
};

}   // namespace

// Upward / downward shifts through the reference's taylor<4, double> operators.
struct RefShift {
    static void run(const double A[20], const double X[3], double B[20], bool down) {
        taylor<4, double> t;
        for (int j = 0; j < 20; ++j) t[j] = A[j];
        const std::array<double, 3> x{X[0], X[1], X[2]};
        if (down) t <<= x;
        else t >>= x;
        for (int j = 0; j < 20; ++j) B[j] = t[j];
    }
    void up(const double A[20], const double X[3], double B[20]) const { run(A, X, B, false); }
    void down(const double A[20], const double X[3], double B[20]) const { run(A, X, B, true); }
};

extern "C" {

int ref_shift(const double* A, const double* X, double* B, int down) {
    RefShift::run(A, X, B, down != 0);
    return 0;
}

int ref_upward(double* M, double* com, const double* mon, const uint8_t* is_leaf, double* com1, int n,
               const ora::TreeNode* nodes, const int32_t* level_start, int n_levels, int rho) {
    ora::TreePool P{M, com, mon, is_leaf, com1, n};
    ora::upward_pass(RefShift{}, P, nodes, level_start, n_levels, rho != 0);
    return 0;
}

int ref_downward(const double* com, const uint8_t* is_leaf, const double* com1, int n, const ora::TreeNode* nodes,
                 const int32_t* level_start, int n_levels, double* L, double* Lc, double* G, double gconst,
                 int correct_am, int rho) {
    ora::TreePool P{nullptr, const_cast<double*>(com), nullptr, is_leaf, const_cast<double*>(com1), n};
    ora::downward_pass(RefShift{}, P, nodes, level_start, n_levels, L, Lc, G, gconst, correct_am != 0, rho != 0);
    return 0;
}

// simd_mode: 0 = scalar lanes, 1 = native SIMD lanes of this build.
int ref_simd_width(int simd_mode) { return simd_mode ? int(native_simd::size()) : 1; }

int ref_build_stencil(double theta, uint8_t* mpole_mask, uint8_t* mpole_phase, uint8_t* p2p_mask, double* four) {
    if (theta < ora::THETA_MIN) return -1;
    const RefStencil& st = ref_stencil(theta);
    for (int i = 0; i < ora::FULL; ++i) {
        mpole_mask[i] = uint8_t(st.masks[i]);
        mpole_phase[i] = uint8_t(st.indicators[i]);
        p2p_mask[i] = uint8_t(st.p2p_masks[i]);
        for (int c = 0; c < 4; ++c) four[4 * i + c] = st.four[4 * i + c];
    }
    return 0;
}

int ref_m2l_soa(int simd_mode, double theta, const double* mon, const double* M, const double* com, double* L,
                double* Lc, int rho, int root) {
    if (theta < ora::THETA_MIN) return -1;
    const RefStencil& st = ref_stencil(theta);
    if (simd_mode) {
        if (root) sweep_m2l_root<native_simd>(st, com, M, L, Lc, rho != 0);
        else sweep_m2l_nonroot<native_simd>(st, mon, com, M, L, Lc, rho != 0);
    } else {
        if (root) sweep_m2l_root<scalar_simd>(st, com, M, L, Lc, rho != 0);
        else sweep_m2l_nonroot<scalar_simd>(st, mon, com, M, L, Lc, rho != 0);
    }
    return 0;
}

int ref_p2p_soa(int simd_mode, double theta, const double* mon, double dx, double* L4) {
    if (theta < ora::THETA_MIN) return -1;
    const RefStencil& st = ref_stencil(theta);
    if (simd_mode) sweep_p2p<native_simd>(st, mon, dx, L4);
    else sweep_p2p<scalar_simd>(st, mon, dx, L4);
    return 0;
}

int ref_p2m_dir(int simd_mode, double theta, int d, const double* nM, const double* ncom, int stride,
                const double* icom, double* L4, double* Lc, int rho, int reset) {
    if (theta < ora::THETA_MIN) return -1;
    const RefStencil& st = ref_stencil(theta);
    if (simd_mode) sweep_p2m<native_simd>(st, d, nM, ncom, stride, icom, L4, Lc, rho != 0, reset != 0);
    else sweep_p2m<scalar_simd>(st, d, nM, ncom, stride, icom, L4, Lc, rho != 0, reset != 0);
    return 0;
}

int ref_batch(int simd_mode, double theta, const double* M, const double* com, const double* mon,
              const uint8_t* is_leaf, int n_sub, const ora::WorkItem* items, int n_items, int rho, double* L_out,
              double* Lc_out, int nthreads) {
    if (theta < ora::THETA_MIN) return -1;
    ref_stencil(theta);
    ora::Pool pool{M, com, mon, is_leaf, n_sub};
    if (simd_mode)
        ora::run_batch(RefKernels<native_simd>{}, theta, pool, items, n_items, rho, L_out, Lc_out, nthreads);
    else
        ora::run_batch(RefKernels<scalar_simd>{}, theta, pool, items, n_items, rho, L_out, Lc_out, nthreads);
    return 0;
}

}   // extern "C"
