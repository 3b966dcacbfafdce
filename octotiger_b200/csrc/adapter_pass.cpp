// Drives the C++ drop-in adapter (include/otfmm_octotiger.hpp) the way
// node_server::compute_fmm drives the reference's interaction interfaces
// (src/node_server.cpp:711-723): one call per node, from several host threads
// at once, with AoS inputs (taylor<4> multipoles, space_vector centres of mass)
// and neighbour payloads that alias the neighbours' own data, the grid's L and
// L_c updated in place. Built as libotfmm_adapter_pass.so; used by bench.py
// (the end-to-end figure through the reference's interfaces) and by the GPU
// tests of the aggregated adapter.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <memory>
#include <thread>
#include <vector>

#include "octotiger_standins.hpp"

namespace {

struct Node {
    std::shared_ptr<std::vector<multipole>> M;
    std::shared_ptr<std::vector<space_vector>> com;
    std::shared_ptr<std::vector<double>> mon;
};

}   // namespace

extern "C" {

/* One or more passes over a work list through the adapter. The pool arrays
 * (M[n][20][512], com[n][3][512], mon[n][512], is_leaf[n]) and the work items
 * are host arrays in the library's batch layout; they are converted to the
 * reference's AoS node data once, outside the timed passes. mode 1: the
 * aggregated interfaces (an otfmm_aggregator of max_subgrids / max_items /
 * idle_us; each thread submits calls_in_flight calls, then finishes them: an
 * HPX task that waits on a future is suspended and its worker thread runs
 * other nodes' tasks, so many calls per thread are in flight), the batch
 * writing the grids' cells
 * itself; mode 2: the same with SoA results that finish() adds to the grids on
 * the caller's thread; mode 3: as mode 1, but a thread polls its calls
 * (otfmm_octotiger::ready) and yields in between instead of blocking in
 * finish(), as an HPX task would; mode 0: the per-call interfaces on
 * the context (one blocking host-buffer call per node). seconds[p] = wall time of pass p (all threads, first call to
 * last return). After the last pass L_out[n][20][512] / Lc_out[n][3][512]
 * hold the grids of the work items' subgrids (zero elsewhere). Returns the
 * first non-zero status of any call. */
int otfmm_adapter_pass(otfmm_context* ctx, int32_t n_sub, const double* M, const double* com, const double* mon,
                       const uint8_t* is_leaf, const otfmm_work_item* items, int32_t n_items, int gsolve_type,
                       int precision, int32_t mode, int32_t threads, int32_t max_subgrids, int32_t max_items,
                       int32_t idle_us, int32_t passes, int32_t calls_in_flight, double* L_out, double* Lc_out,
                       double* seconds) {
    if (!ctx || !M || !com || !mon || !is_leaf || !items || !L_out || !Lc_out || !seconds || n_sub < 1 ||
        n_items < 1 || threads < 1 || passes < 1 || mode < 0 || mode > 3 || calls_in_flight < 1)
        return OTFMM_ERR_INVALID;
    for (int i = 0; i < n_items; ++i)
        if (items[i].subgrid < 0 || items[i].subgrid >= n_sub) return OTFMM_ERR_INVALID;
    std::vector<Node> nodes(n_sub);
    for (int s = 0; s < n_sub; ++s) {
        Node& nd = nodes[s];
        nd.M = std::make_shared<std::vector<multipole>>(512);
        nd.com = std::make_shared<std::vector<space_vector>>(512);
        nd.mon = std::make_shared<std::vector<double>>(512);
        for (int u = 0; u < 512; ++u) {
            for (int c = 0; c < 20; ++c) (*nd.M)[u][c] = M[((size_t)s * 20 + c) * 512 + u];
            for (int c = 0; c < 3; ++c) (*nd.com)[u][c] = com[((size_t)s * 3 + c) * 512 + u];
            (*nd.mon)[u] = mon[(size_t)s * 512 + u];
        }
    }
    // per item: the 26 neighbour payloads (leaf neighbours as masses, refined
    // ones as multipoles and centres of mass; empty directions without data)
    std::vector<std::vector<neighbor_gravity_type>> nbs(n_items, std::vector<neighbor_gravity_type>(26));
    std::vector<grid> grids(n_items);
    std::vector<std::vector<std::shared_ptr<std::vector<space_vector>>>> com_ptrs(n_items);
    std::vector<char> has_refined(n_items, 0);
    for (int i = 0; i < n_items; ++i) {
        for (int d = 0; d < 26; ++d) {
            const int g = items[i].neighbors[d];
            if (g < 0 || g >= n_sub) continue;
            neighbor_gravity_type& nb = nbs[i][d];
            nb.is_monopole = is_leaf[g] != 0;
            if (nb.is_monopole) {
                nb.data.m = nodes[g].mon;
            } else {
                nb.data.M = nodes[g].M;
                nb.data.x = nodes[g].com;
                has_refined[i] = 1;
            }
        }
        com_ptrs[i] = {nodes[items[i].subgrid].com};
    }
    otfmm_aggregator* agg = nullptr;
    if (mode >= 1) {
        const int rc = otfmm_aggregator_create(ctx, max_subgrids, max_items, idle_us, gsolve_type, precision, &agg);
        if (rc != OTFMM_OK) return rc;
    }
    std::atomic<int> first_rc{OTFMM_OK};
    const std::array<bool, 26> empty{};
    for (int p = 0; p < passes; ++p) {
        for (auto& gr : grids) {
            for (auto& l : gr.L) l = multipole{};
            for (auto& l : gr.L_c) l = space_vector{};
        }
        std::atomic<int> next{0};
        auto note = [&](int rc) {
            if (rc != OTFMM_OK) {
                int expect = OTFMM_OK;
                first_rc.compare_exchange_strong(expect, rc);
            }
        };
        // aggregated: a thread takes calls_in_flight nodes at a time, submits all
        // their calls, then finishes them; per-call: one blocking call after the
        // other
        auto agg_worker = [&]() {
            std::vector<otfmm_octotiger::AggregatedCall<grid*>> calls(calls_in_flight);
            for (auto& c : calls) c.in_place = (mode != 2);
            std::vector<int> ok(calls_in_flight);
            for (;;) {
                const int i0 = next.fetch_add(calls_in_flight);
                if (i0 >= n_items) return;
                const int i1 = std::min(n_items, i0 + calls_in_flight);
                for (int i = i0; i < i1; ++i) {
                    const otfmm_work_item& w = items[i];
                    const Node& nd = nodes[w.subgrid];
                    const std::array<double, 3> xb{w.xbase[0], w.xbase[1], w.xbase[2]};
                    int rc;
                    if (w.kind == OTFMM_KIND_LEAF)
                        rc = otfmm_octotiger::monopole_kernel_interface_submit(agg, *nd.mon, com_ptrs[i], nbs[i],
                                                                               gsolve_type, w.dx, empty, &grids[i],
                                                                               has_refined[i] != 0, calls[i - i0]);
                    else
                        rc = otfmm_octotiger::multipole_kernel_interface_submit(
                            agg, *nd.mon, *nd.M, com_ptrs[i], nbs[i], gsolve_type, w.dx, empty, xb, &grids[i],
                            w.kind == OTFMM_KIND_M2L_ROOT, calls[i - i0]);
                    note(rc);
                    ok[i - i0] = rc == OTFMM_OK;
                }
                if (mode == 3) {
                    // poll the calls in order, yielding while one is not ready (the
                    // calls after it are in the same batch or a later one)
                    for (int i = i0; i < i1; ++i) {
                        if (!ok[i - i0]) continue;
                        while (otfmm_octotiger::ready(calls[i - i0]) == 0) std::this_thread::yield();
                        note(otfmm_octotiger::finish(calls[i - i0]));   // returns at once (or the error)
                        ok[i - i0] = 0;
                    }
                }
                for (int i = i0; i < i1; ++i)
                    if (ok[i - i0]) note(otfmm_octotiger::finish(calls[i - i0]));
            }
        };
        auto worker = [&]() {
            if (agg) return agg_worker();
            for (;;) {
                const int i = next.fetch_add(1);
                if (i >= n_items) return;
                const otfmm_work_item& w = items[i];
                const Node& nd = nodes[w.subgrid];
                grid* gp = &grids[i];
                const std::array<double, 3> xb{w.xbase[0], w.xbase[1], w.xbase[2]};
                int rc;
                if (w.kind == OTFMM_KIND_LEAF) {
                    rc = otfmm_octotiger::monopole_kernel_interface(ctx, *nd.mon, com_ptrs[i], nbs[i], gsolve_type,
                                                                    w.dx, empty, gp, has_refined[i] != 0, precision);
                } else {
                    const bool root = w.kind == OTFMM_KIND_M2L_ROOT;
                    rc = otfmm_octotiger::multipole_kernel_interface(ctx, *nd.mon, *nd.M, com_ptrs[i], nbs[i],
                                                                     gsolve_type, w.dx, empty, xb, gp, root,
                                                                     precision);
                }
                note(rc);
            }
        };
        const auto t0 = std::chrono::steady_clock::now();
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
        for (auto& t : pool) t.join();
        seconds[p] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    if (agg) otfmm_aggregator_destroy(agg);
    std::fill(L_out, L_out + (size_t)n_sub * 20 * 512, 0.0);
    std::fill(Lc_out, Lc_out + (size_t)n_sub * 3 * 512, 0.0);
    for (int i = 0; i < n_items; ++i) {
        const size_t s = items[i].subgrid;
        for (int u = 0; u < 512; ++u) {
            for (int c = 0; c < 20; ++c) L_out[(s * 20 + c) * 512 + u] = grids[i].L[u][c];
            for (int c = 0; c < 3; ++c) Lc_out[(s * 3 + c) * 512 + u] = grids[i].L_c[u][c];
        }
    }
    return first_rc.load();
}

}   // extern "C"
