// Aggregation of concurrent per-node interaction calls into batched solves
// (host side of libotfmm.so; included once by otfmm.cu after the context).
//
// node_server::compute_fmm calls the reference's interaction interfaces once
// per node, from many HPX worker threads at once (src/node_server.cpp:717-722).
// The reference's Kokkos backend fuses concurrent monopole calls into one
// launch (monopole_kernel_agg, octotiger/monopole_interactions/kernel/
// kokkos_kernel.hpp:1357-1405) and its CUDA backend spreads callers over a
// per-GPU stream pool (src/multipole_interactions/legacy/
// cuda_multipole_interaction_interface.cpp:64-70). Here every kind of call
// (multipole, root, monopole with P2M) joins one open batch:
//   * otfmm_aggregator_reserve gives the call pool slots for its own subgrid and
//     its neighbours' records in pinned host memory; a record whose key (the
//     address of the caller's data, the same for a node and for the payloads
//     that alias it) is already in the batch is not copied again;
//   * the caller writes the parts it was asked to fill, without any lock;
//   * otfmm_aggregator_submit adds its work item and returns at once;
//     otfmm_aggregator_wait blocks until the call's batch has run (so a caller
//     can have many calls in flight, as HPX tasks do);
//   * a batch runs (otfmm_batch_host on the aggregator's own stream) once it is
//     full and every reserved call has submitted, or once it has been idle for
//     `idle_us` with no call between reserve and submit; a waiting caller runs
//     it and copies every call's results to the caller's buffers (with up to
//     AGG_COPY_THREADS_MAX helper threads), the others sleep on a condition
//     variable;
//   * two batch buffers: one collects while the other runs.
#pragma once

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <string>
#include <system_error>
#include <thread>
#include <unordered_map>
#include <vector>

constexpr size_t AGG_COPY_CHUNK = 32;         // calls a copy thread takes at a time
constexpr size_t AGG_COPY_THREADS_MAX = 16;   // threads that copy a batch's results

// The aggregator's state lock: held for well under a microsecond at a time,
// by every caller of every host thread, several times per call, so a
// contended acquire first retries for a few microseconds (a blocked thread's
// wake-up takes longer than the critical section) and only then blocks.
struct AggLock {
    std::mutex m;
    void lock() {
        for (int i = 0; i < 512; ++i) {
            if (m.try_lock()) return;
#if defined(__x86_64__) || defined(__i386__)
            __builtin_ia32_pause();
#endif
        }
        m.lock();
    }
    bool try_lock() { return m.try_lock(); }
    void unlock() { m.unlock(); }
};

// The record keys of one batch -> pool slot: open addressing with linear
// probing over at least twice the batch's slots (so a probe always ends),
// 0 = empty; cleared through the list of used buckets. Looked up 27 times per
// call under the aggregator's lock, hence no node-based map.
struct AggKeyMap {
    std::vector<uint64_t> key;
    std::vector<int32_t> val;
    std::vector<uint32_t> used;
    uint32_t mask = 0;
    void init(size_t cap) {
        size_t n = 64;
        while (n < 2 * cap) n <<= 1;
        key.assign(n, 0);
        val.assign(n, -1);
        used.reserve(cap);
        mask = (uint32_t)(n - 1);
    }
    static uint32_t bucket(uint64_t k) { return (uint32_t)((k * 0x9E3779B97F4A7C15ull) >> 32); }
    int32_t find(uint64_t k) const {
        for (uint32_t h = bucket(k) & mask;; h = (h + 1) & mask) {
            if (key[h] == k) return val[h];
            if (key[h] == 0) return -1;
        }
    }
    void insert(uint64_t k, int32_t v) {
        uint32_t h = bucket(k) & mask;
        while (key[h] != 0) h = (h + 1) & mask;
        key[h] = k;
        val[h] = v;
        used.push_back(h);
    }
    void clear() {
        for (uint32_t h : used) key[h] = 0;
        used.clear();
    }
};

struct otfmm_aggregator {
    enum State { FREE, OPEN, CLOSED, RUNNING };
    struct Out {
        double* L;
        double* Lc;
        int slot;
        int kind;
        int l_stride;    // 0: L gets the SoA rows; else L[u * l_stride + c] += component c of cell u
        int lc_stride;   // 0: Lc gets the SoA rows; else Lc[u * lc_stride + c] = component c of cell u
    };
    struct Batch {
        // written under the lock; epoch and done_epoch are also read without it
        // (otfmm_aggregator_record, the fast path of otfmm_aggregator_wait)
        std::atomic<State> state{FREE};
        std::atomic<long long> epoch{0}, done_epoch{0};   // the batch collecting now / the last one that ran
        int n_sub = 0, pending = 0;
        AggKeyMap keys;
        std::vector<uint8_t> claimed;   // per slot: parts some caller fills (OTFMM_AGG_*)
        std::vector<otfmm_work_item> staged;
        std::vector<Out> outs;
        std::chrono::steady_clock::time_point last;
        double *M = nullptr, *com = nullptr, *mon = nullptr, *L = nullptr, *Lc = nullptr;
        uint8_t* is_leaf = nullptr;
        otfmm_work_item* items = nullptr;
    };
    otfmm_context* ctx = nullptr;
    int gsolve = OTFMM_RHO, precision = OTFMM_FP64, cap_sub = 0, cap_items = 0;
    std::chrono::microseconds idle{200};
    cudaStream_t stream = nullptr;
    AggLock mu;          // batch states
    std::mutex run_mu;   // one batch on the GPU at a time (the context's host-path buffers)
    std::condition_variable_any cv;
    std::atomic<bool> any_failed{false};   // some batch run failed (waits take the lock to find out which)
    Batch b[2];
    long long epochs = 0;
    std::unordered_map<long long, std::pair<int, std::string>> failed;   // epoch -> status of a failed run
};

namespace {

void agg_free_buffers(otfmm_aggregator::Batch& b) {
    cudaFreeHost(b.M);
    cudaFreeHost(b.com);
    cudaFreeHost(b.mon);
    cudaFreeHost(b.L);
    cudaFreeHost(b.Lc);
    cudaFreeHost(b.is_leaf);
    cudaFreeHost(b.items);
}

// dst[u * stride + c] += src[c * NCELL + u] for c < ncomp, 8 cells at a time
// (whole cache lines of every source row).
void agg_aos_add(double* dst, int stride, const double* src, int ncomp) {
    for (int u0 = 0; u0 < NCELL; u0 += 8)
        for (int c = 0; c < ncomp; ++c)
            for (int u = u0; u < u0 + 8; ++u) dst[(size_t)u * stride + c] += src[c * NCELL + u];
}

// dst[u * stride + c] = src[c * NCELL + u] for c < 3, zeros when src is NULL.
void agg_aos_set3(double* dst, int stride, const double* src) {
    for (int u0 = 0; u0 < NCELL; u0 += 8)
        for (int c = 0; c < 3; ++c)
            for (int u = u0; u < u0 + 8; ++u) dst[(size_t)u * stride + c] = src ? src[c * NCELL + u] : 0.0;
}

// Runs a batch (the caller holds no lock; the batch is RUNNING) and copies
// every call's results to its buffers: multipole items L (20 x 512) and L_c
// (3 x 512), leaves L0..L3 and L_c (L_c only where the caller asked for it);
// as SoA rows, or added (L) / written (L_c) into the caller's AoS cells.
int agg_run(otfmm_aggregator* a, otfmm_aggregator::Batch& b, std::string& msg) {
    // multipole items first, as order_work_list does: the long tiles start first
    std::vector<otfmm_work_item> items(b.staged);
    std::stable_partition(items.begin(), items.end(),
                          [](const otfmm_work_item& w) { return w.kind != OTFMM_KIND_LEAF; });
    std::copy(items.begin(), items.end(), b.items);
    std::lock_guard<std::mutex> run(a->run_mu);
    int rc = otfmm_batch_host(a->ctx, b.M, b.com, b.mon, b.is_leaf, b.n_sub, b.items, (int32_t)items.size(), b.L,
                              b.Lc, a->gsolve, a->precision, a->stream);
    if (rc == OTFMM_OK) rc = otfmm_batch_status(a->ctx, a->stream);   // synchronises the stream
    if (rc != OTFMM_OK) {
        msg = otfmm_last_error();
        return rc;
    }
    // leaves with a refined neighbour (the only leaves whose L_c the solve writes)
    std::vector<uint8_t> p2m_leaf(b.n_sub, 0);
    for (const otfmm_work_item& w : items) {
        if (w.kind != OTFMM_KIND_LEAF) continue;
        for (int d = 0; d < 26; ++d)
            if (w.neighbors[d] >= 0 && !b.is_leaf[w.neighbors[d]]) p2m_leaf[w.subgrid] = 1;
    }
    auto copy_out = [&](const otfmm_aggregator::Out& o) {
        const int ncomp = (o.kind == OTFMM_KIND_LEAF) ? 4 : 20;
        const double* rL = b.L + (size_t)o.slot * 20 * NCELL;
        if (o.l_stride == 0) std::copy(rL, rL + (size_t)ncomp * NCELL, o.L);
        else agg_aos_add(o.L, o.l_stride, rL, ncomp);
        if (!o.Lc) return;
        const double* rLc = (o.kind == OTFMM_KIND_LEAF && !p2m_leaf[o.slot]) ? nullptr : b.Lc + (size_t)o.slot * 3 * NCELL;
        if (o.lc_stride != 0) agg_aos_set3(o.Lc, o.lc_stride, rLc);
        else if (rLc) std::copy(rLc, rLc + 3 * NCELL, o.Lc);
        else std::fill(o.Lc, o.Lc + 3 * NCELL, 0.0);
    };
    // A full batch holds a few hundred MB of results (up to 92 KB per call),
    // and the batch's callers sleep while they are copied, so the copy is split
    // over host threads, AGG_COPY_CHUNK calls at a time. A helper that cannot
    // be started leaves its share to the others.
    const size_t nout = b.outs.size();
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (;;) {
            const size_t i0 = next.fetch_add(AGG_COPY_CHUNK);
            if (i0 >= nout) return;
            for (size_t i = i0; i < std::min(nout, i0 + AGG_COPY_CHUNK); ++i) copy_out(b.outs[i]);
        }
    };
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nthr = std::min<size_t>({hw, AGG_COPY_THREADS_MAX, (nout + AGG_COPY_CHUNK - 1) / AGG_COPY_CHUNK});
    std::vector<std::thread> helpers;
    for (size_t t = 1; t < nthr; ++t) {
        try {
            helpers.emplace_back(work);
        } catch (const std::system_error&) {
            break;
        }
    }
    work();
    for (auto& h : helpers) h.join();
    return OTFMM_OK;
}

// Runs buffer k if it can run now (full, or idle with no call between
// reserve and submit); called with the lock held, returns with it held.
// True if it ran.
bool agg_try_run(otfmm_aggregator* a, int k, std::unique_lock<AggLock>& lock) {
    otfmm_aggregator::Batch& b = a->b[k];
    const bool idle = b.state == otfmm_aggregator::OPEN && std::chrono::steady_clock::now() - b.last >= a->idle;
    if (!((b.state == otfmm_aggregator::CLOSED || idle) && b.pending == 0)) return false;
    const long long e = b.epoch;
    b.state = otfmm_aggregator::RUNNING;
    lock.unlock();
    std::string msg;
    const int rc = b.staged.empty() ? OTFMM_OK : agg_run(a, b, msg);
    lock.lock();
    if (rc != OTFMM_OK) {
        a->failed[e] = {rc, msg};
        a->any_failed = true;   // before done_epoch: a wait that sees the epoch done sees this too
    }
    b.done_epoch = e;
    b.staged.clear();
    b.outs.clear();
    b.state = otfmm_aggregator::FREE;
    a->cv.notify_all();
    return true;
}

}   // namespace

extern "C" {

int otfmm_aggregator_create(otfmm_context* ctx, int32_t max_subgrids, int32_t max_items, int32_t idle_us,
                            int gsolve_type, int precision, otfmm_aggregator** out) {
    if (!ctx || !out) return fail(OTFMM_ERR_INVALID, "NULL argument");
    *out = nullptr;
    if (max_subgrids < 27 || max_items < 1 || idle_us < 0)
        return fail(OTFMM_ERR_INVALID, "aggregator: max_subgrids >= 27, max_items >= 1, idle_us >= 0");
    if (gsolve_type != OTFMM_RHO && gsolve_type != OTFMM_DRHODT) return fail(OTFMM_ERR_INVALID, "bad gsolve_type");
    if (precision != OTFMM_FP64_EXACT && precision != OTFMM_FP64 && precision != OTFMM_FP32_SPLIT)
        return fail(OTFMM_ERR_INVALID, "unknown precision");
    DeviceGuard g(ctx->device);
    auto* a = new otfmm_aggregator;
    a->ctx = ctx;
    a->gsolve = gsolve_type;
    a->precision = precision;
    a->cap_sub = max_subgrids;
    a->cap_items = max_items;
    a->idle = std::chrono::microseconds(idle_us);
    cudaError_t e = cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking);
    const size_t n = (size_t)max_subgrids;
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        otfmm_aggregator::Batch& b = a->b[k];
        if ((e = cudaHostAlloc((void**)&b.M, sizeof(double) * n * 20 * NCELL, cudaHostAllocDefault)) != cudaSuccess ||
            (e = cudaHostAlloc((void**)&b.com, sizeof(double) * n * 3 * NCELL, cudaHostAllocDefault)) != cudaSuccess ||
            (e = cudaHostAlloc((void**)&b.mon, sizeof(double) * n * NCELL, cudaHostAllocDefault)) != cudaSuccess ||
            (e = cudaHostAlloc((void**)&b.L, sizeof(double) * n * 20 * NCELL, cudaHostAllocDefault)) != cudaSuccess ||
            (e = cudaHostAlloc((void**)&b.Lc, sizeof(double) * n * 3 * NCELL, cudaHostAllocDefault)) != cudaSuccess ||
            (e = cudaHostAlloc((void**)&b.is_leaf, n, cudaHostAllocDefault)) != cudaSuccess ||
            (e = cudaHostAlloc((void**)&b.items, sizeof(otfmm_work_item) * (size_t)max_items, cudaHostAllocDefault)) !=
                cudaSuccess)
            break;
        b.claimed.reserve(n);
        b.keys.init(n);
    }
    if (e != cudaSuccess) {
        for (auto& b : a->b) agg_free_buffers(b);
        if (a->stream) cudaStreamDestroy(a->stream);
        delete a;
        return cuda_fail(e, "aggregator buffers");
    }
    *out = a;
    return OTFMM_OK;
}

int otfmm_aggregator_destroy(otfmm_aggregator* a) {
    if (!a) return OTFMM_OK;
    {
        std::lock_guard<AggLock> lock(a->mu);
        for (auto& b : a->b)
            if (b.state != otfmm_aggregator::FREE && (b.pending > 0 || !b.staged.empty()))
                return fail(OTFMM_ERR_INVALID, "aggregator destroyed with calls in flight");
    }
    DeviceGuard g(a->ctx->device);
    cudaStreamSynchronize(a->stream);
    for (auto& b : a->b) agg_free_buffers(b);
    cudaStreamDestroy(a->stream);
    delete a;
    return OTFMM_OK;
}

int otfmm_aggregator_reserve(otfmm_aggregator* a, int32_t n, const uint64_t* keys, const uint8_t* is_leaf,
                             const uint8_t* need, int32_t* slots, uint8_t* fill, int64_t* ticket) {
    if (!a || !keys || !is_leaf || !need || !slots || !fill || !ticket) return fail(OTFMM_ERR_INVALID, "NULL argument");
    if (n < 1 || n > 27 || n > a->cap_sub) return fail(OTFMM_ERR_INVALID, "a call reserves 1..27 records");
    std::unique_lock<AggLock> lock(a->mu);
    for (;;) {
        int k = -1;
        for (int i = 0; i < 2 && k < 0; ++i)
            if (a->b[i].state == otfmm_aggregator::OPEN) k = i;
        for (int i = 0; i < 2 && k < 0; ++i)
            if (a->b[i].state == otfmm_aggregator::FREE) {
                otfmm_aggregator::Batch& nb = a->b[i];
                nb.state = otfmm_aggregator::OPEN;
                nb.epoch = ++a->epochs;
                nb.n_sub = nb.pending = 0;
                nb.keys.clear();
                nb.claimed.clear();
                nb.staged.clear();
                nb.outs.clear();
                nb.last = std::chrono::steady_clock::now();
                k = i;
            }
        if (k < 0) {
            // both buffers busy: run one that can run (its callers may not be
            // waiting yet), else wait for one to come free
            if (!agg_try_run(a, 0, lock) && !agg_try_run(a, 1, lock)) a->cv.wait_for(lock, a->idle);
            continue;
        }
        otfmm_aggregator::Batch& b = a->b[k];
        // each key looked up once: found[i] = its slot in the batch, -1 = new,
        // -2 - j = the same key as record j of this call
        int found[27];
        int fresh = 0;
        for (int i = 0; i < n; ++i) {
            found[i] = -1;
            if (keys[i] != 0) {
                for (int j = 0; j < i && found[i] == -1; ++j)
                    if (keys[j] == keys[i]) found[i] = -2 - j;
                if (found[i] == -1) found[i] = b.keys.find(keys[i]);
            }
            if (found[i] == -1) ++fresh;
        }
        if (b.n_sub + fresh > a->cap_sub || (int)b.staged.size() + b.pending + 1 > a->cap_items) {
            // full: no more calls join it; it runs once its reserved calls have submitted
            b.state = otfmm_aggregator::CLOSED;
            if (b.pending == 0 && b.staged.empty()) b.state = otfmm_aggregator::FREE;
            a->cv.notify_all();
            continue;
        }
        for (int i = 0; i < n; ++i) {
            int s = found[i] >= 0 ? found[i] : found[i] <= -2 ? slots[-2 - found[i]] : -1;
            if (s < 0) {
                s = b.n_sub++;
                b.claimed.push_back(0);
                b.is_leaf[s] = is_leaf[i] ? 1 : 0;
                if (keys[i] != 0) b.keys.insert(keys[i], s);
            } else if ((b.is_leaf[s] != 0) != (is_leaf[i] != 0)) {
                return fail(OTFMM_ERR_INVALID, "a record key is used for a leaf and for a refined subgrid");
            }
            slots[i] = s;
            fill[i] = (uint8_t)(need[i] & ~b.claimed[s]);
            b.claimed[s] |= need[i];
        }
        ++b.pending;
        b.last = std::chrono::steady_clock::now();
        *ticket = (int64_t)((b.epoch << 1) | k);
        return OTFMM_OK;
    }
}

int otfmm_aggregator_record(otfmm_aggregator* a, int64_t ticket, int32_t slot, double** M, double** com,
                            double** mon) {
    if (!a || !M || !com || !mon) return fail(OTFMM_ERR_INVALID, "NULL argument");
    // no lock: the batch buffers are fixed for the aggregator's life, and a
    // ticket's batch keeps its epoch until every reserved call has submitted
    otfmm_aggregator::Batch& b = a->b[ticket & 1];
    if (b.epoch.load(std::memory_order_acquire) != (ticket >> 1) || slot < 0 || slot >= a->cap_sub)
        return fail(OTFMM_ERR_INVALID, "stale ticket or slot out of range");
    *M = b.M + (size_t)slot * 20 * NCELL;
    *com = b.com + (size_t)slot * 3 * NCELL;
    *mon = b.mon + (size_t)slot * NCELL;
    return OTFMM_OK;
}

}   // extern "C"

namespace {

// Ends a call's reservation and, if its item and output description are
// valid, adds it to its batch.
int agg_submit(otfmm_aggregator* a, int64_t ticket, const otfmm_work_item* item, double* L, int l_stride,
               double* L_c, int lc_stride) {
    if (!a || !item) return fail(OTFMM_ERR_INVALID, "NULL argument");
    std::lock_guard<AggLock> lock(a->mu);
    otfmm_aggregator::Batch& b = a->b[ticket & 1];
    if (b.epoch != (ticket >> 1) || (b.state != otfmm_aggregator::OPEN && b.state != otfmm_aggregator::CLOSED))
        return fail(OTFMM_ERR_INVALID, "stale ticket");
    const int ncomp = (item->kind == OTFMM_KIND_LEAF) ? 4 : 20;
    bool ok = L != nullptr && item->subgrid >= 0 && item->subgrid < b.n_sub && item->kind >= 0 && item->kind <= 2 &&
              (l_stride == 0 || l_stride >= ncomp) && (lc_stride == 0 || lc_stride >= 3);
    for (int d = 0; d < 26; ++d) ok = ok && item->neighbors[d] >= -1 && item->neighbors[d] < b.n_sub;
    --b.pending;   // the reservation ends either way, so the batch can run without this call
    b.last = std::chrono::steady_clock::now();
    // waiters can only act on a batch with no reservation left (it may run)
    if (b.pending == 0) a->cv.notify_all();
    if (!ok) return fail(OTFMM_ERR_INVALID, "bad work item or output strides (call withdrawn)");
    b.staged.push_back(*item);
    b.outs.push_back({L, L_c, item->subgrid, item->kind, l_stride, lc_stride});
    return OTFMM_OK;
}

}   // namespace

extern "C" {

int otfmm_aggregator_submit(otfmm_aggregator* a, int64_t ticket, const otfmm_work_item* item, double* L,
                            double* L_c) {
    return agg_submit(a, ticket, item, L, 0, L_c, 0);
}

int otfmm_aggregator_submit_aos(otfmm_aggregator* a, int64_t ticket, const otfmm_work_item* item, double* L,
                                int32_t l_stride, double* L_c, int32_t lc_stride) {
    if (l_stride < 1 || (L_c && lc_stride < 1)) {
        // still end the reservation, with an item that is refused
        otfmm_work_item bad{};
        bad.subgrid = -1;
        agg_submit(a, ticket, &bad, nullptr, 0, nullptr, 0);
        return fail(OTFMM_ERR_INVALID, "aggregator: AoS strides must be positive (call withdrawn)");
    }
    return agg_submit(a, ticket, item, L, l_stride, L_c, L_c ? lc_stride : 0);
}

int otfmm_aggregator_poll(otfmm_aggregator* a, int64_t ticket) {
    if (!a) return fail(OTFMM_ERR_INVALID, "NULL argument");
    const long long e = ticket >> 1;
    const int k = (int)(ticket & 1);
    otfmm_aggregator::Batch& b = a->b[k];
    if (b.done_epoch.load(std::memory_order_acquire) >= e) return 1;
    // no lock while the batch runs on another thread: pollers spin on this
    if (b.epoch.load(std::memory_order_relaxed) == e && b.state.load(std::memory_order_relaxed) == otfmm_aggregator::RUNNING)
        return 0;
    std::unique_lock<AggLock> lock(a->mu);
    if (b.done_epoch >= e) return 1;
    if (b.epoch != e) return fail(OTFMM_ERR_INVALID, "unknown ticket");
    // a batch that can run now runs on this thread, as in a wait
    agg_try_run(a, k, lock);
    return b.done_epoch >= e ? 1 : 0;
}

int otfmm_aggregator_wait(otfmm_aggregator* a, int64_t ticket) {
    if (!a) return fail(OTFMM_ERR_INVALID, "NULL argument");
    const long long e = ticket >> 1;
    otfmm_aggregator::Batch& b = a->b[ticket & 1];
    // the call's batch has run (its results are in place) and no run failed
    if (b.done_epoch.load(std::memory_order_acquire) >= e && !a->any_failed.load(std::memory_order_acquire))
        return OTFMM_OK;
    std::unique_lock<AggLock> lock(a->mu);
    for (;;) {
        if (b.done_epoch >= e) break;
        if (b.epoch != e) return fail(OTFMM_ERR_INVALID, "unknown ticket");
        if (agg_try_run(a, (int)(ticket & 1), lock)) continue;
        a->cv.wait_for(lock, a->idle);
    }
    auto it = a->failed.find(e);
    if (it == a->failed.end()) return OTFMM_OK;
    const auto f = it->second;
    lock.unlock();
    return fail(f.first, f.second);
}

}   // extern "C"
