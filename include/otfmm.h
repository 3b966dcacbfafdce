/*
 * otfmm.h — C ABI of the B200-native FMM cell-interaction kernels for
 * Octo-Tiger (libotfmm.so).
 *
 * These entry points are what a new `interaction_device_kernel_type` backend
 * inside Octo-Tiger binds. They replace, for one GPU:
 *   - the multipole (M2L) launch path
 *     octotiger::fmm::multipole_interactions::launch_interface
 *     (octotiger/multipole_interactions/kernel/kokkos_kernel.hpp:768-863,
 *      called from multipole_kernel at :944-983, itself behind
 *      multipole_kernel_interface, src/multipole_interactions/multipole_kernel_interface.cpp:73-169);
 *   - the monopole (P2P + P2M) launch path
 *     octotiger::fmm::monopole_interactions::launch_interface_p2p_p2m / launch_interface_p2p
 *     (octotiger/monopole_interactions/kernel/kokkos_kernel.hpp:1051-1165,
 *      called from monopole_kernel at :1279-1354, behind monopole_kernel_interface,
 *      src/monopole_interactions/monopole_kernel_interface.cpp:97-198);
 *   - the stencil set-up those paths do on first use
 *     (get_device_masks / get_device_constants, kokkos_kernel.hpp:58-82 and
 *      monopole kokkos_kernel.hpp:78-114; calculate_stencil,
 *      src/multipole_interactions/util/calculate_stencil.cpp:23-160).
 * Beyond the reference, a batched entry point runs a whole gravity solve's
 * work list (every refined and leaf subgrid of the octree) in one launch from
 * subgrid data resident in GPU memory.
 *
 * Conventions
 *   - All functions return an int status: OTFMM_OK (0) or a negative error
 *     code; otfmm_last_error() gives a message for the calling thread. No C++
 *     exception crosses this boundary. The reference aborts on misuse
 *     (multipole_kernel_interface.cpp:107-158); here the caller decides.
 *   - Thread-safe: a context may be used from several host threads; each call
 *     is enqueued on the stream the caller passes (cudaStream_t as void*,
 *     NULL = the calling thread's default stream: the library is built with
 *     per-thread default streams, which synchronise with the legacy default
 *     stream as any blocking stream does, and calls from several threads on
 *     their own default streams run concurrently).
 *   - Layouts: "SoA" is the reference's per-subgrid kernel layout
 *     (mon[5832], M[20][5851], com[3][5851] over the 18^3 padded halo;
 *     L[20][531], L_c[3][531]); "pool" is M[n][20][512], com[n][3][512],
 *     mon[n][512] per subgrid. Cell order is x-major (x*64 + y*8 + z).
 *   - Precision: OTFMM_FP64_EXACT reproduces the reference's arithmetic bit
 *     for bit (IEEE operations in the reference's order, no contraction);
 *     OTFMM_FP64 is the fast FP64 kernel (fused multiply-adds, reordered
 *     constants; within 1e-12 of the reference); OTFMM_FP32_SPLIT builds the
 *     derivative tensors and contracts them in FP32 with FP64 chunk sums,
 *     and keeps centre-of-mass differences, the angular correction L_c and
 *     the final accumulation in FP64.
 */
#ifndef OTFMM_H
#define OTFMM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OTFMM_OK 0
#define OTFMM_ERR_INVALID (-1)     /* bad argument (null pointer, size, kind, id) */
#define OTFMM_ERR_THETA (-2)       /* theta below the compiled minimum 0.34 */
#define OTFMM_ERR_CUDA (-3)        /* CUDA runtime error */
#define OTFMM_ERR_DEVICE (-4)      /* kernel reported a bad work item on the device */
#define OTFMM_ERR_UNSUPPORTED (-5) /* combination not built (e.g. precision for theta) */

/* gsolve_type (octotiger/defs.hpp): RHO carries the angular correction L_c */
#define OTFMM_RHO 0
#define OTFMM_DRHODT 1

#define OTFMM_FP64_EXACT 0
#define OTFMM_FP64 1
#define OTFMM_FP32_SPLIT 2

/* Work-item kinds, as node_server::compute_fmm dispatches them (src/node_server.cpp:711-723). */
#define OTFMM_KIND_M2L 0      /* refined node: multipole_kernel_interface, use_root_stencil = false */
#define OTFMM_KIND_M2L_ROOT 1 /* level-0 node: multipole_kernel_interface, use_root_stencil = true */
#define OTFMM_KIND_LEAF 2     /* leaf: monopole_kernel_interface (P2P, plus P2M per refined neighbour) */

/* One work item (144 bytes). neighbors[d] is the pool index of the same-level
 * neighbour in geo::direction flat order d = 0..25 (octotiger/geometry.hpp:91-197),
 * or -1 for an empty direction (is_direction_empty). dx and xbase as passed to
 * multipole_kernel_interface (xbase = centre of inner cell (0,0,0),
 * src/node_server.cpp:712-715). */
typedef struct otfmm_work_item {
    int32_t subgrid;
    int32_t kind;
    int32_t neighbors[26];
    double dx;
    double xbase[3];
} otfmm_work_item;

typedef struct otfmm_context otfmm_context;

/* Creates a context on `device` for opening angle theta (opts().theta,
 * src/options_processing.cpp:119; must be >= 0.34, :234-236). Builds the
 * multipole two-phase stencil and the monopole stencil with its constants and
 * uploads them. Replaces calculate_stencil + get_device_masks. theta >= 0.5
 * runs the shared-memory tile kernels, 0.34 <= theta < 0.5 (partners up to
 * two coarse cells away) global-memory kernels of the same results. */
int otfmm_create(int device, double theta, otfmm_context** out);
int otfmm_destroy(otfmm_context* ctx);

/* Stencil sizes of the context: counts[0] multipole offsets, [1] of which
 * full multipole (phase one), [2] monopole offsets; masks may be NULL, else
 * 1331 bytes each (11^3 box, x-major) like stencil_masks / inner_stencil_masks
 * and the P2P mask. */
int otfmm_stencil_info(const otfmm_context* ctx, int32_t counts[3], uint8_t* mpole_mask, uint8_t* mpole_phase,
                       uint8_t* p2p_mask);

/* Multipole interactions of one subgrid from the reference's SoA buffers
 * (device pointers). Equivalent of launch_interface (kokkos_kernel.hpp:768-863)
 * followed by its partial-sum reduction: writes L (20 x 531) and, for RHO,
 * L_c (3 x 531). use_root_stencil selects the root kernel
 * (multipole_kernel_root_*_impl); mon is not read then and may be NULL. */
int otfmm_m2l_soa(otfmm_context* ctx, const double* mon, const double* M, const double* com, double* L,
                  double* L_c, int gsolve_type, int use_root_stencil, int precision, void* stream);

/* Same with host buffers: copies in, computes, copies out and waits, like the
 * reference's launch_interface with host_buffer arguments and fut.get(). */
int otfmm_m2l_soa_host(otfmm_context* ctx, const double* mon, const double* M, const double* com, double* L,
                       double* L_c, int gsolve_type, int use_root_stencil, int precision);

/* No counterpart in the reference. Same as otfmm_m2l_soa_host for up to
 * OTFMM_NOALLOC_MAX_SUBGRIDS subgrids per call (host buffers laid out one
 * subgrid after the other: mon[n][5832], M[n][20*5851], com[n][3*5851] in,
 * L[n][20*531], L_c[n][3*531] out), but it allocates nothing: its device
 * staging is a fixed static array of OTFMM_NOALLOC_MAX_SUBGRIDS x 1.22 MB that
 * every GPU loading the library holds until the process exits. For callers
 * that must not allocate device memory while they run: code inside a
 * pre-sized memory budget, threads that must not trigger the implicit device
 * synchronisation of cudaMalloc/cudaFree, or HPX tasks on a hot path where the
 * reference uses recycled buffers. The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress). With CUDA's lazy module
 * loading the library's device code, and the array with it, is placed on a
 * device when the library is first used there, so make that first call at
 * set-up time, before the code that must not allocate runs. Larger n_subgrids is rejected (OTFMM_ERR_INVALID). All calls
 * share the one array: calls that overlap on the GPU would race, so calls
 * from this library are serialised and each waits for its stream before it
 * returns, on error returns too. */
#define OTFMM_NOALLOC_MAX_SUBGRIDS 4
int otfmm_m2l_soa_host_noalloc(otfmm_context* ctx, int32_t n_subgrids, const double* mon, const double* M,
                               const double* com, double* L, double* L_c, int gsolve_type, int use_root_stencil,
                               int precision, void* stream);

/* P2P of one leaf subgrid from its staged monopole buffer (mon[5832], device
 * pointer), p2p_kernel_impl + sum_p2p_results (monopole kokkos_kernel.hpp:118-320):
 * writes L4 (4 x 531). */
int otfmm_p2p_soa(otfmm_context* ctx, const double* mon, double dx, double* L4, int precision, void* stream);

/* P2M of one leaf subgrid against the refined neighbour in direction d
 * (0..25): p2m_kernel_impl_rho / _non_rho (monopole kokkos_kernel.hpp:517-942).
 * neighbor_M / neighbor_com hold the neighbour's slab in the layout of
 * update_neighbor_input (20 / 3 components, stride = slab cells + 19),
 * inner_com the leaf's centres of mass (3 x 531). Adds to L4 (4 x 531) and
 * L_c (3 x 531); reset_lc zeroes L_c first (first P2M call of a subgrid). */
int otfmm_p2m_soa(otfmm_context* ctx, int d, const double* neighbor_M, const double* neighbor_com,
                  const double* inner_com, double* L4, double* L_c, int gsolve_type, int reset_lc, int precision,
                  void* stream);

/* Halo staging for the per-subgrid entry points, on the device from the
 * resident pool: the reference's update_input restated
 * (octotiger/multipole_interactions/legacy/multipole_interaction_interface.hpp:88-281
 * for refined and root items -> mon[5832], M[20][5851], com[3][5851];
 * octotiger/monopole_interactions/legacy/monopole_interaction_interface.hpp:64-143
 * for leaf items -> mon[5832], M and com unused and may be NULL). `item` is a
 * host pointer; the output buffers are device pointers. Asynchronous. */
int otfmm_stage_soa(otfmm_context* ctx, const double* pool_M, const double* pool_com, const double* pool_mon,
                    const uint8_t* pool_is_leaf, int32_t n_subgrids, const otfmm_work_item* item, double* mon,
                    double* M, double* com, void* stream);

/* Slab of refined neighbour `neighbor` seen in direction d (0..25) by a leaf,
 * in the layout otfmm_p2m_soa reads (update_neighbor_input,
 * octotiger/monopole_interactions/legacy/p2m_interaction_interface.hpp:102-160):
 * 20 / 3 components of stride *stride = cells + 19 (at most 320 cells, stride 339). */
int otfmm_stage_p2m_soa(otfmm_context* ctx, const double* pool_M, const double* pool_com, int32_t n_subgrids,
                        int32_t neighbor, int d, double* neighbor_M, double* neighbor_com, int32_t* stride,
                        void* stream);

/* Batched solve: every work item of `items` (device array of n_items),
 * reading the resident pool (device pointers, n_subgrids records) and writing
 * per subgrid into L[n][20][512] and L_c[n][3][512]:
 *   refined items: all 20 L components and the 3 L_c components (zeros for DRHODT);
 *   leaf items:    L[0..3] (P2P + P2M), and L_c when a neighbour is refined.
 * Everything else is left untouched: as node_server::compute_fmm does before
 * the reference's kernels (src/node_server.cpp:701-705), the caller zeroes L
 * and L_c once; later solves of work lists with the same kinds overwrite the
 * same entries. Enqueues a classification kernel that builds device-side work
 * lists, then persistent launches for the multipole tiles of refined items,
 * P2P of the leaves and P2M of leaves with refined neighbours (the reference's
 * P2P-then-P2M order); the two leaf launches run on the context's second
 * stream, forked from `stream` after the classification and joined back into
 * it, so that they use the SMs the tiles leave idle. Work-list storage lives in the context and grows (a
 * device allocation) when a larger work list arrives. Asynchronous; work items
 * are validated on the device and a bad one is reported by otfmm_batch_status
 * (its outputs are left unwritten). Every subgrid may appear in at most one
 * work item. Calls that overlap on the GPU must use distinct contexts. */
int otfmm_batch(otfmm_context* ctx, const double* pool_M, const double* pool_com, const double* pool_mon,
                const uint8_t* pool_is_leaf, int32_t n_subgrids, const otfmm_work_item* items, int32_t n_items,
                double* L, double* L_c, int gsolve_type, int precision, void* stream);

/* Kernel variants of the batched solve. Every variant computes the same
 * interactions within its precision's tolerance; they differ in speed only.
 * No counterpart in the reference (its kernels have fixed launch shapes). */
#define OTFMM_SPLIT_WARP_SPECIALISED 0 /* FP32-split RHO tiles: FP32 contraction warps + FP64 L_c warps */
#define OTFMM_SPLIT_SINGLE_ROLE 1      /* FP32-split RHO tiles: every warp does both */
#define OTFMM_SPLIT_WARP_SPECIALISED_PACKED 2 /* warp-specialised, contraction in packed FP32 pairs */
#define OTFMM_SPLIT_FUSED 3 /* FP32-split RHO tiles: each thread interleaves the FP32 contraction and the FP64 L_c of its pairs */
#define OTFMM_P2P_BOX 0     /* leaf P2P over the 6x6x6 partner box, four cells per thread */
#define OTFMM_P2P_STENCIL 1 /* leaf P2P in stencil order, two cells per thread */
#define OTFMM_P2M_COARSE 0  /* fast-form P2M: one lane per cell, the 8 cells of a coarse cell share partner loads */
#define OTFMM_P2M_LANES 1   /* fast-form P2M: p2m_lanes lanes share one cell's partners */
#define OTFMM_P2M_OCTANT 2  /* P2M by leaf octant, partner slabs in shared memory (the split precision contracts in FP32) */
typedef struct otfmm_tuning {
    int32_t split_m2l_form;  /* one of the OTFMM_SPLIT_* forms above */
    int32_t split_m2l_chunk; /* FP32 partial sums of the warp-specialised tiles promoted every 8 or 16 partners
                              * (the fused form promotes every 16 whatever this field holds) */
    int32_t split_p2p_chunk; /* FP32 P2P partial sums promoted every 16 or 32 partners (box form: every 18 or 36) */
    int32_t p2m_lanes;       /* fast-form P2M: at most 4, 8 or 16 lanes share one cell's entries */
    int32_t p2p_form;        /* OTFMM_P2P_BOX or OTFMM_P2P_STENCIL (fast and split forms, theta >= 0.5) */
    int32_t p2m_form;        /* OTFMM_P2M_COARSE, OTFMM_P2M_LANES or OTFMM_P2M_OCTANT (fast and split forms,
                              * theta >= 0.5) */
} otfmm_tuning;

/* One otfmm_batch with CUDA events between its launches: kernel_ms receives the
 * device time of the classification, multipole-tile, P2P and P2M kernels of
 * this solve (roofline reporting). Synchronises the stream. No counterpart in
 * the reference. */
int otfmm_batch_profile(otfmm_context* ctx, const double* pool_M, const double* pool_com, const double* pool_mon,
                        const uint8_t* pool_is_leaf, int32_t n_subgrids, const otfmm_work_item* items,
                        int32_t n_items, double* L, double* L_c, int gsolve_type, int precision, float kernel_ms[4],
                        void* stream);

/* The context's current variants (defaults: fused, 16, 32, 4, box, octant). */
int otfmm_get_tuning(const otfmm_context* ctx, otfmm_tuning* out);
int otfmm_set_tuning(otfmm_context* ctx, const otfmm_tuning* t);

/* Autotuner: times the variants on the caller's own batch (same arguments as
 * otfmm_batch; L and L_c are overwritten) by coordinate descent, median of
 * `repeats` solves per candidate, keeps the fastest in the context and
 * returns it in *chosen (may be NULL). Synchronises the stream. */
int otfmm_autotune(otfmm_context* ctx, const double* pool_M, const double* pool_com, const double* pool_mon,
                   const uint8_t* pool_is_leaf, int32_t n_subgrids, const otfmm_work_item* items, int32_t n_items,
                   double* L, double* L_c, int gsolve_type, int precision, int repeats, otfmm_tuning* chosen,
                   void* stream);

/* A batched solve captured once into a CUDA graph (the counter resets, the
 * classification and the three persistent launches of otfmm_batch with the
 * context's variants at creation), replayed by otfmm_plan_launch with one
 * graph launch. The plan binds the given device pointers and owns its own
 * work-list storage and error flag, so plans of one context may run
 * concurrently when their outputs are disjoint; otfmm_plan_status reads the
 * flag of the last launch. No counterpart in the reference. */
typedef struct otfmm_plan otfmm_plan;
int otfmm_plan_create(otfmm_context* ctx, const double* pool_M, const double* pool_com, const double* pool_mon,
                      const uint8_t* pool_is_leaf, int32_t n_subgrids, const otfmm_work_item* items, int32_t n_items,
                      double* L, double* L_c, int gsolve_type, int precision, otfmm_plan** out);
/* A plan of otfmm_batch_host: the whole host-buffer solve (chunked uploads,
 * kernels, downloads) captured once for fixed pinned host buffers and work
 * list, replayed by otfmm_plan_launch with one graph launch; every launch reads
 * the host inputs' current contents and writes the host outputs (same contract
 * as otfmm_batch_host). It uses the context's host-path buffers and work
 * lists: an otfmm_batch_host call after it was made, or a solve of the context
 * with more work items, invalidates it (its launch then returns
 * OTFMM_ERR_INVALID). No counterpart in the reference. */
int otfmm_plan_create_host(otfmm_context* ctx, const double* pool_M, const double* pool_com, const double* pool_mon,
                           const uint8_t* pool_is_leaf, int32_t n_subgrids, const otfmm_work_item* items,
                           int32_t n_items, double* L, double* L_c, int gsolve_type, int precision,
                           otfmm_plan** out);
int otfmm_plan_launch(otfmm_plan* plan, void* stream);
int otfmm_plan_status(otfmm_plan* plan, void* stream);
int otfmm_plan_destroy(otfmm_plan* plan);

/* Batched solve from host buffers (pinned memory lets the copies overlap):
 * pool and work list as for otfmm_batch but in host memory; writes the host
 * outputs L[n][20][512] and L_c[n][3][512]: the solve's results, zeros where
 * it computes nothing, as node_server::compute_fmm zeroes L / L_c before the
 * reference's kernels (src/node_server.cpp:701-705) - except L[4..19] of leaf
 * subgrids, which no kernel writes (the reference's monopole kernels output
 * L[0..3] and L_c), and L_c of leaves without a refined neighbour (which only
 * the P2M writes), both left as the caller set them. The pool is uploaded in
 * chunks of consecutive subgrids (the moments of refined subgrids, the masses
 * of chunks with leaves and the centres of mass: what the kernels read); each work item runs once the records it
 * reads have arrived and each output range is copied back once final, on two
 * copy streams, so uploads, kernels and downloads overlap when neighbours have
 * nearby pool indices. When pool_M, pool_com, L and L_c are page-locked host
 * memory mapped into the device's address space (cudaHostAlloc /
 * cudaMallocHost, 16-byte aligned) the scattered records move by one SM-copy
 * launch per chunk instead of one DMA copy per run of subgrids, and only the
 * centres of mass of refined subgrids and of leaves with a refined neighbour
 * are uploaded; other buffers take the copy engines. Device copies live in the context (grown on demand).
 * Asynchronous: the outputs are valid once `stream` has completed; a later
 * call waits for the earlier call's uploads. Calls of one context share its
 * device copies: consecutive calls on the same stream run in order, calls on
 * different streams must not overlap on the GPU (wait for the earlier call's
 * stream first, or use distinct contexts). Work items are re-validated on the
 * device (otfmm_batch_status). No counterpart in the reference. */
int otfmm_batch_host(otfmm_context* ctx, const double* pool_M, const double* pool_com, const double* pool_mon,
                     const uint8_t* pool_is_leaf, int32_t n_subgrids, const otfmm_work_item* items, int32_t n_items,
                     double* L, double* L_c, int gsolve_type, int precision, void* stream);

/* ------------------------------------------------------------------ tree passes
 * The two passes around the interaction kernels of a gravity solve, on the
 * device from the resident pool. One node of the octree (48 bytes): */
typedef struct otfmm_tree_node {
    int32_t subgrid;  /* pool index of the node */
    int32_t parent;   /* pool index of its parent, -1 for the root */
    int32_t octant;   /* its octant in the parent: x + 2y + 4z (geo::octant) */
    int32_t reserved;
    double dx;        /* cell size */
    double xbase[3];  /* centre of inner cell (0,0,0) */
} otfmm_tree_node;

/* Upward pass (M2M): grid::compute_multipoles (src/grid_fmm.cpp:1639-1803)
 * with the octant gather of node_server::compute_fmm (src/node_server.cpp:613-640).
 * `nodes` (device) are ordered by level, root first; level l is
 * [level_start[l], level_start[l+1]) (host array of n_levels + 1). Levels run
 * finest first: every node forms the centres of mass of its 4^3 coarse cells
 * (RHO; written to com1[n][3][64]) and the multipoles of its children shifted
 * to them (taylor::operator>>=), written into its parent's cells of its octant
 * (pool M and com). Leaves take pool mon as their cell masses and, for RHO,
 * their cell centres as centres of mass. DRHODT reuses com / com1 of the
 * preceding RHO pass. Arithmetic in the reference's order (bit-identical to
 * the oracle). Asynchronous; malformed nodes raise the flag otfmm_batch_status
 * reports. */
int otfmm_upward(otfmm_context* ctx, double* pool_M, double* pool_com, const double* pool_mon,
                 const uint8_t* pool_is_leaf, double* com1, int32_t n_subgrids, const otfmm_tree_node* nodes,
                 const int32_t* level_start, int32_t n_levels, int gsolve_type, void* stream);

/* Downward pass (L2L): grid::compute_expansions (src/grid_fmm.cpp:1525-1637)
 * with the octant scatter of node_server (src/node_server.cpp:756-786), root
 * first: every fine cell adds its parent cell's expansion shifted to the cell's
 * centre of mass (taylor::operator<<=) and the parent's L_c (RHO) to L / L_c
 * (the interaction outputs, [n][20][512] / [n][3][512]); leaves then write
 * G[n][4][512]: RHO phi = gconst L0, g = -gconst (L1..3 + L_c if
 * correct_am_grav); DRHODT d(phi)/dt = gconst L0 in slot 0. */
int otfmm_downward(otfmm_context* ctx, const double* pool_com, const uint8_t* pool_is_leaf, const double* com1,
                   int32_t n_subgrids, const otfmm_tree_node* nodes, const int32_t* level_start, int32_t n_levels,
                   double* L, double* L_c, double* G, double gconst, int correct_am_grav, int gsolve_type,
                   void* stream);

/* Cell-interactions a work list evaluates (host-side count, no device
 * work): the (cell, partner) pairs that pass the stencil and coarse-distance
 * masks, which is what the reference's kernels evaluate. per_class (may be
 * NULL) receives [M2L, root M2L, P2P, P2M]. is_leaf and items are host
 * arrays. Returns the total, or a negative status. */
long long otfmm_count_pairs(const otfmm_context* ctx, const uint8_t* is_leaf, int32_t n_subgrids,
                            const otfmm_work_item* items, int32_t n_items, long long per_class[4]);

/* Aggregation of per-node calls (no single counterpart in the reference, whose
 * node_server::compute_fmm calls the interaction interfaces once per node from
 * many threads at once, src/node_server.cpp:717-722; its Kokkos backend fuses
 * concurrent monopole calls, octotiger/monopole_interactions/kernel/
 * kokkos_kernel.hpp:1357-1405, and its CUDA backend spreads callers over a
 * stream pool, src/multipole_interactions/legacy/
 * cuda_multipole_interaction_interface.cpp:64-70). Concurrent calls of every
 * kind join one batched solve (otfmm_batch_host on the aggregator's own stream):
 *   1. otfmm_aggregator_reserve(n records: own subgrid first, then neighbours):
 *      slots[i] is record i's pool slot in the open batch; fill[i] the parts
 *      (OTFMM_AGG_* bits of need[i]) this caller must write - a record whose
 *      non-zero key is already in the batch needs none (key = an address that
 *      identifies the data, the same for a node's own call and for the
 *      payloads that alias it; 0 = never shared). Blocks while both batch
 *      buffers are busy.
 *   2. otfmm_aggregator_record: host pointers to a slot's pinned storage
 *      (M[20][512], com[3][512], mon[512]); write the parts of fill[i].
 *   3. otfmm_aggregator_submit: the call's work item (subgrid and neighbour
 *      fields are slots, -1 = empty) and its output buffers; returns at once.
 *      Every reserved call must be submitted (a bad item withdraws the call
 *      and returns OTFMM_ERR_INVALID).
 *      otfmm_aggregator_submit_aos instead: the results go into the caller's
 *      array-of-structures cells when the batch runs, L[u * l_stride + c] +=
 *      component c of cell u (the reference's L += result) and, when L_c is
 *      not NULL, L_c[u * lc_stride + c] = component c (L_c = result); no
 *      intermediate buffer, and the caller leaves those cells alone until its
 *      wait returns (two calls in flight must not name the same cells: the
 *      results of one batch are written by several threads).
 *   4. otfmm_aggregator_wait(ticket): blocks until the call's batch has run
 *      (otfmm_aggregator_poll(ticket) instead returns at once: 1 once the
 *      batch has run, 0 before, so that a task can yield to its scheduler in
 *      between; a poll that finds the batch ready to run runs it);
 *      then L holds 20 x 512 (multipole items) or 4 x 512 (leaves) values and
 *      L_c, when not NULL, 3 x 512 (SoA), or the AoS cells are updated. A
 *      caller may have many calls submitted before it waits (as HPX tasks do).
 * A batch runs when it is full and all its reserved calls have submitted, or
 * when it has been idle for idle_us with no call between reserve and submit;
 * a caller in otfmm_aggregator_wait or _poll (or in a reserve that finds both
 * batch buffers busy) runs it. All calls of an aggregator share its solve type and
 * precision. Thread-safe; no context-wide lock is held while callers copy their
 * data. Destroy only with no call in flight. */
#define OTFMM_AGG_M 1
#define OTFMM_AGG_COM 2
#define OTFMM_AGG_MON 4
typedef struct otfmm_aggregator otfmm_aggregator;
int otfmm_aggregator_create(otfmm_context* ctx, int32_t max_subgrids, int32_t max_items, int32_t idle_us,
                            int gsolve_type, int precision, otfmm_aggregator** out);
int otfmm_aggregator_destroy(otfmm_aggregator* agg);
int otfmm_aggregator_reserve(otfmm_aggregator* agg, int32_t n, const uint64_t* keys, const uint8_t* is_leaf,
                             const uint8_t* need, int32_t* slots, uint8_t* fill, int64_t* ticket);
int otfmm_aggregator_record(otfmm_aggregator* agg, int64_t ticket, int32_t slot, double** M, double** com,
                            double** mon);
int otfmm_aggregator_submit(otfmm_aggregator* agg, int64_t ticket, const otfmm_work_item* item, double* L,
                            double* L_c);
/* l_stride >= the components of the item's kind (20 multipole, 4 leaf),
 * lc_stride >= 3, in doubles. A leaf without a refined neighbour has no P2M
 * part: its L_c cells are set to zero, as otfmm_aggregator_submit's L_c. */
int otfmm_aggregator_submit_aos(otfmm_aggregator* agg, int64_t ticket, const otfmm_work_item* item, double* L,
                                int32_t l_stride, double* L_c, int32_t lc_stride);
int otfmm_aggregator_poll(otfmm_aggregator* agg, int64_t ticket);
int otfmm_aggregator_wait(otfmm_aggregator* agg, int64_t ticket);

/* Checks a device-side error flag written by the last otfmm_batch on `stream`
 * without synchronizing the whole device: returns OTFMM_OK or OTFMM_ERR_DEVICE. */
int otfmm_batch_status(otfmm_context* ctx, void* stream);

/* Device memory helpers for host adapters that do not link the CUDA runtime
 * themselves (include/otfmm_octotiger.hpp): allocate / free on the context's
 * device, and blocking copies between host and device. */
int otfmm_device_alloc(otfmm_context* ctx, size_t bytes, void** ptr);
int otfmm_device_free(void* ptr);
int otfmm_copy_to_device(otfmm_context* ctx, void* dst, const void* src, size_t bytes);
int otfmm_copy_to_host(otfmm_context* ctx, void* dst, const void* src, size_t bytes);

/* Message for the last error on the calling thread ("" if none). */
const char* otfmm_last_error(void);

/* Library build information ("sm_100a ..."). */
const char* otfmm_build_info(void);

/* Measures the FP64 and FP32 FMA issue rates of the current device with a
 * register-resident FMA loop (lanes x FMAs x 2 flops / time); results in
 * TFLOP/s. Used as the roofline denominators. */
int otfmm_measure_fma_peaks(int device, double* fp64_tflops, double* fp32_tflops);

#ifdef __cplusplus
}
#endif

#endif /* OTFMM_H */
