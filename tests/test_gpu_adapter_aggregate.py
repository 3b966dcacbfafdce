"""The C++ drop-in adapter driven like node_server::compute_fmm: one call per
node of a small AMR tree (multipole, P2P and P2M nodes) from several host
threads at once, AoS inputs, neighbour payloads aliasing the neighbours' data
(libotfmm_adapter_pass.so). The aggregated interfaces gather the concurrent
calls into batched solves; the grids after the pass must equal the oracle:
bit-identical in the exact FP64 form, within 1e-12 in the fast form. Small
batch capacities force many batches (full batches close while others run);
the per-call interfaces on the context give the same results. The batch
writes the grids' cells itself (otfmm_aggregator_submit_aos), or, with
in_place off, finish() adds SoA results on the caller's thread."""
from __future__ import annotations

import numpy as np
import pytest

from octotiger_b200.layout import DRHODT, KIND_LEAF, RHO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from octotiger_b200.otfmm import Context
    c = Context(0, 0.5)
    yield c
    c.close()


@pytest.fixture(scope="module")
def tree():
    from octotiger_b200 import amr
    return amr.polytrope_batch(radius=0.05, max_level=5, seed=81)


def expected(tree, oracle, solve):
    """The grids node_server::compute_fmm leaves: multipole nodes L (20) and
    L_c (RHO); leaves L0..L3 and, with a refined neighbour in the RHO solve,
    the P2M L_c; everything else zero."""
    b = tree
    Lo, Lco = oracle.batch(0.5, b.pool, b.items, rho=(solve == RHO), nthreads=4)
    L = np.zeros_like(Lo)
    Lc = np.zeros_like(Lco)
    for it in b.items:
        s = int(it["subgrid"])
        if int(it["kind"]) == KIND_LEAF:
            L[s, :4] = Lo[s, :4]
            nb = [int(g) for g in it["neighbors"] if g >= 0]
            if solve == RHO and any(b.pool.is_leaf[g] == 0 for g in nb):
                Lc[s] = Lco[s]
        else:
            L[s] = Lo[s]
            if solve == RHO:
                Lc[s] = Lco[s]
    return L, Lc


def scaled(a, ref):
    num = np.abs(a - ref).max(axis=(0, 2))
    den = np.abs(ref).max(axis=(0, 2))
    return np.where(den > 0, num / np.where(den > 0, den, 1), num)


@pytest.mark.parametrize("in_place", [True, False])
@pytest.mark.parametrize("solve", [RHO, DRHODT])
@pytest.mark.parametrize("max_subgrids,threads,in_flight", [(64, 8, 64), (4096, 16, 512)])
def test_aggregated_adapter_exact_matches_oracle(ctx, oracle, tree, solve, max_subgrids, threads, in_flight,
                                                 in_place):
    from octotiger_b200.otfmm import adapter_pass
    L, Lc, sec = adapter_pass(ctx, tree.pool, tree.items, solve, "fp64_exact", aggregate=True, threads=threads,
                              max_subgrids=max_subgrids, max_items=max_subgrids // 2, passes=2, in_place=in_place,
                              calls_in_flight=in_flight)
    Le, Lce = expected(tree, oracle, solve)
    np.testing.assert_array_equal(L, Le)
    np.testing.assert_array_equal(Lc, Lce)
    assert (sec > 0).all()


@pytest.mark.parametrize("max_subgrids,in_flight", [(64, 16), (4096, 512)])
def test_aggregated_adapter_polling(ctx, oracle, tree, max_subgrids, in_flight):
    """Threads poll their calls (otfmm_octotiger::ready) and yield instead of
    blocking in finish(); a poll runs a batch that is ready to run."""
    from octotiger_b200.otfmm import adapter_pass
    L, Lc, _ = adapter_pass(ctx, tree.pool, tree.items, RHO, "fp64_exact", aggregate=True, threads=8,
                            max_subgrids=max_subgrids, max_items=max_subgrids // 2, passes=2,
                            calls_in_flight=in_flight, poll=True)
    Le, Lce = expected(tree, oracle, RHO)
    np.testing.assert_array_equal(L, Le)
    np.testing.assert_array_equal(Lc, Lce)


def test_aggregated_adapter_fast_and_split(ctx, oracle, tree):
    from octotiger_b200.otfmm import adapter_pass
    Le, Lce = expected(tree, oracle, RHO)
    L, Lc, _ = adapter_pass(ctx, tree.pool, tree.items, RHO, "fp64", threads=8, max_subgrids=256, max_items=128)
    assert scaled(L, Le).max() <= 1e-12 and scaled(Lc, Lce).max() <= 1e-12
    L, Lc, _ = adapter_pass(ctx, tree.pool, tree.items, RHO, "fp32_split", threads=8, max_subgrids=256,
                            max_items=128)
    e = scaled(L, Le)
    assert e[:4].max() <= 1e-6 and e[4:].max() <= 1e-5 and scaled(Lc, Lce).max() <= 1e-10


def test_per_call_adapter_matches_aggregated(ctx, oracle, tree):
    """The per-node host-buffer calls on the context, from several threads."""
    from octotiger_b200.otfmm import adapter_pass
    L, Lc, _ = adapter_pass(ctx, tree.pool, tree.items, RHO, "fp64_exact", aggregate=False, threads=4)
    Le, Lce = expected(tree, oracle, RHO)
    np.testing.assert_array_equal(L, Le)
    np.testing.assert_array_equal(Lc, Lce)


def test_aggregator_rejects_bad_arguments(ctx):
    import ctypes

    from octotiger_b200.otfmm import load_library
    lib = load_library()
    agg = ctypes.c_void_p()
    lib.otfmm_aggregator_create.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    assert lib.otfmm_aggregator_create(ctx.handle, 8, 4, 100, RHO, 1, ctypes.byref(agg)) == -1   # < 27 slots
    assert lib.otfmm_aggregator_create(ctx.handle, 64, 4, 100, 7, 1, ctypes.byref(agg)) == -1    # bad solve type
    assert lib.otfmm_aggregator_create(ctx.handle, 64, 4, 100, RHO, 1, ctypes.byref(agg)) == 0
    # AoS outputs with strides below a cell's components: the call is withdrawn
    # (its reservation ends, so the aggregator can be destroyed afterwards)
    from octotiger_b200.layout import WORK_ITEM_DTYPE
    lib.otfmm_aggregator_reserve.argtypes = [ctypes.c_void_p, ctypes.c_int32] + [ctypes.c_void_p] * 6
    lib.otfmm_aggregator_submit_aos.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32]
    keys = np.zeros(1, np.uint64)
    leaf = np.zeros(1, np.uint8)
    need = np.array([3], np.uint8)   # moments and centres of mass
    slots = np.zeros(1, np.int32)
    fill = np.zeros(1, np.uint8)
    cells = np.zeros(512 * 20)
    for l_stride, lc_stride in [(10, 3), (20, 2), (0, 3)]:
        ticket = ctypes.c_int64()
        assert lib.otfmm_aggregator_reserve(agg, 1, keys.ctypes.data, leaf.ctypes.data, need.ctypes.data,
                                            slots.ctypes.data, fill.ctypes.data, ctypes.byref(ticket)) == 0
        item = np.zeros(1, WORK_ITEM_DTYPE)
        item["subgrid"] = slots[0]
        item["neighbors"] = -1
        item["dx"] = 1.0
        assert lib.otfmm_aggregator_submit_aos(agg, ticket, item.ctypes.data, cells.ctypes.data, l_stride,
                                               cells.ctypes.data, lc_stride) == -1
    lib.otfmm_aggregator_destroy.argtypes = [ctypes.c_void_p]
    assert lib.otfmm_aggregator_destroy(agg) == 0
