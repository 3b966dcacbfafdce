"""CUDA-graph plans and kernel variants of the batched solve:
* a plan replays exactly the launches of otfmm_batch (bit-identical results);
* every variant the autotuner may choose stays within its precision's
  tolerance against the oracle (FP64 fast: 1e-12; FP32 split: 1e-6 potential
  and force, 1e-10 L_c);
* the autotuner returns one of the allowed variants and the context keeps it;
* invalid variants are rejected."""
from __future__ import annotations

import itertools

import numpy as np
import pytest

from octotiger_b200 import synthetic as syn
from octotiger_b200.layout import DRHODT, RHO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from octotiger_b200.otfmm import Context
    c = Context(0, 0.5)
    yield c
    c.close()


def amr_small():
    from octotiger_b200 import amr
    return amr.polytrope_batch(radius=0.05, max_level=5, seed=71)


def scaled(a, ref):
    num = np.abs(a - ref).max(axis=(0, 2))
    den = np.abs(ref).max(axis=(0, 2))
    return np.where(den > 0, num / np.where(den > 0, den, 1), num)


@pytest.mark.parametrize("precision", ["fp64_exact", "fp64", "fp32_split"])
@pytest.mark.parametrize("solve", [RHO, DRHODT])
def test_plan_replays_batch(ctx, precision, solve):
    import torch
    from octotiger_b200.otfmm import BatchSolver
    b = amr_small()
    s = BatchSolver(ctx, b.pool, b.items)
    s.run(solve, precision)
    L0, Lc0 = s.results()
    s.L.zero_()
    s.Lc.zero_()
    plan = s.plan(solve, precision)
    for _ in range(2):
        plan.launch()
    plan.status()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(s.L.cpu().numpy(), L0)
    np.testing.assert_array_equal(s.Lc.cpu().numpy(), Lc0)
    plan.close()


# (split M2L form, M2L chunk, P2P chunk, P2M lanes): the warp-specialised,
# single-role and packed forms with chunks 8 / 16, the fused form with 16
VARIANTS = (list(itertools.product([0, 1, 2], [8, 16], [16, 32], [4, 8, 16]))
            + list(itertools.product([3], [16], [16, 32], [4, 8])))
ALLOWED = list(itertools.product([0, 1, 2, 3], [8, 16], [16, 32], [4, 8, 16]))
P2P_FORMS = (0, 1)   # OTFMM_P2P_BOX, OTFMM_P2P_STENCIL
P2M_FORMS = (0, 1, 2)   # OTFMM_P2M_COARSE, OTFMM_P2M_LANES, OTFMM_P2M_OCTANT


@pytest.mark.parametrize("form,m2l_chunk,p2p_chunk,lanes", VARIANTS)
def test_every_variant_within_tolerance(ctx, oracle, form, m2l_chunk, p2p_chunk, lanes):
    from octotiger_b200.otfmm import BatchSolver, Tuning
    b = amr_small()
    Lo, Lco = oracle.batch(0.5, b.pool, b.items, rho=True)
    keep = ctx.get_tuning()
    try:
        ctx.set_tuning(Tuning(form, m2l_chunk, p2p_chunk, lanes, 0, 1))
        s = BatchSolver(ctx, b.pool, b.items)
        s.run(RHO, "fp32_split")
        L, Lc = s.results()
        e = scaled(L, Lo)
        assert e[:4].max() <= 1e-6 and e[4:].max() <= 1e-5, e
        assert scaled(Lc, Lco).max() <= 1e-10
        s.run(RHO, "fp64")
        L, Lc = s.results()
        assert scaled(L, Lo).max() <= 1e-12 and scaled(Lc, Lco).max() <= 1e-12
    finally:
        ctx.set_tuning(keep)


@pytest.mark.parametrize("solve", [RHO, DRHODT])
@pytest.mark.parametrize("theta", [0.5, 0.7])
@pytest.mark.parametrize("p2p_form,p2m_form", list(itertools.product(P2P_FORMS, P2M_FORMS)))
@pytest.mark.parametrize("precision,p2p_chunk", [("fp64", 32), ("fp32_split", 16), ("fp32_split", 32)])
def test_leaf_forms_within_tolerance(oracle, solve, theta, p2p_form, p2m_form, precision, p2p_chunk):
    """The leaf P2P and P2M forms, with the partner box full (theta = 0.5: every
    parity's stencil is its whole 6^3 box, one table of offsets) and partial
    (theta = 0.7: the coarse corners drop out, per-parity masked tables)."""
    from octotiger_b200.otfmm import BatchSolver, Context, Tuning
    b = amr_small()
    Lo, Lco = oracle.batch(theta, b.pool, b.items, rho=(solve == RHO))
    c = Context(0, theta)
    try:
        c.set_tuning(Tuning(0, 16, p2p_chunk, 8, p2p_form, p2m_form))
        s = BatchSolver(c, b.pool, b.items)
        s.run(solve, precision)
        L, Lc = s.results()
        e = scaled(L, Lo)
        if precision == "fp64":
            assert e.max() <= 1e-12 and scaled(Lc, Lco).max() <= 1e-12, e
        else:
            assert e[:4].max() <= 1e-6 and e[4:].max() <= 1e-5, e
            assert scaled(Lc, Lco).max() <= 1e-10
    finally:
        c.close()


@pytest.mark.parametrize("solve", [RHO, DRHODT])
@pytest.mark.parametrize("case", ["all_refined", "mixed"])
@pytest.mark.parametrize("precision", ["fp64", "fp32_split"])
def test_p2m_octant_form_against_oracle(oracle, solve, case, precision):
    """The octant P2M on a leaf whose 26 neighbours are all refined (every
    octant has its 3 faces, 3 edges and corner: the largest slab set), and on
    a leaf with leaf and empty neighbours mixed in; against the oracle and
    against the lane form."""
    from octotiger_b200.otfmm import BatchSolver, Context, Tuning
    b = (syn.single_subgrid(seed=95, leaf_centre=True) if case == "all_refined"
         else syn.single_subgrid(seed=96, leaf_centre=True, leaf_dirs=(0, 4, 12, 21), empty_dirs=(7, 25)))
    Lo, Lco = oracle.batch(0.5, b.pool, b.items, rho=(solve == RHO))
    c = Context(0, 0.5)
    try:
        got = {}
        for form in (1, 2):
            c.set_tuning(Tuning(3, 16, 32, 4, 0, form))
            s = BatchSolver(c, b.pool, b.items)
            s.run(solve, precision)
            got[form] = s.results()
        L, Lc = got[2]
        e = scaled(L, Lo)
        if precision == "fp64":
            assert e.max() <= 1e-12 and scaled(Lc, Lco).max() <= 1e-12, e
            assert scaled(L, got[1][0]).max() <= 1e-13
        else:
            assert e[:4].max() <= 1e-6, e
            assert scaled(Lc, Lco).max() <= 1e-10
        sub = int(b.items[0]["subgrid"])
        assert np.isfinite(L[sub, :4]).all() and (np.abs(L[sub, :4]) > 0).all()
        # the octant kernel ran (a fallback to the lane form would give its bits)
        assert not np.array_equal(L, got[1][0])
    finally:
        c.close()


def test_autotune_keeps_an_allowed_variant(ctx, oracle):
    from octotiger_b200.otfmm import BatchSolver
    b = amr_small()
    keep = ctx.get_tuning()
    try:
        s = BatchSolver(ctx, b.pool, b.items)
        t = s.autotune(RHO, "fp32_split", repeats=2)
        assert (t.split_m2l_form, t.split_m2l_chunk, t.split_p2p_chunk, t.p2m_lanes) in ALLOWED
        assert t.p2p_form in P2P_FORMS and t.p2m_form in P2M_FORMS
        got = ctx.get_tuning()
        assert got.as_dict() == t.as_dict()
        s.run(RHO, "fp32_split")
        L, Lc = s.results()
        Lo, Lco = oracle.batch(0.5, b.pool, b.items, rho=True)
        assert scaled(L, Lo)[:4].max() <= 1e-6 and scaled(Lc, Lco).max() <= 1e-10
    finally:
        ctx.set_tuning(keep)


def test_invalid_variants_rejected(ctx):
    from octotiger_b200.otfmm import OtfmmError, Tuning
    keep = ctx.get_tuning()
    for bad in (Tuning(4, 16, 32, 16), Tuning(0, 12, 32, 16), Tuning(0, 16, 8, 16), Tuning(0, 16, 32, 3),
                Tuning(0, 16, 32, 16, 2), Tuning(0, 16, 32, 16, 0, 3)):
        with pytest.raises(OtfmmError):
            ctx.set_tuning(bad)
    assert ctx.get_tuning().as_dict() == keep.as_dict()


def test_batch_profile_times_each_kernel_and_matches_batch(ctx):
    from octotiger_b200.otfmm import BatchSolver
    b = amr_small()
    s = BatchSolver(ctx, b.pool, b.items)
    s.run(RHO, "fp64")
    L0, Lc0 = s.results()
    ms = s.profile(RHO, "fp64")
    assert set(ms) == {"classify", "m2l", "p2p", "p2m"}
    assert all(v > 0.0 for v in ms.values()), ms
    L, Lc = s.results()
    np.testing.assert_array_equal(L, L0)
    np.testing.assert_array_equal(Lc, Lc0)


def _writes_lc(b):
    """Subgrids whose L_c a solve writes: the refined ones and the leaves with a
    refined neighbour."""
    w = b.pool.is_leaf == 0
    for it in b.items:
        nb = it["neighbors"][it["neighbors"] >= 0]
        if it["kind"] == 2 and (b.pool.is_leaf[nb] == 0).any():
            w[it["subgrid"]] = True
    return w


@pytest.mark.parametrize("precision", ["fp64_exact", "fp32_split"])
@pytest.mark.parametrize("pinned", [False, True, "inputs"])
def test_batch_host_matches_device_batch(ctx, precision, pinned):
    """otfmm_batch_host (chunked uploads, kernels and downloads) gives the
    device batch's results, zeros where the solve writes nothing, and leaves
    L[4..19] of leaf subgrids and L_c of leaves without a refined neighbour (no
    kernel writes them) as the caller set them:
    with pageable buffers (copy engines), page-locked ones (the SMs move the
    moments in and the outputs out) and page-locked inputs with pageable
    outputs."""
    import torch
    from octotiger_b200.otfmm import BatchSolver, order_work_list
    b = amr_small()
    s = BatchSolver(ctx, b.pool, b.items)
    s.run(RHO, precision)
    L0, Lc0 = s.results()
    n = b.pool.n
    items = order_work_list(b.items)
    if pinned:   # True or "inputs"
        arrs = {k: torch.from_numpy(getattr(b.pool, k)).pin_memory() for k in ("M", "com", "mon", "is_leaf")}
        it = torch.from_numpy(items.view(np.uint8).reshape(-1).copy()).pin_memory()
    else:
        arrs = {k: np.ascontiguousarray(getattr(b.pool, k)) for k in ("M", "com", "mon", "is_leaf")}
        it = items
    pinned = pinned is True
    if pinned:
        L = torch.full((n, 20, 512), np.nan, dtype=torch.float64).pin_memory()
        Lc = torch.full((n, 3, 512), np.nan, dtype=torch.float64).pin_memory()
    else:
        L = np.full((n, 20, 512), np.nan)
        Lc = np.full((n, 3, 512), np.nan)
    for _ in range(2):   # the second call reuses the context's buffers
        ctx.batch_host(arrs["M"], arrs["com"], arrs["mon"], arrs["is_leaf"], n, it, len(items), L, Lc, RHO,
                       precision)
        torch.cuda.synchronize()
        ctx.batch_status()
        Lh = L.numpy() if pinned else L
        Lch = Lc.numpy() if pinned else Lc
        leaf = b.pool.is_leaf == 1
        np.testing.assert_array_equal(Lh[~leaf], L0[~leaf])
        np.testing.assert_array_equal(Lh[leaf, :4], L0[leaf, :4])
        assert np.isnan(Lh[leaf, 4:]).all()
        writes_lc = _writes_lc(b)
        np.testing.assert_array_equal(Lch[writes_lc], Lc0[writes_lc])
        assert np.isnan(Lch[~writes_lc]).all()


@pytest.mark.parametrize("precision", ["fp64", "fp32_split"])
def test_host_plan_replays_batch_host(ctx, precision):
    """otfmm_plan_create_host: the host-buffer solve captured once replays
    with the results of the device batch (each launch reads the current host
    inputs); an otfmm_batch_host call afterwards invalidates it."""
    import torch
    from octotiger_b200.otfmm import BatchSolver, OtfmmError, order_work_list
    b = amr_small()
    s = BatchSolver(ctx, b.pool, b.items)
    s.run(RHO, precision)
    L0, Lc0 = s.results()
    n = b.pool.n
    items = order_work_list(b.items)
    arrs = {k: torch.from_numpy(getattr(b.pool, k)).pin_memory() for k in ("M", "com", "mon", "is_leaf")}
    it = torch.from_numpy(items.view(np.uint8).reshape(-1).copy()).pin_memory()
    L = torch.zeros((n, 20, 512), dtype=torch.float64).pin_memory()
    Lc = torch.zeros((n, 3, 512), dtype=torch.float64).pin_memory()
    plan = ctx.plan_host(arrs["M"], arrs["com"], arrs["mon"], arrs["is_leaf"], n, it, len(items), L, Lc, RHO,
                         precision)
    leaf = b.pool.is_leaf == 1
    for _ in range(2):
        L.fill_(np.nan)
        Lc.fill_(np.nan)
        L[torch.from_numpy(leaf)] = 0.0   # the caller zeroes L (leaves' L4..L19 are not written)
        Lc[torch.from_numpy(~_writes_lc(b))] = 0.0   # and L_c (only P2M writes a leaf's)
        plan.launch()
        torch.cuda.synchronize()
        plan.status()
        np.testing.assert_array_equal(L.numpy()[~leaf], L0[~leaf])
        np.testing.assert_array_equal(L.numpy()[leaf, :4], L0[leaf, :4])
        np.testing.assert_array_equal(Lc.numpy(), Lc0)
    ctx.batch_host(arrs["M"], arrs["com"], arrs["mon"], arrs["is_leaf"], n, it, len(items), L, Lc, RHO, precision)
    torch.cuda.synchronize()
    with pytest.raises(OtfmmError):
        plan.launch()
    plan.close()
