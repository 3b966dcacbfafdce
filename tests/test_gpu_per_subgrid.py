"""Device-side halo staging (otfmm_stage_soa / otfmm_stage_p2m_soa) against the
oracle's restatement of update_input / update_neighbor_input (bit for bit), and
the per-subgrid call pattern (one entry-point call per node over a stream pool)
against the batched solve of the same work list."""
from __future__ import annotations

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


STAGE_CASES = {
    "mixed": lambda: syn.single_subgrid(seed=51, leaf_dirs=(0, 4, 12, 13, 25), empty_dirs=(1, 7, 20)),
    "root": lambda: syn.root_subgrid(seed=52),
    "leaf": lambda: syn.single_subgrid(seed=53, leaf_centre=True, leaf_dirs=tuple(range(0, 26, 3)), empty_dirs=(4,)),
}


@pytest.mark.parametrize("name", sorted(STAGE_CASES))
def test_device_staging_matches_oracle(ctx, oracle, name):
    import torch
    from octotiger_b200.layout import COMPONENT_LENGTH, ENTRIES
    from octotiger_b200.otfmm import P2M_SLAB_STRIDE_MAX, DevicePool
    b = STAGE_CASES[name]()
    dev = DevicePool.upload(b.pool, 0)
    d = torch.device("cuda", 0)
    item = b.items[0]
    mon = torch.full((ENTRIES,), np.nan, dtype=torch.float64, device=d)
    if int(item["kind"]) == 2:
        ctx.stage_soa(dev, item, mon)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(mon.cpu().numpy(), oracle.stage_p2p(b.pool, item))
        for dd in range(26):
            nb = int(item["neighbors"][dd])
            if nb < 0 or b.pool.is_leaf[nb]:
                continue
            nM = torch.full((20 * P2M_SLAB_STRIDE_MAX,), np.nan, dtype=torch.float64, device=d)
            nc = torch.full((3 * P2M_SLAB_STRIDE_MAX,), np.nan, dtype=torch.float64, device=d)
            stride = ctx.stage_p2m_soa(dev, nb, dd, nM, nc)
            torch.cuda.synchronize()
            eM, ec, es = oracle.stage_p2m(b.pool, nb, dd)
            assert stride == es
            np.testing.assert_array_equal(nM.cpu().numpy()[:20 * stride], eM[:20 * stride])
            np.testing.assert_array_equal(nc.cpu().numpy()[:3 * stride], ec[:3 * stride])
    else:
        M = torch.full((20 * COMPONENT_LENGTH,), np.nan, dtype=torch.float64, device=d)
        com = torch.full((3 * COMPONENT_LENGTH,), np.nan, dtype=torch.float64, device=d)
        ctx.stage_soa(dev, item, mon, M, com)
        torch.cuda.synchronize()
        emon, eM, ecom = oracle.stage_m2l(b.pool, item)
        np.testing.assert_array_equal(mon.cpu().numpy(), emon)
        np.testing.assert_array_equal(M.cpu().numpy(), eM)
        np.testing.assert_array_equal(com.cpu().numpy(), ecom)


@pytest.mark.parametrize("solve", [RHO, DRHODT])
def test_per_subgrid_calls_match_batched(ctx, solve):
    from octotiger_b200 import amr
    from octotiger_b200.otfmm import BatchSolver, PerSubgridSolver
    b = amr.polytrope_batch(radius=0.05, max_level=5, seed=61)
    batched = BatchSolver(ctx, b.pool, b.items)
    batched.run(solve, "fp64_exact")
    Lb, Lcb = batched.results()
    plain = PerSubgridSolver(ctx, b.pool, b.items, n_streams=8)
    plain.run(solve, "fp64_exact")
    L, Lc = plain.results()
    sub = b.items["subgrid"]
    leaf = b.items["kind"] == 2
    # refined nodes: all 20 L and L_c; leaves: L0..L3 (L_c where a neighbour is refined)
    np.testing.assert_array_equal(L[sub[~leaf]], Lb[sub[~leaf]])
    np.testing.assert_array_equal(L[sub[leaf], :4], Lb[sub[leaf], :4])
    if solve == RHO:
        np.testing.assert_array_equal(Lc[sub[~leaf]], Lcb[sub[~leaf]])
    has_p2m = np.array([len(x) > 0 for x in plain.p2m_by_leaf], dtype=bool)
    np.testing.assert_array_equal(Lc[sub[leaf][has_p2m]], Lcb[sub[leaf][has_p2m]])
