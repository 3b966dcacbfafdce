"""Opening angle below 0.5 (theta = 0.34, coarse reach 2, the reference's
production setting of its rotating-star runs): the plane-streaming kernels
against the oracle. Exact form bit-identical, fast form within 1e-12; the
FP32-split form (fused split tiles in the RHO solve, FP32 P2P, the fast FP64
form for the d(rho)/dt tiles and P2M) within 1e-6 on the potential and force, 1e-5 on
L4..L19 and 1e-10 on L_c, also on the full-size AMR polytrope."""
from __future__ import annotations

import numpy as np
import pytest

from octotiger_b200 import synthetic as syn
from octotiger_b200.layout import COMPONENT_LENGTH_UNPADDED, DRHODT, NCELL, RHO

pytestmark = pytest.mark.gpu

THETA = 0.34


@pytest.fixture(scope="module")
def ctx34():
    from octotiger_b200.otfmm import Context
    c = Context(0, THETA)
    yield c
    c.close()


def scaled(a, ref):
    axes = (0, 2)
    num = np.abs(a - ref).max(axis=axes)
    den = np.abs(ref).max(axis=axes)
    return np.where(den > 0, num / np.where(den > 0, den, 1), num)


CASES = {
    "single": lambda: syn.single_subgrid(seed=91, theta=THETA),
    "root": lambda: syn.root_subgrid(seed=92, theta=THETA),
    "mixed": lambda: syn.single_subgrid(seed=93, theta=THETA, leaf_dirs=(0, 4, 12, 13, 25), empty_dirs=(1, 7, 20)),
    "leaf": lambda: syn.single_subgrid(seed=94, theta=THETA, leaf_centre=True, leaf_dirs=tuple(range(0, 26, 2)),
                                       empty_dirs=(5,)),
    "amr_small": lambda: __import__("octotiger_b200.amr", fromlist=["amr"]).polytrope_batch(
        radius=0.05, max_level=5, seed=95, theta=THETA),
}


@pytest.mark.parametrize("solve", [RHO, DRHODT])
@pytest.mark.parametrize("name", sorted(CASES))
def test_batch_theta034(ctx34, oracle, name, solve):
    from octotiger_b200.otfmm import BatchSolver
    b = CASES[name]()
    s = BatchSolver(ctx34, b.pool, b.items)
    Lo, Lco = oracle.batch(THETA, b.pool, b.items, rho=(solve == RHO))
    sel = b.items["subgrid"]
    s.run(solve, "fp64_exact")
    L, Lc = s.results()
    np.testing.assert_array_equal(L[sel], Lo[sel])
    np.testing.assert_array_equal(Lc[sel], Lco[sel])
    s.run(solve, "fp64")
    L, Lc = s.results()
    assert scaled(L[sel], Lo[sel]).max() <= 1e-12
    if np.abs(Lco[sel]).max() > 0:
        assert scaled(Lc[sel], Lco[sel]).max() <= 1e-12
    check_split(s, solve, sel, Lo, Lco)


def check_split(s, solve, sel, Lo, Lco):
    s.run(solve, "fp32_split")
    L, Lc = s.results()
    e = scaled(L[sel], Lo[sel])
    assert e[:4].max() <= 1e-6 and e[4:].max() <= 1e-5, e
    if np.abs(Lco[sel]).max() > 0:
        assert scaled(Lc[sel], Lco[sel]).max() <= 1e-10


def test_amr_polytrope_full_size_theta034(ctx34, oracle):
    import os

    from octotiger_b200 import amr
    from octotiger_b200.otfmm import BatchSolver
    b = amr.polytrope_batch(theta=THETA)
    Lo, Lco = oracle.batch(THETA, b.pool, b.items, rho=True, nthreads=os.cpu_count() or 1)
    s = BatchSolver(ctx34, b.pool, b.items)
    check_split(s, RHO, b.items["subgrid"], Lo, Lco)


@pytest.mark.parametrize("precision", ["fp64_exact", "fp64"])
@pytest.mark.parametrize("solve", [RHO, DRHODT])
def test_soa_entry_point_theta034(ctx34, oracle, precision, solve):
    import torch
    b = syn.single_subgrid(seed=96, theta=THETA, leaf_dirs=(2, 17), empty_dirs=(9,))
    mon, M, com = oracle.stage_m2l(b.pool, b.items[0])
    Lo, Lco = oracle.m2l_soa(THETA, mon, M, com, rho=(solve == RHO), root=False)
    d = torch.device("cuda", 0)
    tm, tM, tc = (torch.from_numpy(x).to(d) for x in (mon, M, com))
    L = torch.zeros(20 * COMPONENT_LENGTH_UNPADDED, dtype=torch.float64, device=d)
    Lc = torch.zeros(3 * COMPONENT_LENGTH_UNPADDED, dtype=torch.float64, device=d)
    ctx34.m2l_soa(tm, tM, tc, L, Lc, solve, False, precision)
    torch.cuda.synchronize()
    Lh = L.cpu().numpy().reshape(20, -1)[:, :NCELL]
    Lo = Lo.reshape(20, -1)[:, :NCELL]
    if precision == "fp64_exact":
        np.testing.assert_array_equal(Lh, Lo)
    else:
        err = np.abs(Lh - Lo).max(axis=1) / np.abs(Lo).max(axis=1)
        assert err.max() <= 1e-12


def test_pair_count_theta034(ctx34, oracle):
    b = CASES["amr_small"]()
    tot, per = ctx34.count_pairs(b.pool.is_leaf, b.items)
    tot_o, per_o = oracle.count_pairs(THETA, b.pool, b.items)
    assert tot == tot_o and list(per) == list(per_o)
