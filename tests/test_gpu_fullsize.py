"""GPU solves of the full-size AMR work lists against the oracle.

* the ragged AMR batch: an n = 1.5 polytrope refined to levels 3-6 (4,809
  subgrids; multipole, P2P and P2M items in one solve);
* the uneven binary: two polytropes (mass ratio 0.7, separation 3 radii)
  refined to level 7 (21,865 subgrids).

Bars, per output component relative to its largest magnitude over the batch:
the exact FP64 form bit-identical, the fast FP64 form <= 1e-12, the FP32-split
form <= 1e-6 on the potential and the force, <= 1e-5 on L4..L19 and <= 1e-10
on L_c. Also cells of zero mass: the non-finite values the reference's
arithmetic gives for L_c there (it divides by the target's mass) appear in the
same places in every form, and the finite values meet the same bars.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from octotiger_b200 import amr
from octotiger_b200 import synthetic as syn
from octotiger_b200.layout import DRHODT, RHO

pytestmark = pytest.mark.gpu

NTHREADS = os.cpu_count() or 1


@pytest.fixture(scope="module")
def ctx():
    from octotiger_b200.otfmm import Context
    c = Context(0, 0.5)
    yield c
    c.close()


def scaled_err(a, ref):
    """max |a - ref| / max |ref| per component over the batch ([n, comp, cells])."""
    num = np.abs(a - ref).max(axis=(0, 2))
    den = np.abs(ref).max(axis=(0, 2))
    return np.where(den > 0, num / np.where(den > 0, den, 1), num)


def check(L, Lc, Lo, Lco, precision, solve):
    if precision == "fp64_exact":
        np.testing.assert_array_equal(L, Lo)
        np.testing.assert_array_equal(Lc, Lco)
        return
    e = scaled_err(L, Lo)
    if precision == "fp64":
        assert e.max() <= 1e-12, e
        if solve == RHO:
            assert scaled_err(Lc, Lco).max() <= 1e-12
        return
    assert e[0] <= 1e-6 and e[1:4].max() <= 1e-6, e
    assert e[4:].max() <= 1e-5, e
    if solve == RHO:
        assert scaled_err(Lc, Lco).max() <= 1e-10


@pytest.fixture(scope="module")
def polytrope():
    return amr.polytrope_batch()


@pytest.fixture(scope="module")
def binary():
    return amr.binary_batch()


def _solve_all(ctx, b, solve, precisions):
    from octotiger_b200.otfmm import BatchSolver
    s = BatchSolver(ctx, b.pool, b.items)
    out = {}
    for p in precisions:
        s.run(solve, p)
        out[p] = s.results()
    del s
    return out


@pytest.mark.parametrize("solve", [RHO, DRHODT])
def test_amr_polytrope_full_size(ctx, oracle, polytrope, solve):
    b = polytrope
    assert b.pool.n > 4000 and (b.pool.is_leaf == 1).sum() > 3000
    Lo, Lco = oracle.batch(0.5, b.pool, b.items, rho=(solve == RHO), nthreads=NTHREADS)
    got = _solve_all(ctx, b, solve, ["fp64_exact", "fp64", "fp32_split"])
    for p, (L, Lc) in got.items():
        check(L, Lc, Lo, Lco, p, solve)


def test_amr_binary_full_size(ctx, oracle, binary):
    b = binary
    assert b.pool.n > 20000
    Lo, Lco = oracle.batch(0.5, b.pool, b.items, rho=True, nthreads=NTHREADS)
    got = _solve_all(ctx, b, RHO, ["fp64_exact", "fp64", "fp32_split"])
    for p, (L, Lc) in got.items():
        check(L, Lc, Lo, Lco, p, RHO)


def test_amr_polytrope_graph_plan_matches_oracle(ctx, oracle, polytrope):
    """The production path of a solve: autotuned variants captured in a CUDA
    graph (otfmm_plan), replayed twice."""
    from octotiger_b200.otfmm import BatchSolver
    b = polytrope
    Lo, Lco = oracle.batch(0.5, b.pool, b.items, rho=True, nthreads=NTHREADS)
    s = BatchSolver(ctx, b.pool, b.items)
    s.autotune(RHO, "fp32_split", repeats=1)
    plan = s.plan(RHO, "fp32_split")
    for _ in range(2):
        s.L.zero_()
        s.Lc.zero_()
        plan.launch()
        plan.status()
        L, Lc = s.results()
        check(L, Lc, Lo, Lco, "fp32_split", RHO)
    plan.close()


@pytest.mark.parametrize("precision", ["fp64_exact", "fp64", "fp32_split"])
def test_zero_mass_cells(ctx, oracle, precision):
    """Massless cells in a refined target, in a refined neighbour and in a leaf
    target: same non-finite places as the oracle (the reference's arithmetic),
    finite values within the form's bars."""
    for b, mutate in ((syn.single_subgrid(seed=17), "refined"),
                      (syn.single_subgrid(seed=18, leaf_centre=True, leaf_dirs=tuple(range(0, 26, 3))), "leaf")):
        s = int(b.items[0]["subgrid"])
        cells = [0, 77, 300, 511]
        if mutate == "refined":
            b.pool.M[s][:, cells] = 0.0
            nb = int(b.items[0]["neighbors"][4])
            b.pool.M[nb][:, [5, 6, 7]] = 0.0
        else:
            b.pool.mon[s][cells] = 0.0
            b.pool.M[s][:, cells] = 0.0
        for solve in (RHO, DRHODT):
            Lo, Lco = oracle.batch(0.5, b.pool, b.items, rho=(solve == RHO), nthreads=2)
            (L, Lc), = _solve_all(ctx, b, solve, [precision]).values()
            sel = [s]
            L, Lc, Lo, Lco = L[sel], Lc[sel], Lo[sel], Lco[sel]
            np.testing.assert_array_equal(np.isfinite(L), np.isfinite(Lo))
            np.testing.assert_array_equal(np.isfinite(Lc), np.isfinite(Lco))
            if mutate == "refined" and solve == RHO:
                assert not np.isfinite(Lco).all()
            fin, finc = np.isfinite(Lo), np.isfinite(Lco)
            check(np.where(fin, L, 0.0), np.where(finc, Lc, 0.0), np.where(fin, Lo, 0.0), np.where(finc, Lco, 0.0),
                  precision, solve)
