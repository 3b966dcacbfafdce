"""Adaptive-octree work lists: tree invariants (Octo-Tiger's refinement
rules) and oracle parity on a mixed M2L / root / P2P / P2M batch."""
from __future__ import annotations

import numpy as np
import pytest

from octotiger_b200 import amr
from octotiger_b200.layout import KIND_LEAF, KIND_M2L, KIND_M2L_ROOT, direction_offsets


def test_lane_emden_first_zero():
    xi, theta = amr.lane_emden(1.5)
    assert abs(xi[-1] - 3.65375) < 1e-4     # known first zero for n = 1.5
    assert theta[0] == 1.0 and np.all(np.diff(theta) <= 0)


def small_tree():
    poly = amr.Polytrope((0.5, 0.5, 0.5), 0.05)
    return amr.build_tree(poly, 5, rho_max=1.0)


def test_tree_invariants():
    levels, pos, ref = small_tree()
    nodes = {(int(l), *map(int, p)): bool(r) for l, p, r in zip(levels, pos, ref)}
    for (l, x, y, z), r in nodes.items():
        if l > 0:
            assert nodes.get((l - 1, x // 2, y // 2, z // 2)) is True, "parent must be refined"
        if r:
            # a refined node sees all 26 same-level neighbours inside the domain
            for d in range(26):
                o = direction_offsets(d)
                q = (x + o[0], y + o[1], z + o[2])
                if min(q) >= 0 and max(q) < 2 ** l:
                    assert (l, *q) in nodes, "refined node with a missing neighbour"
    assert max(levels) == 5 and (~ref).sum() > 0


def test_small_amr_batch_kinds():
    b = amr.polytrope_batch(radius=0.05, max_level=5)
    kinds = set(int(k) for k in b.items["kind"])
    assert kinds == {KIND_M2L, KIND_M2L_ROOT, KIND_LEAF}
    leaves = b.items[b.items["kind"] == KIND_LEAF]
    has_refined_nb = [any(nb >= 0 and not b.pool.is_leaf[nb] for nb in it["neighbors"]) for it in leaves]
    has_empty = [any(nb < 0 for nb in it["neighbors"]) for it in leaves]
    assert any(has_refined_nb) and any(has_empty)


@pytest.mark.parametrize("theta", [0.5, 0.34])
def test_small_amr_oracle_matches_reference_math(oracle, refmath, theta):
    """A ragged AMR work list (refined, root and leaf items, P2M at the
    refinement boundaries) at the default opening angle and at 0.34, whose
    partners reach two coarse cells."""
    b = amr.polytrope_batch(radius=0.05, max_level=5, theta=theta)
    for rho in (True, False):
        L, Lc = oracle.batch(theta, b.pool, b.items, rho=rho)
        L2, Lc2 = refmath.batch(theta, b.pool, b.items, rho=rho)
        np.testing.assert_array_equal(L, L2)
        np.testing.assert_array_equal(Lc, Lc2)
