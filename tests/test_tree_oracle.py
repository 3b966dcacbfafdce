"""Oracle of the tree passes (upward M2M, downward L2L) on the CPU:
* pinned bit for bit to the reference's own taylor<4> shift operators
  (oracle/_ref, built from octotiger/taylor.hpp and src/taylor.cpp) and to the
  committed golden vectors they produced (tests/golden/ref_tree.npz);
* physics: the upward pass conserves mass and centre of mass; a whole solve
  (upward, interactions, downward) gives the potential and acceleration of a
  direct sum over the leaf cells within the order-3 truncation error."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

from octotiger_b200.layout import DRHODT, RHO
from octotiger_b200.tree import TREE_NODE_DTYPE, batch_tree

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
from cases import input_digest, tree_case  # noqa: E402


@pytest.fixture(scope="module")
def tree():
    b = tree_case()
    nodes, ls = batch_tree(b)
    return b, nodes, ls


def test_tree_records(tree):
    b, nodes, ls = tree
    assert nodes.dtype == TREE_NODE_DTYPE and TREE_NODE_DTYPE.itemsize == 48
    assert ls[0] == 0 and ls[-1] == len(nodes) and nodes[0]["parent"] == -1
    lvl = b.levels[nodes["subgrid"]]
    assert np.all(np.diff(lvl) >= 0)
    for nd in nodes[1:]:
        assert b.pool.is_leaf[nd["parent"]] == 0
        assert b.levels[nd["parent"]] == b.levels[nd["subgrid"]] - 1


def test_shift_matches_golden(oracle):
    g = np.load(GOLDEN / "ref_tree.npz")
    for i in range(len(g["shift_A"])):
        assert np.array_equal(oracle.shift(g["shift_A"][i], g["shift_X"][i], False), g["shift_up"][i])
        assert np.array_equal(oracle.shift(g["shift_A"][i], g["shift_X"][i], True), g["shift_down"][i])


def test_shift_matches_reference_taylor(oracle, refmath):
    rng = np.random.default_rng(5)
    for _ in range(200):
        A, X = rng.standard_normal(20), rng.standard_normal(3) * 10.0 ** rng.integers(-3, 2)
        for down in (False, True):
            assert np.array_equal(oracle.shift(A, X, down), refmath.shift(A, X, down))


def test_upward_matches_golden(oracle, tree):
    b, nodes, ls = tree
    g = np.load(GOLDEN / "ref_tree.npz")
    assert str(g["digest"]) == input_digest(b), "tree-case inputs changed: regenerate the goldens"
    M, com, com1 = oracle.upward(b.pool, nodes, ls, rho=True)
    root = int(nodes[0]["subgrid"])
    assert np.array_equal(M[root], g["root_M"])
    assert np.array_equal(com[root], g["root_com"])
    assert np.array_equal(com1[root], g["root_com1"])


@pytest.mark.parametrize("solve", [RHO, DRHODT])
def test_upward_matches_reference(oracle, refmath, tree, solve):
    b, nodes, ls = tree
    M, com, com1 = oracle.upward(b.pool, nodes, ls, rho=True)
    Mr, comr, com1r = refmath.upward(b.pool, nodes, ls, rho=True)
    assert np.array_equal(M, Mr) and np.array_equal(com, comr) and np.array_equal(com1, com1r)
    if solve == DRHODT:
        # d(rho)/dt pass: masses change, centres of mass are the RHO pass's
        from octotiger_b200.layout import SubgridPool
        rng = np.random.default_rng(9)
        p2 = SubgridPool(M=M, com=com, mon=b.pool.mon * rng.uniform(-1, 1, b.pool.mon.shape), is_leaf=b.pool.is_leaf)
        a = oracle.upward(p2, nodes, ls, rho=False, com1=com1)
        r = refmath.upward(p2, nodes, ls, rho=False, com1=com1)
        for x, y in zip(a, r):
            assert np.array_equal(x, y)


def test_downward_matches_reference(oracle, refmath, tree):
    b, nodes, ls = tree
    M, com, com1 = oracle.upward(b.pool, nodes, ls, rho=True)
    rng = np.random.default_rng(11)
    L = rng.standard_normal((b.pool.n, 20, 512))
    Lc = rng.standard_normal((b.pool.n, 3, 512))
    for rho in (True, False):
        a = oracle.downward(com, b.pool.is_leaf, com1, nodes, ls, L, Lc, gconst=1.3, correct_am=True, rho=rho)
        r = refmath.downward(com, b.pool.is_leaf, com1, nodes, ls, L, Lc, gconst=1.3, correct_am=True, rho=rho)
        for x, y in zip(a, r):
            assert np.array_equal(x, y)


def test_upward_conserves_mass_and_centre_of_mass(oracle, tree):
    b, nodes, ls = tree
    M, com, com1 = oracle.upward(b.pool, nodes, ls, rho=True)
    leaf = b.pool.is_leaf == 1
    m = b.pool.mon[leaf]
    x = com[leaf]
    root = int(nodes[0]["subgrid"])
    mtot = m.sum()
    assert abs(M[root][0].sum() - mtot) <= 1e-13 * mtot
    want = (x * m[:, None, :]).sum(axis=(0, 2)) / mtot
    got = (com[root] * M[root][0][None, :]).sum(axis=1) / M[root][0].sum()
    assert np.abs(got - want).max() <= 1e-13


def _solve_errors(oracle, theta):
    """Max errors (relative to the largest value) of phi and g of 400 leaf
    cells from upward + interactions + downward vs a direct sum over the leaf
    cells (masses at their cell centres), G = 1."""
    from octotiger_b200 import amr
    from octotiger_b200.layout import SubgridPool
    b = amr.polytrope_batch(radius=0.05, max_level=4, seed=81, theta=theta)
    nodes, ls = batch_tree(b)
    M, com, com1 = oracle.upward(b.pool, nodes, ls, rho=True)
    pool = SubgridPool(M=M, com=com, mon=b.pool.mon, is_leaf=b.pool.is_leaf)
    L, Lc = oracle.batch(theta, pool, b.items, rho=True)
    L, Lc, G = oracle.downward(com, pool.is_leaf, com1, nodes, ls, L, Lc, gconst=1.0, correct_am=True, rho=True)
    leaf = np.nonzero(pool.is_leaf == 1)[0]
    pos = com[leaf].transpose(0, 2, 1).reshape(-1, 3)
    mass = pool.mon[leaf].reshape(-1)
    pick = np.random.default_rng(3).choice(len(pos), 400, replace=False)
    phi = np.empty(len(pick))
    g = np.empty((len(pick), 3))
    pt = np.ascontiguousarray(pos.T)   # [3][N]
    d = np.empty((3, len(pos)))
    r2 = np.empty(len(pos))
    w = np.empty(len(pos))
    for t, c in enumerate(pick):   # one target at a time, buffers reused
        np.subtract(pos[c][:, None], pt, out=d)   # x_target - x_j
        np.einsum("kn,kn->n", d, d, out=r2)
        r2[c] = np.inf
        np.sqrt(r2, out=w)
        np.divide(mass, w, out=w)                 # m / r
        phi[t] = -w.sum()
        np.divide(w, r2, out=w)                   # m / r^3
        g[t] = -(d @ w)
    Gl = G[leaf].transpose(0, 2, 1).reshape(-1, 4)[pick]
    return np.abs(Gl[:, 0] - phi).max() / np.abs(phi).max(), np.abs(Gl[:, 1:] - g).max() / np.abs(g).max()


def test_whole_solve_against_direct_sum(oracle):
    """Order-3 FMM with the multipole acceptance of theta: the errors are the
    expansion's truncation error, so they are small and shrink with theta
    (measured: phi 7.1e-3 -> 6.2e-4, g 6.2e-2 -> 8.5e-3 from theta 0.5 to 0.34)."""
    p5, g5 = _solve_errors(oracle, 0.5)
    p3, g3 = _solve_errors(oracle, 0.34)
    assert p5 < 1e-2 and g5 < 1e-1, (p5, g5)
    assert p3 < p5 / 5 and g3 < g5 / 5, (p5, p3, g5, g3)
