"""Physics pin of a whole gravity solve (upward M2M, interactions, downward
L2L with the gravity output) on the oracle: a uniform sphere's potential and
acceleration against the analytic ones (measured at max level 4: phi 1.5e-3
max / 5.2e-4 L1, g 1.6e-2 max; phi's L1 error 1.8e-4 one level finer)."""
from __future__ import annotations

from octotiger_b200.layout import SubgridPool
from octotiger_b200.tree import batch_tree

from sphere_case import analytic_errors, sphere_batch


def test_uniform_sphere_against_analytic(oracle):
    b = sphere_batch(max_level=4)
    nodes, ls = batch_tree(b)
    M, com, com1 = oracle.upward(b.pool, nodes, ls, rho=True)
    pool = SubgridPool(M=M, com=com, mon=b.pool.mon, is_leaf=b.pool.is_leaf)
    L, Lc = oracle.batch(0.5, pool, b.items, rho=True)
    L, Lc, G = oracle.downward(com, pool.is_leaf, com1, nodes, ls, L, Lc, gconst=1.0, correct_am=True, rho=True)
    e_phi, l1_phi, e_g = analytic_errors(pool, com, G)
    assert e_phi < 3e-3 and l1_phi < 1e-3 and e_g < 3e-2, (e_phi, l1_phi, e_g)
