"""Device tree passes (otfmm_upward / otfmm_downward) against the oracle
(tests/test_tree_oracle.py pins the oracle to the reference's taylor<4>):
bit-identical, since both use the reference's operation order in FP64; and a
whole device gravity solve (upward, batched interactions, downward) against
the oracle's: bit-identical with the exact interaction form, within the fast
and split tolerances otherwise."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

from octotiger_b200.layout import DRHODT, RHO, SubgridPool
from octotiger_b200.tree import batch_tree

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from cases import tree_case  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from octotiger_b200.otfmm import Context
    c = Context(0, 0.5)
    yield c
    c.close()


@pytest.fixture(scope="module")
def tree():
    b = tree_case()
    nodes, ls = batch_tree(b)
    return b, nodes, ls


def _dev(ctx, b, nodes):
    import torch
    from octotiger_b200.otfmm import DevicePool
    dev = DevicePool.upload(b.pool, 0)
    d = torch.device("cuda", 0)
    nd = torch.from_numpy(np.ascontiguousarray(nodes).view(np.uint8).reshape(-1).copy()).to(d)
    com1 = torch.zeros((b.pool.n, 3, 64), dtype=torch.float64, device=d)
    return dev, nd, com1


def test_upward_bit_identical(ctx, oracle, tree):
    import torch
    b, nodes, ls = tree
    dev, nd, com1 = _dev(ctx, b, nodes)
    ctx.upward(dev, com1, nd, ls, RHO)
    torch.cuda.synchronize()
    ctx.batch_status()
    M, com, c1 = oracle.upward(b.pool, nodes, ls, rho=True)
    np.testing.assert_array_equal(dev.M.cpu().numpy(), M)
    np.testing.assert_array_equal(dev.com.cpu().numpy(), com)
    np.testing.assert_array_equal(com1.cpu().numpy(), c1)
    # d(rho)/dt pass on the same tree: new masses, the RHO pass's centres of mass
    rng = np.random.default_rng(13)
    mon2 = b.pool.mon * rng.uniform(-1.0, 1.0, b.pool.mon.shape)
    dev.mon.copy_(torch.from_numpy(mon2))
    ctx.upward(dev, com1, nd, ls, DRHODT)
    torch.cuda.synchronize()
    p2 = SubgridPool(M=M, com=com, mon=mon2, is_leaf=b.pool.is_leaf)
    M2, com2, c12 = oracle.upward(p2, nodes, ls, rho=False, com1=c1)
    np.testing.assert_array_equal(dev.M.cpu().numpy(), M2)
    np.testing.assert_array_equal(dev.com.cpu().numpy(), com2)
    np.testing.assert_array_equal(com1.cpu().numpy(), c12)


@pytest.mark.parametrize("solve", [RHO, DRHODT])
def test_downward_bit_identical(ctx, oracle, tree, solve):
    import torch
    b, nodes, ls = tree
    dev, nd, com1 = _dev(ctx, b, nodes)
    ctx.upward(dev, com1, nd, ls, RHO)
    rng = np.random.default_rng(17)
    L = rng.standard_normal((b.pool.n, 20, 512))
    Lc = rng.standard_normal((b.pool.n, 3, 512))
    d = torch.device("cuda", 0)
    tL, tLc = torch.from_numpy(L).to(d), torch.from_numpy(Lc).to(d)
    G = torch.zeros((b.pool.n, 4, 512), dtype=torch.float64, device=d)
    ctx.downward(dev, com1, nd, ls, tL, tLc, G, 0.7, True, solve)
    torch.cuda.synchronize()
    ctx.batch_status()
    eL, eLc, eG = oracle.downward(dev.com.cpu().numpy(), b.pool.is_leaf, com1.cpu().numpy(), nodes, ls, L, Lc,
                                  gconst=0.7, correct_am=True, rho=(solve == RHO))
    np.testing.assert_array_equal(tL.cpu().numpy(), eL)
    np.testing.assert_array_equal(tLc.cpu().numpy(), eLc)
    np.testing.assert_array_equal(G.cpu().numpy(), eG)


@pytest.mark.parametrize("precision", ["fp64_exact", "fp64", "fp32_split"])
def test_whole_gravity_solve(ctx, oracle, tree, precision):
    from octotiger_b200.otfmm import GravitySolver
    b, nodes, ls = tree
    gs = GravitySolver(ctx, b.pool, b.items, nodes, ls, gconst=1.0, correct_am_grav=True)
    gs.run(RHO, precision)
    L, Lc, G = gs.results()
    M, com, c1 = oracle.upward(b.pool, nodes, ls, rho=True)
    pool = SubgridPool(M=M, com=com, mon=b.pool.mon, is_leaf=b.pool.is_leaf)
    Lo, Lco = oracle.batch(b.theta, pool, b.items, rho=True)
    eL, eLc, eG = oracle.downward(com, pool.is_leaf, c1, nodes, ls, Lo, Lco, gconst=1.0, correct_am=True, rho=True)
    leaf = b.pool.is_leaf == 1
    if precision == "fp64_exact":
        np.testing.assert_array_equal(G, eG)
        np.testing.assert_array_equal(L, eL)
        return
    tol_phi, tol_g = (1e-12, 1e-12) if precision == "fp64" else (1e-6, 1e-6)
    err_phi = np.abs(G[leaf, 0] - eG[leaf, 0]).max() / np.abs(eG[leaf, 0]).max()
    err_g = np.abs(G[leaf, 1:] - eG[leaf, 1:]).max() / np.abs(eG[leaf, 1:]).max()
    assert err_phi <= tol_phi and err_g <= tol_g, (err_phi, err_g)


@pytest.mark.parametrize("precision", ["fp64_exact", "fp64", "fp32_split"])
def test_device_solve_of_uniform_sphere(ctx, oracle, precision):
    """The whole device solve of a uniform sphere (the analogue of the
    reference's `sphere` gravity scenario): its potential and acceleration
    against the analytic ones within the bounds the oracle meets, and equal to
    the oracle's solve with the exact form."""
    from octotiger_b200.otfmm import GravitySolver
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    from sphere_case import analytic_errors, sphere_batch
    b = sphere_batch(max_level=4)
    nodes, ls = batch_tree(b)
    gs = GravitySolver(ctx, b.pool, b.items, nodes, ls, gconst=1.0, correct_am_grav=True)
    gs.run(RHO, precision)
    L, Lc, G = gs.results()
    M, com, c1 = oracle.upward(b.pool, nodes, ls, rho=True)
    e_phi, l1_phi, e_g = analytic_errors(SubgridPool(M=M, com=com, mon=b.pool.mon, is_leaf=b.pool.is_leaf), com, G)
    assert e_phi < 3e-3 and l1_phi < 1e-3 and e_g < 3e-2, (e_phi, l1_phi, e_g)
    if precision == "fp64_exact":
        pool = SubgridPool(M=M, com=com, mon=b.pool.mon, is_leaf=b.pool.is_leaf)
        Lo, Lco = oracle.batch(b.theta, pool, b.items, rho=True)
        _, _, eG = oracle.downward(com, pool.is_leaf, c1, nodes, ls, Lo, Lco, gconst=1.0, correct_am=True, rho=True)
        np.testing.assert_array_equal(G, eG)
