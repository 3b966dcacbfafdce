"""Pins the oracle (CPU restatement) before anything is checked against it.

* stencil sizes the reference's generators give (src/multipole_interactions/util/calculate_stencil.cpp);
* bit-for-bit equality with the committed golden vectors, which were produced by
  the reference's own kernel arithmetic (tests/golden/make_golden.py);
* bit-for-bit equality with the reference-math build itself, where present;
* physics: the order-3 potential/force against a direct sum over point masses,
  and the mass-weighted pairwise cancellation of the angular correction.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

from octotiger_b200 import synthetic as syn
from octotiger_b200.layout import COMPONENT_LENGTH_UNPADDED, NCELL, RHO, direction_offsets

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from cases import CASES, input_digest  # noqa: E402

GOLDEN = np.load(Path(__file__).resolve().parent / "golden" / "ref_kernels.npz")


def test_stencil_sizes(oracle):
    st = oracle.stencil(0.5)
    assert (st["n_mpole"], st["n_phase_one"], st["n_p2p"]) == (342, 316, 342)
    assert int(st["mpole_mask"].sum()) == 342
    assert int((st["mpole_mask"] & (st["mpole_phase"] == 0)).sum()) == 26
    st34 = oracle.stencil(0.34)
    assert st34["n_mpole"] == 1074


def test_pairs_per_subgrid(oracle):
    b = syn.single_subgrid()
    total, per = oracle.count_pairs(0.5, b.pool, b.items)
    assert per[0] == total
    assert total == 110080 == 215 * NCELL
    b34 = syn.single_subgrid(theta=0.34)
    assert oracle.count_pairs(0.34, b34.pool, b34.items)[0] == 743 * NCELL


def test_stencil_matches_reference_generators(oracle, refmath):
    for theta in (0.34, 0.5, 0.7, 1.0):
        a, b = oracle.stencil(theta), refmath.stencil(theta)
        for k in ("mpole_mask", "mpole_phase", "p2p_mask", "four"):
            assert np.array_equal(a[k], b[k]), (theta, k)


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_golden(oracle, name):
    make, theta, solve = CASES[name]
    b = make()
    assert input_digest(b) == str(GOLDEN[f"{name}/digest"]), "synthetic generator drifted from the fixtures"
    L, Lc = oracle.batch(theta, b.pool, b.items, rho=(solve == RHO), nthreads=2)
    s = int(b.items[0]["subgrid"])
    np.testing.assert_array_equal(L[s], GOLDEN[f"{name}/L"])
    np.testing.assert_array_equal(Lc[s], GOLDEN[f"{name}/Lc"])


@pytest.mark.parametrize("theta", [0.34, 0.5, 0.7, 1.0])
@pytest.mark.parametrize("simd", [False, True])
@pytest.mark.parametrize("rho", [True, False])
def test_oracle_matches_reference_math_soa(oracle, refmath, rho, simd, theta):
    """Every supported stencil: theta 0.34 (partners up to two coarse cells
    away), 0.5, and the smaller stencils of 0.7 and 1.0."""
    b = syn.single_subgrid(seed=7, leaf_dirs=(3, 9, 21), empty_dirs=(11,))
    mon, M, com = oracle.stage_m2l(b.pool, b.items[0])
    for root in (False, True):
        L, Lc = oracle.m2l_soa(theta, mon, M, com, rho=rho, root=root)
        L2, Lc2 = refmath.m2l_soa(theta, mon, M, com, rho=rho, root=root, simd=simd)
        np.testing.assert_array_equal(L, L2)
        np.testing.assert_array_equal(Lc, Lc2)
    bl = syn.single_subgrid(seed=8, leaf_centre=True, leaf_dirs=(0, 1, 2, 13, 24))
    mon = oracle.stage_p2p(bl.pool, bl.items[0])
    np.testing.assert_array_equal(oracle.p2p_soa(theta, mon, 1 / 64),
                                  refmath.p2p_soa(theta, mon, 1 / 64, simd=simd))
    icom = np.zeros(3 * COMPONENT_LENGTH_UNPADDED)
    icom.reshape(3, -1)[:, :NCELL] = bl.pool.com[0]
    for d in (3, 12, 25):   # refined neighbours of the leaf
        nb = int(bl.items[0]["neighbors"][d])
        nM, ncom, stride = oracle.stage_p2m(bl.pool, nb, d)
        outs = []
        for impl in (oracle, refmath):
            L4 = np.arange(4 * COMPONENT_LENGTH_UNPADDED, dtype=np.float64) * 1e-3
            Lc = np.zeros(3 * COMPONENT_LENGTH_UNPADDED)
            kw = {} if impl is oracle else {"simd": simd}
            impl.p2m_dir(theta, d, nM, ncom, stride, icom, L4, Lc, rho=rho, reset=True, **kw)
            outs.append((L4, Lc))
        np.testing.assert_array_equal(outs[0][0], outs[1][0])
        np.testing.assert_array_equal(outs[0][1], outs[1][1])


def test_oracle_matches_reference_math_uniform_batch(oracle, refmath):
    b = syn.uniform_level(2, seed=11)   # 64 subgrids, boundary subgrids included
    for rho in (True, False):
        L, Lc = oracle.batch(0.5, b.pool, b.items, rho=rho)
        L2, Lc2 = refmath.batch(0.5, b.pool, b.items, rho=rho)
        np.testing.assert_array_equal(L, L2)
        np.testing.assert_array_equal(Lc, Lc2)


def _point_mass_case(seed=5, spread=0.005):
    """Single subgrid whose multipoles come from explicit point masses."""
    b = syn.single_subgrid(seed=seed)
    rng = np.random.default_rng(seed)
    n = b.pool.n
    pts = np.zeros((n, NCELL, 4, 4))   # 4 point masses: (m, x, y, z)
    dx = 1 / 64
    for i in range(n):
        m = b.pool.M[i, 0]
        com = b.pool.com[i].T
        w = rng.uniform(0.5, 1.5, (NCELL, 4))
        w = w / w.sum(1, keepdims=True) * m[:, None]
        off = rng.uniform(-spread, spread, (NCELL, 4, 3)) * dx
        off -= (w[:, :, None] * off).sum(1)[:, None, :] / m[:, None, None]
        pts[i, :, :, 0] = w
        pts[i, :, :, 1:] = com[:, None, :] + off
        quad = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
        octs = [(0, 0, 0), (0, 0, 1), (0, 0, 2), (0, 1, 1), (0, 1, 2), (0, 2, 2), (1, 1, 1), (1, 1, 2),
                (1, 2, 2), (2, 2, 2)]
        Mi = np.zeros((NCELL, 20))
        Mi[:, 0] = m
        Mi[:, 1:4] = (w[:, :, None] * off).sum(1)
        for q, (a, c) in enumerate(quad):
            Mi[:, 4 + q] = (w * off[:, :, a] * off[:, :, c]).sum(1)
        for q, (a, c, e) in enumerate(octs):
            Mi[:, 10 + q] = (w * off[:, :, a] * off[:, :, c] * off[:, :, e]).sum(1)
        b.pool.M[i] = Mi.T
    return b, pts


def test_potential_and_force_against_direct_sum(oracle):
    b, pts = _point_mass_case()
    L, _ = oracle.batch(0.5, b.pool, b.items, rho=True)
    st = oracle.stencil(0.5)
    lookup = {}
    for d in range(26):
        lookup[direction_offsets(d)] = int(b.items[0]["neighbors"][d])
    lookup[(0, 0, 0)] = 0
    X = b.pool.com[0].T
    phi = np.zeros(NCELL)
    grad = np.zeros((NCELL, 3))
    for c in range(NCELL):
        cx, cy, cz = c // 64, (c // 8) % 8, c % 8
        for sx in range(-3, 4):
            for sy in range(-3, 4):
                for sz in range(-3, 4):
                    idx = (sx + 5) * 121 + (sy + 5) * 11 + (sz + 5)
                    if not st["mpole_mask"][idx] or not st["mpole_phase"][idx]:
                        continue
                    co = [(q + 8) // 2 - 4 for q in (cx + 8, cy + 8, cz + 8)]
                    pc = [(q + 8) // 2 - 4 for q in (cx + 8 + sx, cy + 8 + sy, cz + 8 + sz)]
                    if sum((a - e) ** 2 for a, e in zip(co, pc)) >= 4:
                        continue
                    p = (cx + sx, cy + sy, cz + sz)
                    key = tuple(q // 8 for q in p)
                    loc = tuple(q % 8 for q in p)
                    sub = lookup[key]
                    pp = pts[sub, loc[0] * 64 + loc[1] * 8 + loc[2]]
                    dvec = X[c][None, :] - pp[:, 1:]
                    r = np.sqrt((dvec ** 2).sum(1))
                    phi[c] += (-pp[:, 0] / r).sum()
                    grad[c] += (pp[:, 0][:, None] * dvec / r[:, None] ** 3).sum(0)
    s = int(b.items[0]["subgrid"])
    np.testing.assert_allclose(L[s, 0], phi, rtol=1e-6)
    for a in range(3):
        assert np.abs(L[s, 1 + a] - grad[:, a]).max() <= 1e-5 * np.abs(grad).max()


def test_angular_correction_cancels_pairwise(oracle):
    """On the root subgrid the interaction set is symmetric, and each pair's
    mass-weighted L_c contributions cancel, so sum_i m_i L_c,i vanishes."""
    b = syn.root_subgrid(seed=3)
    _, Lc = oracle.batch(0.5, b.pool, b.items, rho=True)
    m = b.pool.M[0, 0]
    weighted = m[None, :] * Lc[0]
    total = weighted.sum(axis=1)
    scale = np.abs(weighted).sum(axis=1)
    assert (np.abs(total) <= 1e-12 * scale).all(), (total, scale)


@pytest.mark.parametrize("rho", [True, False])
def test_zero_mass_cells_match_reference_math(oracle, refmath, rho):
    """Cells whose multipoles are all zero (a massless target and massless
    partners): the RHO correction divides by the target's mass, so the
    reference's arithmetic gives non-finite L_c there; the oracle reproduces
    every value, non-finite ones included, bit for bit."""
    b = syn.single_subgrid(seed=17)
    s = int(b.items[0]["subgrid"])
    cells = [0, 77, 300, 511]
    b.pool.M[s][:, cells] = 0.0
    nb = int(b.items[0]["neighbors"][4])
    b.pool.M[nb][:, [5, 6, 7]] = 0.0
    mon, M, com = oracle.stage_m2l(b.pool, b.items[0])
    L, Lc = oracle.m2l_soa(0.5, mon, M, com, rho=rho, root=False)
    L2, Lc2 = refmath.m2l_soa(0.5, mon, M, com, rho=rho, root=False, simd=False)
    np.testing.assert_array_equal(L, L2)
    np.testing.assert_array_equal(Lc, Lc2)
    if rho:
        assert not np.isfinite(Lc).all() and np.isfinite(L).all()
    Lb, Lcb = oracle.batch(0.5, b.pool, b.items, rho=rho, nthreads=2)
    Lb2, Lcb2 = refmath.batch(0.5, b.pool, b.items, rho=rho)
    np.testing.assert_array_equal(Lb, Lb2)
    np.testing.assert_array_equal(Lcb, Lcb2)
    # a leaf target with massless cells: P2P and the P2M of its refined neighbours
    bl = syn.single_subgrid(seed=18, leaf_centre=True, leaf_dirs=tuple(range(0, 26, 3)))
    sl = int(bl.items[0]["subgrid"])
    bl.pool.mon[sl][cells] = 0.0
    bl.pool.M[sl][:, cells] = 0.0
    Lb, Lcb = oracle.batch(0.5, bl.pool, bl.items, rho=rho, nthreads=2)
    Lb2, Lcb2 = refmath.batch(0.5, bl.pool, bl.items, rho=rho)
    np.testing.assert_array_equal(Lb, Lb2)
    np.testing.assert_array_equal(Lcb, Lcb2)
