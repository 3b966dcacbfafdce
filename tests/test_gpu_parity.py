"""GPU kernels (through the C ABI) against the oracle on the same seeded inputs.

* OTFMM_FP64_EXACT: bit-for-bit equal to the oracle (which is bit-for-bit the
  reference's own kernel arithmetic, tests/test_oracle.py);
* OTFMM_FP64: within 1e-12 of the oracle, per output component relative to that
  component's largest magnitude over the batch (L components cross zero).
"""
from __future__ import annotations

import numpy as np
import pytest

from octotiger_b200 import synthetic as syn
from octotiger_b200.layout import COMPONENT_LENGTH_UNPADDED, DRHODT, NCELL, RHO

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


@pytest.fixture(scope="module")
def ctx():
    from octotiger_b200.otfmm import Context
    c = Context(0, 0.5)
    yield c
    c.close()


def scaled_err(a, ref):
    """max |a - ref| / max |ref| per leading component axis."""
    a = np.asarray(a)
    ref = np.asarray(ref)
    axes = tuple(i for i in range(ref.ndim) if i != ref.ndim - 2) if ref.ndim >= 2 else None
    num = np.abs(a - ref).max(axis=axes)
    den = np.abs(ref).max(axis=axes)
    return np.where(den > 0, num / np.where(den > 0, den, 1), num)


def run_batch(ctx, b, solve, precision):
    from octotiger_b200.otfmm import BatchSolver
    s = BatchSolver(ctx, b.pool, b.items)
    s.run(solve, precision)
    return s.results()


CASES = {
    "single": lambda: syn.single_subgrid(seed=21),
    "root": lambda: syn.root_subgrid(seed=22),
    "mixed": lambda: syn.single_subgrid(seed=23, leaf_dirs=(0, 4, 12, 13, 25), empty_dirs=(1, 7, 20)),
    "leaf": lambda: syn.single_subgrid(seed=24, leaf_centre=True, leaf_dirs=tuple(range(0, 26, 2)),
                                       empty_dirs=(5,)),
    "leaf_all_refined": lambda: syn.single_subgrid(seed=25, leaf_centre=True),
    "leaf_only_leaves": lambda: syn.single_subgrid(seed=26, leaf_centre=True, leaf_dirs=tuple(range(26))),
    "uniform_level2": lambda: syn.uniform_level(2, seed=27),
    "amr_small": lambda: __import__("octotiger_b200.amr", fromlist=["amr"]).polytrope_batch(radius=0.05, max_level=5,
                                                                                             seed=28),
}


@pytest.mark.parametrize("solve", [RHO, DRHODT])
@pytest.mark.parametrize("name", sorted(CASES))
def test_batch_exact_is_bit_identical(ctx, oracle, name, solve):
    b = CASES[name]()
    L, Lc = run_batch(ctx, b, solve, "fp64_exact")
    Lo, Lco = oracle.batch(0.5, b.pool, b.items, rho=(solve == RHO))
    sel = b.items["subgrid"]
    np.testing.assert_array_equal(L[sel], Lo[sel])
    np.testing.assert_array_equal(Lc[sel], Lco[sel])


@pytest.mark.parametrize("solve", [RHO, DRHODT])
@pytest.mark.parametrize("name", sorted(CASES))
def test_batch_fast_fp64_within_1e12(ctx, oracle, name, solve):
    b = CASES[name]()
    L, Lc = run_batch(ctx, b, solve, "fp64")
    Lo, Lco = oracle.batch(0.5, b.pool, b.items, rho=(solve == RHO))
    sel = b.items["subgrid"]
    assert scaled_err(L[sel], Lo[sel]).max() <= FP64_TOL
    if solve == RHO:
        assert scaled_err(Lc[sel], Lco[sel]).max() <= FP64_TOL
    else:
        assert not Lc[sel].any()


def test_uniform_level3_full_size_fast(ctx, oracle):
    """The 512-subgrid batch (64^3 cells) at full size."""
    b = syn.uniform_level(3)
    L, Lc = run_batch(ctx, b, RHO, "fp64")
    Lo, Lco = oracle.batch(0.5, b.pool, b.items, rho=True)
    assert scaled_err(L, Lo).max() <= FP64_TOL
    assert scaled_err(Lc, Lco).max() <= FP64_TOL


@pytest.mark.parametrize("precision", ["fp64_exact", "fp64"])
@pytest.mark.parametrize("root", [False, True])
@pytest.mark.parametrize("solve", [RHO, DRHODT])
def test_soa_entry_points(ctx, oracle, precision, root, solve):
    import torch
    b = syn.root_subgrid(seed=31) if root else syn.single_subgrid(seed=31, leaf_dirs=(2, 17), empty_dirs=(9,))
    mon, M, com = oracle.stage_m2l(b.pool, b.items[0])
    Lo, Lco = oracle.m2l_soa(0.5, mon, M, com, rho=(solve == RHO), root=root)
    d = torch.device("cuda", 0)
    tm, tM, tc = (torch.from_numpy(x).to(d) for x in (mon, M, com))
    L = torch.zeros(20 * COMPONENT_LENGTH_UNPADDED, dtype=torch.float64, device=d)
    Lc = torch.zeros(3 * COMPONENT_LENGTH_UNPADDED, dtype=torch.float64, device=d)
    ctx.m2l_soa(tm, tM, tc, L, Lc, solve, root, precision)
    torch.cuda.synchronize()
    Lh = L.cpu().numpy().reshape(20, -1)[:, :NCELL]
    Lch = Lc.cpu().numpy().reshape(3, -1)[:, :NCELL]
    Lo = Lo.reshape(20, -1)[:, :NCELL]
    Lco = Lco.reshape(3, -1)[:, :NCELL]
    if precision == "fp64_exact":
        np.testing.assert_array_equal(Lh, Lo)
        if solve == RHO:
            np.testing.assert_array_equal(Lch, Lco)
    else:
        assert scaled_err(Lh, Lo).max() <= FP64_TOL
        if solve == RHO:
            assert scaled_err(Lch, Lco).max() <= FP64_TOL
    # host-buffer variant of the same call
    Lh2, Lch2 = ctx.m2l_soa_host(None if root else mon, M, com, solve, root, precision)
    np.testing.assert_array_equal(Lh2.reshape(20, -1)[:, :NCELL], Lh)
    if solve == RHO:
        np.testing.assert_array_equal(Lch2.reshape(3, -1)[:, :NCELL], Lch)


@pytest.mark.parametrize("precision", ["fp64_exact", "fp64"])
@pytest.mark.parametrize("solve", [RHO, DRHODT])
def test_p2p_p2m_soa_entry_points(ctx, oracle, precision, solve):
    import torch
    b = syn.single_subgrid(seed=41, leaf_centre=True, leaf_dirs=(0, 1, 2, 13, 24))
    mon = oracle.stage_p2p(b.pool, b.items[0])
    dx = float(b.items[0]["dx"])
    L4o = oracle.p2p_soa(0.5, mon, dx)
    d = torch.device("cuda", 0)
    L4 = torch.zeros(4 * COMPONENT_LENGTH_UNPADDED, dtype=torch.float64, device=d)
    ctx.p2p_soa(torch.from_numpy(mon).to(d), dx, L4, precision)
    torch.cuda.synchronize()
    got = L4.cpu().numpy().reshape(4, -1)[:, :NCELL]
    exp = L4o.reshape(4, -1)[:, :NCELL]
    if precision == "fp64_exact":
        np.testing.assert_array_equal(got, exp)
    else:
        assert scaled_err(got, exp).max() <= FP64_TOL
    icom = np.zeros(3 * COMPONENT_LENGTH_UNPADDED)
    icom.reshape(3, -1)[:, :NCELL] = b.pool.com[0]
    Lco = np.zeros(3 * COMPONENT_LENGTH_UNPADDED)
    Lc = torch.zeros(3 * COMPONENT_LENGTH_UNPADDED, dtype=torch.float64, device=d)
    ticom = torch.from_numpy(icom).to(d)
    first = True
    for dd in range(26):
        nb = int(b.items[0]["neighbors"][dd])
        if nb < 0 or b.pool.is_leaf[nb]:
            continue
        nM, ncom, stride = oracle.stage_p2m(b.pool, nb, dd)
        oracle.p2m_dir(0.5, dd, nM, ncom, stride, icom, L4o, Lco, rho=(solve == RHO), reset=first)
        ctx.p2m_soa(dd, torch.from_numpy(nM).to(d), torch.from_numpy(ncom).to(d), ticom, L4, Lc, solve, first,
                    precision)
        first = False
    torch.cuda.synchronize()
    got = L4.cpu().numpy().reshape(4, -1)[:, :NCELL]
    exp = L4o.reshape(4, -1)[:, :NCELL]
    gotc = Lc.cpu().numpy().reshape(3, -1)[:, :NCELL]
    expc = Lco.reshape(3, -1)[:, :NCELL]
    if precision == "fp64_exact":
        np.testing.assert_array_equal(got, exp)
        if solve == RHO:
            np.testing.assert_array_equal(gotc, expc)
    else:
        assert scaled_err(got, exp).max() <= FP64_TOL
        if solve == RHO:
            assert scaled_err(gotc, expc).max() <= FP64_TOL


def test_device_rejects_bad_work_item(ctx):
    """A neighbour id outside the pool is caught by the kernel's own checks
    (no access is made with it) and reported as OTFMM_ERR_DEVICE."""
    import torch
    from octotiger_b200.otfmm import DevicePool, OtfmmError
    b = syn.single_subgrid(seed=51)
    dev = DevicePool.upload(b.pool)
    items = b.items.copy()
    items[0]["neighbors"][3] = b.pool.n + 100
    raw = torch.from_numpy(items.view(np.uint8).reshape(-1).copy()).cuda()
    L = torch.full((b.pool.n, 20, NCELL), 7.0, dtype=torch.float64, device="cuda")
    Lc = torch.zeros((b.pool.n, 3, NCELL), dtype=torch.float64, device="cuda")
    ctx.batch(dev, raw, 1, L, Lc, RHO, "fp64")
    with pytest.raises(OtfmmError) as e:
        ctx.batch_status()
    assert e.value.code == -4
    assert bool((L == 7.0).all())   # outputs of the rejected item untouched
    # the context stays usable
    good = torch.from_numpy(b.items.view(np.uint8).reshape(-1).copy()).cuda()
    ctx.batch(dev, good, 1, L, Lc, RHO, "fp64")
    ctx.batch_status()


def test_empty_work_list(ctx, oracle):
    """No work items: the device and host-buffer batched calls return at once
    and write nothing; the next non-empty solve is unaffected."""
    import torch
    from octotiger_b200.otfmm import DevicePool
    b = syn.single_subgrid(seed=52)
    dev = DevicePool.upload(b.pool)
    raw = torch.from_numpy(b.items.view(np.uint8).reshape(-1).copy()).cuda()
    L = torch.full((b.pool.n, 20, NCELL), 7.0, dtype=torch.float64, device="cuda")
    Lc = torch.full((b.pool.n, 3, NCELL), 7.0, dtype=torch.float64, device="cuda")
    for precision in ("fp64_exact", "fp64", "fp32_split"):
        ctx.batch(dev, raw, 0, L, Lc, RHO, precision)
        ctx.batch_status()
    assert bool((L == 7.0).all()) and bool((Lc == 7.0).all())
    Lh = np.full((b.pool.n, 20, NCELL), 7.0)
    Lch = np.full((b.pool.n, 3, NCELL), 7.0)
    ctx.batch_host(b.pool.M, b.pool.com, b.pool.mon, b.pool.is_leaf, b.pool.n, b.items, 0, Lh, Lch, RHO,
                   "fp32_split")
    ctx.batch_status()
    assert (Lh == 7.0).all() and (Lch == 7.0).all()
    # the same context then solves the item as usual (bit-identical to the oracle)
    Lo, Lco = oracle.batch(0.5, b.pool, b.items, rho=True)
    L.zero_()
    Lc.zero_()
    ctx.batch(dev, raw, 1, L, Lc, RHO, "fp64_exact")
    ctx.batch_status()
    s = int(b.items[0]["subgrid"])
    np.testing.assert_array_equal(L.cpu().numpy()[s], Lo[s])
    np.testing.assert_array_equal(Lc.cpu().numpy()[s], Lco[s])


def test_fma_peaks_measurable():
    from octotiger_b200.otfmm import measure_fma_peaks
    f64, f32 = measure_fma_peaks(0)
    assert 5.0 < f64 < 200.0 and 10.0 < f32 < 400.0


def split_errors(L, Lc, Lo, Lco):
    """Scaled max error per group: potential L0, force L1..3, higher L4..19, L_c."""
    e = scaled_err(L, Lo)
    out = {"L0": float(e[0]), "force": float(e[1:4].max()), "higher": float(e[4:].max())}
    out["Lc"] = float(scaled_err(Lc, Lco).max()) if np.abs(Lco).max() > 0 else 0.0
    return out


SPLIT_CASES = ["single", "mixed", "uniform_level2", "leaf", "amr_small"]


@pytest.mark.parametrize("solve", [RHO, DRHODT])
@pytest.mark.parametrize("name", SPLIT_CASES)
def test_batch_fp32_split_accuracy(ctx, oracle, name, solve):
    """FP32 split form: <= 1e-6 on potential and force, <= 1e-10 on L_c
    (which stays FP64), per component relative to its largest magnitude."""
    b = CASES[name]()
    L, Lc = run_batch(ctx, b, solve, "fp32_split")
    Lo, Lco = oracle.batch(0.5, b.pool, b.items, rho=(solve == RHO))
    sel = b.items["subgrid"]
    err = split_errors(L[sel], Lc[sel], Lo[sel], Lco[sel])
    assert err["L0"] <= 1e-6 and err["force"] <= 1e-6, err
    assert err["higher"] <= 1e-5, err
    assert err["Lc"] <= 1e-10, err


def test_fp32_split_full_size_accuracy(ctx, oracle):
    b = syn.uniform_level(3)
    L, Lc = run_batch(ctx, b, RHO, "fp32_split")
    Lo, Lco = oracle.batch(0.5, b.pool, b.items, rho=True)
    err = split_errors(L, Lc, Lo, Lco)
    assert err["L0"] <= 1e-6 and err["force"] <= 1e-6 and err["Lc"] <= 1e-10, err


@pytest.mark.parametrize("name", sorted(CASES))
def test_library_pair_count_matches_oracle(ctx, oracle, name):
    b = CASES[name]()
    tot, per = ctx.count_pairs(b.pool.is_leaf, b.items)
    tot_o, per_o = oracle.count_pairs(0.5, b.pool, b.items)
    assert tot == tot_o and list(per) == list(per_o)


@pytest.mark.parametrize("theta", [0.7, 1.0])
@pytest.mark.parametrize("solve", [RHO, DRHODT])
@pytest.mark.parametrize("name", ["mixed", "amr_small"])
def test_other_opening_angles(oracle, theta, solve, name):
    """Opening angles above 0.5 (smaller multipole stencils, larger P2P boxes
    relative to them): exact form bit-identical, fast form within 1e-12,
    FP32-split form within its bars, against the oracle at the same theta."""
    from octotiger_b200.otfmm import BatchSolver, Context
    b = CASES[name]()
    Lo, Lco = oracle.batch(theta, b.pool, b.items, rho=(solve == RHO))
    sel = b.items["subgrid"]
    c = Context(0, theta)
    try:
        s = BatchSolver(c, b.pool, b.items)
        s.run(solve, "fp64_exact")
        L, Lc = s.results()
        np.testing.assert_array_equal(L[sel], Lo[sel])
        np.testing.assert_array_equal(Lc[sel], Lco[sel])
        s.run(solve, "fp64")
        L, Lc = s.results()
        assert scaled_err(L[sel], Lo[sel]).max() <= FP64_TOL
        s.run(solve, "fp32_split")
        L, Lc = s.results()
        e = scaled_err(L[sel], Lo[sel])
        assert e[:4].max() <= 1e-6 and e[4:].max() <= 1e-5, e
        if solve == RHO:
            assert scaled_err(Lc[sel], Lco[sel]).max() <= 1e-10
    finally:
        c.close()
