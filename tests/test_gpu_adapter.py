"""The C++ drop-in adapter (include/otfmm_octotiger.hpp), driven like
node_server::compute_fmm drives the reference's interaction interfaces:
AoS inputs in, the grid's L / L_c after the call, against the oracle
(bit-identical for the exact form)."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from octotiger_b200 import synthetic as syn
from octotiger_b200.layout import DRHODT, KIND_LEAF, RHO

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def adapter_bin(tmp_path_factory):
    out = tmp_path_factory.mktemp("adapter") / "adapter_test"
    lib = ROOT / "octotiger_b200"
    cmd = ["g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"), "-I", str(ROOT / "octotiger_b200" / "csrc"),
           str(ROOT / "tests" / "cpp" / "adapter_test.cpp"),
           "-L", str(lib), "-lotfmm", f"-Wl,-rpath,{lib}", "-o", str(out)]
    subprocess.run(cmd, check=True)
    return out


def run_adapter(adapter_bin, tmp_path, b, solve, precision, mode=0, expect_rc=0):
    it = b.items[0]
    p = b.pool
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        np.array([p.n, it["kind"], solve, it["subgrid"]], np.int32).tofile(f)
        np.asarray(it["neighbors"], np.int32).tofile(f)
        np.array([it["dx"]], np.float64).tofile(f)
        np.asarray(it["xbase"], np.float64).tofile(f)
        p.M.tofile(f)
        p.com.tofile(f)
        p.mon.tofile(f)
        p.is_leaf.tofile(f)
    outp = tmp_path / "out.bin"
    r = subprocess.run([str(adapter_bin), str(inp), str(outp), str(precision), str(b.theta), str(mode)])
    assert r.returncode == expect_rc
    if expect_rc != 0:
        return None
    raw = np.fromfile(outp, np.float64)
    return raw[:512 * 20].reshape(512, 20).T, raw[512 * 20:].reshape(512, 3).T


CASES = {
    "refined_mixed": lambda: syn.single_subgrid(seed=71, leaf_dirs=(0, 9, 25), empty_dirs=(4,)),
    "root": lambda: syn.root_subgrid(seed=72),
    "leaf_p2m": lambda: syn.single_subgrid(seed=73, leaf_centre=True, leaf_dirs=tuple(range(0, 26, 3)),
                                           empty_dirs=(2,)),
}


@pytest.mark.parametrize("solve", [RHO, DRHODT])
@pytest.mark.parametrize("name", sorted(CASES))
def test_adapter_exact_matches_oracle(adapter_bin, tmp_path, oracle, name, solve):
    b = CASES[name]()
    L, Lc = run_adapter(adapter_bin, tmp_path, b, solve, 0)
    Lo, Lco = oracle.batch(b.theta, b.pool, b.items, rho=(solve == RHO))
    s = int(b.items[0]["subgrid"])
    ncomp = 4 if int(b.items[0]["kind"]) == KIND_LEAF else 20
    np.testing.assert_array_equal(L[:ncomp], Lo[s][:ncomp])
    if solve == RHO:
        np.testing.assert_array_equal(Lc, Lco[s])


NEIGHBOURED = ("refined_mixed", "leaf_p2m")


@pytest.mark.parametrize("solve", [RHO, DRHODT])
@pytest.mark.parametrize("name", NEIGHBOURED)
def test_adapter_compressed_payloads(adapter_bin, tmp_path, oracle, name, solve):
    """Remote neighbours' compressed payloads (grid::get_gravity_boundary packs
    the cells of grid::get_ilist_n_bnd(dir)) through the overloads that take the
    grid: the whole band listed gives the full-size result bit for bit; a list
    with cells left out gives the result of full payloads with those cells
    zeroed; without a grid the compressed payloads are rejected."""
    b = CASES[name]()
    full = run_adapter(adapter_bin, tmp_path, b, solve, 0, mode=0)
    whole = run_adapter(adapter_bin, tmp_path, b, solve, 0, mode=1)
    subset = run_adapter(adapter_bin, tmp_path, b, solve, 0, mode=2)
    zeroed = run_adapter(adapter_bin, tmp_path, b, solve, 0, mode=3)
    for a, c in zip(whole, full):
        np.testing.assert_array_equal(a, c)
    for a, c in zip(subset, zeroed):
        np.testing.assert_array_equal(a, c)
    assert not np.array_equal(subset[0], full[0])
    run_adapter(adapter_bin, tmp_path, b, solve, 0, mode=4, expect_rc=7)
