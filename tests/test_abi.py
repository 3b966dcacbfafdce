"""The C-ABI library loads and exports every entry point include/otfmm.h
declares; host-side validation rejects malformed inputs before any launch.
No GPU compute is called here."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from octotiger_b200 import synthetic as syn
from octotiger_b200.layout import WORK_ITEM_DTYPE, validate_work_list

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols() -> list[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        names.update(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(otfmm_\w+)\s*\(", text, re.M))
    return sorted(names)


def test_library_exports_declared_symbols():
    from octotiger_b200.otfmm import LIB_PATH, load_library
    if not LIB_PATH.exists():
        pytest.fail("libotfmm.so not built (run python -m octotiger_b200.build)")
    lib = load_library()
    names = declared_symbols()
    assert "otfmm_batch" in names and "otfmm_m2l_soa" in names
    for n in names:
        assert hasattr(lib, n), n


def test_work_item_layout_matches_header():
    assert WORK_ITEM_DTYPE.itemsize == 144
    assert WORK_ITEM_DTYPE.fields["dx"][1] == 112
    assert WORK_ITEM_DTYPE.fields["xbase"][1] == 120


def test_work_list_validation_rejects_bad_items():
    b = syn.single_subgrid()
    validate_work_list(b.items, b.pool.n)
    bad = b.items.copy()
    bad[0]["neighbors"][0] = b.pool.n
    with pytest.raises(ValueError):
        validate_work_list(bad, b.pool.n)
    bad = b.items.copy()
    bad[0]["kind"] = 7
    with pytest.raises(ValueError):
        validate_work_list(bad, b.pool.n)
    bad = b.items.copy()
    bad[0]["dx"] = 0.0
    with pytest.raises(ValueError):
        validate_work_list(bad, b.pool.n)
    dup = np.concatenate([b.items, b.items])
    with pytest.raises(ValueError):
        validate_work_list(dup, b.pool.n)


def test_work_list_order_puts_multipole_items_first():
    """order_work_list: refined and root items before leaves, each group in
    its input order, every item kept once."""
    from octotiger_b200 import amr
    from octotiger_b200.otfmm import order_work_list
    b = amr.polytrope_batch(max_level=4)
    items = b.items[::-1].copy()   # leaves and multipole items interleaved differently
    out = order_work_list(items)
    assert len(out) == len(items) and out.flags["C_CONTIGUOUS"]
    kinds = out["kind"]
    n_multi = int((items["kind"] != 2).sum())
    assert (kinds[:n_multi] != 2).all() and (kinds[n_multi:] == 2).all()
    for group in (items[items["kind"] != 2], items[items["kind"] == 2]):
        got = out[np.isin(out["subgrid"], group["subgrid"])]
        np.testing.assert_array_equal(got["subgrid"], group["subgrid"])
    assert sorted(out["subgrid"].tolist()) == sorted(items["subgrid"].tolist())


def test_create_rejects_small_theta_without_gpu():
    """theta below 0.34 is rejected before any device call."""
    from octotiger_b200.otfmm import LIB_PATH, load_library
    if not LIB_PATH.exists():
        pytest.fail("libotfmm.so not built")
    lib = load_library()
    h = ctypes.c_void_p()
    assert lib.otfmm_create(0, 0.2, ctypes.byref(h)) == -2
    assert b"theta" in lib.otfmm_last_error()


def test_entry_points_reject_missing_context_without_gpu():
    """Every entry point that takes a context refuses a NULL one (and NULL
    buffers) with OTFMM_ERR_INVALID before any device call."""
    from octotiger_b200.otfmm import LIB_PATH, Tuning, load_library
    if not LIB_PATH.exists():
        pytest.fail("libotfmm.so not built")
    lib = load_library()
    null = None
    inv = -1
    assert lib.otfmm_batch(null, null, null, null, null, 1, null, 1, null, null, 0, 1, null) == inv
    assert lib.otfmm_batch_host(null, null, null, null, null, 1, null, 1, null, null, 0, 1, null) == inv
    assert lib.otfmm_batch_profile(null, null, null, null, null, 1, null, 1, null, null, 0, 1, null, null) == inv
    assert lib.otfmm_autotune(null, null, null, null, null, 1, null, 1, null, null, 0, 1, 3, null, null) == inv
    plan = ctypes.c_void_p()
    assert lib.otfmm_plan_create(null, null, null, null, null, 1, null, 1, null, null, 0, 1,
                                 ctypes.byref(plan)) == inv
    assert lib.otfmm_plan_launch(null, null) == inv
    assert lib.otfmm_plan_destroy(null) == 0
    t = Tuning()
    assert lib.otfmm_get_tuning(null, ctypes.byref(t)) == inv
    assert lib.otfmm_set_tuning(null, ctypes.byref(t)) == inv
    ls = (ctypes.c_int32 * 2)(0, 1)
    assert lib.otfmm_upward(null, null, null, null, null, null, 1, null, ls, 1, 0, null) == inv
    assert lib.otfmm_downward(null, null, null, null, 1, null, ls, 1, null, null, null, 1.0, 1, 0, null) == inv
    stride = ctypes.c_int32()
    assert lib.otfmm_stage_soa(null, null, null, null, null, 1, null, null, null, null, null) == inv
    assert lib.otfmm_stage_p2m_soa(null, null, null, 1, 0, 0, null, null, ctypes.byref(stride), null) == inv
    assert lib.otfmm_m2l_soa_host_noalloc(null, 1, null, null, null, null, null, 0, 0, 1, null) == inv
    assert lib.otfmm_destroy(null) == 0
    assert lib.otfmm_last_error() != b""


def test_tree_records_reject_missing_parent():
    from octotiger_b200.tree import tree_nodes
    with pytest.raises(ValueError):
        tree_nodes([0, 2], [[0, 0, 0], [1, 1, 1]])
    nodes, ls = tree_nodes([0, 1, 1], [[0, 0, 0], [1, 0, 0], [0, 1, 1]])
    assert list(ls) == [0, 1, 3]
    assert list(nodes["parent"]) == [0 - 1, 0, 0] and sorted(nodes["octant"][1:]) == [1, 6]


def test_struct_layouts_match_header(tmp_path):
    """Sizes and field offsets of the C structs of include/otfmm.h, from a
    probe compiled against the header, equal the Python side's (numpy dtypes
    of the work item and tree node, ctypes otfmm_tuning)."""
    import subprocess
    from octotiger_b200.otfmm import Tuning
    from octotiger_b200.tree import TREE_NODE_DTYPE
    src = tmp_path / "layout_probe.c"
    src.write_text(r"""
#include <stddef.h>
#include <stdio.h>
#include "otfmm.h"
#define F(T, f) printf(#T " " #f " %zu\n", offsetof(T, f))
int main(void) {
    printf("otfmm_work_item size %zu\n", sizeof(otfmm_work_item));
    F(otfmm_work_item, subgrid); F(otfmm_work_item, kind); F(otfmm_work_item, neighbors);
    F(otfmm_work_item, dx); F(otfmm_work_item, xbase);
    printf("otfmm_tree_node size %zu\n", sizeof(otfmm_tree_node));
    F(otfmm_tree_node, subgrid); F(otfmm_tree_node, parent); F(otfmm_tree_node, octant);
    F(otfmm_tree_node, dx); F(otfmm_tree_node, xbase);
    printf("otfmm_tuning size %zu\n", sizeof(otfmm_tuning));
    F(otfmm_tuning, split_m2l_form); F(otfmm_tuning, split_m2l_chunk); F(otfmm_tuning, split_p2p_chunk);
    F(otfmm_tuning, p2m_lanes); F(otfmm_tuning, p2p_form); F(otfmm_tuning, p2m_form);
    return 0;
}
""")
    exe = tmp_path / "layout_probe"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        t, f, v = line.split()
        got[(t, f)] = int(v)
    for t, dt in (("otfmm_work_item", WORK_ITEM_DTYPE), ("otfmm_tree_node", TREE_NODE_DTYPE)):
        assert got[(t, "size")] == dt.itemsize, t
        for f in ("subgrid", "dx", "xbase") + (("kind", "neighbors") if t == "otfmm_work_item" else ("parent", "octant")):
            assert got[(t, f)] == dt.fields[f][1], (t, f)
    assert got[("otfmm_tuning", "size")] == ctypes.sizeof(Tuning)
    for name, _ in Tuning._fields_:
        assert got[("otfmm_tuning", name)] == getattr(Tuning, name).offset, name
