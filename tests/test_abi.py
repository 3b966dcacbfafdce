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


def test_create_rejects_small_theta_without_gpu():
    """theta below 0.34 is rejected before any device call."""
    from octotiger_b200.otfmm import LIB_PATH, load_library
    if not LIB_PATH.exists():
        pytest.fail("libotfmm.so not built")
    lib = load_library()
    h = ctypes.c_void_p()
    assert lib.otfmm_create(0, 0.2, ctypes.byref(h)) == -2
    assert b"theta" in lib.otfmm_last_error()
