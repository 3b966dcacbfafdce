"""The C++ adapter's halo staging (include/otfmm_octotiger.hpp) on the CPU:
compressed neighbour payloads (the cells of grid::get_ilist_n_bnd(dir), as
grid::get_gravity_boundary packs remote neighbours) expand to the same
buffers as full-size payloads, left-out cells read as update_input's zeros,
and malformed lists are rejected (tests/cpp/staging_test.cpp). Also: which
grid cell types the aggregated calls write in place (flat_cells)."""
from __future__ import annotations

import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_compressed_payload_staging(tmp_path):
    exe = tmp_path / "staging_test"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", str(ROOT / "include"),
                    "-I", str(ROOT / "octotiger_b200" / "csrc"),
                    str(ROOT / "tests" / "cpp" / "staging_test.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "staging ok"
