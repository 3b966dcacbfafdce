"""Regenerates tests/golden/ref_tree.npz from the reference's own taylor<4>
shift operators (octotiger/taylor.hpp, src/taylor.cpp, compiled into
oracle/_ref by oracle/build_ref.sh): seeded shifts in both directions and the
upward pass of a small polytrope tree (root multipoles and coarse centres of
mass). Run from the repository root:  python tests/golden/make_golden_tree.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))

from cases import input_digest, tree_case  # noqa: E402
from oracle.pyoracle import RefMath  # noqa: E402
from octotiger_b200.tree import batch_tree  # noqa: E402


def main() -> None:
    ref = RefMath()
    rng = np.random.default_rng(20261203)
    A = rng.standard_normal((64, 20))
    X = rng.uniform(-1.0, 1.0, (64, 3))
    up = np.stack([ref.shift(A[i], X[i], False) for i in range(64)])
    down = np.stack([ref.shift(A[i], X[i], True) for i in range(64)])
    b = tree_case()
    nodes, ls = batch_tree(b)
    M, com, com1 = ref.upward(b.pool, nodes, ls, rho=True)
    root = int(nodes[0]["subgrid"])
    commit = ROOT / "oracle" / "_ref" / "REFERENCE_COMMIT"
    np.savez_compressed(Path(__file__).resolve().parent / "ref_tree.npz",
                        reference_commit=np.array(commit.read_text().strip() if commit.exists() else "unknown"),
                        shift_A=A, shift_X=X, shift_up=up, shift_down=down, digest=np.array(input_digest(b)),
                        root_M=M[root], root_com=com[root], root_com1=com1[root])
    print("wrote ref_tree.npz")


if __name__ == "__main__":
    main()
