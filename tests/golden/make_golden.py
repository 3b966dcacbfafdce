"""Regenerates tests/golden/ref_kernels.npz from the reference's own kernel
arithmetic (oracle/_ref, built by oracle/build_ref.sh from the Octo-Tiger
source tree). Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))

from cases import CASES, input_digest  # noqa: E402
from oracle.pyoracle import RefMath  # noqa: E402
from octotiger_b200.layout import RHO  # noqa: E402


def main() -> None:
    ref = RefMath()
    out = {}
    commit = (ROOT / "oracle" / "_ref" / "REFERENCE_COMMIT")
    out["reference_commit"] = np.array(commit.read_text().strip() if commit.exists() else "unknown")
    out["simd_width"] = np.array(ref.simd_width())
    for name, (make, theta, solve) in CASES.items():
        b = make()
        L, Lc = ref.batch(theta, b.pool, b.items, rho=(solve == RHO), nthreads=4, simd=True)
        s = int(b.items[0]["subgrid"])
        out[f"{name}/L"] = L[s]
        out[f"{name}/Lc"] = Lc[s]
        out[f"{name}/digest"] = np.array(input_digest(b))
    np.savez_compressed(Path(__file__).resolve().parent / "ref_kernels.npz", **out)
    print("wrote", len(CASES), "cases")


if __name__ == "__main__":
    main()
