"""Golden-vector cases: seeded inputs (regenerated, checked by checksum) and
the outputs the reference's own kernel arithmetic produced for them."""
from __future__ import annotations

import hashlib

from octotiger_b200 import synthetic as syn
from octotiger_b200.layout import DRHODT, RHO

# name -> (batch factory, theta, solve type)
CASES = {
    "c1_rho": (lambda: syn.single_subgrid(), 0.5, RHO),
    "c1_drhodt": (lambda: syn.single_subgrid(), 0.5, DRHODT),
    "c1_theta034_rho": (lambda: syn.single_subgrid(theta=0.34), 0.34, RHO),
    "root_rho": (lambda: syn.root_subgrid(), 0.5, RHO),
    "root_drhodt": (lambda: syn.root_subgrid(), 0.5, DRHODT),
    "mixed_rho": (lambda: syn.single_subgrid(leaf_dirs=(0, 4, 12, 13, 25), empty_dirs=(1, 7, 20)), 0.5, RHO),
    "leaf_rho": (lambda: syn.single_subgrid(leaf_centre=True, leaf_dirs=tuple(range(0, 26, 2)), empty_dirs=(5,)),
                 0.5, RHO),
    "leaf_drhodt": (lambda: syn.single_subgrid(leaf_centre=True, leaf_dirs=tuple(range(0, 26, 2)),
                                               empty_dirs=(5,)), 0.5, DRHODT),
}


def input_digest(batch) -> str:
    h = hashlib.sha256()
    for a in (batch.pool.M, batch.pool.com, batch.pool.mon, batch.pool.is_leaf, batch.items):
        h.update(a.tobytes())
    return h.hexdigest()


def tree_case():
    """A small polytrope octree (levels 0-4) for the tree-pass goldens."""
    from octotiger_b200 import amr
    return amr.polytrope_batch(radius=0.05, max_level=4, seed=81)
