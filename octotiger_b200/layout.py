"""Data layouts shared by the host code, the C ABI and the tests.

Constants follow Octo-Tiger's interaction constants for GRIDDIM 8 and
theta_min 0.34 (octotiger/common_kernel/interaction_constants.hpp:173-214).

Two layouts exist:

* the reference's per-subgrid kernel buffers ("SoA" layout): monopoles
  ``mon[ENTRIES]``, multipoles ``M[20][ENTRIES + SOA_PADDING]`` and centres of
  mass ``com[3][ENTRIES + SOA_PADDING]`` over the 18^3 padded halo; outputs
  ``L[20][INNER_CELLS + SOA_PADDING]`` and ``L_c[3][INNER_CELLS + SOA_PADDING]``
  (octotiger/multipole_interactions/kernel/kokkos_kernel.hpp:953-958);
* the resident subgrid pool of the batched path: per subgrid
  ``M[20][512]``, ``com[3][512]``, ``mon[512]`` and one leaf flag, with a
  work list of :data:`WORK_ITEM_DTYPE` records.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

INX = 8
NCELL = INX ** 3                       # 512 inner cells
STENCIL_MAX = 5
STENCIL_INX = 2 * STENCIL_MAX + 1      # 11
FULL_STENCIL_SIZE = STENCIL_INX ** 3   # 1331
PADDED_STRIDE = INX + 2 * STENCIL_MAX  # 18
ENTRIES = PADDED_STRIDE ** 3           # 5832
SOA_PADDING = 19
COMPONENT_LENGTH = ENTRIES + SOA_PADDING            # 5851
COMPONENT_LENGTH_UNPADDED = NCELL + SOA_PADDING     # 531
THETA_MIN = 0.34

# gsolve_type (octotiger/defs.hpp): RHO carries the angular-momentum correction.
RHO = 0
DRHODT = 1

# Work-item kinds: what node_server::compute_fmm runs per subgrid
# (src/node_server.cpp:711-723).
KIND_M2L = 0        # refined node: multipole stencil sweep
KIND_M2L_ROOT = 1   # level-0 node: root stencil
KIND_LEAF = 2       # leaf node: P2P, plus P2M for refined neighbours

WORK_ITEM_DTYPE = np.dtype([
    ("subgrid", "<i4"),
    ("kind", "<i4"),
    ("neighbors", "<i4", (26,)),
    ("dx", "<f8"),
    ("xbase", "<f8", (3,)),
])
assert WORK_ITEM_DTYPE.itemsize == 144


def direction_offsets(d: int) -> tuple[int, int, int]:
    """Offsets of flat neighbour index ``d`` (0..25), geo::direction order
    (octotiger/geometry.hpp:111-122,181-186)."""
    r = d if d < 13 else d + 1
    return (r % 3 - 1, (r // 3) % 3 - 1, r // 9 - 1)


def direction_index(ox: int, oy: int, oz: int) -> int:
    """Inverse of :func:`direction_offsets`."""
    r = (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)
    if r == 13:
        raise ValueError("centre is not a direction")
    return r if r < 13 else r - 1


@dataclass
class SubgridPool:
    """Resident inputs of a batch: one record per subgrid."""

    M: np.ndarray        # [n, 20, 512] float64, raw multipoles about the cell COM
    com: np.ndarray      # [n, 3, 512] float64
    mon: np.ndarray      # [n, 512] float64, cell masses (leaf subgrids)
    is_leaf: np.ndarray  # [n] uint8

    @property
    def n(self) -> int:
        return int(self.M.shape[0])

    def validate(self) -> None:
        n = self.n
        if self.M.shape != (n, 20, NCELL) or self.com.shape != (n, 3, NCELL) or \
                self.mon.shape != (n, NCELL) or self.is_leaf.shape != (n,):
            raise ValueError("inconsistent subgrid pool shapes")
        for a, dt in ((self.M, np.float64), (self.com, np.float64), (self.mon, np.float64),
                      (self.is_leaf, np.uint8)):
            if a.dtype != dt or not a.flags.c_contiguous:
                raise ValueError("subgrid pool arrays must be C-contiguous with the documented dtypes")


def validate_work_list(items: np.ndarray, n_subgrids: int) -> None:
    if items.dtype != WORK_ITEM_DTYPE or not items.flags.c_contiguous:
        raise ValueError("work list must be a C-contiguous WORK_ITEM_DTYPE array")
    if len(items) == 0:
        return
    if (items["subgrid"] < 0).any() or (items["subgrid"] >= n_subgrids).any():
        raise ValueError("work item subgrid out of range")
    nb = items["neighbors"]
    if ((nb < -1) | (nb >= n_subgrids)).any():
        raise ValueError("neighbour id out of range")
    if not np.isin(items["kind"], (KIND_M2L, KIND_M2L_ROOT, KIND_LEAF)).all():
        raise ValueError("unknown work item kind")
    if (items["dx"] <= 0).any():
        raise ValueError("dx must be positive")
    if len(np.unique(items["subgrid"])) != len(items):
        raise ValueError("a subgrid appears in more than one work item")


def cell_flat(x: int, y: int, z: int) -> int:
    return x * INX * INX + y * INX + z
