"""Octree description for the tree passes (upward M2M, downward L2L).

A tree node record (``TREE_NODE_DTYPE``, 48 bytes, the C struct
``otfmm_tree_node`` of include/otfmm.h) names a node's pool index, its
parent's pool index (-1 for the root), its octant in the parent
(x + 2 y + 4 z, geo::octant, octotiger/geometry.hpp:199-226), its cell size
and the centre of its inner cell (0,0,0). Records are ordered by level, root
first; ``level_start[l]`` is the first record of level l. The upward pass runs
the levels finest first (node_server::compute_fmm gathers the children's
multipoles before its own M2M, src/node_server.cpp:613-640), the downward pass
root first (src/node_server.cpp:756-786).
"""
from __future__ import annotations

import numpy as np

from .layout import INX

TREE_NODE_DTYPE = np.dtype([
    ("subgrid", np.int32),
    ("parent", np.int32),
    ("octant", np.int32),
    ("reserved", np.int32),
    ("dx", np.float64),
    ("xbase", np.float64, (3,)),
], align=True)
assert TREE_NODE_DTYPE.itemsize == 48


def tree_nodes(levels, positions) -> tuple[np.ndarray, np.ndarray]:
    """Tree records of nodes given by level and integer position (every
    ancestor of every node must be present). Returns (nodes, level_start)."""
    levels = np.asarray(levels, dtype=np.int64)
    positions = np.asarray(positions, dtype=np.int64).reshape(-1, 3)
    lookup = {(int(levels[i]), *map(int, positions[i])): i for i in range(len(levels))}
    order = np.lexsort((np.arange(len(levels)), levels))
    nodes = np.zeros(len(levels), dtype=TREE_NODE_DTYPE)
    for k, i in enumerate(order):
        lvl = int(levels[i])
        p = positions[i]
        dx = 1.0 / (INX * 2 ** lvl)
        nodes[k]["subgrid"] = i
        nodes[k]["dx"] = dx
        nodes[k]["xbase"] = p * INX * dx + 0.5 * dx
        if lvl == 0:
            nodes[k]["parent"] = -1
            nodes[k]["octant"] = 0
        else:
            key = (lvl - 1, *map(int, p // 2))
            if key not in lookup:
                raise ValueError(f"node {(lvl, *map(int, p))} has no parent in the tree")
            nodes[k]["parent"] = lookup[key]
            nodes[k]["octant"] = int((p[0] & 1) + 2 * (p[1] & 1) + 4 * (p[2] & 1))
    n_levels = int(levels.max()) + 1 if len(levels) else 0
    level_start = np.searchsorted(levels[order], np.arange(n_levels + 1)).astype(np.int32)
    return nodes, level_start


def batch_tree(batch) -> tuple[np.ndarray, np.ndarray]:
    """Tree records of a generated batch (synthetic / amr), which keeps the
    levels and positions of its nodes."""
    return tree_nodes(batch.levels, batch.positions)
