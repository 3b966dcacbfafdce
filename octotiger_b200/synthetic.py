"""Seeded synthetic inputs for the FMM interaction kernels.

No dataset is involved: every workload is generated here from a seed.

* cell masses: log-uniform on [1e-3, 1] (single-subgrid case) or
  ``rho * dx^3`` from a density profile, floored at 1e-12 of the batch maximum
  (the RHO kernel divides by the target cell mass,
  octotiger/multipole_interactions/kernel/compute_kernel_templates.hpp:228);
* refined-node cells: centre of mass = cell centre + U[-0.4, 0.4] dx per axis;
  raw multipoles (octotiger/taylor.hpp:222-255 convention: sum m x_a x_b ...,
  no factorials) of 8 point masses with weights U[0.5, 1.5] normalised to the
  cell mass and offsets U[-0.1, 0.1] dx re-centred on the centre of mass;
* leaf-node cells: mass only, centre of mass = cell centre.

Subgrid ``level`` has ``dx = 1 / (8 * 2**level)`` in the unit domain.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .layout import (INX, KIND_LEAF, KIND_M2L, KIND_M2L_ROOT, NCELL, WORK_ITEM_DTYPE,
                     SubgridPool, direction_offsets)

BASE_SEED = 20261203

_QUAD = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
_OCT = [(0, 0, 0), (0, 0, 1), (0, 0, 2), (0, 1, 1), (0, 1, 2), (0, 2, 2), (1, 1, 1), (1, 1, 2),
        (1, 2, 2), (2, 2, 2)]


@dataclass
class Batch:
    """A pool of subgrids plus the work list of one gravity solve."""

    pool: SubgridPool
    items: np.ndarray            # WORK_ITEM_DTYPE
    theta: float = 0.5
    name: str = ""
    levels: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    positions: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int64))


def cell_centres(level: int, pos) -> np.ndarray:
    """[512, 3] cell centres of the subgrid at integer position ``pos``."""
    dx = 1.0 / (INX * 2 ** level)
    i = np.arange(INX)
    gx, gy, gz = np.meshgrid(i, i, i, indexing="ij")
    idx = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1).astype(np.float64)
    origin = np.asarray(pos, dtype=np.float64) * INX * dx
    return origin[None, :] + (idx + 0.5) * dx


def point_mass_moments(rng: np.random.Generator, m: np.ndarray, dx: float) -> np.ndarray:
    """[n, 20] raw moments of 8 point masses per cell about their centre of mass."""
    n = m.shape[0]
    w = rng.uniform(0.5, 1.5, size=(n, 8))
    w = w / w.sum(axis=1, keepdims=True) * m[:, None]
    off = rng.uniform(-0.1, 0.1, size=(n, 8, 3)) * dx
    mean = (w[:, :, None] * off).sum(axis=1) / w.sum(axis=1)[:, None]
    off = off - mean[:, None, :]
    M = np.zeros((n, 20))
    M[:, 0] = m
    M[:, 1:4] = (w[:, :, None] * off).sum(axis=1)
    for q, (a, b) in enumerate(_QUAD):
        M[:, 4 + q] = (w * off[:, :, a] * off[:, :, b]).sum(axis=1)
    for o, (a, b, c) in enumerate(_OCT):
        M[:, 10 + o] = (w * off[:, :, a] * off[:, :, b] * off[:, :, c]).sum(axis=1)
    return M


def sphere_profile(x: np.ndarray, centre=(0.5, 0.5, 0.5), radius: float = 0.5) -> np.ndarray:
    """rho = (1 - r^2)^1.5 inside r < 1, r in units of ``radius``."""
    r2 = (((x - np.asarray(centre)) / radius) ** 2).sum(axis=-1)
    return np.where(r2 < 1.0, np.clip(1.0 - r2, 0.0, None) ** 1.5, 0.0)


def build_batch(levels, positions, refined, *, theta: float = 0.5, seed: int = BASE_SEED,
                density=None, loguniform_mass: bool = False, noise: float = 0.0,
                work: np.ndarray | None = None, name: str = "") -> Batch:
    """Builds pool + work list from octree nodes.

    ``levels[i]``, ``positions[i]`` (integer subgrid coordinates at that level)
    and ``refined[i]`` describe node i. Neighbours are the same-level nodes at
    the 26 adjacent positions (-1 where none exists). ``work`` selects which
    nodes get a work item (default: all). ``density(x)`` gives the density at
    cell centres; ``loguniform_mass`` draws masses on [1e-3, 1] instead.
    """
    levels = np.asarray(levels, dtype=np.int32)
    positions = np.asarray(positions, dtype=np.int64).reshape(-1, 3)
    refined = np.asarray(refined, dtype=bool)
    n = len(levels)
    M = np.zeros((n, 20, NCELL))
    com = np.zeros((n, 3, NCELL))
    mon = np.zeros((n, NCELL))
    is_leaf = (~refined).astype(np.uint8)
    masses = np.zeros((n, NCELL))
    rngs = [np.random.default_rng(seed + i) for i in range(n)]
    for i in range(n):
        lvl = int(levels[i])
        dx = 1.0 / (INX * 2 ** lvl)
        x = cell_centres(lvl, positions[i])
        if loguniform_mass:
            masses[i] = np.exp(rngs[i].uniform(np.log(1e-3), np.log(1.0), size=NCELL))
        else:
            rho = density(x)
            if noise > 0:
                rho = rho * np.exp(noise * rngs[i].standard_normal(NCELL))
            masses[i] = rho * dx ** 3
    floor = 1e-12 * masses.max()
    masses = np.maximum(masses, floor)
    for i in range(n):
        lvl = int(levels[i])
        dx = 1.0 / (INX * 2 ** lvl)
        x = cell_centres(lvl, positions[i])
        m = masses[i]
        mon[i] = m
        if refined[i]:
            c = x + rngs[i].uniform(-0.4, 0.4, size=(NCELL, 3)) * dx
            com[i] = c.T
            M[i] = point_mass_moments(rngs[i], m, dx).T
        else:
            com[i] = x.T
            M[i, 0] = m
    pool = SubgridPool(M=M, com=com, mon=mon, is_leaf=is_leaf)
    lookup = {(int(levels[i]), *map(int, positions[i])): i for i in range(n)}
    sel = np.arange(n) if work is None else np.asarray(work, dtype=np.int64)
    items = np.zeros(len(sel), dtype=WORK_ITEM_DTYPE)
    for k, i in enumerate(sel):
        lvl = int(levels[i])
        dx = 1.0 / (INX * 2 ** lvl)
        items[k]["subgrid"] = i
        if refined[i]:
            items[k]["kind"] = KIND_M2L_ROOT if lvl == 0 else KIND_M2L
        else:
            items[k]["kind"] = KIND_LEAF
        items[k]["dx"] = dx
        items[k]["xbase"] = positions[i] * INX * dx + 0.5 * dx
        for d in range(26):
            o = direction_offsets(d)
            key = (lvl, int(positions[i][0]) + o[0], int(positions[i][1]) + o[1], int(positions[i][2]) + o[2])
            items[k]["neighbors"][d] = lookup.get(key, -1)
    return Batch(pool=pool, items=items, theta=theta, name=name, levels=levels, positions=positions)


def single_subgrid(seed: int = BASE_SEED, theta: float = 0.5, leaf_dirs=(), empty_dirs=(),
                   leaf_centre: bool = False) -> Batch:
    """One 8^3 subgrid at level 3 with its 26 neighbours present.

    Log-uniform cell masses. ``leaf_dirs`` turns those neighbours into leaf
    (monopole) subgrids, ``empty_dirs`` removes them; ``leaf_centre`` makes the
    centre subgrid a leaf (P2P / P2M work item).
    """
    centre = np.array([3, 3, 3])
    pos, refined = [centre], [not leaf_centre]
    for d in range(26):
        if d in empty_dirs:
            continue
        pos.append(centre + np.array(direction_offsets(d)))
        refined.append(d not in leaf_dirs)
    levels = np.full(len(pos), 3)
    return build_batch(levels, np.array(pos), np.array(refined), theta=theta, seed=seed,
                       loguniform_mass=True, work=[0], name="single_subgrid")


def root_subgrid(seed: int = BASE_SEED, theta: float = 0.5) -> Batch:
    """The level-0 subgrid (root stencil), log-uniform masses."""
    return build_batch([0], [[0, 0, 0]], [True], theta=theta, seed=seed, loguniform_mass=True,
                       name="root")


def uniform_level(level: int = 3, seed: int = BASE_SEED, theta: float = 0.5, noise: float = 0.01) -> Batch:
    """Every subgrid of one octree level, all refined (M2L work items), with the
    (1 - r^2)^1.5 sphere profile and lognormal density noise."""
    k = 2 ** level
    g = np.arange(k)
    gx, gy, gz = np.meshgrid(g, g, g, indexing="ij")
    pos = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)
    levels = np.full(len(pos), level)
    refined = np.ones(len(pos), dtype=bool)
    return build_batch(levels, pos, refined, theta=theta, seed=seed, density=sphere_profile, noise=noise,
                       name=f"uniform_level{level}")
