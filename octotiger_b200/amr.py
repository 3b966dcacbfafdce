"""Adaptive-octree work lists for the batched solve (seeded, synthetic).

Tree rules follow Octo-Tiger's regrid: levels below ``base_level`` are fully
refined; a node at level >= base_level refines where the density inside it
exceeds ``threshold`` times the peak; and whenever a node refines, its 26
same-level neighbours are forced to exist (node_server::check_for_refinement
and force_nodes_to_exist, src/node_server_actions_2.cpp:36-75,387-430), which
refines their parents in turn. Refined nodes therefore always see all 26
neighbours at their level; leaves may face empty directions.

Density: n = 1.5 polytropes from a Lane-Emden integration (the reference has
its own integrator in src/lane_emden.cpp:32-103; this one is an RK4 march of
theta'' + 2 theta'/xi + theta^n = 0).
"""
from __future__ import annotations

import numpy as np

from .synthetic import BASE_SEED, Batch, build_batch


def lane_emden(n: float = 1.5, h: float = 1e-4):
    """Returns (xi, theta) sampled up to the first zero xi_1 of theta."""
    def rhs(x, y):
        th, dth = y
        th_n = np.power(max(th, 0.0), n)
        if x == 0.0:
            return np.array([dth, -th_n / 3.0])
        return np.array([dth, -th_n - 2.0 * dth / x])

    xs, ths = [0.0], [1.0]
    y = np.array([1.0, 0.0])
    x = 0.0
    while y[0] > 0.0:
        k1 = rhs(x, y)
        k2 = rhs(x + h / 2, y + h / 2 * k1)
        k3 = rhs(x + h / 2, y + h / 2 * k2)
        k4 = rhs(x + h, y + h * k3)
        y = y + h / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
        x += h
        xs.append(x)
        ths.append(y[0])
    xs, ths = np.array(xs), np.array(ths)
    # linear zero crossing
    x1 = xs[-2] + (xs[-1] - xs[-2]) * ths[-2] / (ths[-2] - ths[-1])
    xs[-1], ths[-1] = x1, 0.0
    return xs, ths


class Polytrope:
    def __init__(self, centre, radius, rho_c=1.0, n=1.5):
        self.centre = np.asarray(centre, dtype=np.float64)
        self.radius = float(radius)
        self.rho_c = float(rho_c)
        self.n = n
        self.xi, self.theta = lane_emden(n)
        self.xi1 = float(self.xi[-1])

    def __call__(self, x: np.ndarray) -> np.ndarray:
        r = np.sqrt(((x - self.centre) ** 2).sum(axis=-1)) / self.radius
        xi = np.clip(r * self.xi1, 0.0, self.xi1)
        th = np.interp(xi, self.xi, self.theta)
        return np.where(r < 1.0, self.rho_c * np.power(np.clip(th, 0.0, None), self.n), 0.0)


def _node_max_density(density, level: int, pos) -> float:
    """Density maximum over a node's cells (sampled at 4^3 points per node)."""
    size = 1.0 / 2 ** level
    g = (np.arange(4) + 0.5) / 4
    gx, gy, gz = np.meshgrid(g, g, g, indexing="ij")
    pts = (np.asarray(pos, dtype=np.float64)[None, :] +
           np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)) * size
    return float(density(pts).max())


def build_tree(density, max_level: int, base_level: int = 3, threshold: float = 1e-2, rho_max: float | None = None):
    """Returns (levels, positions, refined) of every existing node."""
    refined: set[tuple] = set()

    def refine(level: int, p: tuple) -> None:
        key = (level, *p)
        if key in refined:
            return
        if level > 0:
            refine(level - 1, tuple(c // 2 for c in p))   # the node itself must exist
        refined.add(key)
        n = 2 ** level
        for ox in (-1, 0, 1):
            for oy in (-1, 0, 1):
                for oz in (-1, 0, 1):
                    q = (p[0] + ox, p[1] + oy, p[2] + oz)
                    if q == p or min(q) < 0 or max(q) >= n:
                        continue
                    if level > 0:
                        refine(level - 1, tuple(c // 2 for c in q))   # neighbours must exist

    for lvl in range(base_level):
        n = 2 ** lvl
        for x in range(n):
            for y in range(n):
                for z in range(n):
                    refine(lvl, (x, y, z))
    if rho_max is None:
        rho_max = _node_max_density(density, 0, (0, 0, 0))
    thr = threshold * rho_max
    for _sweep in range(2):
        for lvl in range(base_level, max_level):
            existing = [k[1:] for k in _existing(refined, lvl)]
            for p in existing:
                if (lvl, *p) not in refined and _node_max_density(density, lvl, p) > thr:
                    refine(lvl, p)
    nodes = sorted(_all_existing(refined, max_level))
    levels = np.array([k[0] for k in nodes], dtype=np.int32)
    positions = np.array([k[1:] for k in nodes], dtype=np.int64)
    is_ref = np.array([k in refined for k in nodes], dtype=bool)
    return levels, positions, is_ref


def _existing(refined: set, level: int):
    if level == 0:
        return [(0, 0, 0, 0)]
    out = []
    for k in refined:
        if k[0] == level - 1:
            for c in range(8):
                out.append((level, 2 * k[1] + (c >> 2 & 1), 2 * k[2] + (c >> 1 & 1), 2 * k[3] + (c & 1)))
    return out


def _all_existing(refined: set, max_level: int):
    out = {(0, 0, 0, 0)}
    for lvl in range(1, max_level + 1):
        out.update(_existing(refined, lvl))
    return out


def polytrope_batch(radius: float = 0.12, max_level: int = 6, seed: int = BASE_SEED, theta: float = 0.5,
                    noise: float = 0.01) -> Batch:
    """One n = 1.5 polytrope at the domain centre, levels 3-6 refined where the
    density exceeds 1e-2 of its peak."""
    poly = Polytrope((0.5, 0.5, 0.5), radius)
    levels, pos, ref = build_tree(poly, max_level=max_level, rho_max=poly.rho_c)
    b = build_batch(levels, pos, ref, theta=theta, seed=seed, density=poly, noise=noise,
                    name=f"amr_polytrope_l{max_level}")
    return b


def binary_batch(radius: float = 0.09, max_level: int = 7, seed: int = BASE_SEED, theta: float = 0.5,
                 noise: float = 0.01) -> Batch:
    """Two n = 1.5 polytropes, mass ratio 0.7, separation 3 radii, refined to
    level 7 around both."""
    # equal radii; the secondary's central density scaled for a 0.7 mass ratio
    sep = 3.0 * radius
    a = Polytrope((0.5 - sep / 2, 0.5, 0.5), radius, rho_c=1.0)
    b = Polytrope((0.5 + sep / 2, 0.5, 0.5), radius, rho_c=0.7)

    def density(x):
        return a(x) + b(x)

    levels, pos, ref = build_tree(density, max_level=max_level, rho_max=1.0)
    return build_batch(levels, pos, ref, theta=theta, seed=seed, density=density, noise=noise,
                       name=f"amr_binary_l{max_level}")
