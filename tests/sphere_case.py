"""A uniform-density sphere on an adaptive octree (the analogue of Octo-Tiger's
`sphere` gravity scenario, test_problems/sphere, whose solid-sphere potential
is checked against the analytic one from src/problem.cpp:371-391): density 1
inside radius R about the domain centre, refined where the density is above 1 %
of its peak (levels 3 to max_level), masses at the cell centres. Shared by the
oracle and the device tests."""
from __future__ import annotations

import numpy as np

R = 0.15
CENTRE = np.array([0.5, 0.5, 0.5])


def density(x):
    r = np.sqrt(((x - CENTRE) ** 2).sum(-1))
    return np.where(r < R, 1.0, 0.0)


def sphere_batch(max_level: int = 4, theta: float = 0.5):
    from octotiger_b200 import amr, synthetic as syn
    levels, pos, ref = amr.build_tree(density, max_level=max_level, rho_max=1.0)
    return syn.build_batch(levels, pos, ref, theta=theta, density=density, noise=0.0, name=f"sphere_l{max_level}")


def analytic_errors(pool, com, G):
    """Errors of the leaves' potential and acceleration (G = 1) against the
    uniform sphere of the same total mass, over the cells within 0.9 R of the
    centre (the staircase surface of the cell masses stays out): max error /
    max |analytic| for phi and g, and the L1 norm of phi's error / L1 of phi."""
    leaf = np.nonzero(pool.is_leaf == 1)[0]
    x = com[leaf].transpose(0, 2, 1).reshape(-1, 3)
    m = pool.mon[leaf].reshape(-1)
    phi = G[leaf][:, 0, :].reshape(-1)
    g = G[leaf][:, 1:, :].transpose(0, 2, 1).reshape(-1, 3)
    mtot = m[m > 1e-6 * m.max()].sum()
    rho0 = mtot / (4.0 / 3.0 * np.pi * R ** 3)
    d = x - CENTRE
    r = np.sqrt((d ** 2).sum(-1))
    phi_a = np.where(r < R, -2.0 * np.pi * rho0 * (R ** 2 - r ** 2 / 3.0), -mtot / r)
    g_a = np.where((r < R)[:, None], -(4.0 / 3.0) * np.pi * rho0 * d, -mtot * d / r[:, None] ** 3)
    sel = r < 0.9 * R
    e_phi = np.abs(phi - phi_a)[sel].max() / np.abs(phi_a[sel]).max()
    l1_phi = np.abs(phi - phi_a)[sel].sum() / np.abs(phi_a[sel]).sum()
    e_g = np.abs(g - g_a)[sel].max() / np.abs(g_a[sel]).max()
    return e_phi, l1_phi, e_g
