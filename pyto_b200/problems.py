"""Synthetic benchmark problems of the hex8 path (seeded; no dataset involved).

Cantilever: all DOFs of the ix = 0 nodes clamped; a unit total -z load split
equally over the nodes of the x = L, z = 0 edge (the grid-problem pattern of
src/hex_structural_examples.py:665-669).  Densities follow the benchmark
recipes: seeded uniform draws in element-id order, optionally passed through
the density filter.
"""
from __future__ import annotations

import numpy as np

from .hex_mesher import HexMesher

CFG1 = (60, 30, 30)     # CPU-runnable OC case
CFG2 = (192, 96, 96)    # ~5.4M DOF deflated solve
CFG4 = (128, 64, 64)    # L-shaped domain


def cantilever(mesh: HexMesher, active=None):
    """(force, fixed_dofs) of the clamped-face / loaded-edge cantilever.  With an
    active mask, nodes touched by no active element are fixed too."""
    ni = mesh.node_indices
    fixed_nodes = mesh.getNodesOnBoundingBoxPlane(0, True)
    if active is not None:
        mesh.set_active_elements(active)
        fixed_nodes = np.union1d(fixed_nodes, mesh.unused_nodes())
    fixed = np.sort(np.concatenate([3 * fixed_nodes + c for c in range(3)])).astype(np.int64)
    load = np.where((ni[:, 0] == mesh.grid[0]) & (ni[:, 2] == 0))[0]
    f = np.zeros(3 * mesh.num_nodes)
    f[3 * load + 2] = -1.0 / len(load)
    return f, fixed


def lshape_active(nel=CFG4):
    """L-domain: the x >= nx/2, z >= nz/2 quadrant of the xz section is void (extruded in y)."""
    nx, ny, nz = nel
    e = np.arange(nx * ny * nz)
    ex, ez = e % nx, e // (nx * ny)
    return ~((ex >= nx // 2) & (ez >= nz // 2))


def uniform_density(nel, lo, hi, seed=0, active=None):
    rng = np.random.default_rng(seed)
    n = int(np.prod(nel)) if active is None else int(np.sum(active))
    x = rng.uniform(lo, hi, n)
    if active is None:
        return x
    full = np.zeros(int(np.prod(nel)))
    full[np.asarray(active, bool)] = x
    return full
