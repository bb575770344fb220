"""Batched structural problems: many independent cantilever designs of uneven
size and several load cases of one design, solved by one CUDA-graph launch.

``batch_problems(...)`` builds the seeded synthetic batch (grid sizes drawn
with nx:ny:nz = 2:1:1, densities uniform in [lo, hi], point loads at random
nodes of the free x = L face with random unit directions, the x = 0 face
clamped); ``BatchSolver`` (engine) captures and launches the solves.
"""
from __future__ import annotations

import numpy as np
import torch

from .deflation import DeflationSolver
from .engine import HexGrid
from .hex_mesher import HexMesher
from .problems import cantilever

F64 = torch.float64


def point_load(mesh: HexMesher, rng):
    """Unit force at a random node of the x = L face, random direction."""
    ni = mesh.node_indices
    face = np.flatnonzero(ni[:, 0] == mesh.grid[0])
    node = int(rng.choice(face))
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    f = np.zeros(3 * mesh.num_nodes)
    f[3 * node:3 * node + 3] = d
    return f


def make_design(nel, rng, lo=0.01, hi=1.0, penal=3.0, emin=1e-9, group_nodes=16, device=None):
    """(grid, defl, s) of one cantilever design with seeded densities."""
    mesh = HexMesher()
    mesh.grid_mesh(nel, (1.0, 1.0, 1.0))
    _, fixed = cantilever(mesh)
    g = HexGrid(nel, device=device).set_fixed_dofs(fixed)
    ds = DeflationSolver(modes=6, shift=1e-14, shift_relative=True)
    agg = tuple(max(1, min(group_nodes, n)) for n in nel)
    ds.create_deflation_groups_box(mesh, agg, modes=6)
    defl = ds.device_deflation(g)
    x = g.tensor(rng.uniform(lo, hi, g.nelem))
    s, _ = g.simp(x, penal, emin, want_ds=False)
    return mesh, g, defl, s


def batch_problems(n_designs=64, min_nx=32, max_nx=96, multi_nel=(128, 64, 64), n_loads=8, seed=0, device=None):
    """The batched workload: n_designs cantilevers with nx drawn in [min_nx, max_nx]
    (even, ny = nz = nx / 2), one point load each, plus one multi_nel design with
    n_loads load cases.  Returns a list of (grid, defl, s, b)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_designs):
        nx = int(rng.integers(min_nx // 2, max_nx // 2 + 1)) * 2
        nel = (nx, nx // 2, nx // 2)
        mesh, g, defl, s = make_design(nel, rng, device=device)
        out.append((g, defl, s, g.tensor(point_load(mesh, rng))))
    if multi_nel is not None and n_loads > 0:
        mesh, g, defl, s = make_design(tuple(multi_nel), rng, device=device)
        for _ in range(n_loads):
            out.append((g, defl, s, g.tensor(point_load(mesh, rng))))
    return out
