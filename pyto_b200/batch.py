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


def partition_by_dof(ndofs, world):
    """Contiguous ranges [start, end) of the problems for each of `world` ranks with
    balanced DOF totals (problems are independent: no communication between ranks).
    Rank r takes the problems whose DOF prefix midpoint falls in its share."""
    nd = np.asarray(ndofs, dtype=np.float64)
    if world <= 1 or nd.size == 0:
        return [(0, int(nd.size))] + [(int(nd.size), int(nd.size))] * max(0, world - 1)
    mid = np.cumsum(nd) - 0.5 * nd
    owner = np.minimum((mid / nd.sum() * world).astype(np.int64), world - 1)
    out = []
    for r in range(world):
        idx = np.flatnonzero(owner == r)
        out.append((int(idx[0]), int(idx[-1]) + 1) if idx.size else (int(np.searchsorted(owner, r)),) * 2)
    return out


def max_over_ranks(seconds, group=None):
    """Slowest rank's time (the job time of independent replicas or partitions)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return float(seconds)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def point_load(mesh: HexMesher, rng, direction=None):
    """Unit force at a random node of the x = L face: along `direction` (e.g. -z), or in
    a random direction."""
    ni = mesh.node_indices
    face = np.flatnonzero(ni[:, 0] == mesh.grid[0])
    node = int(rng.choice(face))
    if direction is None:
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
    else:
        d = np.asarray(direction, dtype=np.float64)
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


def batch_shapes(n_designs=64, min_nx=32, max_nx=96, seed=0):
    """Grid shapes of the batch's designs (nx even in [min_nx, max_nx], ny = nz = nx/2)."""
    rng = np.random.default_rng(seed)
    return [(nx, nx // 2, nx // 2) for nx in (int(rng.integers(min_nx // 2, max_nx // 2 + 1)) * 2
                                              for _ in range(n_designs))]


def batch_problems(n_designs=64, min_nx=32, max_nx=96, multi_nel=(128, 64, 64), n_loads=8, seed=None, device=None,
                   rank=0, world=1):
    """The batched workload: n_designs cantilevers with nx drawn from {min_nx, min_nx+2,
    ..., max_nx} (ny = nz = nx / 2, seed 2), densities U[0.01, 1] (stream (2, k) for
    design k), one unit -z point load each at a random node of the x = L face (stream
    (3, k)), plus one multi_nel design with n_loads load cases, unit point loads in
    random directions on that face (stream (4, k)).  Units of partitioning: each design,
    and the multi-load design as a whole; with world > 1 only this rank's contiguous,
    DOF-balanced share is built.  `seed` replaces all three seeds (tests).  Returns a
    list of (grid, defl, s, b)."""
    s_shape, s_dens, s_load, s_multi = (2, 2, 3, 4) if seed is None else (seed,) * 4
    shapes = batch_shapes(n_designs, min_nx, max_nx, s_shape)
    units = [(nel, 1) for nel in shapes]
    if multi_nel is not None and n_loads > 0:
        units.append((tuple(multi_nel), n_loads))
    ndof = [n * 3 * (a + 1) * (b + 1) * (c + 1) for (a, b, c), n in units]
    lo, hi = partition_by_dof(ndof, world)[rank]
    out = []
    for k in range(lo, hi):
        nel, nloads = units[k]
        # per-unit streams: the same data on any rank count
        mesh, g, defl, s = make_design(nel, np.random.default_rng((s_dens, k)), device=device)
        if nloads == 1:
            out.append((g, defl, s, g.tensor(point_load(mesh, np.random.default_rng((s_load, k)), (0.0, 0.0, -1.0)))))
        else:
            rng = np.random.default_rng((s_multi, k))
            for _ in range(nloads):
                out.append((g, defl, s, g.tensor(point_load(mesh, rng))))
    return out
