"""One deflated PCG solve split across ranks: slabs of node planes along z.

Partition.  The (nelz + 1) node planes of a grid are cut into `world` contiguous
ranges; rank r owns planes [z0, z1) and the element layers [z0, min(z1, nelz)), so
every element belongs to exactly one rank.  A rank's slab grid holds the element
layers touching its nodes, [max(z0 - 1, 0), min(z1, nelz)), hence one halo node
plane below (global z0 - 1, owned by rank r - 1) and one above (global z1, owned by
rank r + 1) where those exist.  z is the slowest grid index, so a slab and each of
its planes are contiguous ranges of the global vectors (no packing).

Per iteration of the reference's DPCG recurrence (src/deflation.py:504-584, two
products with K per iteration: K p and K z) a rank exchanges two halo planes of p
and of z with its neighbours (into each receiver's own halo slots), sums three
things over the ranks (p.Kp; r.r with r.z; the restricted coarse vector W^T K z)
and applies the replicated coarse inverse.  The coarse matrix is summed over the
ranks once per solve (each rank assembles its own element layers) and inverted on
every rank.  A rank marks its halo nodes fixed in the mask it hands the kernels,
so operator outputs, dot products and restrictions cover its own nodes only.

The collectives go through a ``SlabComm``: ``DistComm`` (torch.distributed: NCCL
between GPUs, gloo on CPU) or ``ThreadComm`` (several ranks as threads of one
process, the exchange done by copies: a test of the decomposition on one device).
The arithmetic goes through a backend: ``DeviceSlab`` calls the C ABI of
libpyto_b200 on the rank's slab.
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass

import numpy as np
import torch

from . import _capi as A


# ---------------------------------------------------------------------------
# partition
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class Slab:
    """Rank r's share of a grid with nel = (nx, ny, nz) elements."""
    rank: int
    world: int
    z0: int          # first owned node plane (global)
    z1: int          # one past the last owned node plane
    n0: int          # first node plane of the slab grid (global): z0 - 1 with a lower halo
    n1: int          # one past the last node plane of the slab grid
    nel: tuple       # the slab grid's elements (nx, ny, n1 - n0 - 1)
    halo_lo: bool    # the slab grid's plane 0 is a halo (owned by rank - 1)
    halo_hi: bool    # its last plane is a halo (owned by rank + 1)
    e0: int          # owned element layers [e0, e1) (global)
    e1: int

    @property
    def plane_nodes(self):
        return (self.nel[0] + 1) * (self.nel[1] + 1)

    @property
    def own_planes(self):
        """Owned planes as slab-local plane indices [a, b)."""
        return self.z0 - self.n0, self.z1 - self.n0


def partition(nel, world: int):
    """The slabs of all ranks: node planes split as evenly as contiguous ranges allow."""
    nx, ny, nz = (int(v) for v in nel)
    planes = nz + 1
    if world < 1 or world > planes:
        raise ValueError(f"{world} ranks for {planes} node planes: every rank needs a plane")
    bounds = [(r * planes) // world for r in range(world + 1)]
    out = []
    for r in range(world):
        z0, z1 = bounds[r], bounds[r + 1]
        n0, n1 = max(z0 - 1, 0), min(z1 + 1, planes)
        out.append(Slab(r, world, z0, z1, n0, n1, (nx, ny, n1 - n0 - 1), z0 > 0, z1 < planes, z0, min(z1, nz)))
    return out


def halo_maps(slab: Slab):
    """(send, recv) plane maps of one rank: lists of (neighbour rank, slab-local plane).
    The lowest owned plane goes to rank - 1 (its upper halo), the highest to rank + 1
    (its lower halo); the halos are received from the same neighbours."""
    a, b = slab.own_planes
    send, recv = [], []
    if slab.halo_lo:
        send.append((slab.rank - 1, a))
        recv.append((slab.rank - 1, 0))
    if slab.halo_hi:
        send.append((slab.rank + 1, b - 1))
        recv.append((slab.rank + 1, slab.n1 - slab.n0 - 1))
    return send, recv


def local_fixed_dofs(slab: Slab, nel, fixed_dofs):
    """Global fixed DOFs that fall in the slab grid, renumbered to it."""
    nx, ny, _ = nel
    P = (nx + 1) * (ny + 1)
    fd = np.asarray(fixed_dofs, dtype=np.int64)
    lo, hi = 3 * P * slab.n0, 3 * P * slab.n1
    sel = fd[(fd >= lo) & (fd < hi)]
    return sel - lo


def owned_elements(slab: Slab, nel):
    """uint8 per slab element: 1 for the element layers this rank owns."""
    nx, ny, nzl = slab.nel
    own = np.zeros((nzl, ny, nx), dtype=np.uint8)
    own[slab.e0 - slab.n0:slab.e1 - slab.n0] = 1
    return own.ravel()


def slab_range(slab: Slab, ndofs_per_node=3):
    """(start, stop) of the slab grid's entries in a global node-major vector."""
    P = slab.plane_nodes
    return ndofs_per_node * P * slab.n0, ndofs_per_node * P * slab.n1


# ---------------------------------------------------------------------------
# collectives
# ---------------------------------------------------------------------------
class DistComm:
    """Collectives over torch.distributed (NCCL for CUDA tensors, gloo for CPU ones)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def allreduce_(self, t: torch.Tensor):
        if self.world > 1:
            self.dist.all_reduce(t, group=self.group)
        return t

    def exchange(self, sends, recvs):
        """sends / recvs: lists of (peer rank, contiguous tensor); receives land in place."""
        if self.world == 1 or not (sends or recvs):
            return
        ops = [self.dist.P2POp(self.dist.isend, t, peer, self.group) for peer, t in sends]
        ops += [self.dist.P2POp(self.dist.irecv, t, peer, self.group) for peer, t in recvs]
        for w in self.dist.batch_isend_irecv(ops):
            w.wait()


class ThreadComm:
    """`world` ranks as threads of one process (one SlabComm view per rank, from
    ``views()``).  Sums are formed in rank order on every rank, so all ranks get
    the same bits; halo planes are copied from the sender's buffer into the
    receiver's.  Device work of a rank is synchronised before it is shared."""

    def __init__(self, world: int):
        self.world = world
        self.barrier = threading.Barrier(world)
        self.slots = [None] * world
        self.boxes = {}

    def views(self):
        return [_ThreadView(self, r) for r in range(self.world)]


class _ThreadView:
    def __init__(self, shared: ThreadComm, rank: int):
        self.s, self.rank, self.world = shared, rank, shared.world

    def _sync(self, t):
        if t.is_cuda:
            torch.cuda.current_stream(t.device).synchronize()

    def allreduce_(self, t: torch.Tensor):
        self._sync(t)
        self.s.slots[self.rank] = t.clone()
        self.s.barrier.wait()
        tot = self.s.slots[0].clone()
        for r in range(1, self.world):
            tot += self.s.slots[r]
        self.s.barrier.wait()
        t.copy_(tot)
        self._sync(t)
        return t

    def exchange(self, sends, recvs):
        for peer, t in sends:
            self._sync(t)
            self.s.boxes[(self.rank, peer)] = t.clone()
        self.s.barrier.wait()
        for peer, t in recvs:
            t.copy_(self.s.boxes[(peer, self.rank)])
            self._sync(t)
        self.s.barrier.wait()


# ---------------------------------------------------------------------------
# the solver
# ---------------------------------------------------------------------------
@dataclass
class SlabInfo:
    converged: bool
    iters: int
    rel_res: float


def slab_dpcg(be, comm, b, rtol=1e-8, max_iters=5000, stop_rule=0):
    """The reference's deflated PCG (src/deflation.py:504-584) on one rank's slab.

    ``be`` is the rank's backend (set up for the current densities), ``b`` its slab of
    the load vector.  Stopping rule 0: ||r|| < rtol ||b|| (scipy cg's test); 1: the
    reference's sqrt(r.z / r0.z0) <= rtol.  Returns (x, info); x is valid on the owned
    planes."""
    # coarse operator: each rank's element layers, summed, inverted on every rank
    E = be.coarse_assemble()
    comm.allreduce_(E)
    be.coarse_invert()
    be.jacobi()
    x, r, z, p, q, kz = (be.zeros() for _ in range(6))
    # ||b|| over the free owned DOFs
    be.copy(r, b)
    bb = float(comm.allreduce_(be.cg_update(0.0, None, None, None, r, z))[0])
    # coarse start x = W E^-1 W^T b;  r = b - K x;  z = M r
    v = comm.allreduce_(be.restrict(b))
    be.prolong(be.apply(v.neg_()), 0.0, None, 0.0, x)
    be.halo(comm, x)
    be.matvec(x, q)
    be.copy(r, b)
    d = comm.allreduce_(be.cg_update(1.0, None, q, None, r, z))
    rz = float(d[1])
    rz0 = rz
    # p = z - W E^-1 W^T K z
    be.halo(comm, z)
    be.matvec(z, kz)
    be.prolong(be.apply(comm.allreduce_(be.restrict(kz))), 1.0, z, 0.0, p)
    be.halo(comm, p)
    it, conv = 0, bb == 0.0
    while it < max_iters and not conv:
        pq = float(comm.allreduce_(be.matvec(p, q, dot=True))[0])
        if not (pq > 0.0) or not np.isfinite(pq):
            break
        alpha = rz / pq
        d = comm.allreduce_(be.cg_update(alpha, p, q, x, r, z))
        rr, rz_new = float(d[0]), float(d[1])
        it += 1
        conv = (np.sqrt(rz_new / rz0) <= rtol) if stop_rule == 1 else (np.sqrt(rr) < rtol * np.sqrt(bb))
        if conv:
            break
        beta = rz_new / rz
        be.halo(comm, z)
        be.matvec(z, kz)
        be.prolong(be.apply(comm.allreduce_(be.restrict(kz))), 1.0, z, beta, p)
        be.halo(comm, p)
        rz = rz_new
    rel = np.sqrt(rz_new / rz0) if (stop_rule == 1 and it) else (np.sqrt(rr / bb) if it and bb else 0.0)
    return x, SlabInfo(bool(conv), it, float(rel))


class DeviceSlab:
    """A rank's slab on its GPU, through the C ABI of libpyto_b200.

    nel, h, E, nu: the global grid; fixed_dofs: global fixed DOFs; node_group and
    centers: the global deflation groups (node -> group, group centroids)."""

    def __init__(self, slab: Slab, nel, fixed_dofs, node_group, centers, h=(1.0, 1.0, 1.0), E=1.0, nu=0.3,
                 modes=6, shift=1e-14, shift_relative=True, device=None):
        from .engine import DeviceDeflation, HexGrid
        self.slab = slab
        self.grid = g = HexGrid(slab.nel, h, E, nu, device=device)
        g.set_fixed_dofs(local_fixed_dofs(slab, nel, fixed_dofs))  # the true fixed DOFs: coarse assembly
        P = slab.plane_nodes
        own = g.mask.clone()  # + halo planes fixed: outputs, dots and restrictions on owned nodes only
        if slab.halo_lo:
            own[:P] = 7
        if slab.halo_hi:
            own[g.nnodes - P:g.nnodes] = 7
        self.mask_own = own
        ng_local = np.asarray(node_group, dtype=np.int32)[P * slab.n0:P * slab.n1]
        cen = np.array(centers, dtype=np.float64).reshape(-1, 3).copy()
        cen[:, 2] -= slab.n0 * h[2]  # group centres in slab coordinates
        self.defl = DeviceDeflation(g, ng_local, cen, modes=modes, shift=shift, shift_relative=shift_relative)
        self.own_el = torch.as_tensor(owned_elements(slab, nel), device=g.device)
        self.dot = torch.empty(2, dtype=torch.float64, device=g.device)
        self.v = torch.empty(self.defl.nc, dtype=torch.float64, device=g.device)
        self.mu = torch.empty(self.defl.nc, dtype=torch.float64, device=g.device)
        self.winv = torch.empty(g.nnodes, dtype=torch.float64, device=g.device)
        self.flags = torch.empty(g.nnodes, dtype=torch.uint8, device=g.device)

    # -- state ---------------------------------------------------------------
    def set_scaling(self, s_slab):
        """Element scaling of the slab grid's elements (all local layers)."""
        self.s = self.grid.tensor(s_slab)
        self.s_own = self.s * self.own_el  # this rank's elements only (coarse assembly)

    def zeros(self):
        return torch.zeros(self.grid.ndof, dtype=torch.float64, device=self.grid.device)

    def copy(self, dst, src):
        dst.copy_(src)

    # -- arithmetic (C ABI) ----------------------------------------------------
    def _ws(self, kind, tag):
        return self.grid._ws(kind, tag)

    def coarse_assemble(self):
        g, d = self.grid, self.defl
        d.sync(g)
        wsp, wsn = self._ws(A.WS_DPCG, "krylov")
        A.call("pyto_coarse_assemble", g.opp, A.ptr(self.s_own), A.ptr(g.mask), C.byref(d.struct), wsp, wsn, g._st())
        return d.coarse_inv

    def coarse_invert(self):
        g, d = self.grid, self.defl
        wsp, wsn = self._ws(A.WS_DPCG, "krylov")
        A.call("pyto_coarse_invert", g.opp, C.byref(d.struct), wsp, wsn, g._st())

    def jacobi(self):
        g = self.grid
        A.call("pyto_jacobi", g.opp, A.ptr(self.s), A.ptr(self.mask_own), A.ptr(self.winv), A.ptr(self.flags), None,
               g._st())

    def matvec(self, u, y, dot=False):
        g = self.grid
        wsp, wsn = self._ws(A.WS_REDUCE, "reduce") if dot else (None, 0)
        A.call("pyto_matvec", g.opp, A.ptr(self.s), A.ptr(self.mask_own), A.ptr(u), A.ptr(y), A.MASK_OUT,
               A.ptr(self.dot) if dot else None, wsp, wsn, g._st())
        return self.dot[:1] if dot else y

    def cg_update(self, alpha, p, q, x, r, z):
        g = self.grid
        wsp, wsn = self._ws(A.WS_REDUCE, "reduce")
        A.call("pyto_cg_update", g.opp, A.ptr(self.winv), A.ptr(self.flags), float(alpha), A.ptr(p), A.ptr(q),
               A.ptr(x), A.ptr(r), A.ptr(z), A.ptr(self.dot), wsp, wsn, g._st())
        return self.dot

    def restrict(self, y):
        g, d = self.grid, self.defl
        wsp, wsn = self._ws(A.WS_DPCG, "krylov")
        A.call("pyto_coarse_restrict", g.opp, C.byref(d.struct), A.ptr(self.mask_own), A.ptr(y), A.ptr(self.v),
               wsp, wsn, g._st())
        return self.v

    def apply(self, v):
        A.call("pyto_coarse_apply", C.byref(self.defl.struct), A.ptr(v), A.ptr(self.mu), self.grid._st())
        return self.mu

    def prolong(self, mu, a, z, b, p):
        g = self.grid
        A.call("pyto_coarse_prolong", g.opp, C.byref(self.defl.struct), A.ptr(self.mask_own), A.ptr(mu), float(a),
               A.ptr(z), float(b), A.ptr(p), g._st())

    def halo(self, comm, vec):
        """Send the owned boundary planes of vec to the neighbours; receive their
        planes into vec's halo planes."""
        P3 = 3 * self.slab.plane_nodes
        send, recv = halo_maps(self.slab)
        comm.exchange([(peer, vec[P3 * k:P3 * (k + 1)]) for peer, k in send],
                      [(peer, vec[P3 * k:P3 * (k + 1)]) for peer, k in recv])
