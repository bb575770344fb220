"""Host backend of pyto_b200.slab for the CPU tests of the slab decomposition (test
infrastructure): the same operations as DeviceSlab, computed with the numpy oracle
on the rank's slab, on torch CPU tensors so that gloo can carry them."""
import numpy as np
import torch

import oracle as O
from pyto_b200.slab import halo_maps, local_fixed_dofs, owned_elements


class HostSlab:
    def __init__(self, slab, nel, fixed_dofs, node_group, centers, h=(1.0, 1.0, 1.0), E=1.0, nu=0.3, modes=6,
                 shift=1e-14, shift_relative=True):
        self.slab, self.h, self.modes = slab, tuple(h), modes
        self.shift, self.shift_relative = shift, shift_relative
        self.Ke = O.ke_hex8(E, nu, h)
        nx, ny, nzl = slab.nel
        self.nnodes = (nx + 1) * (ny + 1) * (nzl + 1)
        P = slab.plane_nodes
        self.fixed_true = local_fixed_dofs(slab, nel, fixed_dofs)
        own = np.zeros(3 * self.nnodes, bool)
        own[self.fixed_true] = True
        if slab.halo_lo:
            own[:3 * P] = True
        if slab.halo_hi:
            own[3 * (self.nnodes - P):] = True
        self.fixed_own = np.flatnonzero(own)
        self.mesh = O.grid_mesh(nx, ny, nzl, h)
        grp = np.asarray(node_group, dtype=np.int64)[P * slab.n0:P * slab.n1]
        cen = np.array(centers, dtype=np.float64).reshape(-1, 3).copy()
        cen[:, 2] -= slab.n0 * h[2]
        self.W = O.deflation_W(self.mesh["node_xyz"], grp, cen, cen.shape[0], modes).toarray()
        self.own_el = owned_elements(slab, nel).astype(bool)

    def set_scaling(self, s_slab):
        self.s = np.asarray(s_slab, dtype=np.float64)

    def zeros(self):
        return torch.zeros(3 * self.nnodes, dtype=torch.float64)

    def copy(self, dst, src):
        dst.copy_(torch.as_tensor(src))

    def coarse_assemble(self):
        K = O.assemble_K(self.mesh, self.s * self.own_el, self.Ke).toarray()
        Wf = self.W.copy()
        Wf[self.fixed_true] = 0.0
        self._E = torch.as_tensor(Wf.T @ K @ Wf)
        return self._E

    def coarse_invert(self):
        E = self._E.numpy()
        E = 0.5 * (E + E.T)
        d = np.diag(E).copy()
        sh = self.shift * np.mean(np.abs(d)) if self.shift_relative else self.shift
        d[d == 0.0] = 1.0
        np.fill_diagonal(E, d + sh)
        self.Einv = np.linalg.inv(E)

    def jacobi(self):
        nd = self.s.size
        diag = np.zeros(3 * self.nnodes)
        edof = self.mesh["edof"]
        np.add.at(diag, edof.ravel(), np.repeat(self.s[:nd], 24) * np.tile(np.diag(self.Ke), nd))
        inv = np.where(np.abs(diag) < 1e-12, 1.0, 1.0 / np.where(diag == 0, 1.0, diag))
        inv[self.fixed_own] = 0.0
        self.minv = inv
        self.free = np.ones(3 * self.nnodes, bool)
        self.free[self.fixed_own] = False

    def matvec(self, u, y, dot=False):
        v = O.matvec_ebe(self.slab.nel, self.s, self.Ke, u.numpy(), self.fixed_true)
        v[self.fixed_own] = 0.0
        y.copy_(torch.as_tensor(v))
        if dot:
            return torch.tensor([float(u.numpy() @ v)], dtype=torch.float64)
        return y

    def cg_update(self, alpha, p, q, x, r, z):
        rn = r.numpy()
        if q is not None:
            rn -= alpha * q.numpy()
        if p is not None:
            x.numpy()[:] += alpha * p.numpy()
        zn = self.minv * rn
        z.copy_(torch.as_tensor(zn))
        f = self.free
        return torch.tensor([float(rn[f] @ rn[f]), float(rn[f] @ zn[f])], dtype=torch.float64)

    def restrict(self, y):
        yn = y.numpy().copy()
        yn[self.fixed_own] = 0.0
        return torch.as_tensor(self.W.T @ yn)

    def apply(self, v):
        return torch.as_tensor(self.Einv @ v.numpy())

    def prolong(self, mu, a, z, b, p):
        v = -(self.W @ mu.numpy())
        if z is not None:
            v += a * z.numpy()
        if b != 0.0:
            v += b * p.numpy()
        v[self.fixed_own] = 0.0
        p.copy_(torch.as_tensor(v))

    def halo(self, comm, vec):
        P3 = 3 * self.slab.plane_nodes
        send, recv = halo_maps(self.slab)
        comm.exchange([(peer, vec[P3 * k:P3 * (k + 1)]) for peer, k in send],
                      [(peer, vec[P3 * k:P3 * (k + 1)]) for peer, k in recv])
