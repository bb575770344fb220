"""Aggregation deflation (drop-in for PyTO's deflation.DeflationSolver).

Group construction is host-side set-up and follows src/deflation.py:86-229
exactly (box partition of the node coordinates, merging of groups with fewer
than ``minNodesPerGroup`` nodes into the nearest valid group) -- integer work,
so the assignment is bit-identical to the reference -- minus its interactive
``input()`` prompt.  The deflation matrix W is never stored: the device keeps
the node->group map and the group centres (src/deflation.py:386-457 defines
W from them), and the coarse operator, its inverse and the DPCG iteration run
in libpyto_b200.
"""
from __future__ import annotations

import warnings

import numpy as np
import scipy.sparse as sp

from .engine import DeviceDeflation

DENSE_COARSE_MAX = 24576  # largest coarse space of the dense coarse inverse


class DeflationSolver:
    """Deflation space + deflated PCG (src/deflation.py:36-584).

    ``coarse``: how the coarse system W^T K W is solved on the device -- "dense" (explicit
    FP64 inverse, one GEMV per correction; up to 24,576 unknowns), "nd" (nested
    dissection on the box grid of groups, for the element-box aggregates of
    ``create_deflation_groups_box``) or "auto" (nested dissection when the dense inverse
    would not fit).  ``nd_leaf``: largest box of groups kept as one tree leaf."""

    def __init__(self, minNodesPerGroup: int = 15, use_gpu: bool = True, modes: int = 6, shift: float = 1e-10,
                 shift_relative: bool = False, coarse: str = "auto", nd_leaf: int = 8):
        self.minNodesPerGroup = minNodesPerGroup
        self.maxGroups = 2000
        self.minGroups = 10
        self.dofPerGroup = 500
        self.use_gpu = True  # the solve always runs on the GPU
        self.modes = int(modes)
        self.shift = float(shift)
        self.shift_relative = bool(shift_relative)
        if coarse not in ("auto", "dense", "nd"):
            raise ValueError(f"unknown coarse solver {coarse!r} (auto, dense, nd)")
        self.coarse = coarse
        self.nd_leaf = int(nd_leaf)
        self._dev = {}
        self.last_info = None

    def setPseudoDensity(self, rho):
        self.elemPseudoDensity = np.asarray(rho).copy()

    def getRecommendedNumberOfGroups(self, nDOF: int = 100000) -> int:
        """clamp(nDOF / dofPerGroup, minGroups, maxGroups) (src/deflation.py:70-84)."""
        n = int(nDOF / self.dofPerGroup)
        return max(min(n, self.maxGroups), self.minGroups)

    def create_deflation_groups(self, meshData, nGroupsDesired: int) -> bool:
        """Box partition + small-group merge (src/deflation.py:86-229)."""
        xyz = meshData.node_xyz
        nn = xyz.shape[0]
        nGroupsDesired = min(nGroupsDesired, int(nn / (1 + self.minNodesPerGroup)))
        mins = np.array([np.min(xyz[:, 0]), np.min(xyz[:, 1]), np.min(xyz[:, 2])])
        L = [np.max(xyz[:, i]) - mins[i] for i in range(3)]
        alpha = (nGroupsDesired / (L[0] * L[1] * L[2])) ** (1.0 / 3)
        nX, nY, nZ = (max(round(alpha * L[i]), 1) for i in range(3))
        ntent = nX * nY * nZ
        size = np.array([L[0] / nX, L[1] / nY, L[2] / nZ])
        idx = np.floor((xyz - mins) / size).astype(np.int32)
        idx = np.minimum(idx, np.array([nX - 1, nY - 1, nZ - 1]))
        grp = (idx[:, 0] + nX * idx[:, 1] + nX * nY * idx[:, 2]).astype(np.int32)
        count = np.bincount(grp, minlength=ntent)
        centre = np.zeros((ntent, 3))
        for i in range(3):
            np.add.at(centre[:, i], grp, xyz[:, i])
        nz_ = count > 0
        centre[nz_] = centre[nz_] / count[nz_, None]
        mapping = np.full(ntent, -1, dtype=np.int32)
        valid = count >= self.minNodesPerGroup
        mapping[valid] = np.arange(int(valid.sum()), dtype=np.int32)
        ngroups = int(valid.sum())
        if np.any(mapping == -1):
            small = np.where((mapping == -1) & (count > 0))[0]
            vidx = np.where(valid)[0]
            if len(small) > 0:
                d = np.linalg.norm(centre[small][:, None, :] - centre[vidx][None, :, :], axis=2)
                mapping[small] = mapping[vidx[np.argmin(d, axis=1)]]
            grp = mapping[grp]
            count = np.bincount(grp, minlength=ngroups)
            centre = np.zeros((ngroups, 3))
            for i in range(3):
                np.add.at(centre[:, i], grp, xyz[:, i])
            centre = centre / count[:, None]
        self.ws_nGroups = ngroups
        self.ws_nodeGroupNumber = grp
        self.ws_groupCount = count
        self.ws_groupCenter = centre
        # without merges the partition is a regular nX x nY x nZ box grid (group id
        # ix + nX iy + nX nY iz): the nested-dissection coarse solver applies to it
        self.box = (int(nX), int(nY), int(nZ)) if ngroups == ntent else None
        self._dev = {}
        if np.any(self.ws_groupCount < self.minNodesPerGroup):
            warnings.warn(f"deflation groups with very few nodes (smallest {int(np.min(self.ws_groupCount))})")
        return int(np.sum(self.ws_groupCount)) == nn

    def create_deflation_groups_box(self, meshData, agg=(4, 4, 4), modes: int = 3) -> bool:
        """Aggregates of agg[0] x agg[1] x agg[2] elements: node (ix,iy,iz) joins box
        (ix//ax, iy//ay, iz//az), the last node layer folded into the preceding box;
        ``modes`` = 3 (translations) or 6 (rigid-body modes)."""
        ni = meshData.node_indices
        nb = [max(1, meshData.grid[d] // agg[d]) for d in range(3)]
        gi = [np.minimum(ni[:, d] // agg[d], nb[d] - 1) for d in range(3)]
        grp = (gi[0] + nb[0] * (gi[1] + nb[1] * gi[2])).astype(np.int32)
        ng = nb[0] * nb[1] * nb[2]
        count = np.bincount(grp, minlength=ng)
        centre = np.zeros((ng, 3))
        for i in range(3):
            np.add.at(centre[:, i], grp, meshData.node_xyz[:, i])
        self.ws_nGroups, self.ws_nodeGroupNumber = ng, grp
        self.ws_groupCount, self.ws_groupCenter = count, centre / count[:, None]
        self.modes = int(modes)
        self.box = tuple(int(v) for v in nb)
        self._dev = {}
        return True

    def create_deflation_matrix(self, meshData):
        """W is implicit on the device (src/deflation.py:386-457 defines it from the
        groups); ``self.W`` builds the explicit sparse matrix on demand."""
        self._mesh = meshData

    @property
    def W(self) -> sp.csr_matrix:
        """Explicit (3*nnodes, modes*ngroups) deflation matrix, host-side (compatibility only)."""
        return self.explicit_W(self._mesh)

    def explicit_W(self, meshData) -> sp.csr_matrix:
        xyz = meshData.node_xyz
        grp = self.ws_nodeGroupNumber
        rel = xyz - self.ws_groupCenter[grp]
        nn = xyz.shape[0]
        n = np.arange(nn)
        m = self.modes
        if m == 3:
            rows = np.concatenate([3 * n + c for c in range(3)])
            cols = np.concatenate([3 * grp + c for c in range(3)])
            return sp.coo_matrix((np.ones(3 * nn), (rows, cols)), shape=(3 * nn, 3 * self.ws_nGroups)).tocsr()
        iW = np.concatenate([3 * n, 3 * n, 3 * n, 3 * n + 1, 3 * n + 1, 3 * n + 1, 3 * n + 2, 3 * n + 2, 3 * n + 2])
        jW = np.concatenate([6 * grp, 6 * grp + 4, 6 * grp + 5, 6 * grp + 1, 6 * grp + 3, 6 * grp + 5, 6 * grp + 2,
                             6 * grp + 3, 6 * grp + 4])
        sW = np.concatenate([np.ones(nn), rel[:, 2], -rel[:, 1], np.ones(nn), -rel[:, 2], rel[:, 0], np.ones(nn),
                             rel[:, 1], -rel[:, 0]])
        return sp.coo_matrix((sW, (iW, jW)), shape=(3 * nn, 6 * self.ws_nGroups)).tocsr()

    def device_deflation(self, grid) -> DeviceDeflation:
        """Device data of this deflation space for a HexGrid (cached per grid)."""
        key = id(grid)
        d = self._dev.get(key)
        if d is None:
            box = getattr(self, "box", None)
            coarse = self.coarse
            if coarse == "auto":  # nested dissection where a dense coarse matrix would not fit
                coarse = "nd" if box is not None and self.ws_nGroups * self.modes > DENSE_COARSE_MAX else "dense"
            d = DeviceDeflation(grid, self.ws_nodeGroupNumber, self.ws_groupCenter, self.modes, self.shift,
                                self.shift_relative, coarse=coarse, group_grid=box, leaf=self.nd_leaf)
            self._dev = {key: d}
        return d

    def deflatedPCG(self, K, f, W=None, M=None, rtol=1e-8, maxIters=2000, verbose=False):
        """Deflated PCG on the reduced operator K (a StiffnessOperator) for full-length f;
        returns the full-length solution (fixed DOFs 0).  W and M are implicit
        (src/deflation.py:491-584)."""
        grid = K.grid
        b = grid.tensor(f)
        dd = self.device_deflation(grid)
        u, info = grid.dpcg(K.s, b, dd, rtol=rtol, max_iters=maxIters, stop_rule=1)
        self.last_info = info
        if verbose and info.converged:
            print(f"Converged in {info.iters} iterations")
        if not info.converged:
            print("Warning: Maximum iterations reached in DPCG; relative residual:", info.rel_res)
        return u
