"""Box-grid mesher with PyTO's numbering (drop-in for HexMesher.grid_mesh).

The GPU kernels never read connectivity arrays: node, element and DOF ids are
implicit functions of the grid indices (src/hex_mesher.py:104-124,
:1080-1095).  The arrays the reference builds with Python loops
(``node_xyz``, ``elemArray``, ``edofMatStructural``, ``elemNeighborsArray``,
``elem_centers``) are still available, vectorised and bit-identical, for
callers that use them; they are materialised only on first access.
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np


@dataclasses.dataclass
class Extent:
    min: float
    max: float

    @property
    def range(self) -> float:
        return self.max - self.min

    @property
    def center(self) -> float:
        return 0.5 * (self.min + self.max)


@dataclasses.dataclass
class BoundingBox:
    x: Extent
    y: Extent
    z: Optional[Extent] = None

    @property
    def lx(self) -> float:
        return abs(self.x.range)

    @property
    def ly(self) -> float:
        return abs(self.y.range)

    @property
    def lz(self) -> float:
        return abs(self.z.range) if self.z else 0.0

    @property
    def diag_length(self) -> float:
        return float(np.sqrt(self.lx ** 2 + self.ly ** 2 + self.lz ** 2))


class HexMesher:
    """Structured voxel grid (``grid_mesh``) with an optional active-element mask."""

    def __init__(self):
        self.num_nodes = 0
        self.num_elems = 0
        self.grid = None
        self.elem_size = None
        self.origin = [0, 0, 0]
        self.active_elements = None  # bool mask (None = all active)
        self.elemPseudoDensity = None
        self._cache = {}

    def grid_mesh(self, num_elems, elem_size):
        """Grid of (nelx, nely, nelz) elements of size (dx, dy, dz) (src/hex_mesher.py:72-169)."""
        nelx, nely, nelz = (int(n) for n in num_elems)
        if min(nelx, nely, nelz) < 1:
            raise ValueError("grid needs at least one element per axis")
        self.grid = [nelx, nely, nelz]
        self.elem_size = tuple(float(h) for h in elem_size)
        self.bbox = BoundingBox(x=Extent(0.0, nelx * self.elem_size[0]), y=Extent(0.0, nely * self.elem_size[1]),
                                z=Extent(0.0, nelz * self.elem_size[2]))
        self.num_components = 1
        self.num_elems = nelx * nely * nelz
        self.num_nodes = (nelx + 1) * (nely + 1) * (nelz + 1)
        self.elemPseudoDensity = np.ones(self.num_elems)
        self.volume_error = 0.0
        self._cache = {}

    # ---- implicit numbering, materialised on demand ---------------------------
    def _ijk(self):
        if "ijk" not in self._cache:
            nx, ny, nz = self.grid
            iz, iy, ix = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
            self._cache["ijk"] = (ix.ravel(), iy.ravel(), iz.ravel())
        return self._cache["ijk"]

    @property
    def node_indices(self) -> np.ndarray:
        if "node_indices" not in self._cache:
            ix, iy, iz = self._ijk()
            self._cache["node_indices"] = np.stack([ix, iy, iz, np.zeros_like(ix)], 1).astype(np.int32)
        return self._cache["node_indices"]

    @property
    def node_xyz(self) -> np.ndarray:
        if "node_xyz" not in self._cache:
            ni = self.node_indices
            xyz = np.zeros((self.num_nodes, 3))
            for i in range(3):
                xyz[:, i] = self.origin[i] + self.elem_size[i] * ni[:, i]
            self._cache["node_xyz"] = xyz
        return self._cache["node_xyz"]

    @property
    def elemArray(self) -> np.ndarray:
        if "elemArray" not in self._cache:
            nx, ny, nz = self.grid
            sx, sy = nx + 1, ny + 1
            ez, ey, ex = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
            n0 = ez.ravel() * sx * sy + ey.ravel() * sx + ex.ravel()
            off = np.array([0, 1, 1 + sx, sx, sx * sy, 1 + sx * sy, 1 + sx + sx * sy, sx + sx * sy])
            self._cache["elemArray"] = (n0[:, None] + off[None, :]).astype(np.int32)
        return self._cache["elemArray"]

    @property
    def elem_centers(self) -> np.ndarray:
        if "elem_centers" not in self._cache:
            self._cache["elem_centers"] = np.sum(self.node_xyz[self.elemArray], axis=1) / 8.0
        return self._cache["elem_centers"]

    @property
    def elemNeighborsArray(self) -> np.ndarray:
        """27-neighbour element table with -1 outside (src/hex_mesher.py:126-151)."""
        if "nb" not in self._cache:
            nx, ny, nz = self.grid
            ne = self.num_elems
            e = np.arange(ne)
            ex, ey, ez = e % nx, (e // nx) % ny, e // (nx * ny)
            nb = np.empty((ne, 27), dtype=np.int64)
            k = 0
            for dz in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dx in (-1, 0, 1):
                        nb[:, k] = e + dz * nx * ny + dy * nx + dx
                        k += 1
            nb[ez == 0, 0:9] = -1
            nb[ez == nz - 1, 18:27] = -1
            nb[np.ix_(ey == 0, [0, 1, 2, 9, 10, 11, 18, 19, 20])] = -1
            nb[np.ix_(ey == ny - 1, [6, 7, 8, 15, 16, 17, 24, 25, 26])] = -1
            nb[np.ix_(ex == 0, [0, 3, 6, 9, 12, 15, 18, 21, 24])] = -1
            nb[np.ix_(ex == nx - 1, [2, 5, 8, 11, 14, 17, 20, 23, 26])] = -1
            nb[nb > ne - 1] = ne - 1
            self._cache["nb"] = nb.astype(np.int32)
        return self._cache["nb"]

    def createEdofMatStructural(self):
        """(nelem, 24) DOF map 3*node + {0,1,2} (src/hex_mesher.py:1080-1095)."""
        self.dofs_per_node = 3
        self.edofMatStructural = (3 * self.elemArray[:, :, None].astype(np.int64) + np.arange(3)).reshape(-1, 24)

    @property
    def edofMat(self):
        if not hasattr(self, "edofMatStructural"):
            self.createEdofMatStructural()
        return self.edofMatStructural

    def getNodesOnBoundingBoxPlane(self, axis: int, minLimit: bool) -> np.ndarray:
        """Nodes on a bounding-box plane (src/hex_mesher.py:732-760)."""
        if axis not in (0, 1, 2):
            raise ValueError("Invalid axis. Must be 0, 1, or 2.")
        col = self.node_indices[:, axis]
        return np.where(col == (0 if minLimit else self.grid[axis]))[0]

    def setPseudoDensity(self, rho):
        """Keep a copy of the densities; a device tensor stays on the device and is copied
        to the host only when ``elemPseudoDensity`` is read (the optimisation loops set it
        every iteration)."""
        if hasattr(rho, "detach"):
            self._pseudo_dev = rho.detach().clone()
            self._elemPseudoDensity = None
        else:
            self._pseudo_dev = None
            self._elemPseudoDensity = np.asarray(rho).copy()

    @property
    def elemPseudoDensity(self):
        if getattr(self, "_elemPseudoDensity", None) is None and getattr(self, "_pseudo_dev", None) is not None:
            self._elemPseudoDensity = self._pseudo_dev.cpu().numpy()
        return getattr(self, "_elemPseudoDensity", None)

    @elemPseudoDensity.setter
    def elemPseudoDensity(self, value):
        self._pseudo_dev = None
        self._elemPseudoDensity = value

    def set_active_elements(self, active):
        """Restrict the domain to a subset of the box (e.g. an L-shape); nodes touched by
        no active element must be fixed by the boundary conditions."""
        self.active_elements = None if active is None else np.asarray(active, dtype=bool).ravel().copy()

    def unused_nodes(self) -> np.ndarray:
        """Nodes that belong to no active element."""
        if self.active_elements is None:
            return np.zeros(0, dtype=np.int64)
        used = np.zeros(self.num_nodes, bool)
        used[self.elemArray[self.active_elements].ravel()] = True
        return np.where(~used)[0]
