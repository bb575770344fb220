"""Linear hat smoothing filter (drop-in for PyTO's createSmoothingFilter,
src/topopt_filters.py:8-38) as a matrix-free grid stencil on the GPU.

``createSmoothingFilter(mesh, r)`` returns ``(H, Hs)`` like the reference; H is
a ``StencilFilter`` supporting ``H @ x``, ``H * x`` (the scipy spelling) and
``H.T @ x`` (H is symmetric on a box grid), Hs the row sums.  Symmetry /
extrusion filters of the reference are outside the GPU path.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _capi as A
from .engine import HexGrid


class StencilFilter:
    """H_ij = (r - d_ij)/r for element centres within r = rel * hx."""

    def __init__(self, grid: HexGrid, rel_filter_radius: float):
        self.grid = grid
        self.rel = float(rel_filter_radius)
        self._hs = None

    @property
    def shape(self):
        return (self.grid.nelem, self.grid.nelem)

    @property
    def T(self):
        return self

    def hs(self):
        if self._hs is None:
            self._hs = self.grid.filter(self.rel, A.FILTER_HS)
        return self._hs

    def _apply(self, x, mode, w=None, hs=None):
        to_np = not isinstance(x, torch.Tensor)
        y = self.grid.filter(self.rel, mode, self.grid.tensor(x), w=None if w is None else self.grid.tensor(w),
                             hs=hs)
        return y.cpu().numpy() if to_np else y

    def __matmul__(self, x):
        return self._apply(x, A.FILTER_RAW)

    __mul__ = __matmul__

    def density(self, x):
        """rho = (H x) / Hs (src/topopt_mma.py:255-258)."""
        return self._apply(x, A.FILTER_DENSITY)

    def chain(self, g):
        """df/dx = H^T (df/drho / Hs) (src/topopt_mma.py:341-345)."""
        return self._apply(g, A.FILTER_CHAIN, hs=self.hs())

    def sensitivity(self, g, x):
        """OC sensitivity filter H (x g) / Hs / x (src/topopt_ocm.py:239)."""
        return self._apply(g, A.FILTER_SENS, w=x)

    def sum(self, axis=None):
        if axis not in (0, 1):
            raise NotImplementedError
        return self.hs().cpu().numpy()[:, None]


def grid_of(mesh) -> HexGrid:
    g = getattr(mesh, "_pyto_grid", None)
    if g is None:
        g = HexGrid(mesh.grid, mesh.elem_size)
        g.set_active(getattr(mesh, "active_elements", None))
        mesh._pyto_grid = g
    return g


def createSmoothingFilter(mesh, rel_filter_radius: float = 1.5):
    H = StencilFilter(grid_of(mesh), rel_filter_radius)
    return H, H.hs().cpu().numpy()
