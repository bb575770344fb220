"""Linear hat smoothing filter (drop-in for PyTO's createSmoothingFilter,
src/topopt_filters.py:8-38) as a matrix-free grid stencil on the GPU.

``createSmoothingFilter(mesh, r)`` returns ``(H, Hs)`` like the reference; H is
a ``StencilFilter`` supporting ``H @ x``, ``H * x`` (the scipy spelling) and
``H.T @ x`` (H is symmetric on a box grid), Hs the row sums.  The mirror-symmetry
and extrusion filters (createX/Y/ZSymmetryFilter, createX/Y/ZExtrudeFilter,
src/topopt_filters.py:292-393, :595-716) are element maps on the grid
(``GridMap``); ``H * HX`` composes them as the reference's sparse product does
(src/topopt_common.py:127-159), giving a ``ComposedFilter`` with the same
methods.  The angular-symmetry filters rotate element centres about a
coordinate axis through the origin; on a grid mesh (origin at a corner) the
rotated centres leave the grid, so they stay outside the GPU path.
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
        if isinstance(x, (GridMap, ComposedFilter)):
            return ComposedFilter(self, x)
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


class GridMap:
    """A symmetric element map F of a full box grid: mirror symmetry or the reference's
    extrusion average along an axis (pyto_symmetry_filter)."""

    def __init__(self, grid: HexGrid, kind: int, axis: int):
        if grid.active is not None:
            raise NotImplementedError("symmetry / extrusion filters need a full box grid (no active mask)")
        self.grid, self.kind, self.axis = grid, int(kind), int(axis)

    @property
    def shape(self):
        return (self.grid.nelem, self.grid.nelem)

    @property
    def T(self):
        return self

    def apply(self, x, pre=None, post=None, out=None):
        g = self.grid
        y = out if out is not None else torch.empty(g.nelem, dtype=torch.float64, device=g.device)
        A.call("pyto_symmetry_filter", g.opp, self.kind, self.axis, A.ptr(x), A.ptr(pre), A.ptr(post), A.ptr(y),
               g._st())
        return y

    def __matmul__(self, x):
        if isinstance(x, (GridMap, ComposedFilter)):
            return ComposedFilter(None, self, x)
        to_np = not isinstance(x, torch.Tensor)
        y = self.apply(self.grid.tensor(x))
        return y.cpu().numpy() if to_np else y

    __mul__ = __matmul__


class ComposedFilter:
    """H = H_s F_1 F_2 ... F_k (H_s the smoothing stencil, or none), applied right to
    left: H x = H_s(F_1(...F_k x)); H^T = F_k ... F_1 H_s (every factor is symmetric)."""

    def __init__(self, stencil, *maps):
        flat = []
        for m in maps:
            if isinstance(m, ComposedFilter):
                if m.stencil is not None:
                    raise NotImplementedError("a smoothing stencil only as the leftmost factor")
                flat.extend(m.maps)
            else:
                flat.append(m)
        self.stencil, self.maps = stencil, flat
        self.grid = stencil.grid if stencil is not None else flat[0].grid
        self._hs = None
        self._T = None

    @property
    def shape(self):
        return (self.grid.nelem, self.grid.nelem)

    def __matmul__(self, x):
        if isinstance(x, (GridMap, ComposedFilter)):
            return ComposedFilter(self.stencil, *self.maps, x)
        to_np = not isinstance(x, torch.Tensor)
        y = self._forward(self.grid.tensor(x))
        return y.cpu().numpy() if to_np else y

    __mul__ = __matmul__

    def _maps(self, v, pre=None, reverse=False):
        for i, m in enumerate(reversed(self.maps) if not reverse else self.maps):
            v = m.apply(v, pre=pre if i == 0 else None)
        return v

    def _smooth(self, v):
        if self.stencil is None:
            return v
        return self.grid.filter(self.stencil.rel, A.FILTER_RAW, v)

    def _forward(self, v, pre=None):
        if not self.maps:
            return self._smooth(v)
        return self._smooth(self._maps(v, pre))

    def _scale(self, x, mul=None, div1=None, div2=None):
        y = torch.empty_like(x)
        A.call("pyto_vec_scale", int(x.numel()), A.ptr(x), A.ptr(mul), A.ptr(div1), A.ptr(div2), A.ptr(y),
               self.grid._st())
        return y

    def hs(self):
        """Row sums H 1 (src/topopt_common.py:158)."""
        if self._hs is None:
            self._hs = self._forward(torch.ones(self.grid.nelem, dtype=torch.float64, device=self.grid.device))
        return self._hs

    def sum(self, axis=None):
        if axis not in (0, 1):
            raise NotImplementedError
        return self.hs().cpu().numpy()[:, None]

    @property
    def T(self):
        if self._T is None:
            self._T = _TransposedFilter(self)
        return self._T

    def _io(self, x):
        return (not isinstance(x, torch.Tensor)), self.grid.tensor(x)

    def density(self, x):
        """rho = (H x) / Hs (src/topopt_mma.py:255-258)."""
        to_np, xd = self._io(x)
        y = self._scale(self._forward(xd), div1=self.hs())
        return y.cpu().numpy() if to_np else y

    def chain(self, g):
        """df/dx = H^T (df/drho / Hs) (src/topopt_mma.py:341-345)."""
        to_np, gd = self._io(g)
        v = self._smooth(self._scale(gd, div1=self.hs()))
        y = self._maps(v, reverse=True) if self.maps else v
        return y.cpu().numpy() if to_np else y

    def sensitivity(self, g, x):
        """OC sensitivity filter H (x g) / Hs / x (src/topopt_ocm.py:239)."""
        to_np, gd = self._io(g)
        xd = self.grid.tensor(x)
        t = self._forward(gd, pre=xd) if self.maps else self._smooth(self._scale(gd, mul=xd))
        y = self._scale(t, div1=self.hs(), div2=xd)
        return y.cpu().numpy() if to_np else y


class _TransposedFilter:
    def __init__(self, f: ComposedFilter):
        self.f = f

    def __matmul__(self, x):
        to_np, xd = self.f._io(x)
        v = self.f._smooth(xd)
        y = self.f._maps(v, reverse=True) if self.f.maps else v
        return y.cpu().numpy() if to_np else y

    __mul__ = __matmul__


def _map(mesh, kind, axis):
    return GridMap(grid_of(mesh), kind, axis)


def createXSymmetryFilter(mesh):
    """Mirror symmetry about the X mid-plane (src/topopt_filters.py:292-327)."""
    return _map(mesh, A.SYM_MIRROR, 0)


def createYSymmetryFilter(mesh):
    """Mirror symmetry about the Y mid-plane (src/topopt_filters.py:329-360)."""
    return _map(mesh, A.SYM_MIRROR, 1)


def createZSymmetryFilter(mesh):
    """Mirror symmetry about the Z mid-plane (src/topopt_filters.py:362-393)."""
    return _map(mesh, A.SYM_MIRROR, 2)


def createXExtrudeFilter(mesh):
    """Extrusion through X (src/topopt_filters.py:595-634)."""
    return _map(mesh, A.SYM_EXTRUDE, 0)


def createYExtrudeFilter(mesh):
    """Extrusion through Y (src/topopt_filters.py:635-675)."""
    return _map(mesh, A.SYM_EXTRUDE, 1)


def createZExtrudeFilter(mesh):
    """Extrusion through Z (src/topopt_filters.py:676-716)."""
    return _map(mesh, A.SYM_EXTRUDE, 2)


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
