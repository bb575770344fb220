"""Thermal FEA object (drop-in for PyTO's HexThermalFEA, src/hex_thermal_fea.py:19-117)
on the device: one temperature DOF per node (DOF = node id, src/hex_mesher.py:1120-1133).

``solve(x, material_model)`` scales the 8x8 conduction Ke by the thermal material
model, solves through ``linear_solvers.solve`` with the matrix-free
``ThermalOperator`` and keeps the temperature on the device; numpy in -> numpy
out, CUDA tensor in -> tensor out.  Every solver choice runs the GPU Jacobi PCG
(the direct solvers to rtol 1e-12).
"""
from __future__ import annotations

import numpy as np
import torch

from . import linear_solvers, topopt_material_model as tmm
from .engine import ThermalGrid
from .topopt_material_model import MaterialModel


def _np(t):
    return t.detach().cpu().numpy() if isinstance(t, torch.Tensor) else t


def hex8_stiffness_matrix_thermal(thermal_conductivity, elem_size):
    """8x8 conduction Ke of a box hex8 (src/hex_element_stiffness.py:340-385)."""
    import ctypes as C
    from . import _capi as A
    ke = np.zeros(64)
    A.call("pyto_ke_hex8_thermal", float(thermal_conductivity), float(elem_size[0]), float(elem_size[1]),
           float(elem_size[2]), ke.ctypes.data_as(C.c_void_p))
    return ke.reshape(8, 8)


class HexThermalFEA:
    def __init__(self, mesh, mat_prop, bc, solver, dsolver=None, elem_body_force=None,
                 thermoElasticReferenceTemperature=23.0, **kwargs):
        if isinstance(mat_prop, list):
            if len({m.thermal_conductivity for m in mat_prop}) != 1:
                raise NotImplementedError("per-element materials are outside the GPU path")
            mp = mat_prop[0]
        else:
            mp = mat_prop
        if elem_body_force is not None:
            raise NotImplementedError("element body heat sources are outside the GPU path")
        self.mesh, self.mat_prop, self.bc = mesh, mat_prop, bc
        self.solver, self.dsolver, self.kwargs = solver, dsolver, kwargs
        self.thermoElasticReferenceTemperature = thermoElasticReferenceTemperature
        self.elem_body_force = None
        self.elem_stiff = hex8_stiffness_matrix_thermal(mp.thermal_conductivity, mesh.elem_size)[None]
        self.grid = ThermalGrid(mesh.grid, mesh.elem_size, mp.thermal_conductivity, device=kwargs.get("device"))
        self.grid.set_fixed_nodes(np.asarray(bc.fixed_dofs, dtype=np.int64))
        self.stiff_mtrx = None
        self.sol_dev = None
        self._sol_np = None

    @property
    def sol(self):
        if self._sol_np is None and self.sol_dev is not None:
            self._sol_np = _np(self.sol_dev)
        return self._sol_np

    def scaling(self, x, material_model=None):
        """Conductivity scaling on the device (src/topopt_material_model.py:98-117)."""
        xd = self.grid.tensor(x)
        if material_model == MaterialModel.SIMP:
            s, _ = self.grid.simp(xd, tmm._SIMP_THERMAL_PENALTY, tmm._KVOID_RELATIVE, want_ds=False)
            return s
        return tmm.get_thermal_material_model_scaling(xd, material_model).contiguous()

    def solve(self, x=None, material_model: MaterialModel = None, elem_mat_id=None):
        """Solve K(x) T = q (src/hex_thermal_fea.py:69-117)."""
        to_np = not isinstance(x, torch.Tensor)
        if x is None:
            x = np.ones(self.mesh.num_elems)
        self.x = x
        s = self.scaling(x, material_model)
        self.elem_material_scaling = s
        self.stiff_mtrx = linear_solvers.ThermalOperator(self.grid, s)
        kw = {k: v for k, v in self.kwargs.items() if k != "device"}
        u = linear_solvers.solve(self.stiff_mtrx, self.grid.tensor(self.bc.force), self.solver, self.bc,
                                 dsolver=self.dsolver, **kw)
        self.last_info = linear_solvers.solve.last_info
        self.sol_dev = u
        self._sol_np = None
        return _np(u) if to_np else u
