"""Structural FEA object (drop-in for PyTO's HexStructuralFEA,
src/hex_structural_fea.py:18-234) with device-resident state.

``solve(x)`` scales Ke by the material model on the GPU, solves through
``linear_solvers.solve`` and keeps the displacement on the device; numpy in ->
numpy out (reference semantics), CUDA tensor in -> CUDA tensor out (no copies).
``stiff_mtrx`` is the matrix-free ``StiffnessOperator`` that the adjoint code
passes back to ``linear_solvers.solve`` (src/topopt_obj_cons_sensitivities.py:269).
"""
from __future__ import annotations

import numpy as np
import torch

from . import linear_solvers, topopt_material_model as tmm
from .engine import HexGrid
from .hex_element_stiffness import hex8_stiffness_matrix_structural, isotropic_constitutive_matrix
from .topopt_material_model import MaterialModel


def _np(t):
    return t.detach().cpu().numpy() if isinstance(t, torch.Tensor) else t


class HexStructuralFEA:
    def __init__(self, mesh, mat_prop, bc, solver, dsolver=None, elem_body_force=None, thermo_elastic_force=None,
                 **kwargs):
        if isinstance(mat_prop, list):
            if len({(m.youngs_modulus, m.poissons_ratio) for m in mat_prop}) != 1:
                raise NotImplementedError("per-element materials are outside the GPU path")
            mp = mat_prop[0]
        else:
            mp = mat_prop
        if elem_body_force is not None or thermo_elastic_force is not None:
            raise NotImplementedError("body / thermo-elastic forces are outside the GPU path")
        if getattr(mesh, "externalSprings", None) is not None:
            raise NotImplementedError("external springs are outside the GPU path")
        self.mesh, self.mat_prop, self.bc = mesh, mat_prop, bc
        self.solver, self.dsolver, self.kwargs = solver, dsolver, kwargs
        self.elem_body_force = None
        self.thermo_elastic_force = None
        self.elem_stiff = hex8_stiffness_matrix_structural(mp.youngs_modulus, mp.poissons_ratio, mesh.elem_size)[None]
        self.grid = HexGrid(mesh.grid, mesh.elem_size, mp.youngs_modulus, mp.poissons_ratio,
                            device=kwargs.get("device"))
        self.grid.set_fixed_dofs(np.asarray(bc.fixed_dofs, dtype=np.int64))
        self.grid.set_active(getattr(mesh, "active_elements", None))
        self.stiff_mtrx = None
        self.sol_dev = None
        self._sol_np = None

    @property
    def sol(self):
        if self._sol_np is None and self.sol_dev is not None:
            self._sol_np = _np(self.sol_dev)
        return self._sol_np

    def scaling(self, x, material_model=MaterialModel.SIMP):
        """Element stiffness scaling on the device (inactive elements -> 0)."""
        xd = self.grid.tensor(x)
        if material_model == MaterialModel.SIMP:
            s, _ = self.grid.simp(xd, tmm._SIMP_STRUCTURAL_PENALTY, tmm._EVOID_RELATIVE, want_ds=False)
            return s
        s = tmm.get_structural_material_model_scaling(xd, material_model)
        if self.grid.active is not None:
            s = s * self.grid.active
        return s.contiguous()

    def solve(self, x=None, material_model: MaterialModel = MaterialModel.SIMP):
        """Solve K(x) u = f (src/hex_structural_fea.py:72-149)."""
        to_np = not isinstance(x, torch.Tensor)
        if x is None:
            x = np.ones(self.mesh.num_elems)
        self.x = x
        s = self.scaling(x, material_model)
        self.elem_material_scaling = s
        self.stiff_mtrx = linear_solvers.StiffnessOperator(self.grid, s)
        self.external_force = self.bc.force
        kw = {k: v for k, v in self.kwargs.items() if k not in ("device", "warm_start")}
        if self.kwargs.get("warm_start") and self.solver == linear_solvers.Solvers.DPCG and self.sol_dev is not None:
            kw["x0"] = self.sol_dev  # the previous design's solution
        u = linear_solvers.solve(self.stiff_mtrx, self._force_device(), self.solver, self.bc,
                                 dsolver=self.dsolver, **kw)
        self.last_info = linear_solvers.solve.last_info
        self.sol_dev = u
        self._sol_np = None
        d = u.view(-1, 3)
        self.deformation_dev = torch.sqrt((d * d).sum(1))
        self.max_deformation = float(self.deformation_dev.max())
        self.solElastic = None
        self.total_force = self.external_force
        return _np(u) if to_np else u

    def _force_device(self):
        """bc.force on the device.  Copied at every solve, as the reference reads it
        (an in-place change between solves is seen); a read-only numpy array, which
        cannot change in place, is copied once and kept on the device."""
        f = self.bc.force
        if isinstance(f, torch.Tensor) or not isinstance(f, np.ndarray) or f.flags.writeable:
            return self.grid.tensor(f)
        key = (id(f), f.__array_interface__["data"][0])
        if getattr(self, "_force_key", None) != key:
            self._force_dev = self.grid.tensor(f)
            self._force_key = key
            self._force_ref = f  # keeps the keyed array alive, so its id is not reused
        return self._force_dev

    @property
    def deformation(self):
        return _np(self.deformation_dev)

    def postprocess(self, as_tensor=False):
        """Centroid strain, stress (x^q relaxation), von Mises, p-norm, strain energy
        (src/hex_structural_fea.py:152-234)."""
        out = self.grid.stress(self.sol_dev, self.grid.tensor(self.x), tmm._SIMP_STRESS_RELAXATION)
        P = tmm.get_pNorm_exponent()
        self.pNormStress = float(self.grid.pow_sum(out["vm"], P).item() ** (1.0 / P))
        conv = (lambda t: t) if as_tensor else _np
        self.strainComponents = conv(out["strain"])
        self.stressComponents = conv(out["stress"])
        self.vonMisesStress = conv(out["vm"])
        self.elemStrainEnergy = conv(out["sed"])
        self._post_dev = out

    def constitutive_matrix(self):
        mp = self.mat_prop[0] if isinstance(self.mat_prop, list) else self.mat_prop
        return isotropic_constitutive_matrix(mp.youngs_modulus, mp.poissons_ratio)
