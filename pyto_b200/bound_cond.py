"""Boundary conditions (drop-in for PyTO's bound_cond, src/bound_cond.py:9-70).

On the GPU the fixed DOFs become a per-node 3-bit mask (``pyto_bc_mask``) and
elimination is masking of full-length vectors; the dataclass keeps the
reference's fields and properties.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class BC:
    force: np.ndarray
    fixed_dofs: np.ndarray
    dirichlet_values: np.ndarray
    constraint_matrix: np.ndarray = None
    constraint_rhs: np.ndarray = None

    @property
    def num_dofs(self) -> int:
        return self.force.shape[0]

    @property
    def free_dofs(self) -> np.ndarray:
        return np.setdiff1d(np.arange(self.num_dofs), np.asarray(self.fixed_dofs))

    def set_force(self, force: np.ndarray):
        self.force = force


def impose_dirichlet_bc(A, b, bc: BC):
    """The reference's row/column elimination has no matrix to act on here: the
    GPU operator is matrix-free and masks fixed DOFs (src/bound_cond.py:40-70)."""
    if bc.constraint_matrix is not None:
        raise NotImplementedError("impose_dirichlet_bc not implemented for constraint_matrix BCs; "
                                  "see linear_solvers.solve")
    raise NotImplementedError("pyto_b200 eliminates Dirichlet DOFs by masking inside the GPU solvers; "
                              "use linear_solvers.solve with fe_solver.stiff_mtrx")
