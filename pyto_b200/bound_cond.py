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
    """Dirichlet elimination (src/bound_cond.py:40-70): b - A[:, fixed] g, then the
    free rows (and, for an assembled matrix, the free columns).

    ``A`` may be PyTO's assembled scipy matrix -- the reference's elimination, returning
    (A[free][:, free], b[free]) -- or this library's matrix-free operator
    (``linear_solvers.StiffnessOperator``): the lift A[:, fixed] g is one masked operator
    application on the GPU, and the operator is returned unchanged (the GPU solvers
    eliminate the fixed DOFs by masking full-length vectors), with b[free] as a device
    tensor.  Constraint-matrix BCs raise NotImplementedError, as in the reference."""
    if bc.constraint_matrix is not None:
        raise NotImplementedError("impose_dirichlet_bc not implemented for constraint_matrix BCs; "
                                  "see linear_solvers.solve")
    fixed = np.asarray(bc.fixed_dofs, dtype=np.int64)
    free = bc.free_dofs
    g = np.zeros(np.shape(b)[0]) if bc.dirichlet_values is None else np.asarray(bc.dirichlet_values, dtype=float)
    if getattr(A, "is_pyto_operator", False):
        import torch

        from . import _capi
        grid = A.grid
        bd = grid.tensor(b)
        if g.size and np.any(g != 0):
            lift = torch.zeros(grid.ndof, dtype=torch.float64, device=grid.device)
            lift[grid.tensor(fixed, torch.int64)] = grid.tensor(np.broadcast_to(g, fixed.shape).astype(np.float64))
            bd = bd - grid.matvec(A.s, lift, mode=_capi.MASK_OUT)
        return A, bd[grid.tensor(free, torch.int64)]
    b_mod = np.array(b, dtype=float, copy=True)
    if g.size and np.any(g != 0):
        b_mod -= A[:, fixed] @ np.broadcast_to(g, fixed.shape)
    A_mod = A.tocsr()[free, :][:, free]
    return A_mod, b_mod[free]
