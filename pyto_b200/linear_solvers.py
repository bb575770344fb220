"""Linear-solver dispatch (drop-in for PyTO's linear_solvers,
src/linear_solvers.py:126-225) over the matrix-free GPU operator.

``solve(A0, b0, solver, bc, **kwargs)`` keeps the reference's signature and
result (full-length u with u[fixed] = dirichlet_values).  ``A0`` is the
``StiffnessOperator`` that ``HexStructuralFEA.solve`` leaves in
``fe_solver.stiff_mtrx``; a scipy matrix is refused (no CPU path exists).
Solvers: PCG -> Jacobi PCG, stop on ||r|| < rtol ||b|| (scipy cg semantics);
DPCG -> aggregation-deflated PCG, stop on sqrt(r.z / r0.z0) <= rtol
(src/deflation.py:567).  The reference's direct solvers (SPSOLVE, SPLU,
PARDISO, PETSC) and PYAMG are served by a Jacobi PCG to rtol 1e-12 on the GPU.
"""
from __future__ import annotations

import enum

import numpy as np
import torch

from . import _capi as A
from ._enum import NamedEnum

DEFAULT_TOL = 1.0e-6


class Preconditioners(NamedEnum):
    JACOBI = enum.auto()
    ILU = enum.auto()


class Solvers(NamedEnum):
    SPSOLVE = enum.auto()
    PCG = enum.auto()
    PYAMG = enum.auto()
    DPCG = enum.auto()
    PARDISO = enum.auto()
    SPLU = enum.auto()
    PETSC = enum.auto()


class SolverError(RuntimeError):
    """Raised when a solve breaks down or does not converge (strict mode)."""


class StiffnessOperator:
    """K(s) = sum_e s_e Ke on a HexGrid, applied matrix-free on the GPU."""

    #: marks this library's operator for a PyTO linear_solvers.solve that dispatches here
    is_pyto_operator = True

    def __init__(self, grid, s):
        self.grid = grid
        self.s = s

    @property
    def shape(self):
        return (self.grid.ndof, self.grid.ndof)

    def __matmul__(self, u):
        """Unmasked K u (full operator, like the assembled reference matrix)."""
        to_np = not isinstance(u, torch.Tensor)
        y = self.grid.matvec(self.s, self.grid.tensor(u), mode=0)
        return y.cpu().numpy() if to_np else y

    def diagonal(self):
        diag, _ = self.grid.jacobi(self.s)
        return diag

    def tocsr(self):
        raise TypeError("pyto_b200 operators are matrix-free; no assembled matrix exists")


class ThermalOperator(StiffnessOperator):
    """K(s) = sum_e s_e Ke of the thermal path (8x8 Ke, one DOF per node) on a
    ThermalGrid, applied matrix-free on the GPU."""

    def diagonal(self):
        """diag K = Ke[a][a] sum_{e ni n} s_e; the node sums come from the operator with
        Ke replaced by the all-ones matrix / 8, applied to a vector of ones."""
        from .engine import ThermalGrid
        g = self.grid
        ones = ThermalGrid(g.nel, g.h, 1.0, ke=np.full((8, 8), 0.125), device=g.device)
        sums = ones.matvec(self.s, torch.ones(g.ndof, dtype=torch.float64, device=g.device), mode=0)
        return float(g.th.kxor[0]) * sums


def _prepare_rhs(A0: StiffnessOperator, b0, bc):
    g = A0.grid
    b = g.tensor(b0)
    dv = getattr(bc, "dirichlet_values", None)
    lift = None
    if dv is not None and np.size(dv) and np.any(np.asarray(dv) != 0):
        lift = torch.zeros(g.ndof, dtype=torch.float64, device=g.device)
        lift[g.tensor(np.asarray(bc.fixed_dofs), torch.int64)] = g.tensor(np.asarray(dv, dtype=np.float64))
        b = b - g.matvec(A0.s, lift, mode=A.MASK_OUT)
    return b, lift


def solve(A0, b0, solver: Solvers, bc, **kwargs):
    """Solve K u = b with Dirichlet conditions of bc (src/linear_solvers.py:136-202)."""
    if not isinstance(A0, StiffnessOperator):
        raise TypeError("linear_solvers.solve expects the GPU StiffnessOperator (fe_solver.stiff_mtrx)")
    if getattr(bc, "constraint_matrix", None) is not None:
        raise ValueError("Only Pardiso and DPCG solvers support Lagrange multipliers currently.")
    g = A0.grid
    to_np = not isinstance(b0, torch.Tensor)
    b, lift = _prepare_rhs(A0, b0, bc)
    rtol = kwargs.get("rtol", DEFAULT_TOL)
    strict = kwargs.get("strict", False)
    if isinstance(A0, ThermalOperator):
        # the thermal path has the Jacobi PCG only; the direct solvers run it to 1e-12
        if solver not in tuple(Solvers):
            raise ValueError("Unknown solver type")
        tol = rtol if solver in (Solvers.PCG, Solvers.DPCG, Solvers.PYAMG) else min(rtol, 1e-12)
        u, info = g.pcg(A0.s, b, rtol=tol, max_iters=kwargs.get("maxiter", 10 * g.ndof), stop_rule=0)
    elif solver == Solvers.PCG:
        u, info = g.pcg(A0.s, b, rtol=rtol, max_iters=kwargs.get("maxiter", 10 * g.ndof), stop_rule=0)
    elif solver == Solvers.DPCG:
        dsolver = kwargs["dsolver"]
        dd = dsolver.device_deflation(g)
        # stop_rule 2 (default): the reference's recurrence with FP64 residual replacement
        # and the true residual as the stopping test; the plain recurrence (stop_rule=1,
        # PyTO's sqrt(r.z / r0.z0) test) drifts and can diverge on high-contrast designs,
        # where the reference only warns and returns the last iterate
        # (src/deflation.py:582-583).  precision="mixed": FP32 recurrence, FP64 residual.
        # x0: a warm start (e.g. the previous design's solution; residual-replacement forms only)
        x0 = kwargs.get("x0")
        if x0 is not None:  # the free part of a full solution: prescribed values are added back below
            x0 = g.tensor(x0) if lift is None else g.tensor(x0) - lift
        if kwargs.get("precision", "fp64") == "mixed":
            u, info = g.dpcg_mixed(A0.s, b, dd, rtol=rtol, max_iters=kwargs.get("maxIters", 4000), x0=x0)
        else:
            u, info = g.dpcg(A0.s, b, dd, rtol=rtol, max_iters=kwargs.get("maxIters", 4000),
                             stop_rule=kwargs.get("stop_rule", 2), x0=x0)
        dsolver.last_info = info
    elif solver in (Solvers.SPSOLVE, Solvers.SPLU, Solvers.PARDISO, Solvers.PETSC, Solvers.PYAMG):
        tol = rtol if solver == Solvers.PYAMG else min(rtol, 1e-12)
        u, info = g.pcg(A0.s, b, rtol=tol, max_iters=10 * g.ndof, stop_rule=0)
    else:
        raise ValueError("Unknown solver type")
    solve.last_info = info
    if info.breakdown or (strict and not info.converged):
        raise SolverError(f"{solver.name} did not converge: {info}")
    if lift is not None:
        u = u + lift
    return u.cpu().numpy() if to_np else u


solve.last_info = None
