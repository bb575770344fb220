"""Differentiable structural objectives of the voxel hex8 path.

``StructuralObjectives`` is a ``torch.autograd.Function`` mapping element
densities x to (compliance, p-norm von Mises stress).  Its backward pass is
written by hand, following the reference sensitivities
(src/topopt_obj_cons_sensitivities.py:148-179 for compliance and 181-287 for the
p-norm adjoint):

* dC/dx_e = -ds_e/dx_e * u_e^T Ke u_e (self-adjoint, no extra solve);
* dPN/dx = T1 + T2, where T1 is the explicit term through the stress relaxation
  x^q (pyto_pnorm_adjoint), and T2 = -ds_e/dx_e * lam_e^T Ke u_e with the adjoint
  lam = K^-1 g, g = dPN/du, solved by the same solver as the forward problem.

With ``recompute=True`` the forward keeps only x and the backward solves for u
again (the state of a large grid is not held between forward and backward).
Every operation runs in libpyto_b200 on the GPU; torch provides tensors only.
"""
from __future__ import annotations

import torch

from .engine import DeviceDeflation, HexGrid

F64 = torch.float64


class HexProblem:
    """Grid, load, SIMP parameters and solver of a differentiable structural problem.

    solver: "pcg" (Jacobi PCG), "dpcg" (deflated PCG, FP64, with FP64 residual replacement) or "mixed" (deflated PCG
    with FP32 recurrence and FP64 residual updates); the deflated solvers need
    ``defl`` (a DeviceDeflation of ``grid``)."""

    def __init__(self, grid: HexGrid, force, penal=3.0, emin=1e-9, q=0.5, P=8.0, solver="dpcg",
                 defl: DeviceDeflation | None = None, rtol=1e-10, max_iters=20000, recompute=False):
        if solver not in ("pcg", "dpcg", "mixed"):
            raise ValueError(f"unknown solver {solver!r}")
        if solver != "pcg" and defl is None:
            raise ValueError("deflated solvers need a DeviceDeflation")
        self.grid = grid
        self.f = grid.tensor(force)
        self.penal, self.emin, self.q, self.P = float(penal), float(emin), float(q), float(P)
        self.solver, self.defl, self.rtol, self.max_iters = solver, defl, float(rtol), int(max_iters)
        self.recompute = bool(recompute)
        self.last_info = None

    def scale(self, x):
        """SIMP scaling s = emin + x^p (1 - emin) and ds/dx (inactive elements 0)."""
        return self.grid.simp(x, self.penal, self.emin)

    def solve(self, s, b=None):
        """u with K(s) u = b on the free DOFs (b defaults to the load)."""
        b = self.f if b is None else b
        g = self.grid
        if self.solver == "pcg":
            u, info = g.pcg(s, b, rtol=self.rtol, max_iters=self.max_iters)
        elif self.solver == "dpcg":
            u, info = g.dpcg(s, b, self.defl, rtol=self.rtol, max_iters=self.max_iters, stop_rule=2)
        else:
            u, info = g.dpcg_mixed(s, b, self.defl, rtol=self.rtol, max_iters=self.max_iters)
        if not info.converged:
            raise RuntimeError(f"structural solve did not converge: {info}")
        self.last_info = info
        return u

    def pnorm_parts(self, u, x):
        """von Mises stresses (relaxed by x^q) and S = sum vm^P (device scalar)."""
        vm = self.grid.stress(u, x, self.q, want=("vm",))["vm"]
        return vm, self.grid.pow_sum(vm, self.P)


class StructuralObjectives(torch.autograd.Function):
    """x -> (C, PN): compliance sum_e s_e u_e^T Ke u_e and p-norm von Mises stress
    (sum_e vm_e^P)^(1/P), with hand-written gradients."""

    @staticmethod
    def forward(ctx, x, prob: HexProblem):
        xd = prob.grid.tensor(x)
        s, ds = prob.scale(xd)
        u = prob.solve(s)
        _, C = prob.grid.energy(u, s=s)
        _, S = prob.pnorm_parts(u, xd)
        pn = S ** (1.0 / prob.P)
        ctx.prob = prob
        ctx.save_for_backward(xd)
        ctx.state = None if prob.recompute else (s, ds, u, S)
        return C.reshape(()).clone(), pn.reshape(()).clone()

    @staticmethod
    def backward(ctx, gC, gPN):
        prob = ctx.prob
        (xd,) = ctx.saved_tensors
        g = prob.grid
        if ctx.state is None:  # recompute the forward state
            s, ds = prob.scale(xd)
            u = prob.solve(s)
            _, S = prob.pnorm_parts(u, xd)
        else:
            s, ds, u, S = ctx.state
        grad = torch.zeros_like(xd)
        if gC is not None and bool(gC != 0):
            grad = grad - gC * ds * g.energy(u)
        if gPN is not None and bool(gPN != 0):
            dpn = (S ** (1.0 / prob.P - 1.0)).reshape(1).contiguous()
            T1, gvec = g.pnorm_adjoint(u, xd, prob.q, prob.P, dpn)
            lam = prob.solve(s, gvec)
            _, dsc = prob.scale(torch.clamp(xd, min=1e-12))
            T2 = -dsc * g.energy(lam, u)
            grad = grad + gPN * (T1 + T2)
        if g.active is not None:
            grad = grad * g.active.to(grad.dtype)
        return grad, None


def structural_objectives(x, prob: HexProblem):
    """(compliance, p-norm von Mises stress) of densities x, differentiable in x."""
    return StructuralObjectives.apply(x, prob)


def compliance(x, prob: HexProblem):
    return StructuralObjectives.apply(x, prob)[0]


def pnorm_stress(x, prob: HexProblem):
    return StructuralObjectives.apply(x, prob)[1]
