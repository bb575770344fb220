"""Objectives, constraints and sensitivities of the hex8 path (drop-in for
PyTO's topopt_obj_cons_sensitivities, src/topopt_obj_cons_sensitivities.py).

All element work runs on the GPU (``pyto_elem_energy``, ``pyto_stress``,
``pyto_pnorm_adjoint``); adjoint solves go through ``linear_solvers.solve``
with the FEA object's operator, solver and boundary conditions, as in the
reference (:269-274, :302-307).  numpy x in -> numpy gradient out; CUDA
tensor in -> tensor out.
"""
from __future__ import annotations

import numpy as np
import torch

from . import linear_solvers
from . import topopt_material_model as tmm
from .engine import HexGrid
from .topopt_common import FEA_MODE, TO_QOI

stress_scaling = 1.0


def _out(t, like):
    return t if isinstance(like, torch.Tensor) else t.detach().cpu().numpy()


def _grid(fe_solver, KE) -> HexGrid:
    g = fe_solver.grid
    if KE is None or np.allclose(np.asarray(KE), fe_solver.elem_stiff[0], rtol=1e-14, atol=0):
        return g
    cache = fe_solver.__dict__.setdefault("_ke_grids", {})
    key = np.asarray(KE).tobytes()
    if key not in cache:
        gg = HexGrid(g.nel, g.h, g.op.E, g.op.nu, ke=np.asarray(KE), device=g.device)
        gg.mask.copy_(g.mask)
        gg.active, gg.n_active = g.active, g.n_active
        cache[key] = gg
    return cache[key]


def _u(fe_solver, sol):
    if fe_solver.sol_dev is not None and (sol is fe_solver.sol_dev or sol is fe_solver._sol_np):
        return fe_solver.sol_dev
    return fe_solver.grid.tensor(sol)


def _scale(g, xd, material_model):
    if material_model == tmm.MaterialModel.SIMP:
        return g.simp(xd, tmm._SIMP_STRUCTURAL_PENALTY, tmm._EVOID_RELATIVE)
    s = tmm.get_structural_material_model_scaling(xd, material_model)
    ds = tmm.get_structural_material_model_sensitivity(xd, material_model)
    if g.active is not None:
        s, ds = s * g.active, ds * g.active
    return s.contiguous(), ds.contiguous()


def compute_compliance(sol, x, fe_solver, KE, material_model):
    """C = sum_e s_e u_e^T Ke u_e (src/topopt_obj_cons_sensitivities.py:118-145)."""
    g = _grid(fe_solver, KE)
    s, _ = _scale(g, g.tensor(x), material_model)
    _, C = g.energy(_u(fe_solver, sol), s=s)
    return float(C.item())


def _thermal_compliance_and_gradient(sol, x, fe_solver, KE, material_model):
    """Thermal branch: C = sum_e s_e T_e^T Ke T_e, dC = -ds T_e^T Ke T_e with the
    conductivity scaling (src/topopt_obj_cons_sensitivities.py:162-175)."""
    g = fe_solver.grid
    if KE is not None and not np.allclose(np.asarray(KE), fe_solver.elem_stiff[0], rtol=1e-14, atol=0):
        raise NotImplementedError("the thermal path uses the FEA object's own element matrix")
    u = fe_solver.sol_dev if (fe_solver.sol_dev is not None and (sol is fe_solver.sol_dev or sol is fe_solver._sol_np)) \
        else g.tensor(sol)
    xd = g.tensor(x)
    if material_model == tmm.MaterialModel.SIMP:
        s, ds = g.simp(xd, tmm._SIMP_THERMAL_PENALTY, tmm._KVOID_RELATIVE)
    else:
        s = tmm.get_thermal_material_model_scaling(xd, material_model).contiguous()
        ds = tmm.get_thermal_material_model_sensitivity(xd, material_model).contiguous()
    ce, C = g.energy(u, s=s)
    return float(C.item()), _out(-ds * ce, x)


def compute_compliance_and_gradient(feaMode, sol, x, fe_solver, KE, material_model):
    """(C, dC/dx = -ds u_e^T Ke u_e) (src/topopt_obj_cons_sensitivities.py:148-179)."""
    if feaMode == FEA_MODE.THERMAL:
        return _thermal_compliance_and_gradient(sol, x, fe_solver, KE, material_model)
    if feaMode != FEA_MODE.STRUCTURAL:
        raise NotImplementedError("only the structural and thermal modes are on the GPU path")
    g = _grid(fe_solver, KE)
    s, ds = _scale(g, g.tensor(x), material_model)
    ce, C = g.energy(_u(fe_solver, sol), s=s)
    return float(C.item()), _out(-ds * ce, x)


def compute_volume_constraint_and_gradient(x, volfracUpper):
    """(mean(x)/V - 1, 1/V/n) (src/topopt_obj_cons_sensitivities.py:100-116)."""
    if isinstance(x, torch.Tensor):
        return float(x.mean()) / volfracUpper - 1.0, torch.ones_like(x) / volfracUpper / x.numel()
    return (np.mean(x) / volfracUpper) - 1.0, np.ones_like(x) / volfracUpper / x.size


def compute_pnorm_stress_and_sensitivity(sol, x, fe_solver, KE, material_model):
    """p-norm von Mises and its adjoint sensitivity T1 + T2
    (src/topopt_obj_cons_sensitivities.py:181-287); x is clamped below at 1e-12
    for the sensitivity terms as in the reference.  Returns (pnorm, grad, max vm)."""
    g = _grid(fe_solver, KE)
    u = _u(fe_solver, sol)
    xd = g.tensor(x)
    q, P = tmm._SIMP_STRESS_RELAXATION, float(tmm.get_pNorm_exponent())
    vm = g.stress(u, xd, q, want=("vm",))["vm"]
    ssum = g.pow_sum(vm, P).clone()
    dpn = (ssum ** (1.0 / P - 1.0)).contiguous()
    T1, gvec = g.pnorm_adjoint(u, xd, q, P, dpn)
    lam = linear_solvers.solve(fe_solver.stiff_mtrx, gvec, fe_solver.solver, fe_solver.bc,
                               dsolver=fe_solver.dsolver, **{k: v for k, v in fe_solver.kwargs.items()
                                                             if k != "device"})
    xc = torch.clamp(xd, min=1e-12)
    _, dsc = _scale(g, xc, material_model)
    T2 = -dsc * g.energy(lam, u)
    pn = float(ssum.item() ** (1.0 / P))
    return pn, _out(T1 + T2, x), float(vm.max())


def compute_solution_dotproduct_and_gradient(sol, x, fe_solver, KE, material_model, g):
    """obj = u.g, gradient via lam = -K^-1 g (src/topopt_obj_cons_sensitivities.py:289-319)."""
    gr = _grid(fe_solver, KE)
    u = _u(fe_solver, sol)
    gd = gr.tensor(g)
    obj = float(torch.dot(u, gd))
    lam = -linear_solvers.solve(fe_solver.stiff_mtrx, gd, fe_solver.solver, fe_solver.bc,
                                dsolver=fe_solver.dsolver, **{k: v for k, v in fe_solver.kwargs.items()
                                                              if k != "device"})
    _, ds = _scale(gr, gr.tensor(x), material_model)
    return obj, _out(ds * gr.energy(lam, u), x)


def compute_objective_and_gradient(feaMode, to_params, sol, x, fe_solver, KE):
    """Objective dispatch (src/topopt_obj_cons_sensitivities.py:11-40)."""
    kind, opt = to_params.Objective[0], to_params.Objective[1]
    mm = to_params.materialModel
    if kind == TO_QOI.COMPLIANCE:
        return compute_compliance_and_gradient(feaMode, sol, x, fe_solver, KE, mm)
    if kind == TO_QOI.VOLUME_FRACTION:
        n = x.numel() if isinstance(x, torch.Tensor) else x.size
        return (float(x.mean()) if isinstance(x, torch.Tensor) else np.mean(x)), (x * 0 + 1) / n
    if kind == TO_QOI.MASS:
        ev = float(np.prod(fe_solver.mesh.elem_size))
        rho = fe_solver.mat_prop.mass_density
        return float((x * ev * rho).sum()), x * 0 + ev * rho
    if kind == TO_QOI.PNORM_STRESS:
        pn, dpn, _ = compute_pnorm_stress_and_sensitivity(sol, x, fe_solver, KE, mm)
        return pn, dpn
    if kind == TO_QOI.MAX_VONMISES_STRESS:
        pn, dpn, mvm = compute_pnorm_stress_and_sensitivity(sol, x, fe_solver, KE, mm)
        return mvm, dpn
    if kind == TO_QOI.GVECTOR:
        return compute_solution_dotproduct_and_gradient(sol, x, fe_solver, KE, mm, opt)
    raise NotImplementedError(f"Objective {kind} is not implemented yet.")


def compute_constraint_and_gradient(feaMode, to_params, sol, x, fe_solver, KE):
    """Constraint dispatch with the adaptive stress scaling of
    src/topopt_obj_cons_sensitivities.py:43-96."""
    n = len(to_params.Constraints)
    nx = x.numel() if isinstance(x, torch.Tensor) else x.size
    c = np.zeros((n, 1))
    dc = np.zeros((n, nx))
    mm = to_params.materialModel
    for m, (kind, opt, lim) in enumerate(to_params.Constraints):
        if kind == TO_QOI.COMPLIANCE:
            C, dC = compute_compliance_and_gradient(feaMode, sol, x, fe_solver, KE, mm)
            c[m, 0], dc[m] = C / lim - 1.0, np.asarray(_out(torch.as_tensor(dC), np.zeros(0))) / lim
        elif kind == TO_QOI.VOLUME_FRACTION:
            v, dv = compute_volume_constraint_and_gradient(x, lim)
            c[m, 0], dc[m] = v, np.asarray(dv.cpu() if isinstance(dv, torch.Tensor) else dv)
        elif kind in (TO_QOI.PNORM_STRESS, TO_QOI.MAX_VONMISES_STRESS, TO_QOI.STRESS_FAILURE_FACTOR):
            pn, dpn, mvm = compute_pnorm_stress_and_sensitivity(sol, x, fe_solver, KE, mm)
            dpn = np.asarray(dpn.cpu() if isinstance(dpn, torch.Tensor) else dpn)
            if kind == TO_QOI.PNORM_STRESS:
                c[m, 0], dc[m] = pn / lim - 1.0, dpn / lim
            else:
                sc = compute_constraint_and_gradient.stress_scaling
                ys = fe_solver.mat_prop.yield_strength if kind == TO_QOI.STRESS_FAILURE_FACTOR else 1.0
                c[m, 0] = sc * pn / ys / lim - 1.0
                dc[m] = sc * dpn / ys / lim
                compute_constraint_and_gradient.stress_scaling = 0.25 * mvm / pn + 0.75 * sc
        elif kind == TO_QOI.MASS:
            ev = float(np.prod(fe_solver.mesh.elem_size))
            rho = fe_solver.mat_prop.mass_density
            xs = np.asarray(x.cpu() if isinstance(x, torch.Tensor) else x)
            c[m, 0] = np.sum(xs * ev * rho) / lim - 1.0
            dc[m] = ev * rho / lim
        else:
            raise NotImplementedError(f"Constraint {kind} is not implemented yet.")
    return c, dc


compute_constraint_and_gradient.stress_scaling = 1.0
