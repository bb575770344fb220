"""Density-based topology optimisation with MMA (drop-in for PyTO's topopt_mma,
src/topopt_mma.py:146-476, and its runMMA loop, src/mmaWrapper.py:18-128), with the
design vector, density filter, solves, sensitivities, chain rule and the MMA
subproblem on the GPU (``pyto_mma_update``: Svanberg's mmasub/subsolv in one
cooperative kernel).  The host reads the objective, the m constraint values and the
KKT norm once per iteration.

Supported: FEA_MODE.STRUCTURAL and FEA_MODE.THERMAL (an FEA object of this
package), the objectives and constraints of ``topopt_obj_cons_sensitivities``.
The thermo-structural mode and the body-force term are outside the GPU path.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import torch

from . import _capi as A
from . import topopt_material_model as tmm
from .topopt_common import FEA_MODE, TO_QOI, createFilters, find_elements_with_forces
from .topopt_obj_cons_sensitivities import compute_constraint_and_gradient, compute_objective_and_gradient


class DeviceMMA:
    """The MMA state of n variables and m constraints on one device: asymptotes, the
    two previous designs, and the subproblem workspace (mmasub's parameters as in
    runMMA: c = 100, d = 1, a0 = 1, a = 0; xmin / xmax scalars)."""

    def __init__(self, n, m, xmin, xmax, move, device):
        self.n, self.m, self.move = int(n), int(m), float(move)
        self.xmin, self.xmax = float(xmin), float(xmax)
        self.device = device
        f64 = dict(dtype=torch.float64, device=device)
        self.low = torch.full((n,), self.xmin, **f64)
        self.upp = torch.full((n,), self.xmax, **f64)
        self.xold1 = torch.zeros(n, **f64)
        self.xold2 = torch.zeros(n, **f64)
        self.dual = torch.zeros(3 + 4 * m, **f64)
        nb = int(A.lib().pyto_mma_workspace_bytes(int(n), int(m)))
        self.ws = torch.empty(nb, dtype=torch.uint8, device=device)
        self.a0 = 1.0
        self.a = np.zeros(m)
        self.c = np.full(m, 100.0)
        self.d = np.ones(m)
        self.iter = 0

    @staticmethod
    def _h(v):
        v = np.ascontiguousarray(np.asarray(v, dtype=np.float64).ravel())
        return v, v.ctypes.data_as(C.c_void_p)

    def update(self, x, df0dx, fval, dfdx):
        """One mmasub step: x (device, n) is replaced by the subproblem's solution."""
        self.iter += 1
        if self.iter == 1:
            self.xold1.copy_(x)
            self.xold2.copy_(x)
        xval = x.clone()
        fv, fp = self._h(fval)
        av, ap = self._h(self.a)
        cv, cp = self._h(self.c)
        dv, dp = self._h(self.d)
        dfdx = dfdx.contiguous()
        A.call("pyto_mma_update", self.n, self.m, self.iter, A.ptr(x), A.ptr(self.xold1), A.ptr(self.xold2), None,
               None, self.xmin, self.xmax, A.ptr(df0dx), fp, A.ptr(dfdx), A.ptr(self.low), A.ptr(self.upp),
               self.a0, ap, cp, dp, self.move, A.ptr(self.dual), A.ptr(self.ws), self.ws.numel(),
               A.stream_ptr(self.device))
        self.xold2, self.xold1 = self.xold1, xval
        return x

    def kkt(self, x, df0dx, fval, dfdx):
        """KKT residual norm of the original problem at x (kktcheck)."""
        fv, fp = self._h(fval)
        av, ap = self._h(self.a)
        cv, cp = self._h(self.c)
        dv, dp = self._h(self.d)
        out = np.zeros(2)
        A.call("pyto_mma_kkt", self.n, self.m, A.ptr(x), None, None, self.xmin, self.xmax, A.ptr(df0dx), fp,
               A.ptr(dfdx.contiguous()), self.a0, ap, cp, dp, out.ctypes.data_as(C.c_void_p), A.ptr(self.ws),
               self.ws.numel(), A.stream_ptr(self.device))
        return float(out[0]), float(out[1])


def topopt_mma(feaMode, fe_structural_solver, fe_thermal_solver, to_params, maxiteration: int = 300,
               timeLimitSecs: float = 36000, move_limit: float = 0.05, kkt_tol: float = 1.0e-6,
               objective_tol: float = 1.0e-3, constraint_tol: float = 1.0e-3, print_progress: bool = True,
               plot_progress: bool = False, use_continuation: bool = False, binarize_topology: bool = True,
               progress_callback=None, plotter=None):
    """Returns (sol, history, success, errorMsg, nFEAs) as the reference does."""
    def log(msg):
        if progress_callback:
            progress_callback(str(msg))
        else:
            print(msg)

    if feaMode == FEA_MODE.STRUCTURAL:
        fe_solver, nDOFPerNode = fe_structural_solver, 3
    elif feaMode == FEA_MODE.THERMAL:
        fe_solver, nDOFPerNode = fe_thermal_solver, 1
    elif feaMode == FEA_MODE.THERMO_STRUCTURAL:
        raise NotImplementedError("the thermo-structural mode is outside the GPU path")
    else:
        raise ValueError("Invalid FEA mode.")
    if getattr(fe_solver, "elem_body_force", None) is not None:
        raise NotImplementedError("body forces are outside the GPU path")
    mesh = fe_solver.mesh
    g = fe_solver.grid
    dev = g.device
    material_model = to_params.materialModel
    num_elems = mesh.num_elems
    tStart = time.time()
    history = {"objective": []}
    for idx, _ in enumerate(to_params.Constraints):
        history[f"constraint_{idx + 1}"] = []
    history["volfrac"] = []
    H, Hs = createFilters(fe_solver, to_params)
    loaded = find_elements_with_forces(mesh, fe_solver.bc.force, nDOFPerNode)
    loaded = torch.as_tensor(loaded, device=dev) if np.size(loaded) else None
    keep = None if to_params.ElemsToKeep is None else torch.as_tensor(np.asarray(to_params.ElemsToKeep), device=dev)
    KE = fe_solver.elem_stiff[0]
    if use_continuation:
        tmm.initialize_SIMP_STRUCTURAL_PENALTY(1)
        tmm.initialize_SIMP_THERMAL_PENALTY(1)
    else:
        tmm.initialize_SIMP_STRUCTURAL_PENALTY(3)
    state = {"obj0": None, "iteration": 0, "nFEAs": 0}

    def optimizationFunction(x):
        """(f0, df0/dx, g, dg/dx) of the MMA variables x (src/topopt_mma.py:246-363)."""
        rho = H.density(x) if to_params.APPLY_FILTER_TO_DENSITY else x
        if hasattr(mesh, "setPseudoDensity"):
            mesh.setPseudoDensity(rho)
        sol = fe_solver.solve(rho, material_model)
        obj, grad = compute_objective_and_gradient(feaMode, to_params, sol, rho, fe_solver, KE)
        c, dcdx = compute_constraint_and_gradient(feaMode, to_params, sol, rho, fe_solver, KE)
        grad = g.tensor(grad)
        dcdx = g.tensor(np.ascontiguousarray(dcdx))
        if state["obj0"] is None:
            state["obj0"] = obj
        if np.any(c.ravel() > 0.5):
            grad = grad * 0.0
        obj0 = state["obj0"]
        obj, grad = obj / obj0, grad / obj0
        if not to_params.APPLY_FILTER_TO_DENSITY:
            if to_params.Objective[0] == TO_QOI.COMPLIANCE:
                grad = H.sensitivity(grad, rho)
            elif to_params.Objective[0] != TO_QOI.VOLUME_FRACTION:
                grad = H.density(grad)
        if loaded is not None:
            grad[loaded] = grad.min()
        if keep is not None:
            grad[keep] = grad.min()
        if not to_params.APPLY_FILTER_TO_DENSITY:
            for j, (kind, _, _) in enumerate(to_params.Constraints):
                if kind == TO_QOI.COMPLIANCE:
                    dcdx[j] = H.sensitivity(dcdx[j], rho)
                elif kind != TO_QOI.VOLUME_FRACTION:
                    dcdx[j] = H.density(dcdx[j])
        else:  # chain rule back to the MMA variables: df/dx = H^T (df/drho / Hs)
            grad = H.chain(grad)
            for j in range(dcdx.shape[0]):
                dcdx[j] = H.chain(dcdx[j].contiguous())
        history["objective"].append(obj * obj0)
        history["volfrac"].append(float(rho.mean()))
        for idx, val in enumerate(c.ravel()):
            history[f"constraint_{idx + 1}"].append(float(val))
        if print_progress:
            log(f"Iteration: {state['iteration']}, objective {obj * obj0:.4g}")
        state["iteration"] += 1
        state["nFEAs"] += 1
        if use_continuation and state["iteration"] % 10 == 0:
            tmm.increment_SIMP_THERMAL_PENALTY(0.25)
            tmm.increment_SIMP_STRUCTURAL_PENALTY(0.25)
        return obj, grad.contiguous(), c.ravel(), dcdx

    # initial design (src/topopt_mma.py:376-385) and the runMMA loop (src/mmaWrapper.py:64-123)
    x0 = 0.5
    for con in to_params.Constraints:
        if con[0] == TO_QOI.VOLUME_FRACTION:
            x0 = con[2]
            break
    x = torch.full((num_elems,), float(x0), dtype=torch.float64, device=dev)
    m = len(to_params.Constraints)
    mma = DeviceMMA(num_elems, m, 1e-6, 1.0 - 1e-6, move_limit, dev)
    f0val, df0dx, gval, dgdx = optimizationFunction(x)
    f0Scaling = f0val if abs(f0val) > 1e-6 else 1.0
    f0valPrev = f0val / f0Scaling
    kktnorm, outit = kkt_tol + 10.0, 0
    success, errorMsg = True, "No errors."
    while kktnorm > kkt_tol and outit < maxiteration:
        outit += 1
        mma.update(x, df0dx, gval, dgdx)
        f0val, df0dx, gval, dgdx = optimizationFunction(x)
        f0val, df0dx = f0val / f0Scaling, df0dx / f0Scaling
        kktnorm, _ = mma.kkt(x, df0dx, gval, dgdx)
        fErr = abs(f0val - f0valPrev) / (1e-10 + abs(f0val))
        gErr = float(np.max(gval))
        if fErr < objective_tol and gErr < constraint_tol:
            break
        f0valPrev = f0val
        if time.time() - tStart > timeLimitSecs:
            errorMsg = "Time limit reached"
            break
        if np.isnan(kktnorm):
            success, errorMsg = False, "kktnorm is nan"
            break
    if outit >= maxiteration:
        errorMsg = "Maximum iterations reached"
    rho = H.density(x) if to_params.APPLY_FILTER_TO_DENSITY else x
    if binarize_topology:
        r = rho.cpu().numpy()
        thr = np.sort(r)[int((1 - np.mean(r)) * len(r))]
        rho = g.tensor(np.where(r < thr, 0.0, 1.0))
    sol = fe_solver.solve(rho, material_model)
    obj, _ = compute_objective_and_gradient(feaMode, to_params, sol, rho, fe_solver, KE)
    c, _ = compute_constraint_and_gradient(feaMode, to_params, sol, rho, fe_solver, KE)
    history["objective"].append(obj)
    history["volfrac"].append(float(rho.mean()))
    for idx, val in enumerate(c.ravel()):
        history[f"constraint_{idx + 1}"].append(float(val))
    if print_progress:
        log(f"Final objective: {obj:.4g}, vf: {float(rho.mean()):.3f}")
        log(f"Total Time: {time.time() - tStart:.2f} s")
        log(f"Error: {errorMsg}")
    fe_solver.mma_design = x
    return (sol.cpu().numpy() if isinstance(sol, torch.Tensor) else np.asarray(sol)), history, success, errorMsg, \
        state["nFEAs"]
