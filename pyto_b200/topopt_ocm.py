"""Optimality-criteria topology optimisation (drop-in for PyTO's
topopt_optimality_criteria, src/topopt_ocm.py:107-345) with the design vector,
solves, sensitivities, sensitivity filter and OC bisection on the GPU; the
host reads one scalar set per iteration for history and convergence.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from . import topopt_material_model as tmm
from .topopt_common import TO_QOI, createFilters, find_elements_with_forces
from .topopt_obj_cons_sensitivities import compute_objective_and_gradient


def topopt_optimality_criteria(feaMode, fe_solver, to_params, maxIterations: int = 250, move: float = 0.2,
                               move_tol: float = 0.05, rel_conv_tol: float = 1.e-4, print_progress: bool = True,
                               plot_progress: bool = False, debug: bool = False, binarize_topology: bool = True,
                               use_continuation: bool = False, progress_callback=None, plotter=None):
    """Returns (sol, history, success, errorMsg, nFEAs) as the reference does.
    The connected-component clean-up after the loop (src/topopt_ocm.py:319-329)
    runs only when the mesh provides ``find_connected_components``."""
    if to_params.Objective[0] != TO_QOI.COMPLIANCE:
        raise ValueError(f"Unsupported objective type: {to_params.Objective[0]}")
    if to_params.Constraints[0][0] != TO_QOI.VOLUME_FRACTION:
        raise ValueError(f"Unsupported constraint type: {to_params.Constraints[0][0]}")
    volfrac = to_params.Constraints[0][2]

    def log(msg):
        if progress_callback:
            progress_callback(str(msg))
        else:
            print(msg)
    g = fe_solver.grid
    mesh = fe_solver.mesh
    ne = mesh.num_elems
    H, Hs = createFilters(fe_solver, to_params)
    loaded = torch.as_tensor(find_elements_with_forces(mesh, fe_solver.bc.force, 3), device=g.device)
    keep = None if to_params.ElemsToKeep is None else torch.as_tensor(np.asarray(to_params.ElemsToKeep),
                                                                       device=g.device)
    x = torch.full((ne,), float(volfrac), dtype=torch.float64, device=g.device)
    if g.active is not None:
        x = x * g.active
    history = {"objective": [], "volfrac": [], "change": []}
    KE = fe_solver.elem_stiff[0]
    success, errorMsg = True, "No errors."
    tmm.initialize_SIMP_STRUCTURAL_PENALTY(1 if use_continuation else 3)
    tStart = time.time()
    objScaling = None
    change = 0.0
    iteration = 0
    for iteration in range(maxIterations):
        mesh.setPseudoDensity(x)
        sol = fe_solver.solve(x, to_params.materialModel)
        obj, grad = compute_objective_and_gradient(feaMode, to_params, sol, x, fe_solver, KE)
        if objScaling is None:
            objScaling = abs(obj)
        obj = obj / objScaling
        grad = grad / objScaling
        grad = H.sensitivity(grad, x)
        if loaded.numel() > 0:
            grad[loaded] = grad.min()
        if keep is not None:
            grad[keep] = grad.min()
        ch = g.oc_update(x, grad.contiguous(), volfrac, move, 0.001, 1.0)
        change = float(ch.item())
        vol = float(x.sum()) / g.n_active
        history["objective"].append(obj * objScaling)
        history["volfrac"].append(vol)
        history["change"].append(change)
        xa = x if g.active is None else x[g.active.bool()]
        fraction_grey = float(((xa > 0.05) & (xa < 0.95)).sum()) / g.n_active
        if print_progress:
            log(f"Iteration: {iteration:d}, obj.: {(obj * objScaling):.3g}, vol.: {vol:.3g}, grey: "
                f"{fraction_grey:.3f}")
        if np.isnan(obj):
            log("Objective function became NaN. Exiting optimization.")
            errorMsg, success = "Objective is diverging", False
            break
        volc = vol / volfrac - 1.0
        if len(history["objective"]) >= 2:
            dJ = abs((history["objective"][-1] - history["objective"][-2]) / history["objective"][-2])
            if (dJ < rel_conv_tol) and (volc < rel_conv_tol) and (change < 0.2) and (fraction_grey < 0.1):
                log("OC optimization converged.")
                break
            if (dJ < rel_conv_tol) and (volc < rel_conv_tol) and (change < move_tol):
                log("OC optimization converged.")
                break
        if use_continuation and iteration % 10 == 0:
            tmm.increment_SIMP_STRUCTURAL_PENALTY(0.5)
    if iteration == maxIterations - 1:
        errorMsg, success = "Maximum iterations reached", False
        log(errorMsg)
    totalTime = time.time() - tStart
    if binarize_topology:
        xs, _ = torch.sort(x)
        threshold = xs[int((1 - float(x.mean())) * ne)]
        x = torch.where(x < threshold, 0.0, 1.0).to(torch.float64)
    mesh.setPseudoDensity(x)
    finder = getattr(mesh, "find_connected_components", None)
    if finder is not None:
        comps = finder()
        if len(comps) > 1:
            largest = max(comps, key=len)
            x = torch.zeros_like(x)
            x[torch.as_tensor(np.asarray(list(largest)), device=g.device)] = 1.0
    volfrac_final = float(x.mean())
    sol = fe_solver.solve(x, to_params.materialModel)
    obj, _ = compute_objective_and_gradient(feaMode, to_params, sol, x, fe_solver, KE)
    history["objective"].append(obj)
    history["volfrac"].append(volfrac_final)
    history["change"].append(change)
    if volfrac_final > 1.1 * volfrac:
        errorMsg, success = f"vf {volfrac:0.3f} not reached", False
    log(f"Final objective: {obj:.4g}, vf: {volfrac_final:.3f}")
    log(f"Total Time: {totalTime:.2f} s")
    log(f"Error: {errorMsg}")
    return sol, history, success, errorMsg, iteration + 1
