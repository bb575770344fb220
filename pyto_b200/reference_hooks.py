"""Routing PyTO's own callers to this library.

PyTO's modules import one another by flat module name (``import linear_solvers``,
``from topopt_material_model import *``, ``import deflation``; src/hex_structural_fea.py:
3-13, src/topopt_obj_cons_sensitivities.py:1-7).  Its optimisers and demos build a
``HexStructuralFEA``, call ``fe.solve(x)``, and reach ``linear_solvers.solve`` again
for every adjoint solve with ``fe_solver.stiff_mtrx`` (src/topopt_obj_cons_sensitivities.py:
269-274, src/topopt_mma.py:282, src/topopt_levelset.py:343).  Two ways to send those
calls to the GPU:

* ``install()`` -- before PyTO's modules are imported, register this package's
  ``linear_solvers``, ``deflation``, ``hex_structural_fea`` and ``topopt_material_model``
  under PyTO's module names.  PyTO's unmodified optimisers, sensitivity routines and
  demos then construct this package's ``HexStructuralFEA`` and solve on the device;
  their own host code (objective assembly, filters, OC/MMA updates) is unchanged.
* ``patch_linear_solvers(module)`` / ``patch_hex_structural_fea(module)`` -- for PyTO
  modules already imported: ``solve`` sends a call whose matrix is this library's
  ``StiffnessOperator`` here and every other call (an assembled scipy matrix) to
  PyTO's own code; ``HexStructuralFEA`` becomes this package's class.

PyTO's enum members (``Solvers.DPCG``, ``MaterialModel.SIMP``, ...) compare equal to
this package's same-named members, so callers may keep passing theirs.
"""
from __future__ import annotations

import sys

from . import deflation, hex_structural_fea, linear_solvers, topopt_material_model

#: PyTO module name -> this package's module that replaces it under install()
ALIASES = {
    "linear_solvers": linear_solvers,
    "deflation": deflation,
    "hex_structural_fea": hex_structural_fea,
    "topopt_material_model": topopt_material_model,
}


def install(replace_imported: bool = False) -> dict:
    """Register this package's modules under PyTO's module names (sys.modules).

    A PyTO module of one of those names that is already imported is left in place
    unless ``replace_imported`` (modules that imported it earlier keep their
    reference); use the patch functions for that case.  Returns the previous
    sys.modules entries, for ``uninstall``."""
    previous = {}
    for name, mod in ALIASES.items():
        cur = sys.modules.get(name)
        if cur is not None and cur is not mod and not replace_imported:
            continue
        previous[name] = cur
        sys.modules[name] = mod
    return previous


def uninstall(previous: dict) -> None:
    """Undo ``install`` (restores the given sys.modules entries)."""
    for name, mod in previous.items():
        if mod is None:
            sys.modules.pop(name, None)
        else:
            sys.modules[name] = mod


def patch_linear_solvers(module):
    """Wrap an imported PyTO ``linear_solvers`` module's ``solve``: this library's
    operator goes to the GPU solve, anything else to PyTO's own path
    (src/linear_solvers.py:136-202).  Idempotent; returns the module."""
    ref_solve = module.solve
    if getattr(ref_solve, "pyto_wrapped", False):
        return module

    def solve(A0, b0, solver, bc, **kwargs):
        if getattr(A0, "is_pyto_operator", False):
            return linear_solvers.solve(A0, b0, solver, bc, **kwargs)
        return ref_solve(A0, b0, solver, bc, **kwargs)

    solve.pyto_wrapped = True
    solve.__wrapped__ = ref_solve
    solve.__doc__ = ref_solve.__doc__
    module.solve = solve
    return module


def patch_hex_structural_fea(module):
    """Point an imported PyTO ``hex_structural_fea`` module's ``HexStructuralFEA`` at this
    package's class (src/hex_structural_fea.py:18-234).  Returns the module."""
    module.HexStructuralFEA = hex_structural_fea.HexStructuralFEA
    return module
