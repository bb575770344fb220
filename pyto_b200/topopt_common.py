"""Shared TO definitions (drop-in for the parts of PyTO's topopt_common used by
the hex8 path, src/topopt_common.py:21-159)."""
from __future__ import annotations

import enum
from dataclasses import dataclass, field
from typing import Tuple

import numpy as np

from ._enum import NamedEnum
from .topopt_material_model import MaterialModel

DIRECT_SOLVER_DOF_CUTOFF = 100000


class TO_METHODS(NamedEnum):
    DENSITYMMA = enum.auto()
    DENSITYOCM = enum.auto()
    PARETO = enum.auto()
    LEVELSET = enum.auto()


class FEA_MODE(NamedEnum):
    STRUCTURAL = enum.auto()
    THERMAL = enum.auto()
    THERMO_STRUCTURAL = enum.auto()


class TO_QOI(NamedEnum):
    VOLUME_FRACTION = enum.auto()
    VOLUME = enum.auto()
    MASS = enum.auto()
    COMPLIANCE = enum.auto()
    PNORM_STRESS = enum.auto()
    MAX_VONMISES_STRESS = enum.auto()
    STRESS_FAILURE_FACTOR = enum.auto()
    GVECTOR = enum.auto()
    GFUNCTION = enum.auto()
    COST = enum.auto()
    TEMPERATURE_FAILURE_FACTOR = enum.auto()
    MAX_CRITICALITY = enum.auto()
    MEAN_CRITICALITY = enum.auto()
    FATIGUE_FAILURE_FACTOR = enum.auto()
    PBR = enum.auto()


@dataclass(slots=True)
class TOParams:
    Comment: str = ""
    Objective: Tuple[TO_QOI, None] = (TO_QOI.COMPLIANCE, None)
    Constraints: list = field(default_factory=lambda: [(TO_QOI.VOLUME_FRACTION, None, 0.5)])
    nDOFDesired: int = 25000
    APPLY_FILTER_TO_DENSITY: bool = True
    RelativeFilterRadius: float = 1.5
    XSymmetry: bool = False
    YSymmetry: bool = False
    ZSymmetry: bool = False
    XAxisAngularSymmetry: int = 0
    YAxisAngularSymmetry: int = 0
    ZAxisAngularSymmetry: int = 0
    ExtrudeX: bool = False
    ExtrudeY: bool = False
    ExtrudeZ: bool = False
    KeepFixedElems: bool = False
    RemoveHangingElems: bool = False
    AMBuildDir: str = ""
    ElemsToKeep: list = None
    MaxIterations: int = 150
    Enforce_Constraints_MMA: bool = False
    Eliminate_Hanging_Elements: bool = False
    MaterialsExcelFile: str = ""
    materialModel: MaterialModel = MaterialModel.SIMP


def find_elements_with_forces(mesh, force, nDOFPerNode) -> np.ndarray:
    """Elements with a loaded node (src/topopt_common.py:79-100)."""
    forced = np.unique(np.where(np.asarray(force) != 0)[0] // nDOFPerNode)
    return np.where(np.isin(mesh.elemArray, forced).any(axis=1))[0]


def find_elements_with_fixedDOF(mesh, bc, nDOFPerNode) -> np.ndarray:
    fixed = np.unique(np.asarray(bc.fixed_dofs) // nDOFPerNode)
    return np.where(np.isin(mesh.elemArray, fixed).any(axis=1))[0]


def createFilters(fe_solver, to_params):
    """Smoothing filter composed with the symmetry / extrusion filters the flags ask for,
    in the reference's order (src/topopt_common.py:127-159); returns (H, Hs).  Angular
    symmetry is outside the GPU path (see topopt_filters)."""
    from . import topopt_filters as tf
    if to_params.XAxisAngularSymmetry or to_params.YAxisAngularSymmetry or to_params.ZAxisAngularSymmetry:
        raise NotImplementedError("angular symmetry filters are outside the GPU path")
    H, Hs = tf.createSmoothingFilter(fe_solver.mesh, rel_filter_radius=to_params.RelativeFilterRadius)
    maps = []
    for flag, fn in (("XSymmetry", tf.createXSymmetryFilter), ("YSymmetry", tf.createYSymmetryFilter),
                     ("ZSymmetry", tf.createZSymmetryFilter), ("ExtrudeY", tf.createYExtrudeFilter),
                     ("ExtrudeX", tf.createXExtrudeFilter), ("ExtrudeZ", tf.createZExtrudeFilter)):
        if getattr(to_params, flag):
            maps.append(fn(fe_solver.mesh))
    if not maps:
        return H, Hs
    for m in maps:
        H = H * m
    return H, H.hs().cpu().numpy()
