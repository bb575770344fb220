"""Material interpolation (drop-in for PyTO's topopt_material_model,
src/topopt_material_model.py:1-209).

The reference keeps the penalties as module globals changed through setters;
they are kept here with the same names and defaults.  The functions accept
numpy arrays (evaluated with numpy, as the reference does) or CUDA tensors
(SIMP on the device through ``pyto_simp``; the others as device tensor
expressions).
"""
from __future__ import annotations

import enum

import numpy as np

from ._enum import NamedEnum

_SIMP_STRUCTURAL_PENALTY_MIN = 1
_SIMP_STRUCTURAL_PENALTY_MAX = 6.0
_SIMP_THERMAL_PENALTY_MIN = 1
_SIMP_THERMAL_PENALTY_MAX = 3
_SIMP_STRUCTURAL_PENALTY = 3.0
_SIMP_THERMAL_PENALTY = 1
_SIMP_STRESS_RELAXATION = 0.5
_EVOID_RELATIVE = 1e-8
_KVOID_RELATIVE = 1e-8
_RAMP_PENALTY = 5
_MASS_PENALTY = 1
_MASS_LOW = 0
_PNORM_EXPONENT = 6


class MaterialModel(NamedEnum):
    SIMP = enum.auto()
    RAMP = enum.auto()
    SIMPPLUS = enum.auto()


def set_SIMP_STRUCTURAL_PENALTY(value: float) -> None:
    global _SIMP_STRUCTURAL_PENALTY
    _SIMP_STRUCTURAL_PENALTY = value


def update_SIMP_STUCTURAL_PENALTY_for_body_force(fraction_grey: float) -> None:
    global _SIMP_STRUCTURAL_PENALTY
    _SIMP_STRUCTURAL_PENALTY = (_SIMP_STRUCTURAL_PENALTY_MIN * (1 - fraction_grey)
                                + _SIMP_STRUCTURAL_PENALTY_MAX * fraction_grey)


def increment_SIMP_STRUCTURAL_PENALTY(value):
    global _SIMP_STRUCTURAL_PENALTY
    _SIMP_STRUCTURAL_PENALTY = max(min(_SIMP_STRUCTURAL_PENALTY + value, _SIMP_STRUCTURAL_PENALTY_MAX),
                                   _SIMP_STRUCTURAL_PENALTY_MIN)
    return _SIMP_STRUCTURAL_PENALTY


def increment_SIMP_THERMAL_PENALTY(value):
    global _SIMP_THERMAL_PENALTY
    _SIMP_THERMAL_PENALTY = max(min(_SIMP_THERMAL_PENALTY + value, _SIMP_THERMAL_PENALTY_MAX),
                                _SIMP_THERMAL_PENALTY_MIN)
    return _SIMP_THERMAL_PENALTY


def initialize_SIMP_STRUCTURAL_PENALTY(value=None) -> None:
    global _SIMP_STRUCTURAL_PENALTY
    _SIMP_STRUCTURAL_PENALTY = 3.0 if value is None else value


def initialize_SIMP_THERMAL_PENALTY(value=None) -> None:
    global _SIMP_THERMAL_PENALTY
    _SIMP_THERMAL_PENALTY = 1.0 if value is None else value


def _is_dev(x):
    return hasattr(x, "is_cuda") and x.is_cuda


def get_structural_material_model_scaling(x, material_model: MaterialModel):
    """E scaling (src/topopt_material_model.py:76-95)."""
    if material_model is None:
        return x
    if material_model == MaterialModel.SIMP:
        if _is_dev(x):
            from . import _capi as A
            import torch
            xc = x.contiguous()
            s = torch.empty_like(xc)
            A.call("pyto_simp", A.ptr(xc), None, int(xc.numel()), float(_SIMP_STRUCTURAL_PENALTY),
                   float(_EVOID_RELATIVE), A.ptr(s), None, A.stream_ptr(xc.device))
            return s
        return _EVOID_RELATIVE + (x ** _SIMP_STRUCTURAL_PENALTY) * (1 - _EVOID_RELATIVE)
    if material_model == MaterialModel.RAMP:
        return _EVOID_RELATIVE + x * (1 - _EVOID_RELATIVE) / (1 + (1 - x) * _RAMP_PENALTY)
    if material_model == MaterialModel.SIMPPLUS:
        return ((_EVOID_RELATIVE + (x ** _SIMP_STRUCTURAL_PENALTY) * (1 - _EVOID_RELATIVE)) + _EVOID_RELATIVE * x) / 2
    raise ValueError("Invalid material model specified.")


def get_structural_material_model_sensitivity(x, material_model: MaterialModel):
    """d(E scaling)/dx (src/topopt_material_model.py:119-139)."""
    if material_model is None:
        return x * 0 + 1
    if material_model == MaterialModel.SIMP:
        if _is_dev(x):
            from . import _capi as A
            import torch
            xc = x.contiguous()
            s, ds = torch.empty_like(xc), torch.empty_like(xc)
            A.call("pyto_simp", A.ptr(xc), None, int(xc.numel()), float(_SIMP_STRUCTURAL_PENALTY),
                   float(_EVOID_RELATIVE), A.ptr(s), A.ptr(ds), A.stream_ptr(xc.device))
            return ds
        return _SIMP_STRUCTURAL_PENALTY * (x ** (_SIMP_STRUCTURAL_PENALTY - 1)) * (1 - _EVOID_RELATIVE)
    if material_model == MaterialModel.RAMP:
        return ((1 - _EVOID_RELATIVE) / (1 + (1 - x) * _RAMP_PENALTY) ** 2) * (1 + _RAMP_PENALTY * (1 - x))
    if material_model == MaterialModel.SIMPPLUS:
        return (_SIMP_STRUCTURAL_PENALTY * (x ** (_SIMP_STRUCTURAL_PENALTY - 1)) * (1 - _EVOID_RELATIVE)
                + _EVOID_RELATIVE) / 2
    raise ValueError("Invalid material model specified.")


def get_thermal_material_model_scaling(x, material_model: MaterialModel):
    """Conductivity scaling (src/topopt_material_model.py:98-117); None: x itself."""
    if material_model is None:
        return x
    if material_model == MaterialModel.SIMP:
        return _KVOID_RELATIVE + (x ** _SIMP_THERMAL_PENALTY) * (1 - _KVOID_RELATIVE)
    if material_model == MaterialModel.RAMP:
        return _KVOID_RELATIVE + x * (1 - _KVOID_RELATIVE) / (1 + (1 - x) * _RAMP_PENALTY)
    if material_model == MaterialModel.SIMPPLUS:
        return ((_KVOID_RELATIVE + (x ** _SIMP_THERMAL_PENALTY) * (1 - _KVOID_RELATIVE)) + _KVOID_RELATIVE * x) / 2
    raise ValueError("Invalid material model specified.")


def get_thermal_material_model_sensitivity(x, material_model: MaterialModel):
    """d(conductivity scaling)/dx (src/topopt_material_model.py:142-161)."""
    if material_model is None:
        return x * 0 + 1
    if material_model == MaterialModel.SIMP:
        return _SIMP_THERMAL_PENALTY * (x ** (_SIMP_THERMAL_PENALTY - 1)) * (1 - _KVOID_RELATIVE)
    if material_model == MaterialModel.RAMP:
        return ((1 - _KVOID_RELATIVE) / (1 + (1 - x) * _RAMP_PENALTY) ** 2) * (1 + _RAMP_PENALTY * (1 - x))
    if material_model == MaterialModel.SIMPPLUS:
        return (_SIMP_THERMAL_PENALTY * (x ** (_SIMP_THERMAL_PENALTY - 1)) * (1 - _KVOID_RELATIVE)
                + _KVOID_RELATIVE) / 2
    raise ValueError("Invalid material model specified.")


def get_stress_relaxation_factor() -> float:
    return _SIMP_STRESS_RELAXATION


def get_stress_relaxation_correction(x):
    return (x ** _SIMP_STRESS_RELAXATION).reshape((-1, 1))


def get_stress_relaxation_factor_sensitivity(x):
    return (_SIMP_STRESS_RELAXATION * (x ** (_SIMP_STRESS_RELAXATION - 1))).reshape((-1, 1))


def get_pNorm_exponent() -> float:
    return _PNORM_EXPONENT
