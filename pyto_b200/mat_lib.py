"""Material data (drop-in for PyTO's mat_lib, src/mat_lib.py:9-175)."""
from __future__ import annotations

import dataclasses
import difflib


@dataclasses.dataclass
class Material:
    name: str
    youngs_modulus: float
    poissons_ratio: float
    mass_density: float = 7850.0
    thermal_conductivity: float = 50.0
    specific_heat: float = 0.0
    thermal_expansion_coefficient: float = 12e-6
    cost: float = 0.1
    yield_strength: float = 30e6


materials = [Material(name="Steel", youngs_modulus=2.1e11, poissons_ratio=0.3, mass_density=7850,
                      thermal_conductivity=50, specific_heat=0.0, thermal_expansion_coefficient=12e-6, cost=0.1,
                      yield_strength=30e6)]


def get_material(name: str) -> Material:
    for m in materials:
        if m.name.lower() == name.lower():
            return m
    close = difflib.get_close_matches(name.lower(), [m.name.lower() for m in materials])
    if close:
        sug = next(m for m in materials if m.name.lower() == close[0])
        raise ValueError(f"Material '{name}' not found. Did you mean '{sug.name}'?")
    raise ValueError(f"Material '{name}' not found")


def create_material_with_defaults(name: str, **kwargs) -> Material:
    props = dataclasses.asdict(get_material("Steel"))
    props["name"] = name
    props.update(kwargs)
    return Material(**props)
