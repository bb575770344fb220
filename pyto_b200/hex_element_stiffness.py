"""Element matrices (drop-in for the structural part of PyTO's
hex_element_stiffness, src/hex_element_stiffness.py:221-286); computed by the
library's host code (``pyto_ke_hex8``)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A


def isotropic_constitutive_matrix(E, nu):
    """Isotropic D, shear rows xy, yz, xz (src/hex_element_stiffness.py:221-228)."""
    c = E / ((1.0 + nu) * (1.0 - 2.0 * nu))
    D = np.zeros((6, 6))
    D[:3, :3] = nu
    np.fill_diagonal(D[:3, :3], 1.0 - nu)
    D[3, 3] = D[4, 4] = D[5, 5] = (1.0 - 2.0 * nu) / 2.0
    return c * D


def hex8_stiffness_matrix_structural(E, nu, elem_size, gauss_order: int = 2) -> np.ndarray:
    """24x24 Ke of a box hex8 with 2x2x2 Gauss integration."""
    if gauss_order != 2:
        raise NotImplementedError("only the 2x2x2 rule of the reference's structural Ke is provided")
    ke = np.zeros(576)
    A.call("pyto_ke_hex8", float(E), float(nu), *(float(h) for h in elem_size), ke.ctypes.data_as(C.c_void_p))
    return ke.reshape(24, 24)
