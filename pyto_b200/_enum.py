"""Enum base of the reference-named modules.

PyTO's callers pass their own enum members (``linear_solvers.Solvers.DPCG``,
``topopt_material_model.MaterialModel.SIMP``, ``topopt_common.FEA_MODE...``) to
the functions they call.  The members of these enums compare equal to, and hash
like, the same-named members of a same-named enum class from another module, so
a caller that still imports the reference's enums reaches the same branch here.
"""
from __future__ import annotations

import enum


class NamedEnum(enum.Enum):
    def __eq__(self, other):
        if self is other:
            return True
        if isinstance(other, enum.Enum):
            return type(other).__name__ == type(self).__name__ and other.name == self.name
        return NotImplemented

    def __hash__(self):  # the hash of enum.Enum members: hash(name)
        return hash(self._name_)
