"""CPU oracle for the hex8 structural-FEA path (TEST INFRASTRUCTURE ONLY).

This package restates, in numpy/scipy, the reference's algorithm for the voxel
hex8 SIMP structural FEA path of PyTO (UW-ERSL/PyTO).  It exists to check the
CUDA product path and to provide the CPU baseline timing; it is never used by
the product.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it.

Parity is pinned: ``tests/golden/gen_golden.py`` ran the reference itself
(``src/*.py`` imported under a test-only mock shim) and committed its outputs
under ``tests/golden/``; ``tests/test_oracle_golden.py`` checks every function
here against those vectors.
"""
from .hex8 import *  # noqa: F401,F403
