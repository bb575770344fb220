"""The C-ABI library loads, exports every declared symbol, and its host-side
set-up (Ke, Hadamard blocks) matches the reference.  No GPU needed."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden
from pyto_b200 import _capi as A


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "pyto_b200.h")).read()
    return sorted(set(re.findall(r"^(?:int|size_t|long long|const char\*|void|pyto_\w+_t\*)\s*(pyto_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_declared_symbol():
    L = A.lib()
    syms = header_symbols()
    assert len(syms) >= 17
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(A.SIGNATURES), "ctypes binding and header disagree"
    assert L.pyto_version() >= 1


def test_ctypes_structs_match_the_c_layout():
    """The ctypes mirrors of the ABI structs have the C compiler's sizes."""
    L = A.lib()
    for which, cls in enumerate((A.Operator, A.SolveCfg, A.SolveStatus, A.Deflation, A.BatchItem, A.Thermal)):
        assert L.pyto_struct_size(which) == C.sizeof(cls), cls.__name__
    assert L.pyto_struct_size(6) == 0


@pytest.mark.parametrize("tag,E,nu,h", [("unit", 1.0, 0.3, (1, 1, 1)), ("box", 1.0, 0.3, (1.0, 0.5, 2.0)),
                                        ("half", 2.5, 0.25, (0.5, 0.5, 0.5))])
def test_ke_matches_reference(tag, E, nu, h):
    ke = np.zeros(576)
    A.call("pyto_ke_hex8", E, nu, *map(float, h), ke.ctypes.data_as(C.c_void_p))
    np.testing.assert_allclose(ke.reshape(24, 24), golden("ke.npz")[f"ke_{tag}"], rtol=1e-13, atol=1e-15)


def test_hadamard_blocks_reproduce_ke():
    """Ke = Phi^T K^ Phi with K^ the eight 3x3 parity blocks."""
    op = A.make_operator(4, 3, 2, (1.0, 0.5, 2.0), 1.0, 0.3)
    bits = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    phi = np.array([[np.prod([(2 * b[d] - 1) for d in range(3) if m >> d & 1]) for b in bits] for m in range(8)])
    kh = np.array(op.khat).reshape(8, 3, 3)
    Khat = np.zeros((24, 24))  # index 8c+m
    for q in range(8):
        for c in range(3):
            for d in range(3):
                Khat[8 * c + (q ^ (1 << c)), 8 * d + (q ^ (1 << d))] = kh[q, c, d]
    Phi = np.zeros((24, 24))  # hat (8c+m) <- dof (3a+c)
    for c in range(3):
        for m in range(8):
            for a in range(8):
                Phi[8 * c + m, 3 * a + c] = phi[m, a]
    ke = np.array(op.ke).reshape(24, 24)
    np.testing.assert_allclose(Phi.T @ Khat @ Phi, ke, rtol=0, atol=1e-14 * np.abs(ke).max())
    assert np.allclose(op.kdiag, np.diag(ke)[:3])


def test_operator_rejects_non_box_ke():
    ke = np.random.default_rng(0).normal(size=(24, 24))
    ke = ke + ke.T
    with pytest.raises(A.PytoError):
        A.make_operator(2, 2, 2, ke=ke)
    with pytest.raises(A.PytoError):
        A.make_operator(0, 2, 2)


def test_workspace_sizes_are_reported():
    op = A.make_operator(12, 6, 6)
    for k in (A.WS_REDUCE, A.WS_PCG, A.WS_DPCG):
        assert A.ws_bytes(op, k) > 0
    assert A.ws_bytes(op, A.WS_PCG) >= 3 * 8 * 3 * 13 * 7 * 7


def test_autotuner_variants_are_the_ones_the_library_accepts():
    """Every operator variant the autotuner times is accepted by pyto_tune, and the
    numbers around them are rejected (host-side check only: no kernel runs)."""
    from pyto_b200.autotune import VARIANTS, VARIANTS_F32
    L = A.lib()
    try:
        for which, listed in ((0, VARIANTS), (1, VARIANTS_F32)):
            for v in range(-1, max(listed) + 3):
                rc = L.pyto_tune(which, v)
                assert (rc == 0) == (v in listed), (which, v, rc)
                if rc:
                    assert rc == A.ERR_ARG, (which, v, rc)
    finally:
        assert L.pyto_tune(0, 2) == 0 and L.pyto_tune(1, 18) == 0  # library defaults


@pytest.mark.parametrize("tag,k,h", [("unit", 1.0, (1.0, 1.0, 1.0)), ("box", 50.0, (1.0, 0.5, 2.0))])
def test_thermal_ke_matches_reference(tag, k, h):
    """pyto_ke_hex8_thermal (host code, no GPU) against the reference's Ke, and the
    operator set-up's box-symmetry check."""
    d = golden("thermal.npz")
    ke = np.zeros(64)
    assert A.lib().pyto_ke_hex8_thermal(k, *h, ke.ctypes.data_as(C.c_void_p)) == 0
    np.testing.assert_allclose(ke.reshape(8, 8), d[f"ke_{tag}"], rtol=1e-13, atol=1e-13)
    t = A.make_thermal(4, 3, 2, h, k)
    np.testing.assert_allclose(np.array(t.ke).reshape(8, 8), d[f"ke_{tag}"], rtol=1e-13, atol=1e-13)
    bad = d[f"ke_{tag}"].copy()
    bad[0, 1] += 0.1 * abs(bad[0, 0])
    with pytest.raises(A.PytoError):
        A.make_thermal(4, 3, 2, h, k, ke=bad)
