"""The allocation-free variant of K(s) u with its fused dot product.

pyto_matvec_dot_noalloc serves callers that cannot allocate device memory (a host
framework that owns all allocations, or a loop that must not allocate after start-up):
its cross-block scratch is a fixed array inside the library instead of a caller
workspace.  This file is collected last so a run that stops at the first failure has
already run every other test; it must also pass alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


def test_noalloc_matvec_matches_workspace_variant_twice():
    from pyto_b200 import _capi as A
    from pyto_b200.engine import HexGrid
    nel = (40, 21, 13)
    m = O.grid_mesh(*nel)
    _, fixed = O.cantilever_bc(m)
    rng = np.random.default_rng(42)
    g = HexGrid(nel).set_fixed_dofs(fixed)
    st = A.stream_ptr()
    for call in range(2):  # two calls in a row: the shared scratch must not carry state
        s = g.tensor(rng.uniform(0.01, 1.0, g.nelem))
        u = g.tensor(rng.normal(size=g.ndof))
        y_ref, d_ref = g.matvec(s, u, dot=True)
        y_ref, d_ref = y_ref.clone(), d_ref.clone()
        y = torch.empty_like(u)
        d = torch.zeros(1, dtype=torch.float64, device=u.device)
        A.call("pyto_matvec_dot_noalloc", C.byref(g.op), A.ptr(s), A.ptr(g.mask), A.ptr(u), A.ptr(y),
               A.MASK_IN | A.MASK_OUT, A.ptr(d), st)
        torch.cuda.synchronize()
        assert torch.allclose(y, y_ref, rtol=1e-13, atol=1e-13 * float(y_ref.abs().max())), call
        assert abs(d.item() - d_ref.item()) <= 1e-12 * abs(d_ref.item()), call
        yo = O.matvec_free(m, s.cpu().numpy(), O.ke_hex8(1.0, 0.3), u.cpu().numpy(), fixed)
        assert np.abs(y.cpu().numpy() - yo).max() <= 1e-13 * np.abs(yo).max()


def test_noalloc_rejects_oversized_grid():
    """Beyond the fixed scratch size the call must refuse before launching anything."""
    from pyto_b200 import _capi as A
    nel = (6000, 300, 2)
    # the matvec launch has at least ceil((nelx+1)/31) * ceil((nely+1)/3) blocks
    min_blocks = -(-(nel[0] + 1) // 31) * -(-(nel[1] + 1) // 3)
    assert min_blocks > 2 * 8192  # far beyond the limit: the call cannot reach a launch
    op = A.make_operator(*nel)
    buf = torch.zeros(4, dtype=torch.float64, device="cuda")
    p = A.ptr(buf)
    rc = A.lib().pyto_matvec_dot_noalloc(C.byref(op), p, None, p, p + 8, 3, p + 16, A.stream_ptr())
    assert rc == A.ERR_TOO_LARGE
