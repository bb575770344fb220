"""PyTO's own modules routed to this library (pyto_b200.reference_hooks), on the CPU.

Each check imports the reference's modules in a fresh interpreter under the same
test-only shim that tests/golden/gen_golden.py uses, so nothing leaks into the
other tests.  Skipped where no reference checkout is present (PYTO_REFERENCE, default
/root/reference).  No GPU work: the device solve is replaced by a recorder."""
import os
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("PYTO_REFERENCE", "/root/reference")
pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src")), reason="no reference checkout")


def _run(body: str):
    code = textwrap.dedent(f"""
        import sys
        sys.path.insert(0, {ROOT!r}); sys.path.insert(0, {os.path.join(ROOT, 'tests', 'golden')!r})
        from gen_golden import install_shim
        install_shim({REF!r})
    """) + textwrap.dedent(body)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_install_routes_reference_callers():
    """After install(), PyTO's unmodified optimiser and sensitivity modules resolve
    linear_solvers, HexStructuralFEA, deflation and the material model to this package."""
    out = _run("""
        from pyto_b200 import reference_hooks, linear_solvers as L, hex_structural_fea as F
        from pyto_b200 import deflation as D, topopt_material_model as T
        reference_hooks.install()
        import topopt_obj_cons_sensitivities as toc   # PyTO's own module
        import topopt_ocm                              # PyTO's own OC driver
        import hex_structural_fea, deflation, linear_solvers
        assert toc.linear_solvers is L
        assert hex_structural_fea.HexStructuralFEA is F.HexStructuralFEA
        assert deflation.DeflationSolver is D.DeflationSolver
        assert topopt_ocm.get_structural_material_model_scaling is T.get_structural_material_model_scaling
        assert toc.__file__.startswith(%r)
        print("ok")
    """ % REF)
    assert "ok" in out


def test_patch_dispatches_operator_and_keeps_reference_path():
    """patch_linear_solvers on PyTO's imported module: this library's operator goes to
    the GPU solve (recorded here), with PyTO's enum member accepted as the solver;
    an assembled matrix still takes PyTO's own scipy path."""
    out = _run("""
        import numpy as np, scipy.sparse as sp
        import linear_solvers as ref_ls, bound_cond        # PyTO's own modules
        from pyto_b200 import reference_hooks, linear_solvers as L
        calls = []
        L.solve = lambda A0, b0, solver, bc, **kw: calls.append((A0, solver, kw)) or np.full(3, 7.0)
        reference_hooks.patch_linear_solvers(ref_ls)
        reference_hooks.patch_linear_solvers(ref_ls)       # idempotent
        op = L.StiffnessOperator(None, None)
        bc = bound_cond.BC(force=np.ones(3), fixed_dofs=np.array([0]), dirichlet_values=np.zeros(1))
        u = ref_ls.solve(op, np.ones(3), ref_ls.Solvers.DPCG, bc, dsolver="d", rtol=1e-8)
        assert len(calls) == 1 and calls[0][0] is op and calls[0][1] == L.Solvers.DPCG
        assert calls[0][2] == {"dsolver": "d", "rtol": 1e-8} and np.all(u == 7.0)
        A = sp.csr_matrix(np.array([[4.0, 1, 0], [1, 3, 1], [0, 1, 2]]))
        u2 = ref_ls.solve(A, np.array([0.0, 1.0, 2.0]), ref_ls.Solvers.SPSOLVE, bc)
        assert len(calls) == 1                              # PyTO's own direct solve ran
        assert u2[0] == 0.0 and np.allclose(A[1:, 1:] @ u2[1:], [1.0, 2.0])
        print("ok")
    """)
    assert "ok" in out


def test_reference_enums_equal_package_enums():
    out = _run("""
        import linear_solvers as ref_ls, topopt_material_model as ref_tmm, topopt_common as ref_tc
        from pyto_b200 import linear_solvers as L, topopt_material_model as T, topopt_common as C
        assert ref_ls.Solvers.PCG == L.Solvers.PCG and L.Solvers.PCG == ref_ls.Solvers.PCG
        assert ref_ls.Solvers.PCG != L.Solvers.DPCG
        assert ref_tmm.MaterialModel.SIMP == T.MaterialModel.SIMP
        assert ref_tc.FEA_MODE.STRUCTURAL == C.FEA_MODE.STRUCTURAL
        assert {L.Solvers.DPCG: 1}[ref_ls.Solvers.DPCG] == 1
        print("ok")
    """)
    assert "ok" in out
