"""The reference-named modules, used the way PyTO code uses them, against the
goldens produced by the reference itself."""
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def _setup(nel=(12, 6, 6), h=(1.0, 1.0, 1.0), solver_name="PCG", dsolver=None, rtol=1e-12):
    from pyto_b200 import bound_cond, hex_mesher, hex_structural_fea, linear_solvers, mat_lib
    from pyto_b200 import topopt_material_model as tmm
    tmm._EVOID_RELATIVE = 1e-9
    m = hex_mesher.HexMesher()
    m.grid_mesh(nel, h)
    m.createEdofMatStructural()
    ni = m.node_indices
    fixed_nodes = m.getNodesOnBoundingBoxPlane(0, True)
    fixed = np.sort(np.concatenate([3 * fixed_nodes + c for c in range(3)]))
    load = np.where((ni[:, 0] == m.grid[0]) & (ni[:, 2] == 0))[0]
    f = np.zeros(3 * m.num_nodes)
    f[3 * load + 2] = -1.0 / len(load)
    bc = bound_cond.BC(force=f, fixed_dofs=fixed, dirichlet_values=np.zeros(len(fixed)))
    mat = mat_lib.create_material_with_defaults("unit", youngs_modulus=1.0, poissons_ratio=0.3)
    solver = getattr(linear_solvers.Solvers, solver_name)
    fe = hex_structural_fea.HexStructuralFEA(mesh=m, mat_prop=mat, bc=bc, solver=solver, dsolver=dsolver, rtol=rtol)
    return m, fe


@pytest.mark.parametrize("solver_name", ["PCG", "SPSOLVE", "PARDISO"])
def test_fea_solve_compliance_gradient(solver_name):
    from pyto_b200 import topopt_common as tc, topopt_obj_cons_sensitivities as toc
    from pyto_b200.topopt_material_model import MaterialModel
    d = golden("cantilever_12x6x6_direct.npz")
    m, fe = _setup(solver_name=solver_name)
    u = fe.solve(d["rho"], MaterialModel.SIMP)
    assert isinstance(u, np.ndarray)
    np.testing.assert_allclose(u, d["u"], rtol=0, atol=1e-9 * np.abs(d["u"]).max())
    assert abs(fe.max_deformation - float(d["max_def"])) <= 1e-9 * float(d["max_def"])
    C, dC = toc.compute_compliance_and_gradient(tc.FEA_MODE.STRUCTURAL, u, d["rho"], fe, fe.elem_stiff[0],
                                                MaterialModel.SIMP)
    assert abs(C - float(d["C"])) <= 1e-10 * float(d["C"])
    np.testing.assert_allclose(dC, d["dC"], rtol=1e-8, atol=1e-11 * np.abs(d["dC"]).max())


def test_force_changes_between_solves_are_seen():
    """As in the reference, every solve reads bc.force: an in-place change between two
    solves changes the displacement (linearly); a read-only load is kept on the device."""
    from pyto_b200.topopt_material_model import MaterialModel
    d = golden("cantilever_12x6x6_direct.npz")
    m, fe = _setup()
    u1 = fe.solve(d["rho"], MaterialModel.SIMP).copy()
    fe.bc.force *= 2.0  # in place
    u2 = fe.solve(d["rho"], MaterialModel.SIMP)
    np.testing.assert_allclose(u2, 2.0 * u1, rtol=0, atol=1e-9 * np.abs(u1).max())
    fe.bc.force = fe.bc.force / 2.0
    fe.bc.force.flags.writeable = False
    u3 = fe.solve(d["rho"], MaterialModel.SIMP)
    u4 = fe.solve(d["rho"], MaterialModel.SIMP)
    np.testing.assert_allclose(u3, u1, rtol=0, atol=1e-9 * np.abs(u1).max())
    np.testing.assert_array_equal(u3, u4)


def test_postprocess_pnorm_and_adjoint():
    from pyto_b200 import topopt_obj_cons_sensitivities as toc
    from pyto_b200 import topopt_material_model as tmm
    d = golden("cantilever_12x6x6_direct.npz")
    m, fe = _setup()
    u = fe.solve(d["rho"], tmm.MaterialModel.SIMP)
    tmm._PNORM_EXPONENT = 8
    try:
        fe.postprocess()
        np.testing.assert_allclose(fe.vonMisesStress, d["vm"], rtol=1e-8)
        np.testing.assert_allclose(fe.stressComponents, d["stress"], rtol=1e-8,
                                   atol=1e-11 * np.abs(d["stress"]).max())
        assert abs(fe.pNormStress - float(d["pnorm"])) <= 1e-9 * float(d["pnorm"])
        pn, dpn, mvm = toc.compute_pnorm_stress_and_sensitivity(u, d["rho"].copy(), fe, fe.elem_stiff[0],
                                                                tmm.MaterialModel.SIMP)
    finally:
        tmm._PNORM_EXPONENT = 6
    assert abs(pn - float(d["pn_val"])) <= 1e-9 * pn
    assert abs(mvm - float(d["pn_maxvm"])) <= 1e-9 * mvm
    np.testing.assert_allclose(dpn, d["pn_grad"], rtol=1e-6, atol=1e-9 * np.abs(d["pn_grad"]).max())
    obj, dobj = toc.compute_solution_dotproduct_and_gradient(u, d["rho"], fe, fe.elem_stiff[0],
                                                             tmm.MaterialModel.SIMP, d["gu_g"])
    assert abs(obj - float(d["gu_obj"])) <= 1e-9 * abs(obj)
    np.testing.assert_allclose(dobj, d["gu_grad"], rtol=1e-6, atol=1e-9 * np.abs(d["gu_grad"]).max())


def test_torch_in_torch_out_no_copies():
    from pyto_b200.topopt_material_model import MaterialModel
    d = golden("cantilever_12x6x6_direct.npz")
    m, fe = _setup()
    x = torch.as_tensor(d["rho"], device="cuda")
    u = fe.solve(x, MaterialModel.SIMP)
    assert isinstance(u, torch.Tensor) and u.is_cuda
    np.testing.assert_allclose(u.cpu().numpy(), d["u"], rtol=0, atol=1e-9 * np.abs(d["u"]).max())


def test_dpcg_through_linear_solvers():
    from pyto_b200 import deflation
    from pyto_b200.topopt_material_model import MaterialModel
    d = golden("cantilever_12x6x6_dpcg.npz")
    rho = golden("cantilever_12x6x6_direct.npz")["rho"]
    ds = deflation.DeflationSolver()
    from pyto_b200 import hex_mesher
    mm = hex_mesher.HexMesher()
    mm.grid_mesh((12, 6, 6), (1.0, 1.0, 1.0))
    ds.create_deflation_groups(mm, 8)
    ds.create_deflation_matrix(mm)
    m, fe = _setup(solver_name="DPCG", dsolver=ds, rtol=1e-10)
    u = fe.solve(rho, MaterialModel.SIMP)
    np.testing.assert_allclose(u, d["u"], rtol=0, atol=1e-7 * np.abs(d["u"]).max())
    assert ds.last_info.converged


def test_smoothing_filter_matches_reference():
    import scipy.sparse as sp
    from pyto_b200 import hex_mesher, topopt_filters
    fd = golden("filter.npz")
    m = hex_mesher.HexMesher()
    m.grid_mesh((12, 6, 6), (1.0, 1.0, 1.0))
    H, Hs = topopt_filters.createSmoothingFilter(m, 1.5)
    Href = sp.coo_matrix((fd["r15_val"], (fd["r15_row"], fd["r15_col"]))).tocsr()
    np.testing.assert_allclose(Hs, fd["r15_Hs"], rtol=1e-14)
    x = np.random.default_rng(0).uniform(size=m.num_elems)
    np.testing.assert_allclose(H @ x, Href @ x, rtol=1e-13)
    np.testing.assert_allclose(H * x, Href * x, rtol=1e-13)


def test_oc_history_matches_reference():
    from pyto_b200 import topopt_common as tc, topopt_ocm
    d = golden("oc_12x6x6.npz")
    m, fe = _setup(solver_name="SPSOLVE")
    params = tc.TOParams(Constraints=[(tc.TO_QOI.VOLUME_FRACTION, None, 0.3)], RelativeFilterRadius=1.5)
    sol, hist, ok, msg, n = topopt_ocm.topopt_optimality_criteria(
        tc.FEA_MODE.STRUCTURAL, fe, params, maxIterations=10, plot_progress=False, print_progress=False,
        binarize_topology=False)
    np.testing.assert_allclose(hist["objective"][:10], d["objective"][:10], rtol=1e-9)
    np.testing.assert_allclose(hist["volfrac"][:10], d["volfrac"][:10], rtol=1e-9)
    np.testing.assert_allclose(hist["objective"][10], d["objective"][10], rtol=1e-8)


def test_cfg1_oc_history_matches_reference():
    """Config 1: 60x30x30 cantilever, rho = 0.3, Jacobi PCG to 1e-8, sensitivity filter
    r = 1.5, volfrac 0.3, move 0.2: the 10-iteration OC objective history and the
    post-loop solve against the reference's own run (PCG tolerance 1e-8 on both sides,
    so the histories agree to the solver accuracy)."""
    from pyto_b200 import topopt_common as tc, topopt_ocm
    d = golden("cfg1_oc10.npz")
    m, fe = _setup(nel=(60, 30, 30), solver_name="PCG", rtol=1e-8)
    params = tc.TOParams(Constraints=[(tc.TO_QOI.VOLUME_FRACTION, None, 0.3)], RelativeFilterRadius=1.5)
    sol, hist, ok, msg, n = topopt_ocm.topopt_optimality_criteria(
        tc.FEA_MODE.STRUCTURAL, fe, params, maxIterations=10, plot_progress=False, print_progress=False,
        binarize_topology=False)
    np.testing.assert_allclose(hist["objective"][:11], d["objective"][:11], rtol=1e-6)
    np.testing.assert_allclose(hist["volfrac"][:10], d["volfrac"][:10], rtol=1e-7)


def test_nonzero_dirichlet_values():
    """Prescribed displacements are lifted into the right-hand side (src/bound_cond.py:58-60)."""
    import oracle as O
    from pyto_b200 import bound_cond, hex_mesher, hex_structural_fea, linear_solvers, mat_lib
    from pyto_b200.topopt_material_model import MaterialModel
    nel = (6, 3, 3)
    m = hex_mesher.HexMesher()
    m.grid_mesh(nel, (1.0, 1.0, 1.0))
    mo = O.grid_mesh(*nel)
    f, fixed = O.cantilever_bc(mo)
    gval = np.random.default_rng(3).normal(size=len(fixed)) * 1e-3
    bc = bound_cond.BC(force=f, fixed_dofs=fixed, dirichlet_values=gval)
    fe = hex_structural_fea.HexStructuralFEA(m, mat_lib.create_material_with_defaults("u", youngs_modulus=1.0,
                                                                                     poissons_ratio=0.3),
                                             bc, linear_solvers.Solvers.PCG, rtol=1e-13)
    rho = np.random.default_rng(4).uniform(0.1, 1.0, m.num_elems)
    u = fe.solve(rho, MaterialModel.SIMP)
    from pyto_b200 import topopt_material_model as tmm
    K = O.assemble_K(mo, O.simp_scaling(rho, 3.0, tmm._EVOID_RELATIVE), O.ke_hex8(1.0, 0.3))
    uref, _ = O.solve_fixed(K, f, fixed, g=gval)
    np.testing.assert_allclose(u, uref, rtol=0, atol=1e-9 * np.abs(uref).max())


def test_caller_enums_from_another_module():
    """A PyTO caller passes its own enum members (PyTO's Solvers, MaterialModel,
    FEA_MODE classes, not this package's): the same-named members select the same
    solver, material model and FEA mode."""
    import enum

    from pyto_b200 import hex_structural_fea, linear_solvers, topopt_obj_cons_sensitivities as toc

    class Solvers(enum.Enum):  # stand-ins with PyTO's class and member names
        SPSOLVE = enum.auto()
        PCG = enum.auto()
        PYAMG = enum.auto()
        DPCG = enum.auto()

    class MaterialModel(enum.Enum):
        SIMP = enum.auto()
        RAMP = enum.auto()

    class FEA_MODE(enum.Enum):
        STRUCTURAL = enum.auto()
        THERMAL = enum.auto()

    d = golden("cantilever_12x6x6_direct.npz")
    m, fe = _setup()
    fe.solver = Solvers.PCG
    u = fe.solve(d["rho"], MaterialModel.SIMP)
    np.testing.assert_allclose(u, d["u"], rtol=0, atol=1e-9 * np.abs(d["u"]).max())
    C, dC = toc.compute_compliance_and_gradient(FEA_MODE.STRUCTURAL, u, d["rho"], fe, fe.elem_stiff[0],
                                                MaterialModel.SIMP)
    assert abs(C - float(d["C"])) <= 1e-10 * float(d["C"])
    v = linear_solvers.solve(fe.stiff_mtrx, d["f"], Solvers.SPSOLVE, fe.bc, rtol=1e-12)
    np.testing.assert_allclose(v, d["u"], rtol=0, atol=1e-9 * np.abs(d["u"]).max())
    assert isinstance(fe, hex_structural_fea.HexStructuralFEA)
