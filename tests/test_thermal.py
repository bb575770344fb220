"""Thermal hex8 path through the C ABI against the oracle and the reference's
goldens (tests/golden/thermal.npz, from PyTO's HexThermalFEA)."""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import golden

pytestmark = pytest.mark.gpu

CASES = [("12x6x6", (12, 6, 6), (1.0, 1.0, 1.0)), ("9x5x4_box", (9, 5, 4), (1.0, 0.5, 2.0))]


@pytest.mark.parametrize("nel,h", [((12, 6, 6), (1.0, 1.0, 1.0)), ((9, 5, 4), (1.0, 0.5, 2.0)),
                                   ((1, 1, 1), (1.0, 1.0, 1.0)), ((40, 17, 23), (0.5, 0.5, 0.5))])
@pytest.mark.parametrize("mode", [0, 3, 2])
def test_thermal_matvec_matches_assembled_K(nel, h, mode):
    from pyto_b200.engine import ThermalGrid
    m = O.grid_mesh(*nel, h)
    rng = np.random.default_rng(4)
    s = rng.uniform(0.01, 1.0, m["num_elems"])
    u = rng.normal(size=m["num_nodes"])
    fixed = np.flatnonzero(m["node_indices"][:, 0] == 0)
    g = ThermalGrid(nel, h, 2.5).set_fixed_nodes(fixed)
    K = O.assemble_K_thermal(m, s, O.ke_hex8_thermal(2.5, h))
    uin = u.copy()
    if mode & 1:
        uin[fixed] = 0.0
    yref = K @ uin
    if mode & 2:
        yref[fixed] = 0.0
    y, dot = g.matvec(g.tensor(s), g.tensor(u), mode=mode, dot=True)
    assert np.abs(y.cpu().numpy() - yref).max() <= 1e-13 * np.abs(yref).max()
    assert abs(dot.item() - uin @ yref) <= 1e-12 * abs(uin @ yref)


@pytest.mark.parametrize("tag,nel,h", CASES)
def test_thermal_pcg_and_compliance_match_reference(tag, nel, h):
    from pyto_b200.engine import ThermalGrid
    d = golden("thermal.npz")
    g = ThermalGrid(nel, h, 1.0).set_fixed_nodes(d[f"{tag}_fixed"])
    s, ds = g.simp(g.tensor(d[f"{tag}_rho"]), float(d["penal"]), float(d["kvoid"]))
    T, info = g.pcg(s, g.tensor(d[f"{tag}_f"]), rtol=1e-12)
    assert info.converged and info.true_rel_res <= 1e-11, info
    np.testing.assert_allclose(T.cpu().numpy(), d[f"{tag}_T"], rtol=0, atol=1e-9 * np.abs(d[f"{tag}_T"]).max())
    ce, C = g.energy(T, s=s)
    assert abs(C.item() - float(d[f"{tag}_C"])) <= 1e-10 * float(d[f"{tag}_C"])
    np.testing.assert_allclose((-ds * ce).cpu().numpy(), d[f"{tag}_dC"], rtol=1e-8,
                               atol=1e-11 * np.abs(d[f"{tag}_dC"]).max())


def test_thermal_pcg_iterations_track_scipy():
    from pyto_b200.engine import ThermalGrid
    d = golden("thermal.npz")
    nel = (12, 6, 6)
    m = O.grid_mesh(*nel)
    s = O.thermal_scaling(d["12x6x6_rho"], float(d["penal"]), float(d["kvoid"]))
    K = O.assemble_K_thermal(m, s, O.ke_hex8_thermal(1.0))
    fixed = d["12x6x6_fixed"]
    free = np.setdiff1d(np.arange(m["num_nodes"]), fixed)
    A_ = K[free][:, free]
    _, it_ref = O.pcg_scipy(A_, d["12x6x6_f"][free], O.jacobi_inverse(A_), 1e-8)
    g = ThermalGrid(nel).set_fixed_nodes(fixed)
    _, info = g.pcg(g.tensor(s), g.tensor(d["12x6x6_f"]), rtol=1e-8, check_every=1)
    assert abs(info.iters - it_ref) <= 2, (info.iters, it_ref)


def test_hex_thermal_fea_dropin():
    """HexThermalFEA / linear_solvers / compute_compliance_and_gradient(THERMAL) used as
    PyTO code uses them, with non-zero prescribed temperatures lifted into the load."""
    from pyto_b200 import bound_cond, hex_mesher, hex_thermal_fea, linear_solvers, mat_lib
    from pyto_b200 import topopt_common as tc, topopt_material_model as tmm, topopt_obj_cons_sensitivities as toc
    d = golden("thermal.npz")
    tag, nel, h = CASES[1]
    kv, pen = tmm._KVOID_RELATIVE, tmm._SIMP_THERMAL_PENALTY
    tmm._KVOID_RELATIVE, tmm._SIMP_THERMAL_PENALTY = float(d["kvoid"]), float(d["penal"])
    try:
        m = hex_mesher.HexMesher()
        m.grid_mesh(nel, h)
        fixed = d[f"{tag}_fixed"]
        bc = bound_cond.BC(force=d[f"{tag}_f"].copy(), fixed_dofs=fixed, dirichlet_values=np.zeros(len(fixed)))
        mat = mat_lib.create_material_with_defaults("unit", thermal_conductivity=1.0)
        fe = hex_thermal_fea.HexThermalFEA(mesh=m, mat_prop=mat, bc=bc, solver=linear_solvers.Solvers.SPSOLVE)
        T = fe.solve(d[f"{tag}_rho"], tmm.MaterialModel.SIMP)
        np.testing.assert_allclose(T, d[f"{tag}_T"], rtol=0, atol=1e-9 * np.abs(d[f"{tag}_T"]).max())
        C, dC = toc.compute_compliance_and_gradient(tc.FEA_MODE.THERMAL, T, d[f"{tag}_rho"], fe, fe.elem_stiff[0],
                                                    tmm.MaterialModel.SIMP)
        assert abs(C - float(d[f"{tag}_C"])) <= 1e-10 * float(d[f"{tag}_C"])
        np.testing.assert_allclose(dC, d[f"{tag}_dC"], rtol=1e-8, atol=1e-11 * np.abs(d[f"{tag}_dC"]).max())
        # prescribed temperature 5 on the clamped face: T - 5 solves the zero-BC problem with
        # the load lifted, so the result is the zero-BC solution shifted by the lift's response
        bc2 = bound_cond.BC(force=d[f"{tag}_f"].copy(), fixed_dofs=fixed, dirichlet_values=np.full(len(fixed), 5.0))
        fe2 = hex_thermal_fea.HexThermalFEA(mesh=m, mat_prop=mat, bc=bc2, solver=linear_solvers.Solvers.PCG,
                                            rtol=1e-12)
        T2 = fe2.solve(d[f"{tag}_rho"], tmm.MaterialModel.SIMP)
        np.testing.assert_allclose(T2[fixed], 5.0)
        # a uniform shift is in the null space of the conduction operator: T2 = T + 5
        np.testing.assert_allclose(T2, T + 5.0, rtol=0, atol=1e-8 * np.abs(T).max())
    finally:
        tmm._KVOID_RELATIVE, tmm._SIMP_THERMAL_PENALTY = kv, pen
