"""Generate golden vectors by running the PyTO reference itself.

Run in a container where the reference checkout is available (it is read-only
and is never needed at test time):

    python tests/golden/gen_golden.py --ref /root/reference [--slow]

The reference's modules are imported from ``<ref>/src`` under a test-only
shim: plotting / optional packages (pyvista, stl, pyamg, matplotlib, ...) are
replaced by ``MagicMock``; ``pypardiso.spsolve`` is provided by a SuperLU
factorisation cached per matrix object (pypardiso reuses the factorisation of
an unchanged matrix); numba JITs from source into a scratch cache.  Outputs are
small ``.npz`` files next to this script.  ``--slow`` also runs the 60x30x30
10-iteration OC history (several minutes).
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile
import types
from unittest import mock

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl

HERE = os.path.dirname(os.path.abspath(__file__))


def install_shim(ref_root: str):
    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "pyto_numba_cache"))
    for m in ["pyvista", "stl", "pyamg", "matplotlib", "matplotlib.pyplot", "matplotlib.colors",
              "pyvistaqt", "mmapy", "trimesh"]:
        sys.modules[m] = mock.MagicMock()
    pard = types.ModuleType("pypardiso")
    cache = {}

    def spsolve(A, b):
        key = id(A)
        if key not in cache or cache[key][0] is not A:
            cache[key] = (A, spl.splu(sp.csc_matrix(A)))
        return cache[key][1].solve(np.asarray(b, dtype=float))
    pard.spsolve = spsolve
    pard.ps = types.SimpleNamespace(free_memory=lambda: None)
    sys.modules["pypardiso"] = pard
    sys.path.insert(0, os.path.join(ref_root, "src"))


def cantilever(mesh):
    ni = mesh.node_indices
    fixed_nodes = mesh.getNodesOnBoundingBoxPlane(0, True)
    fixed = np.sort(np.concatenate([3 * fixed_nodes + c for c in range(3)]))
    load = np.where((ni[:, 0] == mesh.grid[0]) & (ni[:, 2] == 0))[0]
    f = np.zeros(3 * mesh.num_nodes)
    f[3 * load + 2] = -1.0 / len(load)
    return f, fixed


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--slow", action="store_true")
    ap.add_argument("--thermal", action="store_true", help="only the thermal hex8 goldens")
    ap.add_argument("--filters", action="store_true", help="only the symmetry / extrusion filter goldens")
    ap.add_argument("--cfg13", action="store_true",
                    help="only the 60x30x30 tight-tolerance goldens (rho = 0.3 and the OC iterate-5 design)")
    args = ap.parse_args()
    install_shim(args.ref)
    if "--filters" in sys.argv:
        return sym_filters()
    ap_thermal = "--thermal" in sys.argv
    if args.cfg13:
        return cfg13()
    if ap_thermal:
        return thermal()
    import bound_cond
    import deflation
    import hex_element_stiffness as hes
    import hex_mesher
    import hex_structural_fea
    import linear_solvers
    import mat_lib
    import topopt_common
    import topopt_filters
    import topopt_material_model as tmm
    import topopt_obj_cons_sensitivities as toc
    import topopt_ocm

    tmm._EVOID_RELATIVE = 1e-9
    out = {}

    # ---- Ke -------------------------------------------------------------
    for tag, (E, nu, h) in {"unit": (1.0, 0.3, (1.0, 1.0, 1.0)),
                            "box": (1.0, 0.3, (1.0, 0.5, 2.0)),
                            "half": (2.5, 0.25, (0.5, 0.5, 0.5))}.items():
        out[f"ke_{tag}"] = hes.hex8_stiffness_matrix_structural(E, nu, h)
    np.savez_compressed(os.path.join(HERE, "ke.npz"), **out)

    # ---- mesh numbering ---------------------------------------------------
    hm = hex_mesher.HexMesher()
    hm.grid_mesh((3, 2, 4), (1.0, 0.5, 2.0))
    hm.createEdofMatStructural()
    planes = {f"plane_{a}_{int(m)}": hm.getNodesOnBoundingBoxPlane(a, m) for a in range(3) for m in (True, False)}
    np.savez_compressed(os.path.join(HERE, "mesh_3x2x4.npz"), node_xyz=hm.node_xyz, node_indices=hm.node_indices,
                        elemArray=hm.elemArray, elemNeighborsArray=hm.elemNeighborsArray,
                        elem_centers=hm.elem_centers, edof=hm.edofMatStructural, **planes)

    # ---- material model ----------------------------------------------------
    x = np.random.default_rng(7).uniform(0.0, 1.0, 50)
    np.savez_compressed(os.path.join(HERE, "material.npz"), x=x,
                        simp=tmm.get_structural_material_model_scaling(x, tmm.MaterialModel.SIMP),
                        dsimp=tmm.get_structural_material_model_sensitivity(x, tmm.MaterialModel.SIMP),
                        ramp=tmm.get_structural_material_model_scaling(x, tmm.MaterialModel.RAMP),
                        dramp=tmm.get_structural_material_model_sensitivity(x, tmm.MaterialModel.RAMP))

    # ---- cantilever solves, objectives, sensitivities -----------------------
    def fea_case(nel, h, solver, rho, dsolver=None, rtol=1e-10, pnorm=8):
        m = hex_mesher.HexMesher()
        m.grid_mesh(nel, h)
        m.createEdofMatStructural()
        f, fixed = cantilever(m)
        bc = bound_cond.BC(force=f, fixed_dofs=fixed, dirichlet_values=np.zeros(len(fixed)))
        mat = mat_lib.create_material_with_defaults("unit", youngs_modulus=1.0, poissons_ratio=0.3)
        fe = hex_structural_fea.HexStructuralFEA(mesh=m, mat_prop=mat, bc=bc, solver=solver,
                                                 dsolver=dsolver, rtol=rtol)
        u = fe.solve(rho, tmm.MaterialModel.SIMP)
        KE = fe.elem_stiff[0]
        C, dC = toc.compute_compliance_and_gradient(topopt_common.FEA_MODE.STRUCTURAL, u, rho, fe, KE,
                                                    tmm.MaterialModel.SIMP)
        tmm._PNORM_EXPONENT = pnorm
        fe.postprocess()
        res = dict(rho=rho, f=f, fixed=fixed, u=u, C=C, dC=dC, stress=fe.stressComponents,
                   vm=fe.vonMisesStress, pnorm=fe.pNormStress, sed=fe.elemStrainEnergy,
                   strain=fe.strainComponents, max_def=fe.max_deformation)
        pn, dpn, mvm = toc.compute_pnorm_stress_and_sensitivity(u, rho.copy(), fe, KE, tmm.MaterialModel.SIMP)
        res.update(pn_val=pn, pn_grad=dpn, pn_maxvm=mvm)
        g = np.random.default_rng(11).normal(size=u.shape)
        obj, dobj = toc.compute_solution_dotproduct_and_gradient(u, rho, fe, KE, tmm.MaterialModel.SIMP, g)
        res.update(gu_g=g, gu_obj=obj, gu_grad=dobj)
        tmm._PNORM_EXPONENT = 6
        return res, m, fe

    rho = np.random.default_rng(0).uniform(0.01, 1.0, 12 * 6 * 6)
    res, m12, _ = fea_case((12, 6, 6), (1.0, 1.0, 1.0), linear_solvers.Solvers.SPSOLVE, rho)
    np.savez_compressed(os.path.join(HERE, "cantilever_12x6x6_direct.npz"), **res)
    res_pcg, _, _ = fea_case((12, 6, 6), (1.0, 1.0, 1.0), linear_solvers.Solvers.PCG, rho)
    np.savez_compressed(os.path.join(HERE, "cantilever_12x6x6_pcg.npz"), u=res_pcg["u"], C=res_pcg["C"])
    rho_b = np.random.default_rng(3).uniform(0.05, 1.0, 10 * 4 * 6)
    res_b, _, _ = fea_case((10, 4, 6), (1.0, 0.5, 2.0), linear_solvers.Solvers.SPSOLVE, rho_b)
    np.savez_compressed(os.path.join(HERE, "cantilever_10x4x6_box_direct.npz"), **res_b)

    # ---- deflation groups / W / DPCG ----------------------------------------
    defl = {}
    for tag, (nel, h, ng) in {"a": ((12, 6, 6), (1.0, 1.0, 1.0), 8),
                              "b": ((12, 6, 6), (1.0, 1.0, 1.0), 39),
                              "c": ((10, 3, 7), (1.0, 1.0, 1.0), 25),
                              "d": ((9, 5, 4), (1.0, 0.5, 2.0), 20)}.items():
        m = hex_mesher.HexMesher()
        m.grid_mesh(nel, h)
        ds = deflation.DeflationSolver()
        with mock.patch("builtins.input", lambda *a, **k: ""):
            ds.create_deflation_groups(m, ng)
        ds.create_deflation_matrix(m)
        W = ds.W.tocoo()
        defl[f"{tag}_group"] = ds.ws_nodeGroupNumber
        defl[f"{tag}_count"] = ds.ws_groupCount
        defl[f"{tag}_center"] = ds.ws_groupCenter
        defl[f"{tag}_Wrow"], defl[f"{tag}_Wcol"], defl[f"{tag}_Wval"] = W.row, W.col, W.data
        defl[f"{tag}_shape"] = np.array(ds.W.shape)
    np.savez_compressed(os.path.join(HERE, "deflation_groups.npz"), **defl)
    ds = deflation.DeflationSolver()
    ds.create_deflation_groups(m12, 8)
    ds.create_deflation_matrix(m12)
    res_d, _, _ = fea_case((12, 6, 6), (1.0, 1.0, 1.0), linear_solvers.Solvers.DPCG, rho, dsolver=ds)
    np.savez_compressed(os.path.join(HERE, "cantilever_12x6x6_dpcg.npz"), u=res_d["u"], C=res_d["C"])

    # ---- smoothing filter ----------------------------------------------------
    filt = {}
    for tag, (nel, h, r) in {"r15": ((12, 6, 6), (1.0, 1.0, 1.0), 1.5),
                             "r2": ((12, 6, 6), (1.0, 1.0, 1.0), 2.0),
                             "box": ((7, 5, 4), (1.0, 0.5, 2.0), 1.5)}.items():
        m = hex_mesher.HexMesher()
        m.grid_mesh(nel, h)
        H, Hs = topopt_filters.createSmoothingFilter(m, r)
        Hc = H.tocoo()
        filt[f"{tag}_row"], filt[f"{tag}_col"], filt[f"{tag}_val"] = Hc.row, Hc.col, Hc.data
        filt[f"{tag}_Hs"] = Hs
    np.savez_compressed(os.path.join(HERE, "filter.npz"), **filt)

    # ---- OC (12x6x6, direct, r=1.5, volfrac 0.3, 10 iterations) --------------
    def run_oc(nel, solver, iters, dsolver=None):
        m = hex_mesher.HexMesher()
        m.grid_mesh(nel, (1.0, 1.0, 1.0))
        m.createEdofMatStructural()
        m.find_connected_components = lambda *a, **k: [np.arange(m.num_elems)]
        f, fixed = cantilever(m)
        bc = bound_cond.BC(force=f, fixed_dofs=fixed, dirichlet_values=np.zeros(len(fixed)))
        mat = mat_lib.create_material_with_defaults("unit", youngs_modulus=1.0, poissons_ratio=0.3)
        fe = hex_structural_fea.HexStructuralFEA(mesh=m, mat_prop=mat, bc=bc, solver=solver, dsolver=dsolver,
                                                 rtol=1e-8)
        fe.plot_pseudo_density_realtime = lambda *a, **k: None
        params = topopt_common.TOParams(Constraints=[(topopt_common.TO_QOI.VOLUME_FRACTION, None, 0.3)],
                                        RelativeFilterRadius=1.5)
        xs = []
        orig = fe.solve

        def solve_rec(x, mm=tmm.MaterialModel.SIMP):
            xs.append(np.array(x, copy=True))
            return orig(x, mm)
        fe.solve = solve_rec
        sol, hist, ok, msg, n = topopt_ocm.topopt_optimality_criteria(
            topopt_common.FEA_MODE.STRUCTURAL, fe, params, maxIterations=iters, plot_progress=False,
            print_progress=False, binarize_topology=False)
        return np.array(hist["objective"]), np.array(hist["volfrac"]), np.array(hist["change"]), np.array(xs)

    h, v, c, xs = run_oc((12, 6, 6), linear_solvers.Solvers.SPSOLVE, 10)
    np.savez_compressed(os.path.join(HERE, "oc_12x6x6.npz"), objective=h, volfrac=v, change=c, x_iter=xs)

    # ---- L-shaped domain (config-4 shape at 8x4x4): p-norm adjoint -----------
    nel = (8, 4, 4)
    m = hex_mesher.HexMesher()
    m.grid_mesh(nel, (1.0, 1.0, 1.0))
    m.createEdofMatStructural()
    ex = np.arange(m.num_elems) % 8
    ez = np.arange(m.num_elems) // 32
    active = ~((ex >= 4) & (ez >= 2))
    used = np.zeros(m.num_nodes, bool)
    used[m.elemArray[active].ravel()] = True
    f, fixed = cantilever(m)
    unused = np.where(~used)[0]
    fixed = np.union1d(fixed, np.concatenate([3 * unused + c for c in range(3)]))
    sub = types.SimpleNamespace(**{k: getattr(m, k) for k in ("num_nodes", "elem_size", "node_xyz", "grid",
                                                              "node_indices")})
    sub.num_elems = int(active.sum())
    sub.edofMatStructural = m.edofMatStructural[active]
    sub.elemArray = m.elemArray[active]
    bc = bound_cond.BC(force=f, fixed_dofs=fixed, dirichlet_values=np.zeros(len(fixed)))
    mat = mat_lib.create_material_with_defaults("unit", youngs_modulus=1.0, poissons_ratio=0.3)
    fe = hex_structural_fea.HexStructuralFEA(mesh=sub, mat_prop=mat, bc=bc, solver=linear_solvers.Solvers.SPSOLVE)
    rho_l = np.random.default_rng(0).uniform(0.2, 1.0, sub.num_elems)
    u = fe.solve(rho_l, tmm.MaterialModel.SIMP)
    tmm._PNORM_EXPONENT = 8
    fe.postprocess()
    pn, dpn, mvm = toc.compute_pnorm_stress_and_sensitivity(u, rho_l.copy(), fe, fe.elem_stiff[0],
                                                            tmm.MaterialModel.SIMP)
    C, dC = toc.compute_compliance_and_gradient(topopt_common.FEA_MODE.STRUCTURAL, u, rho_l, fe, fe.elem_stiff[0],
                                                tmm.MaterialModel.SIMP)
    tmm._PNORM_EXPONENT = 6
    np.savez_compressed(os.path.join(HERE, "lshape_8x4x4.npz"), active=active, rho=rho_l, f=f, fixed=fixed, u=u,
                        pnorm=pn, pn_grad=dpn, pn_maxvm=mvm, vm=fe.vonMisesStress, C=C, dC=dC)

    # ---- config-1 grid: one PCG solve at rho = 0.3 -------------------------------
    rho1 = 0.3 * np.ones(60 * 30 * 30)
    m = hex_mesher.HexMesher()
    m.grid_mesh((60, 30, 30), (1.0, 1.0, 1.0))
    m.createEdofMatStructural()
    f, fixed = cantilever(m)
    bc = bound_cond.BC(force=f, fixed_dofs=fixed, dirichlet_values=np.zeros(len(fixed)))
    mat = mat_lib.create_material_with_defaults("unit", youngs_modulus=1.0, poissons_ratio=0.3)
    fe = hex_structural_fea.HexStructuralFEA(mesh=m, mat_prop=mat, bc=bc, solver=linear_solvers.Solvers.PCG,
                                             rtol=1e-8)
    u = fe.solve(rho1, tmm.MaterialModel.SIMP)
    C1, _ = toc.compute_compliance_and_gradient(topopt_common.FEA_MODE.STRUCTURAL, u, rho1, fe, fe.elem_stiff[0],
                                                tmm.MaterialModel.SIMP)
    sample = np.arange(0, m.num_nodes * 3, 997)
    np.savez_compressed(os.path.join(HERE, "cfg1_pcg.npz"), C=C1, max_def=fe.max_deformation,
                        sample_idx=sample, u_sample=u[sample])
    if args.slow:
        h, v, c, _ = run_oc((60, 30, 30), linear_solvers.Solvers.PCG, 10)
        np.savez_compressed(os.path.join(HERE, "cfg1_oc10.npz"), objective=h, volfrac=v, change=c)
    print("golden vectors written to", HERE)


def sym_filters():
    """Symmetry and extrusion filters (src/topopt_filters.py:292-393, :595-716) and their
    composition with the smoothing filter by createFilters (src/topopt_common.py:127-159)
    on small full grids."""
    import hex_mesher
    import topopt_common
    import topopt_filters as tf

    out = {}
    for tag, nel, h in (("a", (7, 5, 4), (1.0, 1.0, 1.0)), ("b", (6, 3, 5), (1.0, 0.5, 2.0))):
        m = hex_mesher.HexMesher()
        m.grid_mesh(nel, h)
        for name, fn in (("mx", tf.createXSymmetryFilter), ("my", tf.createYSymmetryFilter),
                         ("mz", tf.createZSymmetryFilter), ("ex", tf.createXExtrudeFilter),
                         ("ey", tf.createYExtrudeFilter), ("ez", tf.createZExtrudeFilter)):
            Hc = fn(m).tocoo()
            out[f"{tag}_{name}_row"], out[f"{tag}_{name}_col"], out[f"{tag}_{name}_val"] = Hc.row, Hc.col, Hc.data
        params = topopt_common.TOParams(RelativeFilterRadius=1.5, XSymmetry=True, ZSymmetry=True, ExtrudeY=True)
        H, Hs = topopt_common.createFilters(types.SimpleNamespace(mesh=m), params)
        Hc = H.tocoo()
        out[f"{tag}_all_row"], out[f"{tag}_all_col"], out[f"{tag}_all_val"] = Hc.row, Hc.col, Hc.data
        out[f"{tag}_all_Hs"] = Hs
    np.savez_compressed(os.path.join(HERE, "sym_filters.npz"), **out)
    print("sym_filters.npz written")


def thermal():
    """Thermal hex8 goldens: Ke (src/hex_element_stiffness.py:340-385) for two element
    sizes, and one HexThermalFEA solve (src/hex_thermal_fea.py:19-117) of a 12x6x6 heat
    sink: temperature 0 on the x = 0 face, a uniform unit heat load shared by all
    nodes, SIMP thermal scaling of rho ~ U[0.01, 1] (seed 0), direct solver; the
    thermal compliance and its gradient (src/topopt_obj_cons_sensitivities.py:148-179)."""
    import bound_cond
    import hex_element_stiffness as hes
    import hex_mesher
    import hex_thermal_fea
    import linear_solvers
    import mat_lib
    import topopt_common
    import topopt_material_model as tmm
    import topopt_obj_cons_sensitivities as toc

    tmm._KVOID_RELATIVE = 1e-3
    tmm._SIMP_THERMAL_PENALTY = 3
    out = {f"ke_{tag}": hes.hex8_stiffness_matrix_thermal(k, h)
           for tag, (k, h) in {"unit": (1.0, (1.0, 1.0, 1.0)), "box": (50.0, (1.0, 0.5, 2.0))}.items()}
    for tag, nel, h in (("12x6x6", (12, 6, 6), (1.0, 1.0, 1.0)), ("9x5x4_box", (9, 5, 4), (1.0, 0.5, 2.0))):
        m = hex_mesher.HexMesher()
        m.grid_mesh(nel, h)
        m.createEdofMatThermal()
        fixed = np.sort(m.getNodesOnBoundingBoxPlane(0, True))
        f = np.full(m.num_nodes, 1.0 / m.num_nodes)
        bc = bound_cond.BC(force=f, fixed_dofs=fixed, dirichlet_values=np.zeros(len(fixed)))
        mat = mat_lib.create_material_with_defaults("unit", thermal_conductivity=1.0)
        fe = hex_thermal_fea.HexThermalFEA(mesh=m, mat_prop=mat, bc=bc, solver=linear_solvers.Solvers.SPSOLVE)
        rho = np.random.default_rng(0).uniform(0.01, 1.0, m.num_elems)
        T = fe.solve(rho, tmm.MaterialModel.SIMP)
        C, dC = toc.compute_compliance_and_gradient(topopt_common.FEA_MODE.THERMAL, T, rho, fe, fe.elem_stiff[0],
                                                    tmm.MaterialModel.SIMP)
        out.update({f"{tag}_rho": rho, f"{tag}_f": f, f"{tag}_fixed": fixed, f"{tag}_T": T, f"{tag}_C": C,
                    f"{tag}_dC": dC, f"{tag}_edof": m.edofMatThermal})
        print(tag, "C =", repr(C))
    np.savez_compressed(os.path.join(HERE, "thermal.npz"), kvoid=1e-3, penal=3.0, **out)


def cfg13():
    """60x30x30 cantilever goldens at rtol 1e-12 (compliance parity to 1e-10):
    rho = 0.3 uniform, and the design after 5 OC updates of the reference's own OC
    loop (PCG at rtol 1e-8, sensitivity filter r = 1.5, volfrac 0.3, move 0.2).
    The reference's PCG path (scipy cg, src/linear_solvers.py:164-168) solves both."""
    import bound_cond
    import hex_mesher
    import hex_structural_fea
    import linear_solvers
    import mat_lib
    import topopt_common
    import topopt_material_model as tmm
    import topopt_obj_cons_sensitivities as toc
    import topopt_ocm

    tmm._EVOID_RELATIVE = 1e-9
    nel = (60, 30, 30)

    def fea(rtol):
        m = hex_mesher.HexMesher()
        m.grid_mesh(nel, (1.0, 1.0, 1.0))
        m.createEdofMatStructural()
        m.find_connected_components = lambda *a, **k: [np.arange(m.num_elems)]
        f, fixed = cantilever(m)
        bc = bound_cond.BC(force=f, fixed_dofs=fixed, dirichlet_values=np.zeros(len(fixed)))
        mat = mat_lib.create_material_with_defaults("unit", youngs_modulus=1.0, poissons_ratio=0.3)
        fe = hex_structural_fea.HexStructuralFEA(mesh=m, mat_prop=mat, bc=bc, solver=linear_solvers.Solvers.PCG,
                                                 rtol=rtol)
        fe.plot_pseudo_density_realtime = lambda *a, **k: None
        return m, fe

    def tight(rho, name):
        m, fe = fea(1e-12)
        u = fe.solve(rho, tmm.MaterialModel.SIMP)
        C, _ = toc.compute_compliance_and_gradient(topopt_common.FEA_MODE.STRUCTURAL, u, rho, fe, fe.elem_stiff[0],
                                                   tmm.MaterialModel.SIMP)
        sample = np.arange(0, m.num_nodes * 3, 997)
        np.savez_compressed(os.path.join(HERE, name), rho=rho, C=C, max_def=fe.max_deformation,
                            u_absmax=np.abs(u).max(), sample_idx=sample, u_sample=u[sample])
        print(name, "C =", repr(C))

    tight(0.3 * np.ones(int(np.prod(nel))), "cfg1_pcg_tight.npz")
    m, fe = fea(1e-8)
    params = topopt_common.TOParams(Constraints=[(topopt_common.TO_QOI.VOLUME_FRACTION, None, 0.3)],
                                    RelativeFilterRadius=1.5)
    xs = []
    orig = fe.solve

    def solve_rec(x, mm=tmm.MaterialModel.SIMP):
        xs.append(np.array(x, copy=True))
        return orig(x, mm)
    fe.solve = solve_rec
    topopt_ocm.topopt_optimality_criteria(topopt_common.FEA_MODE.STRUCTURAL, fe, params, maxIterations=5,
                                          plot_progress=False, print_progress=False, binarize_topology=False)
    # xs[k] is the design of the k-th solve; xs[5] is the design after 5 OC updates
    tight(xs[5], "cfg3_oc5_pcg_tight.npz")


if __name__ == "__main__":
    main()
