"""The CPU oracle against vectors produced by the reference itself."""
import numpy as np
import pytest

import oracle as O
from conftest import golden


def test_ke_matches_reference():
    d = golden("ke.npz")
    for tag, (E, nu, h) in {"unit": (1.0, 0.3, (1, 1, 1)), "box": (1.0, 0.3, (1.0, 0.5, 2.0)),
                            "half": (2.5, 0.25, (0.5, 0.5, 0.5))}.items():
        np.testing.assert_allclose(O.ke_hex8(E, nu, h), d[f"ke_{tag}"], rtol=1e-14, atol=1e-15)


def test_grid_numbering_bit_exact():
    d = golden("mesh_3x2x4.npz")
    m = O.grid_mesh(3, 2, 4, (1.0, 0.5, 2.0))
    for k in ("node_indices", "elemArray", "elemNeighborsArray", "edof"):
        assert np.array_equal(m[k], d[k]), k
    assert np.array_equal(m["node_xyz"], d["node_xyz"])
    np.testing.assert_allclose(m["elem_centers"], d["elem_centers"], rtol=0, atol=1e-15)
    for a in range(3):
        for mn in (True, False):
            assert np.array_equal(O.nodes_on_plane(m, a, mn), d[f"plane_{a}_{int(mn)}"])


def test_material_model():
    d = golden("material.npz")
    x = d["x"]
    np.testing.assert_allclose(O.simp_scaling(x, 3.0, 1e-9), d["simp"], rtol=1e-15)
    np.testing.assert_allclose(O.simp_sensitivity(x, 3.0, 1e-9), d["dsimp"], rtol=1e-15)
    np.testing.assert_allclose(O.ramp_scaling(x, 5.0, 1e-9), d["ramp"], rtol=1e-15)
    np.testing.assert_allclose(O.ramp_sensitivity(x, 5.0, 1e-9), d["dramp"], rtol=1e-15)


def _case(name, nel, h):
    d = golden(name)
    m = O.grid_mesh(*nel, h)
    Ke = O.ke_hex8(1.0, 0.3, h)
    s = O.simp_scaling(d["rho"], 3.0, 1e-9)
    K = O.assemble_K(m, s, Ke)
    return d, m, Ke, K


@pytest.mark.parametrize("name,nel,h", [("cantilever_12x6x6_direct.npz", (12, 6, 6), (1.0, 1.0, 1.0)),
                                        ("cantilever_10x4x6_box_direct.npz", (10, 4, 6), (1.0, 0.5, 2.0))])
def test_direct_solve_objectives(name, nel, h):
    d, m, Ke, K = _case(name, nel, h)
    f, fixed = O.cantilever_bc(m)
    assert np.array_equal(f, d["f"]) and np.array_equal(fixed, d["fixed"])
    u, _ = O.solve_fixed(K, f, fixed, method="direct")
    np.testing.assert_allclose(u, d["u"], rtol=1e-10, atol=1e-12 * np.abs(d["u"]).max())
    C, dC, _ = O.compliance_and_gradient(u, d["rho"], m["edof"], Ke, 3.0, 1e-9)
    assert abs(C - d["C"]) <= 1e-11 * abs(d["C"])
    np.testing.assert_allclose(dC, d["dC"], rtol=1e-9, atol=1e-12 * np.abs(d["dC"]).max())
    post = O.postprocess(u, d["rho"], m["edof"], 1.0, 0.3, h, 0.5, 8.0)
    np.testing.assert_allclose(post["stress"], d["stress"], rtol=1e-9, atol=1e-12 * np.abs(d["stress"]).max())
    np.testing.assert_allclose(post["vm"], d["vm"], rtol=1e-9)
    assert abs(post["pnorm"] - d["pnorm"]) <= 1e-10 * d["pnorm"]
    solve = lambda g: O.solve_fixed(K, g, fixed, method="direct")[0]
    pn, dpn, mvm, _ = O.pnorm_stress_and_sensitivity(u, d["rho"], m["edof"], Ke, 1.0, 0.3, h, solve,
                                                     q=0.5, P=8.0, penal=3.0, emin=1e-9)
    assert abs(pn - d["pn_val"]) <= 1e-10 * pn
    np.testing.assert_allclose(dpn, d["pn_grad"], rtol=1e-7, atol=1e-10 * np.abs(d["pn_grad"]).max())
    obj, dobj = O.solution_dotproduct_and_gradient(u, d["rho"], m["edof"], Ke, d["gu_g"], solve, 3.0, 1e-9)
    assert abs(obj - d["gu_obj"]) <= 1e-10 * abs(obj)
    np.testing.assert_allclose(dobj, d["gu_grad"], rtol=1e-7, atol=1e-10 * np.abs(d["gu_grad"]).max())


def test_pcg_and_dpcg_reference_paths():
    d, m, Ke, K = _case("cantilever_12x6x6_direct.npz", (12, 6, 6), (1.0, 1.0, 1.0))
    f, fixed = O.cantilever_bc(m)
    u, info = O.solve_fixed(K, f, fixed, method="pcg", rtol=1e-10)
    dp = golden("cantilever_12x6x6_pcg.npz")
    assert abs(O.compliance_and_gradient(u, d["rho"], m["edof"], Ke, 3.0, 1e-9)[0] - dp["C"]) <= 1e-12 * dp["C"]
    grp, cnt, cen = O.deflation_groups(m["node_xyz"], 8)
    W = O.deflation_W(m["node_xyz"], grp, cen, len(cnt), 6)
    u2, _ = O.solve_fixed(K, f, fixed, method="dpcg", rtol=1e-10, dsolver={"W": W})
    dd = golden("cantilever_12x6x6_dpcg.npz")
    C2 = O.compliance_and_gradient(u2, d["rho"], m["edof"], Ke, 3.0, 1e-9)[0]
    assert abs(C2 - dd["C"]) <= 1e-10 * dd["C"]


@pytest.mark.parametrize("tag,nel,h,ng", [("a", (12, 6, 6), (1.0, 1.0, 1.0), 8), ("b", (12, 6, 6), (1.0, 1.0, 1.0), 39),
                                          ("c", (10, 3, 7), (1.0, 1.0, 1.0), 25), ("d", (9, 5, 4), (1.0, 0.5, 2.0), 20)])
def test_deflation_groups_bit_exact(tag, nel, h, ng):
    d = golden("deflation_groups.npz")
    m = O.grid_mesh(*nel, h)
    grp, cnt, cen = O.deflation_groups(m["node_xyz"], ng)
    assert np.array_equal(grp, d[f"{tag}_group"])
    assert np.array_equal(cnt, d[f"{tag}_count"])
    assert np.array_equal(cen, d[f"{tag}_center"])
    W = O.deflation_W(m["node_xyz"], grp, cen, len(cnt), 6).tocoo()
    Wr = __import__("scipy.sparse", fromlist=["x"]).coo_matrix(
        (d[f"{tag}_Wval"], (d[f"{tag}_Wrow"], d[f"{tag}_Wcol"])), shape=tuple(d[f"{tag}_shape"])).tocsr()
    assert (abs(W.tocsr() - Wr) > 0).nnz == 0


@pytest.mark.parametrize("tag,nel,h,r", [("r15", (12, 6, 6), (1.0, 1.0, 1.0), 1.5), ("r2", (12, 6, 6), (1.0, 1.0, 1.0), 2.0),
                                         ("box", (7, 5, 4), (1.0, 0.5, 2.0), 1.5)])
def test_filter(tag, nel, h, r):
    import scipy.sparse as sp
    d = golden("filter.npz")
    m = O.grid_mesh(*nel, h)
    H, Hs = O.smoothing_filter(m, r)
    Hr = sp.coo_matrix((d[f"{tag}_val"], (d[f"{tag}_row"], d[f"{tag}_col"])), shape=H.shape).tocsr()
    assert abs(H.tocsr() - Hr).max() <= 1e-15
    np.testing.assert_allclose(Hs, d[f"{tag}_Hs"], rtol=1e-14)


def test_oc_history_12x6x6():
    d = golden("oc_12x6x6.npz")
    m = O.grid_mesh(12, 6, 6)
    Ke = O.ke_hex8(1.0, 0.3)
    f, fixed = O.cantilever_bc(m)
    H, Hs = O.smoothing_filter(m, 1.5)

    def solve(x):
        return O.solve_fixed(O.assemble_K(m, O.simp_scaling(x, 3.0, 1e-9), Ke), f, fixed)[0]
    hist, _ = O.topopt_oc(m, Ke, f, solve, 0.3, 10, H, Hs, 0.2, 3.0, 1e-9)
    np.testing.assert_allclose(hist, d["objective"][:10], rtol=1e-9)


def test_cfg1_known_answers():
    d = golden("cfg1_pcg.npz")
    assert abs(float(d["C"]) - 54.33955968674) < 1e-9
    oc = golden("cfg1_oc10.npz")["objective"]
    np.testing.assert_allclose(oc[:3], [54.33955968674, 30.69814385124, 20.59204409203], rtol=1e-11)


@pytest.mark.parametrize("name,nel,h", [("cantilever_12x6x6_direct.npz", (12, 6, 6), (1.0, 1.0, 1.0)),
                                        ("cantilever_10x4x6_box_direct.npz", (10, 4, 6), (1.0, 0.5, 2.0))])
def test_matvec_ebe_against_reference_solution(name, nel, h):
    """The matrix-free oracle operator (used where an assembled K does not fit the
    host) applied to the reference's direct-solver displacement gives back the load
    on the free DOFs, and equals the assembled reduced operator."""
    d = golden(name)
    m = O.grid_mesh(*nel, h)
    Ke = O.ke_hex8(1.0, 0.3, h)
    s = O.simp_scaling(d["rho"], 3.0, 1e-9)
    y = O.matvec_ebe(nel, s, Ke, d["u"], d["fixed"], chunk=37)
    f = d["f"].copy()
    f[d["fixed"]] = 0.0
    assert np.linalg.norm(y - f) <= 1e-12 * np.linalg.norm(f)
    v = np.random.default_rng(3).normal(size=d["u"].shape)
    yref = O.matvec_free(m, s, Ke, v, d["fixed"])
    assert np.abs(O.matvec_ebe(nel, s, Ke, v, d["fixed"]) - yref).max() <= 1e-13 * np.abs(yref).max()


def test_thermal_ke_and_solve_match_reference():
    """Thermal hex8: the oracle's Ke, assembly and direct solve against the
    reference's HexThermalFEA (tests/golden/thermal.npz)."""
    d = golden("thermal.npz")
    np.testing.assert_allclose(O.ke_hex8_thermal(1.0, (1.0, 1.0, 1.0)), d["ke_unit"], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(O.ke_hex8_thermal(50.0, (1.0, 0.5, 2.0)), d["ke_box"], rtol=1e-13, atol=1e-13)
    import scipy.sparse.linalg as spl
    for tag, nel, h in (("12x6x6", (12, 6, 6), (1.0, 1.0, 1.0)), ("9x5x4_box", (9, 5, 4), (1.0, 0.5, 2.0))):
        m = O.grid_mesh(*nel, h)
        assert np.array_equal(m["elemArray"], d[f"{tag}_edof"])
        Ke = O.ke_hex8_thermal(1.0, h)
        s = O.thermal_scaling(d[f"{tag}_rho"], float(d["penal"]), float(d["kvoid"]))
        K = O.assemble_K_thermal(m, s, Ke)
        fixed = d[f"{tag}_fixed"]
        free = np.setdiff1d(np.arange(m["num_nodes"]), fixed)
        T = np.zeros(m["num_nodes"])
        T[free] = spl.spsolve(K[free][:, free].tocsc(), d[f"{tag}_f"][free])
        np.testing.assert_allclose(T, d[f"{tag}_T"], rtol=1e-10, atol=1e-12 * np.abs(T).max())
        ce = (T[m["elemArray"]] @ Ke * T[m["elemArray"]]).sum(1)
        assert abs(np.sum(s * ce) - float(d[f"{tag}_C"])) <= 1e-10 * float(d[f"{tag}_C"])
        dC = -O.thermal_sensitivity(d[f"{tag}_rho"], float(d["penal"]), float(d["kvoid"])) * ce
        np.testing.assert_allclose(dC, d[f"{tag}_dC"], rtol=1e-9, atol=1e-12 * np.abs(dC).max())


@pytest.mark.parametrize("tag,nel,h", [("a", (7, 5, 4), (1.0, 1.0, 1.0)), ("b", (6, 3, 5), (1.0, 0.5, 2.0))])
def test_symmetry_and_extrusion_filters_match_reference(tag, nel, h):
    """Mirror / extrusion filters and the composed H = H_s HX HZ HEY of createFilters
    against the reference's matrices (tests/golden/sym_filters.npz)."""
    import scipy.sparse as sp
    d = golden("sym_filters.npz")
    m = O.grid_mesh(*nel, h)
    ne = m["num_elems"]

    def ref(name):
        return sp.coo_matrix((d[f"{tag}_{name}_val"], (d[f"{tag}_{name}_row"], d[f"{tag}_{name}_col"])),
                             shape=(ne, ne)).toarray()
    for name, M in (("mx", O.mirror_filter(m, 0)), ("my", O.mirror_filter(m, 1)), ("mz", O.mirror_filter(m, 2)),
                    ("ex", O.extrude_filter(m, 0)), ("ey", O.extrude_filter(m, 1)), ("ez", O.extrude_filter(m, 2))):
        np.testing.assert_allclose(M.toarray(), ref(name), rtol=1e-15, atol=1e-15, err_msg=name)
    H, _ = O.smoothing_filter(m, 1.5)
    Ht = H @ O.mirror_filter(m, 0) @ O.mirror_filter(m, 2) @ O.extrude_filter(m, 1)
    np.testing.assert_allclose(Ht.toarray(), ref("all"), rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(np.asarray(Ht.sum(1)).ravel(), d[f"{tag}_all_Hs"], rtol=1e-13)


def test_mma_restatement_reaches_the_kkt_point():
    """The oracle's MMA (restated from the published algorithm; the reference's mmapy
    is not installed) on a convex separable problem, min sum c_i / x_i s.t.
    sum x_i <= V, reaches the closed-form optimum x_i = sqrt(c_i / lam)."""
    from oracle import mma as M
    rng = np.random.default_rng(0)
    n = 50
    cc = rng.uniform(1, 4, n)
    V = 0.4 * n
    x = np.full(n, 0.5)
    xold1, xold2, low, upp = x.copy(), x.copy(), np.zeros(n), np.ones(n)
    sc = None
    for it in range(1, 80):
        f0, df0 = np.sum(cc / x), -cc / x ** 2
        sc = f0 if sc is None else sc
        out = M.mmasub(1, n, it, x, np.full(n, 1e-3), np.ones(n), xold1, xold2, f0 / sc, df0 / sc,
                       np.array([x.sum() / V - 1]), np.ones((1, n)) / V, low, upp, 1.0, np.zeros(1),
                       np.full(1, 100.0), np.ones(1), 0.2)
        xold2, xold1, x = xold1, x, out[0]
        low, upp = out[-2], out[-1]
    lo, hi = 1e-6, 1e6
    for _ in range(200):
        lam = np.sqrt(lo * hi)
        xs = np.clip(np.sqrt(cc / lam), 1e-3, 1)
        lo, hi = (lam, hi) if xs.sum() > V else (lo, lam)
    assert np.abs(x - xs).max() < 1e-6
