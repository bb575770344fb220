"""The oracle's compiled half (oracle/hex8_cpu.c, the timed CPU baseline) against
the numpy oracle and the reference's goldens: the CSR it assembles is the
reference's reduced matrix, its PCG and DPCG follow the reference's recurrences
(iteration counts and compliance), and its density filter and coarse matrix are
the reference's.  CPU only."""
import numpy as np
import pytest

import oracle as O
from conftest import golden
from oracle import cpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    cpu.build()


@pytest.mark.parametrize("nel,h", [((12, 6, 6), (1.0, 1.0, 1.0)), ((5, 3, 4), (1.0, 0.5, 2.0)),
                                   ((1, 1, 1), (1.0, 1.0, 1.0))])
def test_csr_is_the_reference_reduced_matrix(nel, h):
    m = O.grid_mesh(*nel, h)
    Ke = O.ke_hex8(1.0, 0.3, h)
    s = np.random.default_rng(2).uniform(0.01, 1.0, m["num_elems"])
    f, fixed = O.cantilever_bc(m)
    fea = cpu.CpuFEA(nel, Ke, fixed, h)
    fea.assemble(s)
    A, _, _ = O.impose_dirichlet_bc(O.assemble_K(m, s, Ke), f, fixed, np.zeros(len(fixed)))
    A = A.tocsr()
    A.sort_indices()
    K = fea.csr()
    assert np.array_equal(K.indptr, A.indptr) and np.array_equal(K.indices, A.indices)
    assert np.abs(K.data - A.data).max() <= 1e-15 * np.abs(A.data).max()


def test_pcg_matches_reference_golden():
    d = golden("cantilever_12x6x6_direct.npz")
    nel = (12, 6, 6)
    m = O.grid_mesh(*nel)
    Ke = O.ke_hex8(1.0, 0.3)
    fea = cpu.CpuFEA(nel, Ke, d["fixed"])
    fea.assemble(O.simp_scaling(d["rho"], 3.0, 1e-9))
    u, info = fea.pcg(d["f"], rtol=1e-12)
    assert info["rc"] == 0 and info["true_rel_res"] < 1e-11
    C = O.compliance_and_gradient(u, d["rho"], m["edof"], Ke, 3.0, 1e-9)[0]
    assert abs(C - d["C"]) <= 1e-10 * abs(d["C"])
    # scipy cg's iteration count on the same reduced system
    K = O.assemble_K(m, O.simp_scaling(d["rho"], 3.0, 1e-9), Ke)
    A_, b_, _ = O.impose_dirichlet_bc(K, d["f"], d["fixed"], np.zeros(len(d["fixed"])))
    _, it_ref = O.pcg_scipy(A_, b_, O.jacobi_inverse(A_), 1e-8)
    _, info8 = fea.pcg(d["f"], rtol=1e-8)
    assert abs(info8["iters"] - it_ref) <= 1, (info8["iters"], it_ref)


def test_dpcg_matches_oracle_and_reference():
    d = golden("cantilever_12x6x6_direct.npz")
    nel = (12, 6, 6)
    m = O.grid_mesh(*nel)
    Ke = O.ke_hex8(1.0, 0.3)
    s = O.simp_scaling(d["rho"], 3.0, 1e-9)
    fea = cpu.CpuFEA(nel, Ke, d["fixed"])
    fea.assemble(s)
    grp, cnt, cen = O.deflation_groups(m["node_xyz"], 8)
    # the reference's settings: absolute shift 1e-10, stop on sqrt(r.z / r0.z0)
    u, info = fea.dpcg(d["f"], grp, cen, modes=6, shift=1e-10, shift_relative=False, rtol=1e-10, stop_rule=1)
    K = O.assemble_K(m, s, Ke)
    A_, b_, free = O.impose_dirichlet_bc(K, d["f"], d["fixed"], np.zeros(len(d["fixed"])))
    W = O.deflation_W(m["node_xyz"], grp, cen, len(cnt), 6)[free]
    _, it_ref = O.dpcg(A_, b_, W, O.jacobi_inverse(A_), rtol=1e-10)
    assert info["rc"] == 0 and info["iters"] == it_ref, (info, it_ref)
    C = O.compliance_and_gradient(u, d["rho"], m["edof"], Ke, 3.0, 1e-9)[0]
    assert abs(C - float(golden("cantilever_12x6x6_dpcg.npz")["C"])) <= 1e-9 * abs(d["C"])
    # the bench settings: relative shift, stop on the residual norm
    u2, info2 = fea.dpcg(d["f"], grp, cen, modes=6, rtol=1e-8)
    assert info2["rc"] == 0 and info2["true_rel_res"] <= 1.0001e-8
    C2 = O.compliance_and_gradient(u2, d["rho"], m["edof"], Ke, 3.0, 1e-9)[0]
    assert abs(C2 - d["C"]) <= 1e-8 * abs(d["C"])


@pytest.mark.parametrize("modes", [6, 3])
def test_coarse_matrix_is_wtkw(modes):
    nel = (10, 3, 7)
    m = O.grid_mesh(*nel)
    Ke = O.ke_hex8(1.0, 0.3)
    s = np.random.default_rng(5).uniform(0.01, 1.0, m["num_elems"])
    f, fixed = O.cantilever_bc(m)
    fea = cpu.CpuFEA(nel, Ke, fixed)
    fea.assemble(s)
    grp, cnt, cen = O.deflation_groups(m["node_xyz"], 25)
    A_, _, free = O.impose_dirichlet_bc(O.assemble_K(m, s, Ke), f, fixed, np.zeros(len(fixed)))
    W = O.deflation_W(m["node_xyz"], grp, cen, len(cnt), modes)[free]
    Eo = (W.T @ A_ @ W).toarray()
    E = fea.coarse_matrix(grp, cen, modes)
    assert np.abs(E - Eo).max() <= 1e-13 * np.abs(Eo).max()


@pytest.mark.parametrize("tag,nel,h,r", [("r15", (12, 6, 6), (1.0, 1.0, 1.0), 1.5),
                                         ("r2", (12, 6, 6), (1.0, 1.0, 1.0), 2.0),
                                         ("box", (7, 5, 4), (1.0, 0.5, 2.0), 1.5)])
def test_density_filter_is_the_reference_filter(tag, nel, h, r):
    g = golden("filter.npz")
    import scipy.sparse as sp
    ne = int(np.prod(nel))
    H = sp.coo_matrix((g[f"{tag}_val"], (g[f"{tag}_row"], g[f"{tag}_col"])), shape=(ne, ne)).tocsr()
    x = np.random.default_rng(1).uniform(0.01, 1.0, ne)
    rho = cpu.density_filter(nel, x, r, h)
    np.testing.assert_allclose(rho, (H @ x) / g[f"{tag}_Hs"], rtol=1e-13, atol=0)


def test_cfg1_tight_golden():
    """60x30x30, rho = 0.3: the port's PCG at rtol 1e-12 against the reference's own
    PCG at rtol 1e-12 (tests/golden/cfg1_pcg_tight.npz), compliance to 1e-10."""
    d = golden("cfg1_pcg_tight.npz")
    nel = (60, 30, 30)
    m = O.grid_mesh(*nel)
    f, fixed = O.cantilever_bc(m)
    Ke = O.ke_hex8(1.0, 0.3)
    fea = cpu.CpuFEA(nel, Ke, fixed)
    fea.assemble(O.simp_scaling(d["rho"], 3.0, 1e-9))
    u, info = fea.pcg(f, rtol=1e-12)
    assert info["rc"] == 0
    C = float(f @ u)
    assert abs(C - float(d["C"])) <= 1e-10 * float(d["C"])
    np.testing.assert_allclose(u[d["sample_idx"]], d["u_sample"], rtol=0, atol=1e-9 * float(d["u_absmax"]))
