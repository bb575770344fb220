"""Device MMA (pyto_mma_update / pyto_mma_kkt and the topopt_mma driver) against the
oracle's restatement of Svanberg's mmasub / subsolv / kktcheck (oracle/mma.py; the
reference's mmapy is not installed, so this parity is against the published
algorithm, not a run of the reference)."""
import numpy as np
import pytest
import torch

import oracle as O
from oracle import mma as M

pytestmark = pytest.mark.gpu


def _problem(n, m, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.1, 0.9, n)
    df0 = -rng.uniform(0.0, 2.0, n) * 1e-3 + rng.normal(0, 1e-4, n)
    dfdx = rng.uniform(0.5, 1.5, (m, n)) / n
    fval = rng.uniform(-0.2, 0.3, m)
    return x, df0, fval, dfdx


@pytest.mark.parametrize("m", [1, 2, 4])
@pytest.mark.parametrize("it", [1, 3])
def test_mma_update_matches_oracle(m, it):
    from pyto_b200.topopt_mma import DeviceMMA
    n = 5000
    x, df0, fval, dfdx = _problem(n, m, 7 + m)
    rng = np.random.default_rng(1)
    xold1 = np.clip(x + rng.normal(0, 0.05, n), 0.01, 0.99)
    xold2 = np.clip(xold1 + rng.normal(0, 0.05, n), 0.01, 0.99)
    low0 = x - rng.uniform(0.2, 0.6, n)
    upp0 = x + rng.uniform(0.2, 0.6, n)
    xmin, xmax = 1e-6, 1 - 1e-6
    ref = M.mmasub(m, n, it, x, np.full(n, xmin), np.full(n, xmax), xold1, xold2, 0.0, df0, fval, dfdx, low0, upp0,
                   1.0, np.zeros(m), np.full(m, 100.0), np.ones(m), 0.2)
    dev = torch.device("cuda")
    mm = DeviceMMA(n, m, xmin, xmax, 0.2, dev)
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    mm.iter = it - 1
    mm.xold1, mm.xold2 = T(xold1), T(xold2)
    mm.low.copy_(T(low0))
    mm.upp.copy_(T(upp0))
    xd = T(x)
    mm.update(xd, T(df0), fval, T(dfdx))
    np.testing.assert_allclose(mm.low.cpu().numpy(), ref[-2], rtol=1e-14, atol=1e-15)
    np.testing.assert_allclose(mm.upp.cpu().numpy(), ref[-1], rtol=1e-14, atol=1e-15)
    np.testing.assert_allclose(xd.cpu().numpy(), ref[0], rtol=0, atol=1e-9)
    dual = mm.dual.cpu().numpy()
    np.testing.assert_allclose(dual[1 + m:1 + 2 * m], ref[3], rtol=1e-6, atol=1e-9)  # lam
    # KKT residual of the original problem at the new point, new gradients
    df1 = df0 * 1.1
    f1 = fval + 0.01
    kn, km = mm.kkt(xd, T(df1), f1, T(dfdx))
    _, kref, kmref = M.kktcheck(m, n, ref[0], ref[1], ref[2], ref[3], ref[4], ref[5], ref[6], ref[7], ref[8],
                                np.full(n, xmin), np.full(n, xmax), df1, f1, dfdx, 1.0, np.zeros(m),
                                np.full(m, 100.0), np.ones(m))
    assert abs(kn - kref) <= 1e-6 * kref + 1e-12, (kn, kref)
    assert abs(km - kmref) <= 1e-6 * kmref + 1e-12, (km, kmref)


def test_mma_topology_run_matches_oracle_loop():
    """12x6x6 cantilever, density filter r = 1.5, volume fraction 0.3, move 0.2: the
    device driver's objective history against the same loop on the host with the
    oracle (direct solve, filter matrix, mmasub)."""
    from pyto_b200 import bound_cond, hex_mesher, hex_structural_fea, linear_solvers, mat_lib
    from pyto_b200 import topopt_common as tc, topopt_material_model as tmm
    from pyto_b200.topopt_mma import topopt_mma
    nel, iters, vf = (12, 6, 6), 6, 0.3
    ev = tmm._EVOID_RELATIVE
    tmm._EVOID_RELATIVE = 1e-9
    try:
        m = hex_mesher.HexMesher()
        m.grid_mesh(nel, (1.0, 1.0, 1.0))
        om = O.grid_mesh(*nel)
        f, fixed = O.cantilever_bc(om)
        bc = bound_cond.BC(force=f, fixed_dofs=fixed, dirichlet_values=np.zeros(len(fixed)))
        mat = mat_lib.create_material_with_defaults("unit", youngs_modulus=1.0, poissons_ratio=0.3)
        fe = hex_structural_fea.HexStructuralFEA(mesh=m, mat_prop=mat, bc=bc, solver=linear_solvers.Solvers.PCG,
                                                 rtol=1e-12)
        params = tc.TOParams(Constraints=[(tc.TO_QOI.VOLUME_FRACTION, None, vf)], RelativeFilterRadius=1.5)
        _, hist, ok, msg, nfea = topopt_mma(tc.FEA_MODE.STRUCTURAL, fe, None, params, maxiteration=iters,
                                            move_limit=0.2, kkt_tol=0.0, objective_tol=0.0, constraint_tol=0.0,
                                            print_progress=False, binarize_topology=False)
    finally:
        tmm._EVOID_RELATIVE = ev
    # the same loop on the host with the oracle
    Ke = O.ke_hex8(1.0, 0.3)
    H, Hs = O.smoothing_filter(om, 1.5)
    loaded = O.elements_with_forces(om, f)
    n = om["num_elems"]
    obj0, objs = None, []

    def fun(x):
        nonlocal obj0
        rho = (H @ x) / Hs
        u, _ = O.solve_fixed(O.assemble_K(om, O.simp_scaling(rho, 3.0, 1e-9), Ke), f, fixed)
        C, dC, _ = O.compliance_and_gradient(u, rho, om["edof"], Ke, 3.0, 1e-9)
        c = np.array([np.mean(rho) / vf - 1.0])
        dc = np.full((1, n), 1.0 / vf / n)
        obj0 = C if obj0 is None else obj0
        objs.append(C)
        g = dC / obj0
        g[loaded] = g.min()
        return C / obj0, H.T @ (g / Hs), c, (H.T @ (dc[0] / Hs))[None, :]

    x = np.full(n, vf)
    xmin, xmax = np.full(n, 1e-6), np.full(n, 1 - 1e-6)
    low, upp, xold1, xold2 = xmin.copy(), xmax.copy(), x.copy(), x.copy()
    f0, df0, gv, dg = fun(x)
    for it in range(1, iters + 1):
        out = M.mmasub(1, n, it, x, xmin, xmax, xold1, xold2, f0, df0, gv, dg, low, upp, 1.0, np.zeros(1),
                       np.full(1, 100.0), np.ones(1), 0.2)
        xold2, xold1, x = xold1, x, out[0]
        low, upp = out[-2], out[-1]
        f0, df0, gv, dg = fun(x)
    ref = np.array(objs)
    got = np.array(hist["objective"][:len(ref)])
    print("objective", got, ref)
    np.testing.assert_allclose(got, ref, rtol=1e-7)
    assert nfea == iters + 1
