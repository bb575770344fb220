"""Parity at the sizes of the benchmarked configurations, through the C ABI.

* 60x30x30 cantilever (rho = 0.3, and the design after 5 OC updates of the
  reference's own OC loop): FP64 solves against the reference's PCG at rtol
  1e-12 (compliance to 1e-10), and the mixed-precision solve's compliance,
  maximum displacement and iteration count against the FP64 oracle.
* 192x96x96 (5.4M DOF): the true residual of the GPU solutions recomputed on the
  host by the oracle's matrix-free operator, and f.u against the GPU compliance.
* The batched workload at its full sizes: every problem converged, and the true
  residual of a seeded sample of designs and of all 8 load cases of the
  128x64x64 design recomputed on the host.
"""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import golden
from oracle import cpu

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def _host_true_res(nel, s, u, f, fixed, Ke=None):
    """||f_f - K_ff u|| / ||f_f|| with the oracle's operator, on the host."""
    Ke = O.ke_hex8(1.0, 0.3) if Ke is None else Ke
    ff = np.array(f, dtype=np.float64, copy=True)
    ff[fixed] = 0.0
    r = ff - O.matvec_ebe(nel, s, Ke, u, fixed)
    return np.linalg.norm(r) / np.linalg.norm(ff)


def _cfg1_grid():
    from pyto_b200.deflation import DeflationSolver
    from pyto_b200.engine import HexGrid
    from pyto_b200.hex_mesher import HexMesher
    from pyto_b200.problems import cantilever
    nel = (60, 30, 30)
    mesh = HexMesher()
    mesh.grid_mesh(nel, (1.0, 1.0, 1.0))
    f, fixed = cantilever(mesh)
    g = HexGrid(nel).set_fixed_dofs(fixed)
    ds = DeflationSolver(modes=6, shift=1e-14, shift_relative=True)
    ds.create_deflation_groups(mesh, ds.getRecommendedNumberOfGroups(g.ndof))
    return nel, mesh, f, fixed, g, ds


@pytest.mark.parametrize("name", ["cfg1_pcg_tight.npz", "cfg3_oc5_pcg_tight.npz"])
def test_cfg1_fp64_compliance_1e10(name):
    """FP64 Jacobi PCG and FP64 deflated PCG (residual replacement) at rtol 1e-12
    against the reference's PCG at rtol 1e-12: compliance to 1e-10 relative."""
    d = golden(name)
    nel, mesh, f, fixed, g, ds = _cfg1_grid()
    s, _ = g.simp(_dev(d["rho"]), 3.0, 1e-9)
    F = _dev(f)
    u, info = g.pcg(s, F, rtol=1e-12)
    # the recurrence stops on its own residual (scipy cg's rule); the true one drifts a little
    assert info.converged and info.true_rel_res <= 1e-11, info
    _, C = g.energy(u, s=s)
    assert abs(C.item() - float(d["C"])) <= 1e-10 * float(d["C"]), (C.item(), float(d["C"]))
    np.testing.assert_allclose(u.cpu().numpy()[d["sample_idx"]], d["u_sample"], rtol=0,
                               atol=1e-9 * float(d["u_absmax"]))
    defl = ds.device_deflation(g)
    u2, info2 = g.dpcg(s, F, defl, rtol=1e-12, stop_rule=2, max_iters=5000)
    assert info2.converged and info2.true_rel_res <= 1e-12, info2
    _, C2 = g.energy(u2, s=s)
    assert abs(C2.item() - float(d["C"])) <= 1e-10 * float(d["C"]), (C2.item(), float(d["C"]))


@pytest.mark.parametrize("name", ["cfg1_pcg_tight.npz", "cfg3_oc5_pcg_tight.npz"])
def test_cfg3_mixed_against_fp64_oracle(name):
    """Mixed precision (FP32 deflated PCG inside FP64 residual replacement, FP64
    coarse solve) to true rel-residual 1e-8 on the 60x30x30 grid: its compliance,
    maximum displacement and iteration count against the FP64 oracle (the compiled
    restatement of the reference's deflated PCG, same coarse space, rtol 1e-8) and
    against the reference's tight solve."""
    d = golden(name)
    nel, mesh, f, fixed, g, ds = _cfg1_grid()
    rho = np.asarray(d["rho"])
    s, _ = g.simp(_dev(rho), 3.0, 1e-9)
    defl = ds.device_deflation(g)
    u, info = g.dpcg_mixed(s, _dev(f), defl, rtol=1e-8)
    assert info.converged and info.true_rel_res <= 1e-8, info
    uh = u.cpu().numpy()
    sh = s.cpu().numpy()
    assert _host_true_res(nel, sh, uh, f, fixed) <= 1.0001e-8
    # FP64 oracle solution: the compiled restatement of the reference's Jacobi PCG on the
    # assembled K_ff at rtol 1e-10
    fea = cpu.CpuFEA(nel, O.ke_hex8(1.0, 0.3), fixed)
    fea.assemble(sh)
    uo, _ = fea.pcg(f, rtol=1e-10)
    # FP64 iteration count: the reference's deflated PCG recurrence, same groups, rtol 1e-8
    _, io = fea.dpcg(f, ds.ws_nodeGroupNumber, ds.ws_groupCenter, modes=6, shift=1e-14, shift_relative=True,
                     rtol=1e-8)
    # and the library's FP64 deflated PCG with residual replacement (robust where the
    # reference's recurrence stagnates)
    _, i64 = g.dpcg(s, _dev(f), defl, rtol=1e-8, stop_rule=2, max_iters=5000)
    assert i64.converged
    _, C = g.energy(u, s=s)
    C, Co, Cref = C.item(), float(f @ uo), float(d["C"])
    dmax, dmax_o = np.abs(uh).max(), np.abs(uo).max()
    err = dict(compliance_vs_oracle=abs(C - Co) / Co, compliance_vs_reference_tight=abs(C - Cref) / Cref,
               max_disp_vs_oracle=abs(dmax - dmax_o) / dmax_o,
               max_disp_vs_reference_tight=abs(dmax - float(d["u_absmax"])) / float(d["u_absmax"]),
               iterations=info.iters, oracle_dpcg_iterations=io["iters"] if io["rc"] == 0 else "not converged",
               fp64_gpu_iterations=i64.iters)
    print(name, err)
    assert err["compliance_vs_reference_tight"] <= 1e-8 and err["compliance_vs_oracle"] <= 1e-8, err
    assert err["max_disp_vs_reference_tight"] <= 1e-7 and err["max_disp_vs_oracle"] <= 1e-7, err
    ref_iters = io["iters"] if io["rc"] == 0 else i64.iters
    assert abs(info.iters - ref_iters) <= 0.05 * ref_iters + 2, err


@pytest.fixture(scope="module")
def cfg2():
    import bench
    P = bench.build(torch.device("cuda", 0), bench.NEL, 432, 6)
    return P


@pytest.mark.parametrize("form", ["mixed", "fp64"])
def test_cfg2_true_residual_on_host(cfg2, form):
    """192x96x96 (5.4M DOF), the bench's input: both solver forms reach true
    relative residual 1e-8 as recomputed on the host by the oracle's operator, and
    f.u (the compliance at the solution) matches the GPU's sum_e s_e u_e^T Ke u_e."""
    import bench
    P = cfg2
    g = P["grid"]
    u, info = bench.solve_step(P, form=form)
    assert info.converged and info.true_rel_res <= 1e-8, info
    s, _ = g.simp(P["rho"], 3.0, 1e-9, want_ds=False)
    _, C = g.energy(u, s=s)
    uh, sh = u.cpu().numpy(), s.cpu().numpy()
    fixed = np.flatnonzero(np.repeat(g.mask[:g.nnodes].cpu().numpy()[:, None], 3, 1)
                           & np.array([1, 2, 4], np.uint8))
    res = _host_true_res(bench.NEL, sh, uh, P["f"], fixed)
    Cf = float(P["f"] @ uh)
    print(form, dict(host_true_rel_res=res, gpu_true_rel_res=info.true_rel_res, iters=info.iters,
                     compliance=C.item(), f_dot_u=Cf))
    assert res <= 1.0001e-8
    assert abs(C.item() - Cf) <= 1e-8 * abs(Cf)


def test_cfg5_batch_full_size_residuals():
    """The batched workload at its full sizes (64 designs 32x16x16 ... 96x48x48 plus
    a 128x64x64 design with 8 load cases) in one graph launch: every solve
    converged, and the host-recomputed true residual of 8 seeded designs and of all
    8 load cases is <= 1e-8."""
    from pyto_b200.batch import batch_problems
    from pyto_b200.engine import BatchSolver
    probs = batch_problems(n_designs=64)
    bs = BatchSolver(probs, rtol=1e-8, max_iters=5000)
    bs.launch()
    infos = bs.status()
    assert len(infos) == 72 and all(i.converged and i.true_rel_res <= 1e-8 for i in infos)
    pick = sorted(np.random.default_rng(1).choice(64, 8, replace=False).tolist()) + list(range(64, 72))
    for k in pick:
        g, defl, s, b = probs[k]
        fixed = np.flatnonzero(np.repeat(g.mask[:g.nnodes].cpu().numpy()[:, None], 3, 1)
                               & np.array([1, 2, 4], np.uint8))
        res = _host_true_res(g.nel, s.cpu().numpy(), bs.u[k].cpu().numpy(), b.cpu().numpy(), fixed)
        assert res <= 1.0001e-8, (k, g.nel, res, infos[k])
    bs.close()
