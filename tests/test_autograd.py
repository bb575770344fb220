"""Differentiable objectives: the hand-written backward against the reference's
sensitivities (goldens) and against central finite differences.

The finite differences are exact differences of the discrete objectives,
C(x + h e_i) - C(x - h e_i) and PN(x + h e_i) - PN(x - h e_i), formed without
cancellation: u(x +- h e_i) - u(x) is solved for directly (its right-hand side
(K(x) - K(x +- h e_i)) u(x) lives on the 24 DOFs of element i), and the stress
and p-norm changes are accumulated from it (the stress is linear in u, x^q and
the powers are differenced through expm1/log1p).  A plain difference of two
objective values would lose all digits at h = 1e-6 on a 1.6M-DOF grid.
"""
import math

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def _vm2(a, b):
    """von Mises bilinear form B(a, b) of stress rows [.., 6] (normals first)."""
    n = (a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1] + a[:, 2] * b[:, 2]
         - 0.5 * (a[:, 0] * b[:, 1] + a[:, 1] * b[:, 0] + a[:, 1] * b[:, 2] + a[:, 2] * b[:, 1]
                  + a[:, 2] * b[:, 0] + a[:, 0] * b[:, 2]))
    return n + 3.0 * (a[:, 3] * b[:, 3] + a[:, 4] * b[:, 4] + a[:, 5] * b[:, 5])


def _problem(nel, lshape, solver, seed=0, groups=None, lo=0.2, rtol=1e-11, recompute=False):
    from pyto_b200.autograd import HexProblem
    from pyto_b200.deflation import DeflationSolver
    from pyto_b200.engine import HexGrid
    from pyto_b200.hex_mesher import HexMesher
    from pyto_b200.problems import cantilever, lshape_active, uniform_density
    mesh = HexMesher()
    mesh.grid_mesh(nel, (1.0, 1.0, 1.0))
    active = lshape_active(nel) if lshape else None
    f, fixed = cantilever(mesh, active)
    g = HexGrid(nel).set_fixed_dofs(fixed)
    if active is not None:
        g.set_active(active)
    x = g.tensor(uniform_density(nel, lo, 1.0, seed=seed, active=active))
    defl = None
    if solver != "pcg":
        ds = DeflationSolver(modes=6, shift=1e-14, shift_relative=True)
        ds.create_deflation_groups(mesh, groups)
        defl = ds.device_deflation(g)
    prob = HexProblem(g, f, penal=3.0, emin=1e-9, q=0.5, P=8.0, solver=solver, defl=defl, rtol=rtol,
                      recompute=recompute)
    return prob, x


def _exact_differences(prob, x, i, h):
    """(C(x+h e_i) - C(x-h e_i), PN(x+h e_i) - PN(x-h e_i)) without cancellation."""
    g, q, P = prob.grid, prob.q, prob.P
    s0, _ = prob.scale(x)
    u0 = prob.solve(s0)
    sig0 = g.stress(u0, x, q, want=("stress",))["stress"]
    vm2_0 = _vm2(sig0, sig0)
    S0 = (vm2_0 ** (P / 2)).sum()
    xi = float(x[i])
    out = []
    for sgn in (1.0, -1.0):
        xp = x.clone()
        xp[i] = xi + sgn * h
        sp, _ = prob.scale(xp)
        dse = (1.0 - prob.emin) * sgn * h * (3 * xi * xi + 3 * xi * sgn * h + h * h)  # s(x_i +- h) - s(x_i), p = 3
        sd = torch.zeros_like(s0)
        sd[i] = -dse
        du = prob.solve(sp, g.matvec(sd, u0))  # K(x+-) du = (K(x) - K(x+-)) u(x)
        dC = torch.dot(prob.f, du)
        dsig = g.stress(du, x, q, want=("stress",))["stress"].clone()
        em1 = math.expm1(q * math.log1p(sgn * h / xi))  # (x_i +- h)^q / x_i^q - 1
        dsig[i] = em1 * sig0[i] + (1.0 + em1) * dsig[i]
        dvm2 = _vm2(dsig, 2.0 * sig0 + dsig)
        pos = vm2_0 > 0
        dvmP = torch.zeros_like(vm2_0)
        dvmP[pos] = vm2_0[pos] ** (P / 2) * torch.expm1((P / 2) * torch.log1p(dvm2[pos] / vm2_0[pos]))
        dS = dvmP.sum()
        dPN = S0 ** (1.0 / P) * torch.expm1(torch.log1p(dS / S0) / P)
        out.append((dC.item(), dPN.item()))
    return out[0][0] - out[1][0], out[0][1] - out[1][1]


def test_autograd_matches_reference_sensitivities():
    """12x6x6 cantilever: values and gradients against vectors produced by PyTO."""
    from pyto_b200.autograd import HexProblem, structural_objectives
    from pyto_b200.engine import HexGrid
    d = golden("cantilever_12x6x6_direct.npz")
    g = HexGrid((12, 6, 6)).set_fixed_dofs(d["fixed"])
    prob = HexProblem(g, d["f"], penal=3.0, emin=1e-9, q=0.5, P=8.0, solver="pcg", rtol=1e-13)
    x = torch.tensor(d["rho"], dtype=torch.float64, device="cuda", requires_grad=True)
    C, pn = structural_objectives(x, prob)
    assert abs(C.item() - float(d["C"])) <= 1e-10 * float(d["C"])
    assert abs(pn.item() - float(d["pn_val"])) <= 1e-9 * float(d["pn_val"])
    gC, = torch.autograd.grad(C, x, retain_graph=True)
    gP, = torch.autograd.grad(pn, x)
    np.testing.assert_allclose(gC.cpu().numpy(), d["dC"], rtol=1e-8, atol=1e-11 * np.abs(d["dC"]).max())
    np.testing.assert_allclose(gP.cpu().numpy(), d["pn_grad"], rtol=1e-6,
                               atol=1e-9 * np.abs(d["pn_grad"]).max())


def test_recompute_matches_stored_state():
    from pyto_b200.autograd import structural_objectives
    prob, x = _problem((16, 8, 8), True, "pcg", rtol=1e-12)
    x1 = x.clone().requires_grad_(True)
    (C1, P1) = structural_objectives(x1, prob)
    (C1 + 0.5 * P1).backward()
    prob.recompute = True
    x2 = x.clone().requires_grad_(True)
    (C2, P2) = structural_objectives(x2, prob)
    (C2 + 0.5 * P2).backward()
    assert C1.item() == C2.item() and P1.item() == P2.item()
    torch.testing.assert_close(x1.grad, x2.grad, rtol=1e-9, atol=1e-14)


@pytest.mark.parametrize("nel,groups,nsample,solver,rtol", [((32, 16, 16), 16, 12, "pcg", 1e-12),
                                                            ((32, 16, 16), 16, 12, "dpcg", 1e-10),
                                                            ((128, 64, 64), 128, 64, "mixed", 1e-11)])
def test_gradients_match_central_differences(nel, groups, nsample, solver, rtol):
    """L-shaped domain, p = 8, q = 0.5: adjoint gradients of compliance and of the
    p-norm von Mises stress against central differences (h = 1e-6, FP64) on seeded
    random active elements, to 1e-5 relative."""
    from pyto_b200.autograd import structural_objectives
    prob, x = _problem(nel, True, solver, groups=groups, rtol=rtol)
    xg = x.clone().requires_grad_(True)
    C, pn = structural_objectives(xg, prob)
    gC, = torch.autograd.grad(C, xg, retain_graph=True)
    gP, = torch.autograd.grad(pn, xg)
    act = np.flatnonzero(prob.grid.active.cpu().numpy())
    idx = np.random.default_rng(1).choice(act, nsample, replace=False)  # the FD sample: seed 1
    h = 1e-6
    for i in idx:
        dC, dP = _exact_differences(prob, x, int(i), h)
        fdC, fdP = dC / (2 * h), dP / (2 * h)
        assert abs(fdC - gC[i].item()) <= 1e-5 * abs(fdC), (i, fdC, gC[i].item())
        assert abs(fdP - gP[i].item()) <= 1e-5 * abs(fdP) + 1e-12 * gP.abs().max().item(), (i, fdP, gP[i].item())


def test_stress_components_give_von_mises():
    prob, x = _problem((16, 8, 8), True, "pcg", rtol=1e-12)
    s, _ = prob.scale(x)
    u = prob.solve(s)
    out = prob.grid.stress(u, x, prob.q, want=("stress", "vm"))
    vm2 = _vm2(out["stress"], out["stress"])
    torch.testing.assert_close(vm2, out["vm"] ** 2, rtol=1e-12, atol=1e-30)
