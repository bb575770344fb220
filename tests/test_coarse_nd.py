"""Nested-dissection coarse solver (pyto_coarse_nd_*): the planner on the host, and on
the GPU the factorisation against the dense coarse inverse and the deflated solves with
either coarse solver.

The coarse matrix is W_f^T K_ff W_f + shift I of element-box aggregates (the 4x4x4
aggregation with 3 translations that the 192x96x96 benchmark configuration names), as
the reference forms and solves it directly (src/deflation.py:517-521, 577)."""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle as O


def _nbr_lists(gx, gy, gz):
    nptr, nl = [0], []
    for G in range(gx * gy * gz):
        i, j, k = G % gx, (G // gx) % gy, G // (gx * gy)
        for kk in range(max(0, k - 1), min(gz, k + 2)):
            for jj in range(max(0, j - 1), min(gy, j + 2)):
                for ii in range(max(0, i - 1), min(gx, i + 2)):
                    nl.append(ii + gx * (jj + gy * kk))
        nptr.append(len(nl))
    return np.array(nptr, np.int32), np.array(nl, np.int32)


def _plan(gx, gy, gz, modes, leaf, nptr=None, nl=None):
    from pyto_b200 import _capi as A
    if nptr is None:
        nptr, nl = _nbr_lists(gx, gy, gz)
    p = A.lib().pyto_coarse_nd_plan(gx, gy, gz, modes, leaf, nptr.ctypes.data, nl.ctypes.data)
    if not p:
        return None, None
    info = (C.c_double * 5)()
    nbytes = A.lib().pyto_coarse_nd_bytes(p, info)
    A.lib().pyto_coarse_nd_free(p)
    return nbytes, list(info)


def test_plan_sizes_of_the_benchmark_coarse_space():
    """48x24x24 groups (192x96x96 elements in 4x4x4 aggregates), 3 translations: the tree
    covers all 82,944 unknowns with fronts of at most 4,248."""
    nbytes, info = _plan(48, 24, 24, 3, 8)
    assert nbytes is not None and nbytes > 0
    nodes, depth, max_front = info[0], info[1], info[2]
    assert depth == 12 and max_front == 4248 and nodes > 1000
    # one group, no separator: a single dense front of the whole system
    nbytes1, info1 = _plan(1, 1, 1, 6, 8)
    assert info1[0] == 1 and info1[2] == 6


def test_plan_rejects_lists_off_the_box_grid():
    from pyto_b200 import _capi as A
    nptr, nl = _nbr_lists(4, 3, 2)
    bad = nl.copy()
    bad[5] = 4 * 3 * 2 - 1  # group 0 "touches" the far corner group
    assert _plan(4, 3, 2, 3, 8, nptr, bad) == (None, None)
    assert "adjacent" in A.last_error()
    assert _plan(0, 3, 2, 3, 8, nptr, nl) == (None, None)


def _space(nel, agg, modes, coarse):
    from pyto_b200.deflation import DeflationSolver
    from pyto_b200.engine import HexGrid
    from pyto_b200.hex_mesher import HexMesher
    mesh = HexMesher()
    mesh.grid_mesh(nel, (1.0, 1.0, 1.0))
    m = O.grid_mesh(*nel)
    f, fixed = O.cantilever_bc(m)
    g = HexGrid(nel).set_fixed_dofs(fixed)
    ds = DeflationSolver(modes=modes, shift=1e-14, shift_relative=True, coarse=coarse, nd_leaf=2)
    ds.create_deflation_groups_box(mesh, agg, modes=modes)
    return g, ds.device_deflation(g), f


@pytest.mark.gpu
@pytest.mark.parametrize("nel,modes", [((16, 8, 8), 3), ((24, 16, 12), 3), ((24, 16, 12), 6), ((32, 8, 12), 6)])
def test_nd_factor_matches_dense_inverse(nel, modes):
    """The nested-dissection solve equals the dense coarse inverse of the same assembled
    matrix (both with the relative 1e-14 shift) to 1e-10, and two set-ups give bitwise
    equal solves."""
    rng = np.random.default_rng(5)
    gd, dd, _ = _space(nel, (4, 4, 4), modes, "dense")
    gn, dn, _ = _space(nel, (4, 4, 4), modes, "nd")
    x = rng.uniform(0.01, 1.0, gd.nelem)
    sd, _ = gd.simp(gd.tensor(x), 3.0, 1e-9)
    sn, _ = gn.simp(gn.tensor(x), 3.0, 1e-9)
    gd.dpcg_setup(sd, dd)
    gn.dpcg_setup(sn, dn)
    v = gn.tensor(rng.normal(size=dn.nc))
    mu = dn.nd_solve(v).clone()
    Einv = dd.coarse_inv.view(dd.nc, dd.nc)
    ref = Einv @ v.to(Einv.device)
    err = (mu - ref).abs().max().item()
    assert err <= 1e-10 * ref.abs().max().item(), err
    gn.dpcg_setup(sn, dn)
    assert torch.equal(dn.nd_solve(v), mu)


@pytest.mark.gpu
@pytest.mark.parametrize("modes", [3, 6])
def test_dpcg_with_nd_coarse_solver(modes):
    """Deflated PCG (FP64 residual replacement and the mixed-precision form) with the
    nested-dissection coarse solver: the same iteration counts as with the dense inverse
    and the same solution to the solve tolerance."""
    nel = (32, 16, 12)
    rng = np.random.default_rng(6)
    gd, dd, f = _space(nel, (4, 4, 4), modes, "dense")
    gn, dn, _ = _space(nel, (4, 4, 4), modes, "nd")
    x = rng.uniform(0.01, 1.0, gd.nelem)
    sd, _ = gd.simp(gd.tensor(x), 3.0, 1e-9)
    sn, _ = gn.simp(gn.tensor(x), 3.0, 1e-9)
    ud, idn = gd.dpcg(sd, gd.tensor(f), dd, rtol=1e-10, stop_rule=2, max_iters=3000)
    un, inn = gn.dpcg(sn, gn.tensor(f), dn, rtol=1e-10, stop_rule=2, max_iters=3000)
    assert idn.converged and inn.converged
    assert abs(idn.iters - inn.iters) <= 1, (idn.iters, inn.iters)
    assert (un - ud).abs().max().item() <= 1e-8 * ud.abs().max().item()
    um, im = gn.dpcg_mixed(sn, gn.tensor(f), dn, rtol=1e-8)
    assert im.converged and im.true_rel_res <= 1e-8
    assert (um - ud).abs().max().item() <= 1e-6 * ud.abs().max().item()
