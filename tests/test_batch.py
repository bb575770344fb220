"""Batched solves in one CUDA graph against one-at-a-time solves, and the
per-grid autotuner."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _compliance(g, s, u):
    return g.energy(u, s=s)[1].item()


def test_batch_matches_individual_solves():
    from pyto_b200.batch import batch_problems
    from pyto_b200.engine import BatchSolver
    probs = batch_problems(n_designs=5, min_nx=16, max_nx=32, multi_nel=(24, 12, 12), n_loads=3, seed=3)
    bs = BatchSolver(probs, rtol=1e-10, max_iters=4000)
    bs.launch()
    infos = bs.status()
    for (g, defl, s, b), u, info in zip(probs, bs.u, infos):
        assert info.converged and info.true_rel_res <= 1e-9, info
        u1, i1 = g.dpcg(s, b, defl, rtol=1e-10, max_iters=4000, stop_rule=0)
        assert i1.converged
        assert abs(info.iters - i1.iters) <= 2, (info.iters, i1.iters)
        c0, c1 = _compliance(g, s, u), _compliance(g, s, u1)
        assert abs(c0 - c1) <= 1e-9 * abs(c1)
        assert (u - u1).abs().max().item() <= 1e-7 * u1.abs().max().item()
    bs.close()


def test_batch_relaunch_with_new_data():
    from pyto_b200.batch import batch_problems
    from pyto_b200.engine import BatchSolver
    probs = batch_problems(n_designs=3, min_nx=16, max_nx=24, multi_nel=None, n_loads=0, seed=5)
    bs = BatchSolver(probs, rtol=1e-10)
    bs.launch()
    first = [u.clone() for u in bs.u]
    rng = np.random.default_rng(9)
    for g, defl, s, b in probs:  # new densities and loads, same buffers
        x = torch.as_tensor(rng.uniform(0.05, 1.0, g.nelem), device="cuda")
        s.copy_(g.simp(x, 3.0, 1e-9, want_ds=False)[0])
        b.mul_(-2.0)
    bs.launch()
    for (g, defl, s, b), u, u0, info in zip(probs, bs.u, first, bs.status()):
        assert info.converged
        u1, _ = g.dpcg(s, b, defl, rtol=1e-10, stop_rule=0)
        assert (u - u1).abs().max().item() <= 1e-7 * u1.abs().max().item()
        assert (u - u0).abs().max().item() > 1e-3 * u0.abs().max().item()
    bs.close()


def test_autotune_picks_a_variant_and_keeps_results():
    from pyto_b200.autotune import autotune
    from pyto_b200.engine import HexGrid
    g = HexGrid((40, 20, 24))
    rng = np.random.default_rng(0)
    s = g.tensor(rng.uniform(0.01, 1.0, g.nelem))
    u = g.tensor(rng.normal(size=g.ndof))
    y0 = g.matvec(s, u).clone()
    res = autotune(g, reps=3, use_cache=False)
    assert set(res) == {"f64", "f32"}
    assert (g.op.tune & 0xFF) - 1 == res["f64"][0] and ((g.op.tune >> 8) & 0xFF) - 1 == res["f32"][0]
    y1 = g.matvec(s, u)
    assert (y1 - y0).abs().max().item() <= 1e-13 * y0.abs().max().item()


def test_batch_refuses_launch_after_fixed_dofs_change():
    """The graph holds the addresses of the deflation boundary lists: resetting a
    grid's fixed DOFs (which rebuilds them at the next sync) must stop the launch."""
    from pyto_b200.batch import batch_problems
    from pyto_b200.engine import BatchSolver
    probs = batch_problems(n_designs=2, min_nx=16, max_nx=16, multi_nel=None, n_loads=0, seed=5)
    bs = BatchSolver(probs, rtol=1e-8)
    bs.launch()
    assert all(i.converged for i in bs.status())
    g, defl, s, b = probs[0]
    nx, ny, nz = g.nel
    n = np.arange(g.nnodes)
    fixed = np.concatenate([3 * n[n % (nx + 1) == 0] + c for c in range(3)])
    g.set_fixed_dofs(np.sort(fixed))  # same set, new mask version
    with pytest.raises(RuntimeError, match="create a new BatchSolver"):
        bs.launch()
    bs.close()
