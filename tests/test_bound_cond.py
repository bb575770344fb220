"""bound_cond.impose_dirichlet_bc (src/bound_cond.py:40-70): on PyTO's assembled matrix
(the reference's elimination) and on the library's matrix-free operator (the lift on the
GPU), both against the oracle's elimination with non-zero prescribed values."""
import numpy as np
import pytest

import oracle as O


def _case():
    nel = (6, 3, 4)
    m = O.grid_mesh(*nel)
    f, fixed = O.cantilever_bc(m)
    rng = np.random.default_rng(3)
    x = rng.uniform(0.01, 1.0, m["num_elems"])
    s = O.simp_scaling(x, 3.0, 1e-9)
    g = rng.normal(size=len(fixed))
    return nel, m, f, fixed, s, g


def test_elimination_of_an_assembled_matrix():
    from pyto_b200.bound_cond import BC, impose_dirichlet_bc
    nel, m, f, fixed, s, g = _case()
    K = O.assemble_K(m, s, O.ke_hex8(1.0, 0.3))
    A_, b_ = impose_dirichlet_bc(K, f, BC(f, fixed, g))
    Ar, br, free = O.impose_dirichlet_bc(K, f, fixed, g)
    assert abs(A_ - Ar).max() == 0.0
    np.testing.assert_allclose(b_, br, rtol=0, atol=1e-14 * np.abs(br).max())
    with pytest.raises(NotImplementedError):
        impose_dirichlet_bc(K, f, BC(f, fixed, g, constraint_matrix=np.eye(2)))


@pytest.mark.gpu
def test_elimination_on_the_gpu_operator():
    from pyto_b200.bound_cond import BC, impose_dirichlet_bc
    from pyto_b200.engine import HexGrid
    from pyto_b200.linear_solvers import StiffnessOperator
    nel, m, f, fixed, s, g = _case()
    grid = HexGrid(nel).set_fixed_dofs(fixed)
    op = StiffnessOperator(grid, grid.tensor(s))
    A_, b_ = impose_dirichlet_bc(op, f, BC(f, fixed, g))
    assert A_ is op
    _, br, _ = O.impose_dirichlet_bc(O.assemble_K(m, s, O.ke_hex8(1.0, 0.3)), f, fixed, g)
    np.testing.assert_allclose(b_.cpu().numpy(), br, rtol=0, atol=1e-13 * np.abs(br).max())
