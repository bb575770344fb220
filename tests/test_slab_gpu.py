"""The slab-decomposed deflated PCG (pyto_b200.slab) through the C ABI on one GPU:
1 to 3 ranks run as threads of one process (ThreadComm: halo planes and sums are
exchanged by copies between the ranks' buffers, each rank on its own stream), and
the assembled solution must equal the single-domain solve of the same grid."""
import threading

import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [1, 2, 3])
def test_slab_dpcg_on_virtual_ranks(world):
    from pyto_b200.engine import DeviceDeflation, HexGrid
    from pyto_b200.slab import DeviceSlab, ThreadComm, partition, slab_dpcg, slab_range
    nel = (24, 12, 20)
    m = O.grid_mesh(*nel)
    f, fixed = O.cantilever_bc(m)
    rho = np.random.default_rng(2).uniform(0.01, 1.0, m["num_elems"])
    s = O.simp_scaling(rho, 3.0, 1e-9)
    grp, cnt, cen = O.deflation_groups(m["node_xyz"], 40)
    # single domain: the library's deflated PCG with the same recurrence and stop rule
    g = HexGrid(nel).set_fixed_dofs(fixed)
    defl = DeviceDeflation(g, grp, cen, modes=6, shift=1e-14, shift_relative=True)
    uref, iref = g.dpcg(g.tensor(s), g.tensor(f), defl, rtol=1e-10, stop_rule=0, max_iters=2000)
    assert iref.converged
    uref = uref.cpu().numpy()
    comm = ThreadComm(world)
    views = comm.views()
    out, errs = [None] * world, []

    def rank_main(r):
        try:
            st = torch.cuda.Stream()
            with torch.cuda.stream(st):
                sl = partition(nel, world)[r]
                be = DeviceSlab(sl, nel, fixed, grp, cen)
                nx, ny, _ = nel
                be.set_scaling(s[nx * ny * sl.n0:nx * ny * (sl.n0 + sl.nel[2])])
                a, b = slab_range(sl)
                x, info = slab_dpcg(be, views[r], be.grid.tensor(f[a:b]), rtol=1e-10, max_iters=2000)
                P3 = 3 * sl.plane_nodes
                lo, hi = sl.own_planes
                out[r] = (x[P3 * lo:P3 * hi].cpu().numpy(), info)
        except Exception as ex:  # pragma: no cover
            errs.append(ex)
            comm.barrier.abort()

    th = [threading.Thread(target=rank_main, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=300)
    assert not errs, errs
    u = np.concatenate([o[0] for o in out])
    infos = [o[1] for o in out]
    assert all(i.converged for i in infos) and len({i.iters for i in infos}) == 1
    assert abs(infos[0].iters - iref.iters) <= 2, (infos[0].iters, iref.iters)
    assert np.abs(u - uref).max() <= 1e-8 * np.abs(uref).max()
    assert abs(f @ u - f @ uref) <= 1e-11 * abs(f @ uref)
