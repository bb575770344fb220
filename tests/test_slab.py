"""The slab decomposition of one deflated PCG solve (pyto_b200.slab) on CPU: the
partition and halo maps, and the sharded solve on 2 and 3 gloo ranks (arithmetic
by the host backend tests/slab_host.py) against the single-domain solve of the
oracle's compiled restatement.  No GPU is involved."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("nz,world", [(1, 1), (1, 2), (7, 3), (10, 4), (96, 8), (5, 6)])
def test_partition_covers_planes_and_elements_once(nz, world):
    from pyto_b200.slab import halo_maps, partition
    nel = (6, 3, nz)
    sl = partition(nel, world)
    assert [s.z0 for s in sl][0] == 0 and sl[-1].z1 == nz + 1
    assert all(a.z1 == b.z0 for a, b in zip(sl, sl[1:])) and all(s.z1 > s.z0 for s in sl)
    layers = [e for s in sl for e in range(s.e0, s.e1)]
    assert layers == list(range(nz))  # every element layer owned exactly once
    for s in sl:
        # the slab grid holds every element layer touching an owned node
        assert s.n0 == max(s.z0 - 1, 0) and s.n1 == min(s.z1 + 1, nz + 1) and s.nel[2] == s.n1 - s.n0 - 1
        assert s.e0 >= s.n0 and s.e1 <= s.n1 - 1
        send, recv = halo_maps(s)
        for peer, k in send:  # what rank s sends is what the peer receives, plane for plane
            t = sl[peer]
            _, rk = [m for m in halo_maps(t)[1] if m[0] == s.rank][0]
            assert s.n0 + k == t.n0 + rk
        for peer, k in recv:  # a halo plane is owned by the rank it comes from
            assert sl[peer].z0 <= s.n0 + k < sl[peer].z1


def test_partition_refuses_more_ranks_than_planes():
    from pyto_b200.slab import partition
    with pytest.raises(ValueError):
        partition((4, 4, 2), 4)


def _problem(nel):
    import oracle as O
    m = O.grid_mesh(*nel)
    f, fixed = O.cantilever_bc(m)
    rho = np.random.default_rng(5).uniform(0.05, 1.0, m["num_elems"])
    s = O.simp_scaling(rho, 3.0, 1e-9)
    grp, cnt, cen = O.deflation_groups(m["node_xyz"], 12)
    return m, f, fixed, s, grp, cen


def _worker(rank, world, port, nel, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import sys
        sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
        from slab_host import HostSlab
        from pyto_b200.slab import DistComm, partition, slab_dpcg, slab_range
        m, f, fixed, s, grp, cen = _problem(nel)
        sl = partition(nel, world)[rank]
        be = HostSlab(sl, nel, fixed, grp, cen)
        nx, ny, _ = nel
        be.set_scaling(s[nx * ny * sl.n0:nx * ny * (sl.n0 + sl.nel[2])])
        a, b = slab_range(sl)
        x, info = slab_dpcg(be, DistComm(), torch.as_tensor(f[a:b]), rtol=1e-10, max_iters=500)
        P3 = 3 * sl.plane_nodes
        lo, hi = sl.own_planes
        q.put((rank, sl.z0, x[P3 * lo:P3 * hi].numpy().copy(), info.iters, info.converged))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
@pytest.mark.parametrize("world", [2, 3])
def test_sharded_dpcg_equals_single_domain(world):
    from oracle import cpu
    import oracle as O
    nel = (8, 4, 10)
    m, f, fixed, s, grp, cen = _problem(nel)
    fea = cpu.CpuFEA(nel, O.ke_hex8(1.0, 0.3), fixed)
    fea.assemble(s)
    uref, iref = fea.dpcg(f, grp, cen, modes=6, shift=1e-14, shift_relative=True, rtol=1e-10, stop_rule=0)
    assert iref["rc"] == 0
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, nel, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=240) for _ in range(world)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    u = np.concatenate([r[2] for r in res])
    assert all(r[4] for r in res) and len({r[3] for r in res}) == 1  # every rank took the same steps
    assert abs(res[0][3] - iref["iters"]) <= 2, (res[0][3], iref["iters"])
    assert np.abs(u - uref).max() <= 1e-8 * np.abs(uref).max()
    assert abs(f @ u - f @ uref) <= 1e-12 * abs(f @ uref)
