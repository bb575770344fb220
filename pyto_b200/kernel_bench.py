"""Micro-benchmark of single library kernels (also the command profiled with ncu).

    python -m pyto_b200.kernel_bench --kernel matvec --nel 192,96,96 --reps 20

Prints one JSON line per kernel: average launch time (CUDA events on the
launching stream, after warm-up) and the achieved algorithmic bandwidth.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import _capi as A
from .engine import HexGrid
from .hex_mesher import HexMesher
from .problems import cantilever


def _timeit(fn, reps, warm=3):
    for _ in range(warm):
        fn()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(reps):
        fn()
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps / 1e3


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel", default="matvec", choices=["matvec", "matvec32", "energy", "filter", "jacobi", "stress", "dpcg",
                                                          "mixed", "pcg", "batch", "oc", "adjoint", "ocupdate",
                                                          "thermal", "mma"])
    ap.add_argument("--iters", type=int, default=20, help="--kernel oc: OC iterations")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"], help="--kernel oc: DPCG form")
    ap.add_argument("--warm-start", action="store_true", help="--kernel oc: start each solve from the previous one")
    ap.add_argument("--designs", type=int, default=64, help="--kernel batch: number of designs")
    ap.add_argument("--no-tune", action="store_true", help="--kernel batch: skip the autotuner")
    ap.add_argument("--groups", type=int, default=432, help="deflation groups for --kernel dpcg")
    ap.add_argument("--nel", default="192,96,96")
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--warm", type=int, default=3)
    ap.add_argument("--variant", type=int, default=2, help="matvec tile variant (pyto_tune)")
    ap.add_argument("--variant32", type=int, default=None, help="FP32 matvec tile variant (pyto_tune)")
    ap.add_argument("--delta", type=float, default=1e-1, help="reliable-update threshold for --kernel mixed")
    ap.add_argument("--mode", type=int, default=3, help="--kernel matvec/matvec32: BC mask mode (1 in, 2 out)")
    ap.add_argument("--dot", action="store_true", help="--kernel matvec/matvec32: with the fused u.y (solver form)")
    ap.add_argument("--stop-rule", type=int, default=0, choices=[0, 1, 2], help="--kernel dpcg: stopping rule")
    ap.add_argument("--check-every", type=int, default=20, help="--kernel dpcg/mixed/pcg: iterations between host polls")
    a = ap.parse_args(argv)
    if a.kernel == "batch":
        return batch_bench(a)
    if a.kernel == "oc":
        return oc_bench(a)
    nel = tuple(int(v) for v in a.nel.split(","))
    if a.kernel == "thermal":
        return thermal_bench(a, nel)
    if a.kernel == "mma":
        return mma_bench(a, nel)
    A.call("pyto_tune", 0, a.variant)
    if a.variant32 is not None:
        A.call("pyto_tune", 1, a.variant32)
    mesh = HexMesher()
    mesh.grid_mesh(nel, (1.0, 1.0, 1.0))
    f, fixed = cantilever(mesh)
    g = HexGrid(nel).set_fixed_dofs(fixed)
    rng = np.random.default_rng(0)
    s = g.tensor(rng.uniform(0.01, 1.0, g.nelem))
    u = g.tensor(rng.normal(size=g.ndof))
    y = torch.empty_like(u)
    if a.kernel == "matvec":
        fn, nbytes = (lambda: g.matvec(s, u, mode=a.mode, out=y, dot=a.dot)), 48 * g.nnodes + 8 * g.nelem + g.nnodes
    elif a.kernel == "matvec32":
        s32, u32 = s.float(), u.float()
        y32 = torch.empty_like(u32)
        fn, nbytes = (lambda: g.matvec_f32(s32, u32, mode=a.mode, out=y32, dot=a.dot)), 24 * g.nnodes + 4 * g.nelem + g.nnodes
    elif a.kernel == "energy":
        fn, nbytes = (lambda: g.energy(u, s=s)), 24 * g.nnodes + 16 * g.nelem
    elif a.kernel == "filter":
        out = torch.empty_like(s)
        fn, nbytes = (lambda: g.filter(2.0, A.FILTER_DENSITY, s, out=out)), 16 * g.nelem
    elif a.kernel == "jacobi":
        fn, nbytes = (lambda: g.jacobi(s)), 8 * g.nelem + 33 * g.nnodes
    elif a.kernel in ("dpcg", "mixed", "pcg"):
        from .deflation import DeflationSolver
        F = g.tensor(f)
        if a.kernel in ("dpcg", "mixed"):
            ds = DeflationSolver(shift=1e-14, shift_relative=True)
            ds.create_deflation_groups(mesh, a.groups)
            defl = ds.device_deflation(g)
            if a.kernel == "dpcg":
                fn = lambda: g.dpcg(s, F, defl, rtol=1e-8, max_iters=5000, stop_rule=a.stop_rule,
                                    check_every=a.check_every)
            else:
                fn = lambda: g.dpcg_mixed(s, F, defl, rtol=1e-8, delta=a.delta, max_iters=8000,
                                          check_every=a.check_every)
        else:
            fn = lambda: g.pcg(s, F, rtol=1e-8, check_every=a.check_every)
        nbytes = 0
    elif a.kernel == "adjoint":  # p-norm adjoint: explicit term T1 and the adjoint load g = dPN/du
        x = s  # densities in (0.01, 1]
        dpn = g.tensor(np.array([1.0]))
        # k_pnorm_elem: u, x in; T1 and the 6-vector t per element out; k_pnorm_gather: t in, g out
        fn, nbytes = (lambda: g.pnorm_adjoint(u, x, 0.5, 8.0, dpn)), 48 * g.nnodes + 112 * g.nelem
    elif a.kernel == "ocupdate":  # OC bisection update (reference sequence), x restored each call
        x0 = s.clone()
        xw = torch.empty_like(x0)
        dc = -g.tensor(rng.uniform(0.1, 1.0, g.nelem))

        def fn():
            xw.copy_(x0)
            return g.oc_update(xw, dc, 0.3)
        nbytes = 24 * g.nelem  # per bisection pass
    else:
        fn, nbytes = (lambda: g.stress(u, s, 0.5, want=("vm",))), 24 * g.nnodes + 16 * g.nelem
    t = _timeit(fn, a.reps, a.warm)
    if a.kernel in ("dpcg", "mixed", "pcg"):
        _, info = fn()
        print(json.dumps({"kernel": a.kernel, "nel": nel, "ms": t * 1e3, "iters": info.iters,
                          "true_rel_res": info.true_rel_res}))
        return
    print(json.dumps({"kernel": a.kernel, "variant": a.variant if a.kernel != "matvec32" else a.variant32,
                      "mode": a.mode, "dot": a.dot, "nel": nel, "ms": t * 1e3, "algorithmic_bytes": int(nbytes),
                      "GB_s": nbytes / t / 1e9}))


def oc_bench(a):
    print(json.dumps(run_oc(tuple(int(v) for v in a.nel.split(",")), a.iters, a.precision, a.groups,
                            a.warm_start)))


def run_oc(nel, n_iters=20, precision="mixed", groups=432, warm_start=False):
    """OC topology optimisation through the reference-named driver (topopt_ocm) on the
    cantilever: rho0 = volfrac, sensitivity filter r = 1.5, volfrac 0.3, move 0.2, each
    FEA solve by the deflated PCG (node-box groups x 6 modes, rtol 1e-8).  Returns the
    wall time of n_iters design iterations after a one-iteration warm-up."""
    from . import bound_cond, hex_structural_fea, linear_solvers, mat_lib, topopt_common as tc, topopt_ocm
    from . import topopt_material_model as tmm
    from .deflation import DeflationSolver
    tmm._EVOID_RELATIVE = 1e-9
    mesh = HexMesher()
    mesh.grid_mesh(nel, (1.0, 1.0, 1.0))
    f, fixed = cantilever(mesh)
    f.flags.writeable = False  # a constant load: the FEA keeps its device copy
    bc = bound_cond.BC(force=f, fixed_dofs=fixed, dirichlet_values=np.zeros(len(fixed)))
    mat = mat_lib.create_material_with_defaults("unit", youngs_modulus=1.0, poissons_ratio=0.3)
    ds = DeflationSolver(modes=6, shift=1e-14, shift_relative=True)
    ds.create_deflation_groups(mesh, groups)
    fe = hex_structural_fea.HexStructuralFEA(mesh=mesh, mat_prop=mat, bc=bc, solver=linear_solvers.Solvers.DPCG,
                                             dsolver=ds, rtol=1e-8, precision=precision, warm_start=warm_start)
    params = tc.TOParams(Constraints=[(tc.TO_QOI.VOLUME_FRACTION, None, 0.3)], RelativeFilterRadius=1.5)
    run = lambda n: topopt_ocm.topopt_optimality_criteria(tc.FEA_MODE.STRUCTURAL, fe, params, maxIterations=n,
                                                          plot_progress=False, print_progress=False,
                                                          binarize_topology=False)
    iters = []
    solve = fe.solve

    def counted_solve(*args, **kw):  # records the Krylov iterations of every FEA solve
        out = solve(*args, **kw)
        iters.append(int(fe.last_info.iters))
        return out

    fe.solve = counted_solve
    run(1)  # warm-up: library load, workspaces
    iters.clear()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sol, hist, ok, msg, nfea = run(n_iters)
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    obj = [float(v) for v in hist["objective"]]
    return {"kernel": "oc", "precision": precision, "warm_start": warm_start, "nel": list(nel),
            "iterations": n_iters, "fea_solves": int(nfea), "krylov_iterations": sum(iters), "s": t,
            "ms_per_iteration": 1e3 * t / max(1, nfea), "objective_first": obj[0],
            "objective_last": obj[-1], "volfrac_last": float(hist["volfrac"][-1])}


def thermal_bench(a, nel):
    """Thermal operator K(s) T (8x8 conduction Ke, one DOF per node), output mask only:
    algorithmic bytes = 8 (T read) + 8 (y write) + 1 (mask) per node + 8 per element (s)."""
    from .engine import ThermalGrid
    g = ThermalGrid(nel)
    g.set_fixed_nodes(np.flatnonzero(np.arange(g.nnodes) % (nel[0] + 1) == 0))
    rng = np.random.default_rng(0)
    s = g.tensor(rng.uniform(0.01, 1.0, g.nelem))
    u = g.tensor(rng.normal(size=g.nnodes))
    y = torch.empty_like(u)
    t = _timeit(lambda: g.matvec(s, u, mode=A.MASK_OUT, out=y), a.reps, a.warm)
    nbytes = 17 * g.nnodes + 8 * g.nelem
    print(json.dumps({"kernel": "thermal", "nel": nel, "ms": t * 1e3, "algorithmic_bytes": nbytes,
                      "GB_s": nbytes / t / 1e9}))


def mma_bench(a, nel):
    """One MMA update (one constraint) over the elements of the grid."""
    from .topopt_mma import DeviceMMA
    n = int(np.prod(nel))
    rng = np.random.default_rng(0)
    dev = torch.device("cuda")
    T = lambda v: torch.as_tensor(v, dtype=torch.float64, device=dev)
    x0 = T(rng.uniform(0.1, 0.9, n))
    df0 = T(-rng.uniform(0.0, 2.0, n) / n)
    dfdx = T(np.full((1, n), 1.0 / (0.3 * n)))
    mm = DeviceMMA(n, 1, 1e-6, 1 - 1e-6, 0.2, dev)
    x = x0.clone()

    def fn():
        x.copy_(x0)
        mm.iter = 0
        mm.update(x, df0, np.array([0.05]), dfdx)
    t = _timeit(fn, a.reps, a.warm)
    print(json.dumps({"kernel": "mma", "n": n, "ms": t * 1e3, "newton_steps": float(mm.dual[-1].item())}))


def batch_bench(a):
    print(json.dumps(run_batch(a.designs, a.reps, tune=not a.no_tune)))


def run_batch(designs=64, reps=3, tune=True):
    """Batched workload: designs of uneven size plus one multi-load-case design, solved
    to rel-residual 1e-8 by one CUDA-graph launch (device time per launch, CUDA events),
    against a loop of single host-polled solves of the same problems."""
    from .autotune import autotune
    from .batch import batch_problems
    from .engine import BatchSolver
    t0 = time.perf_counter()
    probs = batch_problems(n_designs=designs)
    tuned = {}
    if tune:
        for g, _, _, _ in probs:
            if g.nel not in tuned:
                tuned[g.nel] = autotune(g, reps=5)
    t_build = time.perf_counter() - t0
    bs = BatchSolver(probs, rtol=1e-8, max_iters=5000)
    bs.launch()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        bs.launch()
    e1.record(st)
    e1.synchronize()
    t_graph = e0.elapsed_time(e1) / 1e3 / reps
    infos = bs.status()
    # the same problems one at a time through the plain (host-polled) solver
    for g, defl, s, b in probs[:2]:
        g.dpcg(s, b, defl, rtol=1e-8, max_iters=5000, stop_rule=0, check_every=20)
    torch.cuda.synchronize()
    e0.record(st)
    loop_iters = 0
    for g, defl, s, b in probs:
        _, info = g.dpcg(s, b, defl, rtol=1e-8, max_iters=5000, stop_rule=0, check_every=20)
        loop_iters += info.iters
    e1.record(st)
    e1.synchronize()
    t_loop = e0.elapsed_time(e1) / 1e3
    n = len(probs)
    bs.close()
    return {"kernel": "batch", "problems": n, "designs": designs,
            "dofs": int(sum(g.ndof for g, _, _, _ in probs)),
            "graph_s": t_graph, "graph_solves_per_s": n / t_graph,
            "loop_s": t_loop, "loop_solves_per_s": n / t_loop, "speedup": t_loop / t_graph,
            "all_converged": all(i.converged for i in infos),
            "max_true_rel_res": max(i.true_rel_res for i in infos),
            "graph_iters": int(sum(i.iters for i in infos)), "loop_iters": int(loop_iters),
            "build_s": t_build,
            "tuned": {f"{k[0]}x{k[1]}x{k[2]}": {p: v[0] for p, v in r.items()} for k, r in tuned.items()}}


if __name__ == "__main__":
    main()
