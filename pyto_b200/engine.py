"""Device-side engine of one voxel grid: every call goes through the C ABI.

``HexGrid`` holds the operator struct (grid + Ke), the per-node Dirichlet mask
and the optional active-element mask on the device, and exposes the library's
entry points on torch CUDA float64 tensors.  Torch provides device memory and
the current stream only; all arithmetic runs in libpyto_b200.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _capi as A

F64 = torch.float64


def _round4(n: int) -> int:
    return (n + 3) // 4 * 4


@dataclass
class SolveInfo:
    """Outcome of one Krylov solve (mirrors pyto_solve_status_t)."""
    converged: bool
    iters: int
    breakdown: bool
    rel_res: float
    true_rel_res: float
    code: int


class HexGrid:
    """A box grid of nelx*nely*nelz hex8 elements on one CUDA device."""

    def __init__(self, nel, elem_size=(1.0, 1.0, 1.0), E=1.0, nu=0.3, ke=None, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("pyto_b200 needs a CUDA device (sm_100a); no CPU path exists")
        self.device = torch.device(device if device is not None else "cuda")
        self.nel = tuple(int(n) for n in nel)
        self.h = tuple(float(v) for v in elem_size)
        self.op = A.make_operator(*self.nel, self.h, E, nu, ke)
        nx, ny, nz = self.nel
        self.nnodes = (nx + 1) * (ny + 1) * (nz + 1)
        self.nelem = nx * ny * nz
        self.ndof = 3 * self.nnodes
        self.mask = torch.zeros(_round4(self.nnodes), dtype=torch.uint8, device=self.device)
        self.active = None
        self.n_active = self.nelem
        self.mask_version = 0

    # ---- helpers -------------------------------------------------------------
    @property
    def opp(self):
        return C.byref(self.op)

    def _st(self):
        return A.stream_ptr(self.device)

    def _ws(self, kind: int, tag: str):
        n = A.ws_bytes(self.op, kind)
        buf = A.workspace(n, self.device, tag)
        return A.ptr(buf), buf.numel()

    def tensor(self, a, dtype=F64):
        """Contiguous device tensor of `a` (numpy or torch)."""
        if isinstance(a, torch.Tensor):
            return a.to(device=self.device, dtype=dtype).contiguous()
        return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=self.device)

    # ---- set-up -----------------------------------------------------------------
    def set_fixed_dofs(self, fixed_dofs):
        fd = self.tensor(np.asarray(fixed_dofs, dtype=np.int64).ravel() if not isinstance(fixed_dofs, torch.Tensor)
                         else fixed_dofs, dtype=torch.int64)
        A.call("pyto_bc_mask", self.opp, A.ptr(fd) if fd.numel() else None, int(fd.numel()), A.ptr(self.mask),
               self._st())
        self.mask_version += 1
        return self

    def set_active(self, active):
        if active is None:
            self.active, self.n_active = None, self.nelem
            return self
        a = np.asarray(active.cpu().numpy() if isinstance(active, torch.Tensor) else active).astype(bool).ravel()
        if a.size != self.nelem:
            raise ValueError("active mask must have one entry per element")
        self.active = torch.as_tensor(a.astype(np.uint8), device=self.device)
        self.n_active = int(a.sum())
        return self

    # ---- material ------------------------------------------------------------------
    def simp(self, x, penal=3.0, emin=1e-9, want_ds=True):
        x = self.tensor(x)
        s = torch.empty_like(x)
        ds = torch.empty_like(x) if want_ds else None
        A.call("pyto_simp", A.ptr(x), A.ptr(self.active), int(x.numel()), float(penal), float(emin), A.ptr(s),
               A.ptr(ds), self._st())
        return s, ds

    # ---- operator -------------------------------------------------------------------
    def matvec(self, s, u, mode=A.MASK_IN | A.MASK_OUT, out=None, dot=False):
        """y = K(s) u on full-length vectors (Dirichlet masking per mode)."""
        y = out if out is not None else torch.empty(self.ndof, dtype=F64, device=self.device)
        d = torch.empty(1, dtype=F64, device=self.device) if dot else None
        wsp, wsn = self._ws(A.WS_REDUCE, "reduce") if dot else (None, 0)
        A.call("pyto_matvec", self.opp, A.ptr(s), A.ptr(self.mask), A.ptr(u), A.ptr(y), int(mode), A.ptr(d), wsp, wsn,
               self._st())
        return (y, d) if dot else y

    def matvec_f32(self, s32, u32, mode=A.MASK_IN | A.MASK_OUT, out=None, dot=False):
        """FP32 y = K(s) u (the operator of the mixed-precision inner cycles); dot: also
        u.y accumulated in FP64."""
        y = out if out is not None else torch.empty(self.ndof, dtype=torch.float32, device=self.device)
        d = torch.empty(1, dtype=F64, device=self.device) if dot else None
        wsp, wsn = self._ws(A.WS_REDUCE, "reduce") if dot else (None, 0)
        A.call("pyto_matvec_f32", self.opp, A.ptr(s32), A.ptr(self.mask), A.ptr(u32), A.ptr(y), int(mode), A.ptr(d),
               wsp, wsn, self._st())
        return (y, d) if dot else y

    def jacobi(self, s):
        winv = torch.empty(self.nnodes, dtype=F64, device=self.device)
        flags = torch.empty(self.nnodes, dtype=torch.uint8, device=self.device)
        diag = torch.empty(self.ndof, dtype=F64, device=self.device)
        A.call("pyto_jacobi", self.opp, A.ptr(s), A.ptr(self.mask), A.ptr(winv), A.ptr(flags), A.ptr(diag),
               self._st())
        return diag, flags

    # ---- solvers ---------------------------------------------------------------------
    @staticmethod
    def _cfg(rtol, max_iters, stop_rule, check_every, x0):
        return A.SolveCfg(float(rtol), int(max_iters), int(stop_rule), int(check_every), 1 if x0 else 0)

    def pcg(self, s, b, rtol=1e-8, max_iters=100000, stop_rule=0, x0=None, check_every=25, out=None):
        """Jacobi PCG on K_ff (fixed DOFs of the result are 0)."""
        u = out if out is not None else torch.empty(self.ndof, dtype=F64, device=self.device)
        if x0 is not None:
            u.copy_(x0)
        cfg = self._cfg(rtol, max_iters, stop_rule, check_every, x0 is not None)
        stt = A.SolveStatus()
        wsp, wsn = self._ws(A.WS_PCG, "krylov")
        rc = A.call("pyto_pcg_solve", self.opp, A.ptr(s), A.ptr(self.mask), A.ptr(b), A.ptr(u), C.byref(cfg),
                    C.byref(stt), wsp, wsn, self._st(), allow=(A.OK, A.NOT_CONVERGED, A.ERR_BREAKDOWN))
        return u, SolveInfo(bool(stt.converged), int(stt.iters), bool(stt.breakdown), float(stt.rel_res),
                            float(stt.true_rel_res), rc)

    def dpcg_setup(self, s, defl):
        defl.sync(self)
        wsp, wsn = self._ws(A.WS_DPCG, "krylov")
        A.call("pyto_dpcg_setup", self.opp, A.ptr(s), A.ptr(self.mask), C.byref(defl.struct), wsp, wsn, self._st())

    def dpcg(self, s, b, defl, rtol=1e-8, max_iters=2000, stop_rule=1, check_every=25, out=None, setup=True,
             x0=None):
        """Deflated PCG (coarse inverse rebuilt for s when setup=True).  x0 (a warm start)
        needs stop_rule=2."""
        if setup:
            self.dpcg_setup(s, defl)
        defl.sync(self)
        u = out if out is not None else torch.empty(self.ndof, dtype=F64, device=self.device)
        if x0 is not None:
            if stop_rule != 2:
                raise ValueError("a warm start needs stop_rule=2 (the other rules start from the coarse solution)")
            u.copy_(x0)
        cfg = self._cfg(rtol, max_iters, stop_rule, check_every, x0 is not None)
        stt = A.SolveStatus()
        wsp, wsn = self._ws(A.WS_DPCG, "krylov")
        rc = A.call("pyto_dpcg_solve", self.opp, A.ptr(s), A.ptr(self.mask), C.byref(defl.struct), A.ptr(b),
                    A.ptr(u), C.byref(cfg), C.byref(stt), wsp, wsn, self._st(),
                    allow=(A.OK, A.NOT_CONVERGED, A.ERR_BREAKDOWN))
        return u, SolveInfo(bool(stt.converged), int(stt.iters), bool(stt.breakdown), float(stt.rel_res),
                            float(stt.true_rel_res), rc)

    def dpcg_mixed(self, s, b, defl, rtol=1e-8, delta=1e-1, max_iters=4000, check_every=10, out=None,
                   setup=True, x0=None):
        """Deflated PCG in mixed precision: an FP32 recurrence whose residual is replaced
        by the FP64 true residual b - K u (u held in FP64) each time it has dropped by
        `delta`; converged when ||b - K u|| <= rtol ||b|| in FP64.  info.cycles is the
        number of FP64 residual updates."""
        wsp, wsn = self._ws(A.WS_DPCG_MIXED, "krylov")
        defl.sync(self)
        if setup:
            A.call("pyto_dpcg_setup", self.opp, A.ptr(s), A.ptr(self.mask), C.byref(defl.struct), wsp, wsn,
                   self._st())
        u = out if out is not None else torch.empty(self.ndof, dtype=F64, device=self.device)
        if x0 is not None:
            u.copy_(x0)
        cfg = self._cfg(rtol, max_iters, 0, check_every, x0 is not None)
        stt = A.SolveStatus()
        rc = A.call("pyto_dpcg_mixed_solve", self.opp, A.ptr(s), A.ptr(self.mask), C.byref(defl.struct), A.ptr(b),
                    A.ptr(u), C.byref(cfg), float(delta), C.byref(stt), wsp, wsn, self._st(),
                    allow=(A.OK, A.NOT_CONVERGED, A.ERR_BREAKDOWN))
        info = SolveInfo(bool(stt.converged), int(stt.iters), bool(stt.breakdown), float(stt.rel_res),
                         float(stt.true_rel_res), rc)
        info.cycles = int(stt.reserved)
        return u, info

    # ---- element quantities ---------------------------------------------------------------
    def energy(self, u, v=None, s=None):
        """ce_e = u_e^T Ke v_e; with s also returns sum_e s_e ce_e (device scalar)."""
        v = u if v is None else v
        ce = torch.empty(self.nelem, dtype=F64, device=self.device)
        tot = torch.empty(1, dtype=F64, device=self.device) if s is not None else None
        wsp, wsn = self._ws(A.WS_REDUCE, "reduce") if s is not None else (None, 0)
        A.call("pyto_elem_energy", self.opp, A.ptr(u), A.ptr(v), A.ptr(s), A.ptr(ce), A.ptr(tot), wsp, wsn,
               self._st())
        return (ce, tot) if s is not None else ce

    def stress(self, u, x, q=0.5, want=("strain", "stress", "vm", "sed")):
        out = {}
        for k, n in (("strain", 6), ("stress", 6), ("vm", 1), ("sed", 1)):
            out[k] = torch.empty(self.nelem * n, dtype=F64, device=self.device) if k in want else None
        A.call("pyto_stress", self.opp, A.ptr(u), A.ptr(self.tensor(x)), float(q), A.ptr(out["strain"]),
               A.ptr(out["stress"]), A.ptr(out["vm"]), A.ptr(out["sed"]), self._st())
        for k in ("strain", "stress"):
            if out[k] is not None:
                out[k] = out[k].view(self.nelem, 6)
        return out

    def pow_sum(self, vm, P):
        out = torch.empty(1, dtype=F64, device=self.device)
        wsp, wsn = self._ws(A.WS_REDUCE, "reduce")
        A.call("pyto_pnorm_sum", self.opp, A.ptr(vm), float(P), A.ptr(out), wsp, wsn, self._st())
        return out

    def pnorm_adjoint(self, u, x, q, P, dpn_dev):
        T1 = torch.empty(self.nelem, dtype=F64, device=self.device)
        g = torch.empty(self.ndof, dtype=F64, device=self.device)
        tvec = torch.empty(6 * self.nelem, dtype=F64, device=self.device)
        A.call("pyto_pnorm_adjoint", self.opp, A.ptr(u), A.ptr(self.tensor(x)), float(q), float(P), A.ptr(dpn_dev),
               A.ptr(T1), A.ptr(g), A.ptr(tvec), self._st())
        return T1, g

    # ---- filter / OC ------------------------------------------------------------------------
    def filter(self, rel_radius, mode, x=None, w=None, hs=None, out=None):
        y = out if out is not None else torch.empty(self.nelem, dtype=F64, device=self.device)
        A.call("pyto_filter", self.opp, float(rel_radius), int(mode), A.ptr(x), A.ptr(w), A.ptr(hs),
               A.ptr(self.active), A.ptr(y), self._st())
        return y

    def oc_update(self, x, dc, volfrac, move=0.2, xmin=0.001, xmax=1.0):
        """In-place OC update of x; returns max |dx| as a device scalar."""
        ch = torch.empty(1, dtype=F64, device=self.device)
        wsp, wsn = self._ws(A.WS_OC, "oc")
        A.call("pyto_oc_update", self.opp, A.ptr(x), A.ptr(dc), A.ptr(self.active), int(self.n_active),
               float(volfrac), float(move), float(xmin), float(xmax), A.ptr(ch), wsp, wsn, self._st())
        return ch


class ThermalGrid:
    """A box grid of hex8 elements with one temperature DOF per node on one CUDA
    device (the thermal path: pyto_thermal_*)."""

    def __init__(self, nel, elem_size=(1.0, 1.0, 1.0), k=1.0, ke=None, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("pyto_b200 needs a CUDA device (sm_100a); no CPU path exists")
        self.device = torch.device(device if device is not None else "cuda")
        self.nel = tuple(int(n) for n in nel)
        self.h = tuple(float(v) for v in elem_size)
        self.th = A.make_thermal(*self.nel, self.h, k, ke)
        nx, ny, nz = self.nel
        self.nnodes = (nx + 1) * (ny + 1) * (nz + 1)
        self.nelem = nx * ny * nz
        self.ndof = self.nnodes
        self.mask = torch.zeros(self.nnodes, dtype=torch.uint8, device=self.device)
        self.active = None

    @property
    def thp(self):
        return C.byref(self.th)

    def _st(self):
        return A.stream_ptr(self.device)

    def _ws(self):
        n = int(A.lib().pyto_thermal_workspace_bytes(self.thp))
        buf = A.workspace(n, self.device, "thermal")
        return A.ptr(buf), buf.numel()

    tensor = HexGrid.tensor

    def set_fixed_nodes(self, nodes):
        nd = self.tensor(np.asarray(nodes, dtype=np.int64).ravel() if not isinstance(nodes, torch.Tensor) else nodes,
                         dtype=torch.int64)
        A.call("pyto_thermal_mask", self.thp, A.ptr(nd) if nd.numel() else None, int(nd.numel()), A.ptr(self.mask),
               self._st())
        return self

    def simp(self, x, penal=1.0, kvoid=1e-8, want_ds=True):
        """Thermal SIMP s = kvoid + x^p (1 - kvoid) (the structural kernel's formula)."""
        x = self.tensor(x)
        s = torch.empty_like(x)
        ds = torch.empty_like(x) if want_ds else None
        A.call("pyto_simp", A.ptr(x), None, int(x.numel()), float(penal), float(kvoid), A.ptr(s), A.ptr(ds),
               self._st())
        return s, ds

    def matvec(self, s, u, mode=A.MASK_IN | A.MASK_OUT, out=None, dot=False):
        y = out if out is not None else torch.empty(self.ndof, dtype=F64, device=self.device)
        d = torch.empty(1, dtype=F64, device=self.device) if dot else None
        wsp, wsn = self._ws() if dot else (None, 0)
        A.call("pyto_thermal_matvec", self.thp, A.ptr(s), A.ptr(self.mask), A.ptr(u), A.ptr(y), int(mode), A.ptr(d),
               wsp, wsn, self._st())
        return (y, d) if dot else y

    def pcg(self, s, b, rtol=1e-8, max_iters=100000, stop_rule=0, x0=None, check_every=25, out=None):
        """Jacobi PCG on the reduced thermal system (fixed nodes of the result are 0)."""
        u = out if out is not None else torch.empty(self.ndof, dtype=F64, device=self.device)
        if x0 is not None:
            u.copy_(x0)
        cfg = HexGrid._cfg(rtol, max_iters, stop_rule, check_every, x0 is not None)
        stt = A.SolveStatus()
        wsp, wsn = self._ws()
        rc = A.call("pyto_thermal_pcg_solve", self.thp, A.ptr(s), A.ptr(self.mask), A.ptr(b), A.ptr(u),
                    C.byref(cfg), C.byref(stt), wsp, wsn, self._st(), allow=(A.OK, A.NOT_CONVERGED, A.ERR_BREAKDOWN))
        return u, SolveInfo(bool(stt.converged), int(stt.iters), bool(stt.breakdown), float(stt.rel_res),
                            float(stt.true_rel_res), rc)

    def energy(self, u, v=None, s=None):
        """ce_e = u_e^T Ke v_e; with s also sum_e s_e ce_e (device scalar)."""
        ce = torch.empty(self.nelem, dtype=F64, device=self.device)
        tot = torch.empty(1, dtype=F64, device=self.device) if s is not None else None
        wsp, wsn = self._ws() if s is not None else (None, 0)
        A.call("pyto_thermal_energy", self.thp, A.ptr(u), A.ptr(v), A.ptr(s), A.ptr(ce), A.ptr(tot), wsp, wsn,
               self._st())
        return (ce, tot) if s is not None else ce


class DeviceDeflation:
    """Device data of a deflation space (node groups + rigid modes).

    Besides the node->group map, the CSR of nodes per group and the group
    centres, set-up derives once per mesh: the box of elements touching each
    group and, per group, the sorted list of groups sharing an element with it
    (the non-zero block pattern of W^T K W).
    """

    def __init__(self, grid: HexGrid, node_group, centers, modes=6, shift=1e-10, shift_relative=False,
                 coarse="dense", group_grid=None, leaf=8):
        node_group = np.asarray(node_group, dtype=np.int32).ravel()
        centers = np.asarray(centers, dtype=np.float64).reshape(-1, 3)
        ng = centers.shape[0]
        order = np.argsort(node_group, kind="stable").astype(np.int32)
        counts = np.bincount(node_group, minlength=ng)
        gptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
        nx, ny, nz = grid.nel
        sx, sy = nx + 1, ny + 1
        n = np.arange(node_group.size)
        ix, iy, iz = n % sx, (n // sx) % sy, n // (sx * sy)
        box = np.zeros((ng, 6), dtype=np.int32)
        for d, (coord, ne) in enumerate(((ix, nx), (iy, ny), (iz, nz))):
            lo = np.full(ng, np.iinfo(np.int64).max)
            hi = np.full(ng, -1)
            np.minimum.at(lo, node_group, coord)
            np.maximum.at(hi, node_group, coord)
            box[:, 2 * d] = np.clip(lo - 1, 0, ne - 1)
            box[:, 2 * d + 1] = np.clip(hi, 0, ne - 1)
        # group pairs sharing an element: corners of every element
        ez, ey, ex = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        n0 = (ex + sx * (ey + sy * ez)).ravel()
        pairs = []
        corner = [0, 1, sx, sx + 1, sx * sy, sx * sy + 1, sx * sy + sx, sx * sy + sx + 1]
        self._corner_nodes = np.stack([n0 + c for c in corner], 1).astype(np.int32)
        cg = node_group[self._corner_nodes]
        self._spans = (cg != cg[:, :1]).any(1)
        for a in range(8):
            for b in range(8):
                pairs.append(cg[:, a].astype(np.int64) * ng + cg[:, b])
        key = np.unique(np.concatenate(pairs))
        ga, gb = (key // ng).astype(np.int32), (key % ng).astype(np.int32)
        nptr = np.concatenate([[0], np.cumsum(np.bincount(ga, minlength=ng))]).astype(np.int32)
        self.max_nbr = int(np.diff(nptr).max())
        if self.max_nbr > 128:
            raise ValueError(f"a deflation group touches {self.max_nbr} groups (limit 128)")
        dev = grid.device
        self.node_group = torch.as_tensor(node_group, device=dev)
        self.group_ptr = torch.as_tensor(gptr, device=dev)
        self.group_nodes = torch.as_tensor(order, device=dev)
        self.group_center = torch.as_tensor(np.ascontiguousarray(centers), device=dev)
        self.group_box = torch.as_tensor(np.ascontiguousarray(box), device=dev)
        self.nbr_ptr = torch.as_tensor(nptr, device=dev)
        self.nbr_list = torch.as_tensor(gb, device=dev)
        self.ngroups, self.modes = ng, int(modes)
        self.nc = ng * self.modes
        if coarse not in ("dense", "nd"):
            raise ValueError(f"unknown coarse solver {coarse!r} (dense, nd)")
        self.coarse = coarse
        self.nd_plan = None
        if coarse == "nd":
            # nested dissection on the box grid of groups: no dense coarse matrix
            if group_grid is None or int(np.prod(group_grid)) != ng:
                raise ValueError("coarse='nd' needs the box grid (gx, gy, gz) of the groups")
            self.box = tuple(int(v) for v in group_grid)
            self._nptr_h, self._nlist_h = np.ascontiguousarray(nptr), np.ascontiguousarray(gb)
            plan = A.lib().pyto_coarse_nd_plan(*self.box, self.modes, int(leaf), self._nptr_h.ctypes.data,
                                               self._nlist_h.ctypes.data)
            if not plan:
                raise ValueError("pyto_coarse_nd_plan: " + A.last_error())
            self.nd_plan = plan
            info = (C.c_double * 5)()
            nbytes = A.lib().pyto_coarse_nd_bytes(plan, info)
            self.nd_info = dict(nodes=int(info[0]), depth=int(info[1]), max_front=int(info[2]),
                                factor_flops=float(info[3]), solve_bytes=float(info[4]), device_bytes=int(nbytes))
            self.nd_buf = torch.empty(int(nbytes), dtype=torch.uint8, device=dev)
            A.call("pyto_coarse_nd_bind", plan, A.ptr(self.nd_buf), int(nbytes), A.stream_ptr(dev))
            self.coarse_inv = None
        else:
            self.coarse_inv = torch.empty(self.nc * self.nc, dtype=F64, device=dev)
        self.struct = A.Deflation(ng, self.modes, A.ptr(self.node_group), A.ptr(self.group_ptr),
                                  A.ptr(self.group_nodes), A.ptr(self.group_center),
                                  A.ptr(self.coarse_inv) if self.coarse_inv is not None else None,
                                  float(shift), 1 if shift_relative else 0, int(counts.max()), A.ptr(self.group_box),
                                  A.ptr(self.nbr_ptr), A.ptr(self.nbr_list), self.max_nbr, 0, None, None)
        if self.nd_plan is not None:
            self.struct.coarse_nd = self.nd_plan
        self._node_group_np = node_group
        self.use_boundary_lists = True
        self.mask_version = None
        self.sync(grid)

    def nd_solve(self, v, out=None):
        """mu = (W_f^T K_ff W_f + shift I)^-1 v with the nested-dissection factors of the
        last set-up (coarse='nd')."""
        if self.nd_plan is None:
            raise ValueError("this deflation space uses the dense coarse inverse")
        mu = out if out is not None else torch.empty_like(v)
        A.call("pyto_coarse_nd_solve", self.nd_plan, A.ptr(v), A.ptr(mu), A.stream_ptr(v.device))
        return mu

    def __del__(self):
        plan = getattr(self, "nd_plan", None)
        if not plan:
            return
        self.nd_plan = None
        try:  # the plan's device buffer is torch's; the host plan must outlive queued work
            torch.cuda.synchronize(self.node_group.device)
            A.lib().pyto_coarse_nd_free(plan)
        except Exception:  # pragma: no cover - interpreter shutdown: the process frees it
            pass

    def sync(self, grid: HexGrid):
        """(Re)build the per-group boundary element lists for the grid's current fixed
        DOFs: elements with a corner in the group and a corner in another group or on a
        fixed DOF (W_f^T K z is formed from these elements only)."""
        if not self.use_boundary_lists:
            if self.nd_plan is not None:
                raise ValueError("the nested-dissection coarse solver needs the boundary element lists")
            self.struct.bel_ptr = self.struct.bel_list = self.struct.bel_meta = None
            self.struct.bel_count = 0
            return self
        if self.mask_version == grid.mask_version:
            self.struct.bel_ptr, self.struct.bel_list = A.ptr(self.bel_ptr), A.ptr(self.bel_list)
            self.struct.bel_meta = A.ptr(self.bel_meta)
            self.struct.bel_count = int(self.bel_list.numel())
            return self
        mask = grid.mask[:grid.nnodes].cpu().numpy()
        fixed_el = ((mask[self._corner_nodes] & 7) != 0).any(1)
        el = np.flatnonzero(self._spans | fixed_el)
        cg = self._node_group_np[self._corner_nodes[el]].astype(np.int64)
        key = np.unique((cg * grid.nelem + el[:, None]).ravel())
        grp, elem = key // grid.nelem, key % grid.nelem
        bptr = np.concatenate([[0], np.cumsum(np.bincount(grp, minlength=self.ngroups))]).astype(np.int32)
        # per entry: which corners of its element lie in its group (bits 0-7), and
        # whether the element has a fixed DOF (bit 8)
        rows = cg[np.searchsorted(el, elem)]
        meta = ((rows == grp[:, None]).astype(np.uint16) << np.arange(8, dtype=np.uint16)).sum(1, dtype=np.uint16)
        meta |= fixed_el[elem].astype(np.uint16) << 8
        self.bel_ptr = torch.as_tensor(bptr, device=grid.device)
        self.bel_list = torch.as_tensor(elem.astype(np.int32), device=grid.device)
        self.bel_meta = torch.as_tensor(meta.astype(np.int16), device=grid.device)  # uint16 bits
        self.struct.bel_ptr, self.struct.bel_list = A.ptr(self.bel_ptr), A.ptr(self.bel_list)
        self.struct.bel_meta = A.ptr(self.bel_meta)
        self.struct.bel_count = int(self.bel_list.numel())
        self.mask_version = grid.mask_version
        return self


class BatchSolver:
    """Many deflated PCG problems solved by one CUDA-graph launch (pyto_batch_*).

    ``problems`` is a list of (grid, defl, s, b): a HexGrid, its DeviceDeflation, the
    element scaling and the right-hand side.  Problems that share one DeviceDeflation
    are load cases of one design (same grid and s): its coarse inverse is built once
    per launch.  ``launch()`` solves all of them; rewrite the s and b tensors in place
    and launch again for new designs and loads.  Solutions are in ``self.u``.

    The graph holds the device addresses of every buffer it reads.  Only the contents
    of s and b may change between launches: a grid whose fixed DOFs were reset (which
    rebuilds its deflation space's boundary lists) or a deflation space whose lists
    were rebuilt makes ``launch()`` raise; build a new BatchSolver then."""

    def __init__(self, problems, rtol=1e-8, max_iters=5000, stop_rule=0):
        self.problems = list(problems)
        n = len(self.problems)
        if n == 0:
            raise ValueError("empty batch")
        self.items = (A.BatchItem * n)()
        self.u, self._ws = [], []
        self._captured = []  # per problem: what the graph's kernel arguments point at
        dev = None
        for k, (grid, defl, s, b) in enumerate(self.problems):
            dev = grid.device
            defl.sync(grid)
            if not defl.use_boundary_lists or defl.struct.bel_count <= 0:
                raise ValueError("batched solves need the boundary element lists of the deflation space")
            # the references keep the captured buffers alive (no address reuse while the
            # graph exists); launch() compares them with the current ones
            self._captured.append((grid, grid.mask_version, defl, defl.bel_ptr, defl.bel_list, defl.bel_meta))
            nb = A.ws_bytes(grid.op, A.WS_DPCG)
            ws = torch.empty(nb, dtype=torch.uint8, device=dev)  # one workspace per problem
            u = torch.zeros(grid.ndof, dtype=F64, device=dev)
            self._ws.append(ws)
            self.u.append(u)
            self.items[k] = A.BatchItem(C.pointer(grid.op), A.ptr(s), A.ptr(grid.mask), C.pointer(defl.struct),
                                        A.ptr(b), A.ptr(u), A.ptr(ws), nb)
        self.device = dev
        self.cfg = A.SolveCfg(float(rtol), int(max_iters), int(stop_rule), 1, 0)
        self.handle = C.c_void_p()
        A.call("pyto_batch_create", self.items, n, C.byref(self.cfg), C.byref(self.handle), A.stream_ptr(dev))

    def _check_captured(self):
        for k, (grid, version, defl, bptr, blist, bmeta) in enumerate(self._captured):
            if grid.mask_version != version or defl.mask_version != version or defl.bel_ptr is not bptr \
                    or defl.bel_list is not blist or defl.bel_meta is not bmeta:
                raise RuntimeError(f"batch problem {k}: the fixed DOFs or the deflation boundary lists changed "
                                   "after the batch was created; create a new BatchSolver")

    def launch(self):
        self._check_captured()
        A.call("pyto_batch_launch", self.handle, A.stream_ptr(self.device))
        return self

    def status(self):
        n = len(self.problems)
        st = (A.SolveStatus * n)()
        A.call("pyto_batch_status", self.handle, st, A.stream_ptr(self.device),
               allow=(A.OK, A.NOT_CONVERGED, A.ERR_BREAKDOWN))
        return [SolveInfo(bool(x.converged), int(x.iters), bool(x.breakdown), float(x.rel_res),
                          float(x.true_rel_res), 0) for x in st]

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            A.call("pyto_batch_destroy", self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass
