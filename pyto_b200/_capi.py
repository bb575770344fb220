"""ctypes binding of libpyto_b200.so (the C ABI declared in include/pyto_b200.h).

The library must be built (``python -m pyto_b200.build``); there is no
fallback: every compute call goes through this binding, and using it on a
machine without the library raises ``PytoLibraryError``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpyto_b200.so")
# library defaults of pyto_tune(PYTO_KERNEL_MATVEC / PYTO_KERNEL_MATVEC32, ...)
MV64_DEFAULT = 2
MV32_DEFAULT = 18

OK, NOT_CONVERGED = 0, 1
ERR_ARG, ERR_CUDA, ERR_WORKSPACE, ERR_BREAKDOWN, ERR_TOO_LARGE = -1, -2, -3, -4, -5
MASK_IN, MASK_OUT = 1, 2
FILTER_RAW, FILTER_DENSITY, FILTER_CHAIN, FILTER_SENS, FILTER_HS = 0, 1, 2, 3, 4
SYM_MIRROR, SYM_EXTRUDE = 0, 1
WS_REDUCE, WS_PCG, WS_DPCG, WS_OC, WS_DPCG_MIXED = 0, 1, 2, 3, 4


class PytoLibraryError(RuntimeError):
    """libpyto_b200.so is missing or failed to load."""


class PytoError(RuntimeError):
    """A C-ABI call returned an error status."""

    def __init__(self, fn: str, rc: int, detail: str = ""):
        names = {ERR_ARG: "invalid argument", ERR_CUDA: "CUDA error", ERR_WORKSPACE: "workspace too small",
                 ERR_BREAKDOWN: "Krylov breakdown", ERR_TOO_LARGE: "size beyond limit"}
        super().__init__(f"{fn} failed: {names.get(rc, rc)} ({rc})" + (f": {detail}" if detail else ""))
        self.rc = rc


class Operator(C.Structure):
    _fields_ = [("nelx", C.c_int32), ("nely", C.c_int32), ("nelz", C.c_int32), ("tune", C.c_int32),
                ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double), ("E", C.c_double), ("nu", C.c_double),
                ("ke", C.c_double * 576), ("khat", C.c_double * 72), ("kdiag", C.c_double * 3)]


class SolveCfg(C.Structure):
    _fields_ = [("rtol", C.c_double), ("max_iters", C.c_int32), ("stop_rule", C.c_int32),
                ("check_every", C.c_int32), ("x0_given", C.c_int32)]


class SolveStatus(C.Structure):
    _fields_ = [("converged", C.c_int32), ("iters", C.c_int32), ("breakdown", C.c_int32), ("reserved", C.c_int32),
                ("rel_res", C.c_double), ("true_rel_res", C.c_double)]


class Deflation(C.Structure):
    _fields_ = [("ngroups", C.c_int32), ("modes", C.c_int32), ("node_group", C.c_void_p), ("group_ptr", C.c_void_p),
                ("group_nodes", C.c_void_p), ("group_center", C.c_void_p), ("coarse_inv", C.c_void_p),
                ("shift", C.c_double), ("shift_relative", C.c_int32), ("max_group_nodes", C.c_int32),
                ("group_box", C.c_void_p), ("nbr_ptr", C.c_void_p), ("nbr_list", C.c_void_p), ("max_nbr", C.c_int32),
                ("bel_count", C.c_int32), ("bel_ptr", C.c_void_p), ("bel_list", C.c_void_p),
                ("bel_meta", C.c_void_p), ("coarse_nd", C.c_void_p)]


class BatchItem(C.Structure):
    _fields_ = [("op", C.POINTER(Operator)), ("s", C.c_void_p), ("mask", C.c_void_p),
                ("defl", C.POINTER(Deflation)), ("b", C.c_void_p), ("u", C.c_void_p), ("ws", C.c_void_p),
                ("ws_bytes", C.c_size_t)]


class Thermal(C.Structure):
    _fields_ = [("nelx", C.c_int32), ("nely", C.c_int32), ("nelz", C.c_int32), ("pad", C.c_int32),
                ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double), ("k", C.c_double),
                ("ke", C.c_double * 64), ("kxor", C.c_double * 8)]


_P = C.c_void_p
_OP = C.POINTER(Operator)
_TH = C.POINTER(Thermal)
SIGNATURES = {
    "pyto_version": (C.c_int, []),
    "pyto_coarse_nd_plan": (C.c_void_p, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P, _P]),
    "pyto_coarse_nd_bytes": (C.c_size_t, [_P, _P]),
    "pyto_coarse_nd_bind": (C.c_int, [_P, _P, C.c_size_t, _P]),
    "pyto_coarse_nd_solve": (C.c_int, [_P, _P, _P, _P]),
    "pyto_coarse_nd_free": (None, [_P]),
    "pyto_struct_size": (C.c_size_t, [C.c_int]),
    "pyto_last_error": (C.c_char_p, []),
    "pyto_launch_count": (C.c_longlong, []),
    "pyto_tune": (C.c_int, [C.c_int, C.c_int]),
    "pyto_workspace_bytes": (C.c_size_t, [_OP, C.c_int]),
    "pyto_ke_hex8": (C.c_int, [C.c_double] * 5 + [_P]),
    "pyto_operator_init": (C.c_int, [_OP, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                     C.c_double, C.c_double, _P]),
    "pyto_simp": (C.c_int, [_P, _P, C.c_int64, C.c_double, C.c_double, _P, _P, _P]),
    "pyto_bc_mask": (C.c_int, [_OP, _P, C.c_int64, _P, _P]),
    "pyto_matvec": (C.c_int, [_OP, _P, _P, _P, _P, C.c_int, _P, _P, C.c_size_t, _P]),
    "pyto_matvec_f32": (C.c_int, [_OP, _P, _P, _P, _P, C.c_int, _P, _P, C.c_size_t, _P]),
    "pyto_tensor_core_status": (C.c_int, [C.c_int]),
    "pyto_jacobi": (C.c_int, [_OP, _P, _P, _P, _P, _P, _P]),
    "pyto_matvec_dot_noalloc": (C.c_int, [_OP, _P, _P, _P, _P, C.c_int, _P, _P]),
    "pyto_pcg_solve": (C.c_int, [_OP, _P, _P, _P, _P, C.POINTER(SolveCfg), C.POINTER(SolveStatus), _P, C.c_size_t,
                                 _P]),
    "pyto_dpcg_setup": (C.c_int, [_OP, _P, _P, C.POINTER(Deflation), _P, C.c_size_t, _P]),
    "pyto_dpcg_solve": (C.c_int, [_OP, _P, _P, C.POINTER(Deflation), _P, _P, C.POINTER(SolveCfg),
                                  C.POINTER(SolveStatus), _P, C.c_size_t, _P]),
    "pyto_dpcg_mixed_solve": (C.c_int, [_OP, _P, _P, C.POINTER(Deflation), _P, _P, C.POINTER(SolveCfg), C.c_double,
                                        C.POINTER(SolveStatus), _P, C.c_size_t, _P]),
    "pyto_coarse_assemble": (C.c_int, [_OP, _P, _P, C.POINTER(Deflation), _P, C.c_size_t, _P]),
    "pyto_coarse_invert": (C.c_int, [_OP, C.POINTER(Deflation), _P, C.c_size_t, _P]),
    "pyto_coarse_restrict": (C.c_int, [_OP, C.POINTER(Deflation), _P, _P, _P, _P, C.c_size_t, _P]),
    "pyto_coarse_apply": (C.c_int, [C.POINTER(Deflation), _P, _P, _P]),
    "pyto_coarse_prolong": (C.c_int, [_OP, C.POINTER(Deflation), _P, _P, C.c_double, _P, C.c_double, _P, _P]),
    "pyto_cg_update": (C.c_int, [_OP, _P, _P, C.c_double, _P, _P, _P, _P, _P, _P, _P, C.c_size_t, _P]),
    "pyto_ke_hex8_thermal": (C.c_int, [C.c_double] * 4 + [_P]),
    "pyto_thermal_init": (C.c_int, [_TH, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                    C.c_double, _P]),
    "pyto_thermal_mask": (C.c_int, [_TH, _P, C.c_int64, _P, _P]),
    "pyto_thermal_workspace_bytes": (C.c_size_t, [_TH]),
    "pyto_thermal_matvec": (C.c_int, [_TH, _P, _P, _P, _P, C.c_int, _P, _P, C.c_size_t, _P]),
    "pyto_thermal_pcg_solve": (C.c_int, [_TH, _P, _P, _P, _P, C.POINTER(SolveCfg), C.POINTER(SolveStatus), _P,
                                         C.c_size_t, _P]),
    "pyto_thermal_energy": (C.c_int, [_TH, _P, _P, _P, _P, _P, _P, C.c_size_t, _P]),
    "pyto_mma_workspace_bytes": (C.c_size_t, [C.c_int64, C.c_int]),
    "pyto_mma_update": (C.c_int, [C.c_int64, C.c_int, C.c_int, _P, _P, _P, _P, _P, C.c_double, C.c_double, _P, _P,
                                  _P, _P, _P, C.c_double, _P, _P, _P, C.c_double, _P, _P, C.c_size_t, _P]),
    "pyto_mma_kkt": (C.c_int, [C.c_int64, C.c_int, _P, _P, _P, C.c_double, C.c_double, _P, _P, _P, C.c_double, _P, _P,
                               _P, _P, _P, C.c_size_t, _P]),
    "pyto_batch_create": (C.c_int, [C.POINTER(BatchItem), C.c_int, C.POINTER(SolveCfg), C.POINTER(C.c_void_p), _P]),
    "pyto_batch_launch": (C.c_int, [_P, _P]),
    "pyto_batch_status": (C.c_int, [_P, C.POINTER(SolveStatus), _P]),
    "pyto_batch_destroy": (C.c_int, [_P]),
    "pyto_elem_energy": (C.c_int, [_OP, _P, _P, _P, _P, _P, _P, C.c_size_t, _P]),
    "pyto_stress": (C.c_int, [_OP, _P, _P, C.c_double, _P, _P, _P, _P, _P]),
    "pyto_pnorm_sum": (C.c_int, [_OP, _P, C.c_double, _P, _P, C.c_size_t, _P]),
    "pyto_pnorm_adjoint": (C.c_int, [_OP, _P, _P, C.c_double, C.c_double, _P, _P, _P, _P, _P]),
    "pyto_filter": (C.c_int, [_OP, C.c_double, C.c_int, _P, _P, _P, _P, _P, _P]),
    "pyto_symmetry_filter": (C.c_int, [_OP, C.c_int, C.c_int, _P, _P, _P, _P, _P]),
    "pyto_vec_scale": (C.c_int, [C.c_int64, _P, _P, _P, _P, _P, _P]),
    "pyto_oc_update": (C.c_int, [_OP, _P, _P, _P, C.c_longlong, C.c_double, C.c_double, C.c_double, C.c_double, _P,
                                 _P, C.c_size_t, _P]),
}

_lib = None


def lib():
    """The loaded library (loads it on first use)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PytoLibraryError(f"{LIB_PATH} not found; build it with `python -m pyto_b200.build`")
        try:
            L = C.CDLL(LIB_PATH)
        except OSError as e:  # pragma: no cover
            raise PytoLibraryError(f"cannot load {LIB_PATH}: {e}") from e
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def call(fn: str, *args, allow=(OK,)) -> int:
    rc = getattr(lib(), fn)(*args)
    if rc not in allow:
        err = PytoError(fn, rc)
        if rc == ERR_CUDA:
            detail = lib().pyto_last_error()
            if detail:
                err = PytoError(fn, rc, detail.decode(errors="replace"))
        raise err
    return rc


def last_error() -> str:
    """The library's description of the last failure of this thread ("" if none)."""
    d = lib().pyto_last_error()
    return d.decode(errors="replace") if d else ""


def ptr(t):
    """Device pointer of a contiguous CUDA tensor (None for None)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t.data_ptr()


def stream_ptr(device=None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


# ---- workspace cache -------------------------------------------------------
_WS: dict = {}


def workspace(nbytes: int, device, tag: str = "ws") -> torch.Tensor:
    """A cached uint8 device buffer of at least nbytes (grows, never shrinks).

    Buffers are keyed by (device, current stream, tag): uses under one tag on one
    stream are ordered by that stream, and a buffer is only ever used on the stream
    it was allocated on, so when a grown buffer replaces it the caching allocator
    reuses the old block only after the work already queued on that stream."""
    key = (str(device), stream_ptr(device), tag)
    buf = _WS.get(key)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
        _WS[key] = buf
    return buf


def make_operator(nelx, nely, nelz, h=(1.0, 1.0, 1.0), E=1.0, nu=0.3, ke=None) -> Operator:
    op = Operator()
    kep = None
    if ke is not None:
        ke = np.ascontiguousarray(np.asarray(ke, dtype=np.float64).reshape(24, 24))
        kep = ke.ctypes.data_as(C.c_void_p)
    call("pyto_operator_init", C.byref(op), int(nelx), int(nely), int(nelz), float(h[0]), float(h[1]), float(h[2]),
         float(E), float(nu), kep)
    return op


def make_thermal(nelx, nely, nelz, h=(1.0, 1.0, 1.0), k=1.0, ke=None) -> Thermal:
    t = Thermal()
    kep = None
    if ke is not None:
        ke = np.ascontiguousarray(np.asarray(ke, dtype=np.float64).reshape(8, 8))
        kep = ke.ctypes.data_as(C.c_void_p)
    call("pyto_thermal_init", C.byref(t), int(nelx), int(nely), int(nelz), float(h[0]), float(h[1]), float(h[2]),
         float(k), kep)
    return t


def ws_bytes(op: Operator, kind: int) -> int:
    return int(lib().pyto_workspace_bytes(C.byref(op), kind))
