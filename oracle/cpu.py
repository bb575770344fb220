"""ctypes binding of the oracle's compiled half, ``oracle/hex8_cpu.c`` (TEST
INFRASTRUCTURE: used by tests/ as a checker and by bench.py's CPU-baseline legs
as the timed restatement of the reference's CPU path; never by the product).

``build()`` compiles it with gcc/OpenMP into ``oracle/libhex8_cpu.so``.
``CpuFEA`` holds one grid with its Dirichlet mask and runs, per call, the
reference's per-solve sequence: CSR assembly of K_ff (src/hex_structural_fea.py:
87-102 and src/bound_cond.py:40-70), then Jacobi PCG (src/linear_solvers.py:
164-168) or deflated PCG (src/deflation.py:504-584).
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "hex8_cpu.c")
LIB = os.path.join(HERE, "libhex8_cpu.so")
CFLAGS = ["-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-Wall"]

_lib = None


def build(force: bool = False) -> str:
    """Compile hex8_cpu.c (gcc, OpenMP, x86-64-v3) into libhex8_cpu.so."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        raise RuntimeError("no C compiler to build the oracle's CPU solver")
    tmp = LIB + ".tmp"
    r = subprocess.run([cc, *CFLAGS, "-o", tmp, SRC, "-lm"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("gcc failed on hex8_cpu.c:\n" + r.stderr)
    os.replace(tmp, LIB)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P = C.c_void_p
        sig = {
            "hex8_cpu_threads": (C.c_int, []),
            "hex8_cpu_create": (P, [C.c_int, C.c_int, C.c_int, P, P]),
            "hex8_cpu_destroy": (None, [P]),
            "hex8_cpu_nfree": (C.c_int64, [P]),
            "hex8_cpu_nnz": (C.c_int64, [P]),
            "hex8_cpu_assemble_seconds": (C.c_double, [P]),
            "hex8_cpu_assemble": (C.c_int, [P, P]),
            "hex8_cpu_csr": (C.c_int, [P, P, P, P]),
            "hex8_cpu_pcg": (C.c_int, [P, P, P, C.c_double, C.c_int, P, P, P]),
            "hex8_cpu_dpcg": (C.c_int, [P, P, C.c_int, P, C.c_int, C.c_double, C.c_int, P, P, P, C.c_double,
                                        C.c_int, C.c_int, P, P, P]),
            "hex8_cpu_density_filter": (C.c_int, [C.c_int, C.c_int, C.c_int, P, C.c_double, P, P]),
            "hex8_cpu_coarse_matrix": (C.c_int, [P, P, C.c_int, P, C.c_int, P, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def threads() -> int:
    """OpenMP threads the solver uses (OMP_NUM_THREADS, default all cores)."""
    return int(lib().hex8_cpu_threads())


def density_filter(nel, x, rel=2.0, h=(1.0, 1.0, 1.0)):
    """rho = (H x)/Hs with the reference's hat weights (src/topopt_filters.py:8-38)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    rho = np.empty_like(x)
    hx = np.ascontiguousarray(h, dtype=np.float64)
    lib().hex8_cpu_density_filter(int(nel[0]), int(nel[1]), int(nel[2]), _p(hx), float(rel), _p(x), _p(rho))
    return rho


class CpuFEA:
    """One grid on the host: K_ff assembled per solve, Jacobi PCG or DPCG."""

    def __init__(self, nel, Ke, fixed_dofs, h=(1.0, 1.0, 1.0)):
        self.nel = tuple(int(v) for v in nel)
        nx, ny, nz = self.nel
        self.nnodes = (nx + 1) * (ny + 1) * (nz + 1)
        self.h = np.ascontiguousarray(h, dtype=np.float64)
        mask = np.zeros(self.nnodes, dtype=np.uint8)
        fd = np.asarray(fixed_dofs, dtype=np.int64)
        np.bitwise_or.at(mask, fd // 3, (1 << (fd % 3)).astype(np.uint8))
        self._ke = np.ascontiguousarray(Ke, dtype=np.float64)
        self._mask = mask
        self.handle = lib().hex8_cpu_create(nx, ny, nz, _p(self._ke), _p(mask))
        if not self.handle:
            raise RuntimeError("hex8_cpu_create failed")
        self.nfree = int(lib().hex8_cpu_nfree(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            lib().hex8_cpu_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def assemble(self, s) -> float:
        """K_ff(s) as CSR plus the Jacobi inverse diagonal; returns seconds."""
        self._s = np.ascontiguousarray(s, dtype=np.float64)
        rc = lib().hex8_cpu_assemble(self.handle, _p(self._s))
        if rc != 0:
            raise RuntimeError(f"hex8_cpu_assemble failed ({rc})")
        return float(lib().hex8_cpu_assemble_seconds(self.handle))

    def csr(self):
        import scipy.sparse as sp
        nnz = int(lib().hex8_cpu_nnz(self.handle))
        rp = np.empty(self.nfree + 1, np.int64)
        col = np.empty(nnz, np.int32)
        val = np.empty(nnz, np.float64)
        lib().hex8_cpu_csr(self.handle, _p(rp), _p(col), _p(val))
        return sp.csr_matrix((val, col, rp), shape=(self.nfree, self.nfree))

    def pcg(self, b, rtol=1e-8, max_iters=100000):
        b = np.ascontiguousarray(b, dtype=np.float64)
        u = np.zeros_like(b)
        it, trr, t = C.c_int(0), C.c_double(0), C.c_double(0)
        rc = lib().hex8_cpu_pcg(self.handle, _p(b), _p(u), float(rtol), int(max_iters), C.byref(it), C.byref(trr),
                                C.byref(t))
        return u, dict(rc=rc, iters=it.value, true_rel_res=trr.value, solve_s=t.value)

    def coarse_matrix(self, node_group, centers, modes=6):
        """W^T K_ff W of the last assembly (dense, unshifted)."""
        ng_arr = np.ascontiguousarray(node_group, dtype=np.int32)
        cen = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, 3)
        nc = cen.shape[0] * modes
        E = np.zeros((nc, nc))
        rc = lib().hex8_cpu_coarse_matrix(self.handle, _p(ng_arr), int(cen.shape[0]), _p(cen), int(modes),
                                          _p(self.h), _p(E))
        if rc != 0:
            raise RuntimeError(f"hex8_cpu_coarse_matrix failed ({rc})")
        return E

    def dpcg(self, b, node_group, centers, modes=6, shift=1e-14, shift_relative=True, rtol=1e-8,
             max_iters=5000, stop_rule=0):
        """Deflated PCG of the last assembly; stop_rule 0: ||r|| < rtol ||b||, 1: the
        reference's sqrt(r.z / r0.z0) <= rtol."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        ng_arr = np.ascontiguousarray(node_group, dtype=np.int32)
        cen = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, 3)
        u = np.zeros_like(b)
        it, trr = C.c_int(0), C.c_double(0)
        times = np.zeros(2)
        rc = lib().hex8_cpu_dpcg(self.handle, _p(ng_arr), int(cen.shape[0]), _p(cen), int(modes), float(shift),
                                 1 if shift_relative else 0, _p(self.h), _p(b), _p(u), float(rtol), int(max_iters),
                                 int(stop_rule), C.byref(it), C.byref(trr), _p(times))
        return u, dict(rc=rc, iters=it.value, true_rel_res=trr.value, setup_s=float(times[0]),
                       solve_s=float(times[1]))
