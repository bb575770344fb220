"""Autotuner of the matrix-free operator's tile shape, per grid.

The matvec kernel has four tile variants (CTA of 32 x TY threads marching up z,
TY in {4, 8, 16}, with 1 to 3 CTAs per SM) and three or four chunk-staged ones
(variants 8-11: node-plane rows copied as 16-byte chunks, faces and pending
accumulators in registers); the FP32 operator has two more that run the element
contraction on the tensor cores.  Which is fastest depends on the grid
(how the (nx+1) x (ny+1) node columns divide into tiles, and the z-slab count).
``autotune(grid)`` times every variant with CUDA events on the grid itself, FP64
and FP32, and stores the choice in the grid's operator (``op.tune``), which every
launch on that grid then uses.  Choices are cached per grid shape.
"""
from __future__ import annotations

import torch

from . import _capi as A

_CACHE: dict = {}
VARIANTS = (0, 1, 2, 3, 8, 9, 10)  # 8-10: chunk-staged planes, faces and accumulators in registers
VARIANTS_F32 = (0, 1, 2, 3, 4, 5, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19)  # 4, 5: tensor-core contraction
# (BF16 split); 12-14: chunk-staged with two element rows per thread; 15-17: the same
# with the two rows as packed FP32x2 lanes


def _time(fn, reps):
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(2):
        fn()
    e0.record(st)
    for _ in range(reps):
        fn()
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def autotune(grid, reps=10, precisions=("f64", "f32"), use_cache=True):
    """Pick the fastest tile variant of K(s)u for this grid; returns
    {precision: (variant, {variant: ms})} and sets grid.op.tune."""
    key = (grid.nel, grid.h)
    if use_cache and key in _CACHE:
        grid.op.tune = _CACHE[key][0]
        return _CACHE[key][1]
    g = torch.Generator(device=grid.device).manual_seed(0)
    s = torch.rand(grid.nelem, dtype=torch.float64, device=grid.device, generator=g) + 0.01
    u = torch.randn(grid.ndof, dtype=torch.float64, device=grid.device, generator=g)
    y = torch.empty_like(u)
    out, tune = {}, 0
    saved = grid.op.tune
    for prec in precisions:
        times = {}
        for v in (VARIANTS if prec == "f64" else VARIANTS_F32):
            if prec == "f64":
                grid.op.tune = (saved & ~0xFF) | (v + 1)
                times[v] = _time(lambda: grid.matvec(s, u, out=y), reps)
            else:
                grid.op.tune = (saved & ~0xFF00) | ((v + 1) << 8)
                s32, u32 = s.float(), u.float()
                y32 = torch.empty_like(u32)
                times[v] = _time(lambda: grid.matvec_f32(s32, u32, out=y32), reps)
        best = min(times, key=times.get)
        out[prec] = (best, times)
        tune |= (best + 1) if prec == "f64" else ((best + 1) << 8)
    grid.op.tune = tune
    _CACHE[key] = (tune, out)
    return out
