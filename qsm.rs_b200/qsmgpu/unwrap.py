"""Phase unwrapping — mirrors the reference's ``unwrap`` module (src/unwrap/laplacian.rs)."""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import Grid, Context, _ctx, _check, _as_f64, _as_u8, _ptr_d, _ptr_u8, _check_len


def laplacian_unwrap(phase, mask, grid: Grid, *, ctx: Optional[Context] = None):
    """unwrap::laplacian_unwrap (src/unwrap/laplacian.rs:135-161)."""
    c = _ctx(ctx)
    ph = _as_f64(phase, grid, "phase")
    m = _as_u8(mask, "mask")
    _check_len(ph, grid, "phase")
    _check_len(m, grid, "mask")
    out = np.empty_like(ph)
    g = grid._c()
    _check(c, c._lib.qsm_laplacian_unwrap(c.handle, _ptr_d(ph), _ptr_u8(m), C.byref(g), _ptr_d(out)))
    return out


def laplacian_unwrap_device(ctx: Context, d_phase: int, d_mask: int, grid: Grid, d_out: int):
    g = grid._c()
    _check(ctx, ctx._lib.qsm_laplacian_unwrap_device(ctx.handle, C.c_void_p(d_phase), C.c_void_p(d_mask),
                                                     C.byref(g), C.c_void_p(d_out)))
