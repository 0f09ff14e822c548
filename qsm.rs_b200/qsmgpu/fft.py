"""Transform primitives (src/fft.rs) exposed for parity testing of the GPU engine."""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import Grid, Context, _ctx, _check, _as_f64, _ptr_d, _check_len


def fft3d_real(x, grid: Grid, *, ctx: Optional[Context] = None) -> np.ndarray:
    """Full complex spectrum of a real volume (src/fft.rs:412, fft3d of real data)."""
    c = _ctx(ctx)
    a = _as_f64(x, grid, "x")
    _check_len(a, grid, "x")
    out = np.empty(2 * a.size, dtype=np.float64)
    g = grid._c()
    _check(c, c._lib.qsm_fft3d_real(c.handle, _ptr_d(a), C.byref(g), _ptr_d(out)))
    return (out[0::2] + 1j * out[1::2]).reshape(a.shape)
