"""Background field removal — mirrors the reference's ``bgremove`` module (src/bgremove/)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Callable, Optional, Sequence

import numpy as np

from . import _lib
from . import Grid, Context, _ctx, _check, _as_f64, _as_u8, _ptr_d, _ptr_u8, _progress, _check_len


@dataclass
class SharpParams:
    """src/bgremove/sharp.rs:22-37."""

    threshold: float = 0.05
    radius: float = 6.0

    def _c(self):
        return _lib.QsmSharpParams(self.threshold, self.radius)


@dataclass
class ResharpParams:
    """src/bgremove/resharp.rs:22-45."""

    radius: float = 6.0
    tik_reg: float = 1e-4
    tol: float = 1e-6
    max_iter: int = 30

    def _c(self):
        return _lib.QsmResharpParams(self.radius, self.tik_reg, self.tol, int(self.max_iter))


@dataclass
class IsmvParams:
    """src/bgremove/ismv.rs:19-35."""

    tol: float = 1e-6
    max_iter: int = 50
    radius: float = 5.0

    def _c(self):
        return _lib.QsmIsmvParams(self.tol, int(self.max_iter), self.radius)


@dataclass
class VsharpParams:
    """src/bgremove/vsharp.rs:22-40."""

    threshold: float = 0.05
    max_radius: float = 12.0
    min_radius: float = 1.0

    def _c(self):
        return _lib.QsmVsharpParams(self.threshold, self.max_radius, self.min_radius)


def _io(field, mask, grid):
    f = _as_f64(field, grid, "field")
    m = _as_u8(mask, "mask")
    _check_len(f, grid, "field")
    _check_len(m, grid, "mask")
    return f, m, np.empty_like(f), np.empty_like(m)


def smv(field, mask, grid: Grid, radius: float, *, ctx: Optional[Context] = None):
    """bgremove::smv (src/bgremove/smv.rs:31-59) -> (local_field, eroded_mask)."""
    c = _ctx(ctx)
    f, m, out, om = _io(field, mask, grid)
    g = grid._c()
    _check(c, c._lib.qsm_smv(c.handle, _ptr_d(f), _ptr_u8(m), C.byref(g), float(radius), _ptr_d(out), _ptr_u8(om)))
    return out, om


def sharp(field, mask, grid: Grid, params: SharpParams = SharpParams(), *, ctx: Optional[Context] = None):
    """bgremove::sharp (src/bgremove/sharp.rs:51-131) -> (local_field, eroded_mask)."""
    c = _ctx(ctx)
    f, m, out, om = _io(field, mask, grid)
    g = grid._c()
    p = params._c()
    _check(c, c._lib.qsm_sharp(c.handle, _ptr_d(f), _ptr_u8(m), C.byref(g), C.byref(p), _ptr_d(out), _ptr_u8(om)))
    return out, om


def vsharp(field, mask, grid: Grid, params: VsharpParams = VsharpParams(),
           progress: Optional[Callable[[int, int], None]] = None, *, ctx: Optional[Context] = None):
    """bgremove::vsharp (src/bgremove/vsharp.rs:55-63) -> (local_field, final_mask)."""
    c = _ctx(ctx)
    f, m, out, om = _io(field, mask, grid)
    g = grid._c()
    p = params._c()
    cb, _keep = _progress(progress)
    _check(c, c._lib.qsm_vsharp(c.handle, _ptr_d(f), _ptr_u8(m), C.byref(g), C.byref(p), cb, None, _ptr_d(out),
                                _ptr_u8(om)))
    return out, om


def vsharp_with_radii(field, mask, grid: Grid, radii: Sequence[float], threshold: float,
                      progress: Optional[Callable[[int, int], None]] = None, *, ctx: Optional[Context] = None):
    """bgremove::vsharp_with_radii (src/bgremove/vsharp.rs:88-199)."""
    c = _ctx(ctx)
    f, m, out, om = _io(field, mask, grid)
    g = grid._c()
    r = np.ascontiguousarray(np.asarray(list(radii), dtype=np.float64))
    cb, _keep = _progress(progress)
    _check(c, c._lib.qsm_vsharp_with_radii(c.handle, _ptr_d(f), _ptr_u8(m), C.byref(g), _ptr_d(r), r.size,
                                           float(threshold), cb, None, _ptr_d(out), _ptr_u8(om)))
    return out, om


def resharp(field, mask, grid: Grid, params: ResharpParams = ResharpParams(),
            progress: Optional[Callable[[int, int], None]] = None, *, ctx: Optional[Context] = None):
    """bgremove::resharp (src/bgremove/resharp.rs:58-125) -> (local_field, eroded_mask)."""
    c = _ctx(ctx)
    f, m, out, om = _io(field, mask, grid)
    g = grid._c()
    p = params._c()
    cb, _keep = _progress(progress)
    _check(c, c._lib.qsm_resharp(c.handle, _ptr_d(f), _ptr_u8(m), C.byref(g), C.byref(p), cb, None, _ptr_d(out),
                                 _ptr_u8(om)))
    return out, om


def ismv(field, mask, grid: Grid, params: IsmvParams = IsmvParams(),
         progress: Optional[Callable[[int, int], None]] = None, *, ctx: Optional[Context] = None):
    """bgremove::ismv (src/bgremove/ismv.rs:48-166) -> (local_field, eroded_mask)."""
    c = _ctx(ctx)
    f, m, out, om = _io(field, mask, grid)
    g = grid._c()
    p = params._c()
    cb, _keep = _progress(progress)
    _check(c, c._lib.qsm_ismv(c.handle, _ptr_d(f), _ptr_u8(m), C.byref(g), C.byref(p), cb, None, _ptr_d(out),
                              _ptr_u8(om)))
    return out, om


def cg_kspace_normal_device(ctx: Context, grid: Grid, d_kernel_spectrum: int, d_weight: int, lam: float, d_b: int,
                            d_x0: int, tol: float, max_iter: int, d_x: int, progress=None):
    """solvers::cg_solve_with_progress (src/solvers/cg.rs:34-101) for
    A x = Re IFFT(K FFT(w Re IFFT(K FFT(x)))) + lam x; device pointers as ints (0 = NULL)."""
    g = grid._c()
    cb, _keep = _progress(progress)
    _check(ctx, ctx._lib.qsm_cg_kspace_normal_device(ctx.handle, C.byref(g), C.c_void_p(d_kernel_spectrum),
                                                     C.c_void_p(d_weight or None), float(lam), C.c_void_p(d_b),
                                                     C.c_void_p(d_x0 or None), float(tol), int(max_iter), cb, None,
                                                     C.c_void_p(d_x)))


def vsharp_radii(params: VsharpParams = VsharpParams()):
    """Descending radii max, max - min, ... while >= min (src/bgremove/vsharp.rs:70-82)."""
    radii, r = [], params.max_radius
    while r >= params.min_radius:
        radii.append(r)
        r -= params.min_radius
    return radii or [params.max_radius]


def vsharp_with_radii_device(ctx: Context, d_field: int, d_mask: int, grid: Grid, radii: Sequence[float],
                             threshold: float, d_out_local: int, d_out_mask: int, progress=None):
    """Device-pointer form of vsharp_with_radii (src/bgremove/vsharp.rs:88-199)."""
    r = np.ascontiguousarray(np.asarray(radii, dtype=np.float64))
    g = grid._c()
    cb, _keep = _progress(progress)
    _check(ctx, ctx._lib.qsm_vsharp_with_radii_device(ctx.handle, C.c_void_p(d_field), C.c_void_p(d_mask), C.byref(g),
                                                      _ptr_d(r), r.size, float(threshold), cb, None,
                                                      C.c_void_p(d_out_local), C.c_void_p(d_out_mask)))
