"""Dipole inversion — mirrors the reference's ``inversion`` module (src/inversion/)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

from . import _lib
from . import Grid, Context, _ctx, _check, _as_f64, _as_u8, _ptr_d, _ptr_u8, _bdir, _progress, _check_len

IDENTITY, GRADIENT, LAPLACIAN = 0, 1, 2  # Regularization, src/inversion/tikhonov.rs:26-34


@dataclass
class TvParams:
    """src/inversion/tv.rs:23-43."""

    lambda_: float = 2e-4
    rho: float = 2e-2
    tol: float = 1e-3
    max_iter: int = 250

    def _c(self):
        return _lib.QsmTvParams(self.lambda_, self.rho, self.tol, int(self.max_iter))


@dataclass
class TkdParams:
    """src/inversion/tkd.rs:23-32."""

    threshold: float = 0.15

    def _c(self):
        return _lib.QsmTkdParams(self.threshold)


@dataclass
class TikhonovParams:
    """src/inversion/tikhonov.rs:38-49."""

    lambda_: float = 0.01
    reg: int = IDENTITY

    def _c(self):
        return _lib.QsmTikhonovParams(self.lambda_, int(self.reg))


@dataclass
class RtsParams:
    """src/inversion/rts.rs:22-51."""

    delta: float = 0.15
    mu: float = 1e5
    rho: float = 10.0
    tol: float = 1e-2
    max_iter: int = 20
    lsmr_iter: int = 4

    def _c(self):
        return _lib.QsmRtsParams(self.delta, self.mu, self.rho, self.tol, int(self.max_iter), int(self.lsmr_iter))


@dataclass
class NltvParams:
    """src/inversion/nltv.rs:24-48."""

    lambda_: float = 1e-3
    mu: float = 1.0
    tol: float = 1e-3
    max_iter: int = 250
    newton_iter: int = 10

    def _c(self):
        return _lib.QsmNltvParams(self.lambda_, self.mu, self.tol, int(self.max_iter), int(self.newton_iter))


@dataclass
class IlsqrParams:
    """src/inversion/ilsqr.rs:20-34."""

    tol: float = 0.01
    max_iter: int = 50

    def _c(self):
        return _lib.QsmIlsqrParams(self.tol, int(self.max_iter))


def _closed(fn_name, local_field, mask, grid: Grid, bdir, params, ctx):
    c = _ctx(ctx)
    f = _as_f64(local_field, grid, "local_field")
    m = _as_u8(mask, "mask")
    _check_len(f, grid, "local_field")
    _check_len(m, grid, "mask")
    out = np.empty_like(f)
    b, _keep = _bdir(bdir)
    g = grid._c()
    p = params._c()
    st = getattr(c._lib, fn_name)(c.handle, _ptr_d(f), _ptr_u8(m), C.byref(g), b, C.byref(p), _ptr_d(out))
    _check(c, st)
    return out


def tkd(local_field, mask, grid: Grid, bdir=(0.0, 0.0, 1.0), params: TkdParams = TkdParams(), *,
        ctx: Optional[Context] = None):
    """inversion::tkd (src/inversion/tkd.rs:48-99)."""
    return _closed("qsm_tkd", local_field, mask, grid, bdir, params, ctx)


def tsvd(local_field, mask, grid: Grid, bdir=(0.0, 0.0, 1.0), params: TkdParams = TkdParams(), *,
         ctx: Optional[Context] = None):
    """inversion::tsvd (src/inversion/tkd.rs:105-153)."""
    return _closed("qsm_tsvd", local_field, mask, grid, bdir, params, ctx)


def tikhonov(local_field, mask, grid: Grid, bdir=(0.0, 0.0, 1.0), params: TikhonovParams = TikhonovParams(), *,
             ctx: Optional[Context] = None):
    """inversion::tikhonov (src/inversion/tikhonov.rs:62-138)."""
    return _closed("qsm_tikhonov", local_field, mask, grid, bdir, params, ctx)


def tv_admm(local_field, mask, grid: Grid, bdir=(0.0, 0.0, 1.0), params: TvParams = TvParams(),
            progress: Optional[Callable[[int, int], None]] = None, *, ctx: Optional[Context] = None,
            out: Optional[np.ndarray] = None):
    """inversion::tv_admm (src/inversion/tv.rs:63-97).

    progress(iter, max_iter) is called once per iteration (delivered in batches between
    CUDA-graph launches) and (iters, iters) on convergence, as in the reference.
    `out` may supply the result buffer (e.g. page-locked host memory).
    """
    c = _ctx(ctx)
    f = _as_f64(local_field, grid, "local_field")
    m = _as_u8(mask, "mask")
    _check_len(f, grid, "local_field")
    _check_len(m, grid, "mask")
    if out is None:
        out = np.empty_like(f)
    elif out.dtype != np.float64 or not out.flags.c_contiguous or out.size != f.size:
        raise ValueError("out must be a contiguous float64 array with one value per voxel")
    b, _keep = _bdir(bdir)
    g = grid._c()
    p = params._c()
    cb, _cbkeep = _progress(progress)
    st = c._lib.qsm_tv_admm(c.handle, _ptr_d(f), _ptr_u8(m), C.byref(g), b, C.byref(p), cb, None, _ptr_d(out))
    _check(c, st)
    return out


def tv_admm_device(ctx: Context, d_local_field: int, d_mask: int, grid: Grid, bdir, params: TvParams,
                   d_out: int, progress=None):
    """Device-pointer variant (inputs/outputs already on ctx's GPU); pointers are ints."""
    b, _keep = _bdir(bdir)
    g = grid._c()
    p = params._c()
    cb, _cbkeep = _progress(progress)
    st = ctx._lib.qsm_tv_admm_device(ctx.handle, C.c_void_p(d_local_field), C.c_void_p(d_mask), C.byref(g), b,
                                     C.byref(p), cb, None, C.c_void_p(d_out))
    _check(ctx, st)


def tkd_device(ctx: Context, d_local_field: int, d_mask: int, grid: Grid, bdir, params: TkdParams, d_out: int):
    b, _keep = _bdir(bdir)
    g = grid._c()
    p = params._c()
    st = ctx._lib.qsm_tkd_device(ctx.handle, C.c_void_p(d_local_field), C.c_void_p(d_mask), C.byref(g), b,
                                 C.byref(p), C.c_void_p(d_out))
    _check(ctx, st)


def dipole_forward(chi, grid: Grid, bdir=(0.0, 0.0, 1.0), *, ctx: Optional[Context] = None):
    """Re IFFT(D * FFT(chi)) (src/fft.rs:214-233)."""
    c = _ctx(ctx)
    x = _as_f64(chi, grid, "chi")
    _check_len(x, grid, "chi")
    out = np.empty_like(x)
    b, _keep = _bdir(bdir)
    g = grid._c()
    _check(c, c._lib.qsm_dipole_forward(c.handle, _ptr_d(x), C.byref(g), b, _ptr_d(out)))
    return out


def dipole_forward_device(ctx: Context, d_chi: int, grid: Grid, bdir, d_out: int):
    """Device-pointer form of dipole_forward."""
    b, _keep = _bdir(bdir)
    g = grid._c()
    _check(ctx, ctx._lib.qsm_dipole_forward_device(ctx.handle, C.c_void_p(d_chi), C.byref(g), b, C.c_void_p(d_out)))


def ilsqr(local_field, mask, grid: Grid, bdir=(0.0, 0.0, 1.0), params: IlsqrParams = IlsqrParams(),
          progress: Optional[Callable[[int, int], None]] = None, *, ctx: Optional[Context] = None):
    """inversion::ilsqr (src/inversion/ilsqr.rs:1307-1351) -> (chi, xsa, xfs, xlsqr).

    progress(step, 4) is called before each of the three steps and after the last one.
    """
    c = _ctx(ctx)
    f = _as_f64(local_field, grid, "local_field")
    m = _as_u8(mask, "mask")
    _check_len(f, grid, "local_field")
    _check_len(m, grid, "mask")
    outs = [np.empty_like(f) for _ in range(4)]
    b, _keep = _bdir(bdir)
    g = grid._c()
    p = params._c()
    cb, _cbkeep = _progress(progress)
    st = c._lib.qsm_ilsqr(c.handle, _ptr_d(f), _ptr_u8(m), C.byref(g), b, C.byref(p), cb, None,
                          *[_ptr_d(o) for o in outs])
    _check(c, st)
    return tuple(outs)


def ilsqr_device(ctx: Context, d_local_field: int, d_mask: int, grid: Grid, bdir, params: IlsqrParams,
                 d_chi: int, d_xsa: int = 0, d_xfs: int = 0, d_xlsqr: int = 0, progress=None):
    """Device-pointer variant; the last three outputs are optional (0 = not wanted)."""
    b, _keep = _bdir(bdir)
    g = grid._c()
    p = params._c()
    cb, _cbkeep = _progress(progress)
    st = ctx._lib.qsm_ilsqr_device(ctx.handle, C.c_void_p(d_local_field), C.c_void_p(d_mask), C.byref(g), b,
                                   C.byref(p), cb, None, C.c_void_p(d_chi), C.c_void_p(d_xsa or None),
                                   C.c_void_p(d_xfs or None), C.c_void_p(d_xlsqr or None))
    _check(ctx, st)


def ilsqr_lsqr_operator_device(ctx: Context, grid: Grid, bdir, d_weights: int, d_x: int, d_y: int):
    """One application of iLSQR's LSQR operator y = D * FFT(w * Re IFFT(D * x))
    (src/inversion/ilsqr.rs:988-1010) on device complex128 vectors of nx*ny*nz values."""
    b, _keep = _bdir(bdir)
    g = grid._c()
    _check(ctx, ctx._lib.qsm_ilsqr_lsqr_operator_device(ctx.handle, C.byref(g), b, C.c_void_p(d_weights),
                                                         C.c_void_p(d_x), C.c_void_p(d_y)))


def prctile_device(ctx: Context, d_vals: int, d_mask: int, n: int, percents):
    """prctile (src/inversion/ilsqr.rs:937-946) of device values where mask != 0 (all when
    d_mask is 0), one result per percent."""
    p = np.ascontiguousarray(np.asarray(percents, dtype=np.float64))
    out = np.zeros_like(p)
    st = ctx._lib.qsm_prctile_device(ctx.handle, C.c_void_p(d_vals), C.c_void_p(d_mask or None), int(n), _ptr_d(p),
                                     p.size, _ptr_d(out))
    _check(ctx, st)
    return out


@dataclass
class TgvParams:
    """src/inversion/tgv.rs:39-76."""

    alpha1: float = 0.0005
    alpha0: float = 0.0015
    iterations: int = 1000
    erosions: int = 3
    step_size: float = 3.0
    fieldstrength: float = 3.0
    te: float = 0.020
    tol: float = 1e-5

    def _c(self):
        return _lib.QsmTgvParams(self.alpha1, self.alpha0, int(self.iterations), int(self.erosions), self.step_size,
                                 self.fieldstrength, self.te, self.tol)


def tgv_qsm(phase, mask, grid: Grid, params: TgvParams = TgvParams(), b0_dir=(0.0, 0.0, 1.0),
            progress: Optional[Callable[[int, int], None]] = None, *, ctx: Optional[Context] = None):
    """inversion::tgv_qsm (src/inversion/tgv.rs:1045-1299): chi (ppm) from wrapped phase.
    Parameters come before the field direction, as in the reference."""
    c = _ctx(ctx)
    f = _as_f64(phase, grid, "phase")
    m = _as_u8(mask, "mask")
    _check_len(f, grid, "phase")
    _check_len(m, grid, "mask")
    out = np.empty_like(f)
    b, _keep = _bdir(b0_dir)
    g = grid._c()
    p = params._c()
    cb, _cbkeep = _progress(progress)
    st = c._lib.qsm_tgv_qsm(c.handle, _ptr_d(f), _ptr_u8(m), C.byref(g), C.byref(p), b, cb, None, _ptr_d(out))
    _check(c, st)
    return out


def tgv_qsm_device(ctx: Context, d_phase: int, d_mask: int, grid: Grid, params: TgvParams, b0_dir, d_out: int,
                   progress=None):
    b, _keep = _bdir(b0_dir)
    g = grid._c()
    p = params._c()
    cb, _cbkeep = _progress(progress)
    st = ctx._lib.qsm_tgv_qsm_device(ctx.handle, C.c_void_p(d_phase), C.c_void_p(d_mask), C.byref(g), C.byref(p), b,
                                     cb, None, C.c_void_p(d_out))
    _check(ctx, st)


def tgv_oblique_stencil(res=(1.0, 1.0, 1.0), b0_dir=(0.0, 0.0, 1.0)):
    """compute_oblique_stencil (src/inversion/tgv.rs:272-479) -> float32 array st[di, dj, dk]."""
    from . import _lib as L
    lib = L.load()
    r = (C.c_double * 3)(*res)
    b = (C.c_double * 3)(*b0_dir)
    out = (C.c_float * 27)()
    if lib.qsm_tgv_oblique_stencil(r, b, out) != 0:
        raise RuntimeError("qsm_tgv_oblique_stencil failed")
    return np.frombuffer(out, dtype=np.float32).reshape(3, 3, 3).copy()


def tv_admm_batch(cases, params: TvParams = TvParams(), progress: Optional[Callable[[int, int], None]] = None, *,
                  ctx: Optional[Context] = None):
    """TV-ADMM over a batch of volumes in one call: cases is a sequence of
    (local_field, mask, grid, bdir).  Returns (list of chi arrays, list of iteration
    counts).  progress(k, n) counts finished volumes."""
    c = _ctx(ctx)
    keep, outs = [], []
    arr = (_lib.QsmVolume * max(len(cases), 1))()
    for b, (field, mask, grid, bdir) in enumerate(cases):
        f = _as_f64(field, grid, "local_field")
        m = _as_u8(mask, "mask")
        _check_len(f, grid, "local_field")
        _check_len(m, grid, "mask")
        o = np.empty_like(f)
        keep += [f, m]
        outs.append(o)
        arr[b].local_field = f.ctypes.data
        arr[b].mask = m.ctypes.data
        arr[b].out_chi = o.ctypes.data
        arr[b].grid = grid._c()
        arr[b].bdir = (C.c_double * 3)(*bdir)
    iters = (C.c_size_t * max(len(cases), 1))()
    p = params._c()
    cb, _cbkeep = _progress(progress)
    _check(c, c._lib.qsm_tv_admm_batch(c.handle, arr, len(cases), C.byref(p), cb, None, iters))
    return outs, [int(iters[b]) for b in range(len(cases))]


def tv_admm_batch_device(ctx: Context, cases, params: TvParams, progress=None):
    """Device form: cases is a sequence of (d_field, d_mask, d_out, grid, bdir) with
    device pointers as ints.  Returns the iteration counts."""
    arr = (_lib.QsmVolume * max(len(cases), 1))()
    for b, (df, dm, do, grid, bdir) in enumerate(cases):
        arr[b].local_field, arr[b].mask, arr[b].out_chi = df, dm, do
        arr[b].grid = grid._c()
        arr[b].bdir = (C.c_double * 3)(*bdir)
    iters = (C.c_size_t * max(len(cases), 1))()
    p = params._c()
    cb, _cbkeep = _progress(progress)
    _check(ctx, ctx._lib.qsm_tv_admm_batch_device(ctx.handle, arr, len(cases), C.byref(p), cb, None, iters))
    return [int(iters[b]) for b in range(len(cases))]


def tkd_batch_device(ctx: Context, cases, params: TkdParams):
    """TKD over a batch: cases as for tv_admm_batch_device."""
    arr = (_lib.QsmVolume * max(len(cases), 1))()
    for b, (df, dm, do, grid, bdir) in enumerate(cases):
        arr[b].local_field, arr[b].mask, arr[b].out_chi = df, dm, do
        arr[b].grid = grid._c()
        arr[b].bdir = (C.c_double * 3)(*bdir)
    p = params._c()
    _check(ctx, ctx._lib.qsm_tkd_batch_device(ctx.handle, arr, len(cases), C.byref(p)))


def tv_admm_unrolled_vjp_device(ctx: Context, d_local_field: int, d_mask: int, grid: Grid, bdir, lam: float,
                                rho: float, iterations: int, checkpoint_every: int, d_grad_chi: int, d_out_chi: int,
                                d_out_grad_field: int = 0):
    """Unrolled TV-ADMM forward (chi into d_out_chi) and, when d_grad_chi is non-zero, its
    vector-Jacobian product: dL/dfield into d_out_grad_field; returns dL/dlambda."""
    b, _keep = _bdir(bdir)
    g = grid._c()
    gl = C.c_double(0.0)
    _check(ctx, ctx._lib.qsm_tv_admm_unrolled_vjp_device(ctx.handle, C.c_void_p(d_local_field), C.c_void_p(d_mask),
                                                         C.byref(g), b, float(lam), float(rho), int(iterations),
                                                         int(checkpoint_every), C.c_void_p(d_grad_chi or None),
                                                         C.c_void_p(d_out_chi), C.c_void_p(d_out_grad_field or None),
                                                         C.byref(gl)))
    return gl.value


def rts(local_field, mask, grid: Grid, bdir=(0.0, 0.0, 1.0), params: RtsParams = RtsParams(),
        progress: Optional[Callable[[int, int], None]] = None, *, ctx: Optional[Context] = None):
    """inversion::rts (src/inversion/rts.rs:72-211)."""
    c = _ctx(ctx)
    f = _as_f64(local_field, grid, "local_field")
    m = _as_u8(mask, "mask")
    _check_len(f, grid, "local_field")
    _check_len(m, grid, "mask")
    out = np.empty_like(f)
    b, _keep = _bdir(bdir)
    g = grid._c()
    p = params._c()
    cb, _cbkeep = _progress(progress)
    _check(c, c._lib.qsm_rts(c.handle, _ptr_d(f), _ptr_u8(m), C.byref(g), b, C.byref(p), cb, None, _ptr_d(out)))
    return out


def nltv(local_field, mask, grid: Grid, bdir=(0.0, 0.0, 1.0), params: NltvParams = NltvParams(),
         progress: Optional[Callable[[int, int], None]] = None, *, ctx: Optional[Context] = None):
    """inversion::nltv (src/inversion/nltv.rs:62-131)."""
    c = _ctx(ctx)
    f = _as_f64(local_field, grid, "local_field")
    m = _as_u8(mask, "mask")
    _check_len(f, grid, "local_field")
    _check_len(m, grid, "mask")
    out = np.empty_like(f)
    b, _keep = _bdir(bdir)
    g = grid._c()
    p = params._c()
    cb, _cbkeep = _progress(progress)
    _check(c, c._lib.qsm_nltv(c.handle, _ptr_d(f), _ptr_u8(m), C.byref(g), b, C.byref(p), cb, None, _ptr_d(out)))
    return out
