"""Pipeline stage dispatchers — mirrors src/pipeline/{inversion,bg_removal,config}.rs."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Callable, Optional, Tuple

import numpy as np

from . import _lib
from . import Context, _ctx, _check, _ptr_d, _ptr_u8, _progress
from .inversion import IlsqrParams, NltvParams, RtsParams, TkdParams, TikhonovParams, TvParams
from .bgremove import IsmvParams, ResharpParams, SharpParams, VsharpParams

# InversionAlgorithm, src/pipeline/config.rs:47-58
TKD, TSVD, TIKHONOV, TV, RTS, NLTV, MEDI, ILSQR, TGV, QSMART = range(10)
# BgRemovalAlgorithm, src/pipeline/config.rs:33-42
VSHARP, PDF, LBV, ISMV, SHARP, RESHARP, HARPERELLA, IHARPERELLA = range(8)


@dataclass
class ScanMetadata:
    """src/pipeline/config.rs:302-324 (echo times are not used on this path)."""

    dims: Tuple[int, int, int]
    voxel_size: Tuple[float, float, float] = (1.0, 1.0, 1.0)
    echo_times: Tuple[float, ...] = ()
    field_strength: float = 3.0
    b0_direction: Tuple[float, float, float] = (0.0, 0.0, 1.0)

    def _c(self):
        b = (C.c_double * 3)(*self.b0_direction)
        return _lib.QsmScanMetadata(self.dims[0], self.dims[1], self.dims[2], *self.voxel_size,
                                    self.field_strength, b)


@dataclass
class InversionConfig:
    """src/pipeline/config.rs:234-264 (default algorithm Rts)."""

    algorithm: int = RTS
    tkd: TkdParams = field(default_factory=TkdParams)
    tsvd: TkdParams = field(default_factory=TkdParams)
    tikhonov: TikhonovParams = field(default_factory=TikhonovParams)
    tv: TvParams = field(default_factory=TvParams)
    ilsqr: IlsqrParams = field(default_factory=IlsqrParams)
    rts: RtsParams = field(default_factory=RtsParams)
    nltv: NltvParams = field(default_factory=NltvParams)

    def _c(self):
        return _lib.QsmInversionConfig(self.algorithm, self.tkd._c(), self.tsvd._c(), self.tikhonov._c(),
                                       self.tv._c(), self.ilsqr._c(), self.rts._c(), self.nltv._c())


@dataclass
class BgRemovalConfig:
    """src/pipeline/config.rs:204-230 (default algorithm Vsharp)."""

    algorithm: int = VSHARP
    vsharp: VsharpParams = field(default_factory=VsharpParams)
    sharp: SharpParams = field(default_factory=SharpParams)
    resharp: ResharpParams = field(default_factory=ResharpParams)
    ismv: IsmvParams = field(default_factory=IsmvParams)

    def _c(self):
        return _lib.QsmBgRemovalConfig(self.algorithm, self.vsharp._c(), self.sharp._c(), self.resharp._c(),
                                       self.ismv._c())


@dataclass
class BgRemovalResult:
    """src/pipeline/config.rs:335-340."""

    local_field_ppm: np.ndarray
    eroded_mask: np.ndarray


def run_dipole_inversion(local_field_ppm, mask, metadata: ScanMetadata, config: InversionConfig,
                         magnitude=None, progress: Optional[Callable[[int, int], None]] = None, *,
                         ctx: Optional[Context] = None):
    """pipeline::run_dipole_inversion (src/pipeline/inversion.rs:28-114)."""
    c = _ctx(ctx)
    f = np.ascontiguousarray(np.asarray(local_field_ppm, dtype=np.float64)).ravel()
    n = metadata.dims[0] * metadata.dims[1] * metadata.dims[2]
    m = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8)).ravel()
    if m.size != n and f.size == n:
        raise ValueError(f"mask has {m.size} values, expected {n}")
    out = np.empty(max(f.size, 1), dtype=np.float64)
    md = metadata._c()
    cfg = config._c()
    cb, _keep = _progress(progress)
    st = c._lib.qsm_run_dipole_inversion(c.handle, _ptr_d(f), f.size, _ptr_u8(m), C.byref(md), C.byref(cfg), cb,
                                         None, _ptr_d(out))
    _check(c, st)
    return out


def run_bg_removal(field_ppm, mask, metadata: ScanMetadata, config: BgRemovalConfig,
                   progress: Optional[Callable[[int, int], None]] = None, *, ctx: Optional[Context] = None):
    """pipeline::run_bg_removal (src/pipeline/bg_removal.rs:20-92)."""
    c = _ctx(ctx)
    f = np.ascontiguousarray(np.asarray(field_ppm, dtype=np.float64)).ravel()
    n = metadata.dims[0] * metadata.dims[1] * metadata.dims[2]
    m = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8)).ravel()
    if m.size != n and f.size == n:
        raise ValueError(f"mask has {m.size} values, expected {n}")
    out = np.empty(max(f.size, 1), dtype=np.float64)
    om = np.empty(max(f.size, 1), dtype=np.uint8)
    md = metadata._c()
    cfg = config._c()
    cb, _keep = _progress(progress)
    st = c._lib.qsm_run_bg_removal(c.handle, _ptr_d(f), f.size, _ptr_u8(m), C.byref(md), C.byref(cfg), cb, None,
                                   _ptr_d(out), _ptr_u8(om))
    _check(c, st)
    return BgRemovalResult(out, om)


REFERENCE_MEAN, REFERENCE_NONE = 0, 1  # QsmReference, src/pipeline/config.rs:69-72


def apply_reference(chi, mask, method: int = REFERENCE_MEAN, *, ctx: Optional[Context] = None):
    """pipeline::referencing::apply_reference (src/pipeline/referencing.rs:12-43)."""
    c = _ctx(ctx)
    x = np.ascontiguousarray(np.asarray(chi, dtype=np.float64)).ravel()
    m = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8)).ravel()
    if m.size != x.size:
        raise ValueError("mask and chi lengths differ")
    out = np.empty_like(x)
    _check(c, c._lib.qsm_apply_reference(c.handle, _ptr_d(x), _ptr_u8(m), x.size, int(method), _ptr_d(out)))
    return out


def run_tgv(phases, mask, metadata: ScanMetadata, tgv_params, reference: int = REFERENCE_MEAN,
            progress: Optional[Callable[[int, int], None]] = None, *, ctx: Optional[Context] = None):
    """pipeline::run_tgv (src/pipeline/inversion.rs:124-157), single echo."""
    c = _ctx(ctx)
    ph = [np.ascontiguousarray(np.asarray(p, dtype=np.float64)).ravel() for p in phases]
    m = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8)).ravel()
    n = metadata.dims[0] * metadata.dims[1] * metadata.dims[2]
    if m.size != n:
        raise ValueError(f"mask has {m.size} values, expected {n}")
    arr = (_lib.c_double_p * max(len(ph), 1))(*[_ptr_d(p) for p in ph])
    out = np.empty(n, dtype=np.float64)
    md = metadata._c()
    p = tgv_params._c()
    cb, _keep = _progress(progress)
    st = c._lib.qsm_run_tgv(c.handle, arr, len(ph), ph[0].size if ph else 0, _ptr_u8(m), C.byref(md), C.byref(p),
                            int(reference), cb, None, _ptr_d(out))
    _check(c, st)
    return out
