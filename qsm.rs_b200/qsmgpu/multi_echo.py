"""Multi-echo field mapping — mirrors the reference's ``utils::multi_echo`` fits
(src/utils/multi_echo.rs:450-804) on the GPU."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from . import Context, _ctx, _check, _ptr_d, _ptr_u8

# B0WeightType, src/utils/multi_echo.rs:78-91
PHASE_SNR, PHASE_VAR, AVERAGE, TES, MAG = range(5)

_WEIGHT_NAMES = {"phase_snr": PHASE_SNR, "phasesnr": PHASE_SNR, "phase_var": PHASE_VAR, "phasevar": PHASE_VAR,
                 "average": AVERAGE, "uniform": AVERAGE, "tes": TES, "te": TES, "mag": MAG, "magnitude": MAG}


def b0_weight_type_from_str(s: str) -> int:
    """B0WeightType::from_str (src/utils/multi_echo.rs:93-104): unknown names -> PhaseSNR."""
    return _WEIGHT_NAMES.get(s.lower(), PHASE_SNR)


@dataclass
class LinearFitParams:
    """src/utils/multi_echo.rs:33-48."""

    estimate_offset: bool = True
    reliability_threshold_percentile: float = 90.0

    def _c(self):
        return _lib.QsmLinearFitParams(1 if self.estimate_offset else 0, self.reliability_threshold_percentile)


@dataclass
class LinearFitResult:
    """src/utils/multi_echo.rs:603-613."""

    field: np.ndarray
    phase_offset: np.ndarray
    fit_residual: np.ndarray
    reliability_mask: np.ndarray


def _stack(volumes, name):
    arr = np.ascontiguousarray(np.stack([np.asarray(v, np.float64).ravel() for v in volumes]))
    return arr


def _inputs(unwrapped_phases, mags, tes, mask):
    ph = _stack(unwrapped_phases, "unwrapped_phases")
    mg = _stack(mags, "mags")
    t = np.ascontiguousarray(np.asarray(tes, np.float64).ravel())
    m = np.ascontiguousarray(np.asarray(mask, np.uint8).ravel())
    ne, n = ph.shape
    if mg.shape != ph.shape or t.size != ne or m.size != n:
        # the reference indexes out of bounds (panics) on mismatched inputs
        raise ValueError(f"inputs disagree: phases {ph.shape}, mags {mg.shape}, tes {t.size}, mask {m.size}")
    return ph, mg, t, m, ne, n


def calculate_b0_weighted(unwrapped_phases: Sequence, mags: Sequence, tes: Sequence[float], mask,
                          weight_type: int = PHASE_SNR, *, ctx: Optional[Context] = None) -> np.ndarray:
    """utils::multi_echo::calculate_b0_weighted (src/utils/multi_echo.rs:450-506): B0 in Hz."""
    c = _ctx(ctx)
    ph, mg, t, m, ne, n = _inputs(unwrapped_phases, mags, tes, mask)
    out = np.empty(n)
    _check(c, c._lib.qsm_calculate_b0_weighted(c.handle, _ptr_d(ph), _ptr_d(mg), _ptr_d(t), ne, _ptr_u8(m), n,
                                               int(weight_type), _ptr_d(out)))
    return out


def multi_echo_linear_fit(unwrapped_phases: Sequence, mags: Sequence, tes: Sequence[float], mask,
                          estimate_offset: bool = True, reliability_threshold_percentile: float = 90.0, *,
                          ctx: Optional[Context] = None) -> LinearFitResult:
    """utils::multi_echo::multi_echo_linear_fit (src/utils/multi_echo.rs:631-768)."""
    c = _ctx(ctx)
    ph, mg, t, m, ne, n = _inputs(unwrapped_phases, mags, tes, mask)
    p = LinearFitParams(estimate_offset, reliability_threshold_percentile)._c()
    f, o, r = np.empty(n), np.empty(n), np.empty(n)
    rm = np.empty(n, np.uint8)
    _check(c, c._lib.qsm_multi_echo_linear_fit(c.handle, _ptr_d(ph), _ptr_d(mg), _ptr_d(t), ne, _ptr_u8(m), n,
                                               C.byref(p), _ptr_d(f), _ptr_d(o), _ptr_d(r), _ptr_u8(rm)))
    return LinearFitResult(f, o, r, rm)


def multi_echo_linear_fit_device(ctx: Context, d_phases: int, d_mags: int, tes: Sequence[float], n_echoes: int,
                                 d_mask: int, n: int, params: LinearFitParams, d_field: int, d_offset: int,
                                 d_residual: int, d_reliability: int):
    """Device-pointer form (ints); phases/mags echo-major, n values per echo."""
    t = np.ascontiguousarray(np.asarray(tes, np.float64).ravel())
    p = params._c()
    _check(ctx, ctx._lib.qsm_multi_echo_linear_fit_device(
        ctx.handle, C.c_void_p(d_phases), C.c_void_p(d_mags), _ptr_d(t), int(n_echoes), C.c_void_p(d_mask), int(n),
        C.byref(p), C.c_void_p(d_field), C.c_void_p(d_offset), C.c_void_p(d_residual), C.c_void_p(d_reliability)))


def calculate_b0_weighted_device(ctx: Context, d_phases: int, d_mags: int, tes: Sequence[float], n_echoes: int,
                                 d_mask: int, n: int, weight_type: int, d_out: int):
    t = np.ascontiguousarray(np.asarray(tes, np.float64).ravel())
    _check(ctx, ctx._lib.qsm_calculate_b0_weighted_device(ctx.handle, C.c_void_p(d_phases), C.c_void_p(d_mags),
                                                          _ptr_d(t), int(n_echoes), C.c_void_p(d_mask), int(n),
                                                          int(weight_type), C.c_void_p(d_out)))

