"""qsmgpu — Python host mirror of QSM.rs's FFT-driven reconstruction API on the B200.

Every call goes through the C ABI of ``libqsmgpu.so`` (``include/qsmgpu.h``); the
names, argument order and defaults follow the reference crate (astewartau/QSM.rs):

    from qsmgpu import Grid, inversion, unwrap, bgremove, pipeline
    chi = inversion.tv_admm(local_field, mask, grid, (0, 0, 1), inversion.TvParams(), progress)

Volumes are numpy arrays in the reference's Fortran order: either flat of length
nx*ny*nz (index i + j*nx + k*nx*ny) or C-ordered arrays of shape (nz, ny, nx), which
have the same memory layout.  Results come back in the shape the input had.
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence, Tuple

import numpy as np

from . import _lib

__all__ = ["Grid", "Context", "QsmError", "DimensionMismatch", "InvalidConfig", "default_context",
           "inversion", "unwrap", "bgremove", "pipeline", "fft"]


class QsmError(RuntimeError):
    """A non-OK status returned by the C ABI."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{_lib.STATUS_NAMES.get(status, status)}: {message}")


class DimensionMismatch(QsmError):
    """PipelineError::DimensionMismatch (src/pipeline/config.rs:343-368)."""


class InvalidConfig(QsmError):
    """PipelineError::InvalidConfig (src/pipeline/config.rs:343-368)."""


@dataclass(frozen=True)
class Grid:
    """src/grid.rs:9-44 — dims (nx, ny, nz) and voxel size in mm."""

    dims: Tuple[int, int, int]
    voxel_size: Tuple[float, float, float] = (1.0, 1.0, 1.0)

    @staticmethod
    def new(nx, ny, nz, vsx=1.0, vsy=1.0, vsz=1.0) -> "Grid":
        return Grid((int(nx), int(ny), int(nz)), (float(vsx), float(vsy), float(vsz)))

    @property
    def nx(self):
        return self.dims[0]

    @property
    def ny(self):
        return self.dims[1]

    @property
    def nz(self):
        return self.dims[2]

    def n_total(self) -> int:
        return self.dims[0] * self.dims[1] * self.dims[2]

    @property
    def shape(self):
        return (self.dims[2], self.dims[1], self.dims[0])

    def _c(self):
        return _lib.QsmGrid(self.dims[0], self.dims[1], self.dims[2], *self.voxel_size)


def _check(ctx: "Context", status: int):
    if status == _lib.QSM_OK:
        return
    msg = ctx.last_error()
    if status == 2:
        raise DimensionMismatch(status, msg)
    if status == 6:
        raise InvalidConfig(status, msg)
    raise QsmError(status, msg)


class Context:
    """Owns a qsm_ctx: CUDA device, stream, precision and cached workspaces.

    precision: "f64" (the reference's arithmetic) or "mixed" (float FFTs/stencils with
    FP64 reductions and FP64 k-space multipliers).
    """

    def __init__(self, device: int = 0, precision: str = "f64"):
        self._lib = _lib.load()
        h = C.c_void_p()
        st = self._lib.qsm_ctx_create(int(device), _prec_code(precision), C.byref(h))
        if st != _lib.QSM_OK:
            raise QsmError(st, f"qsm_ctx_create(device={device}) failed")
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.qsm_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def precision(self) -> str:
        return "mixed" if self._lib.qsm_ctx_get_precision(self._h) == _lib.PRECISION_MIXED else "f64"

    @precision.setter
    def precision(self, p: str):
        _check(self, self._lib.qsm_ctx_set_precision(self._h, _prec_code(p)))

    @property
    def plan_mode(self) -> str:
        """"compiled" (compile-time pass kernels where a length has one) or "runtime"
        (the runtime Stockham engine for every pass)."""
        return "runtime" if self._lib.qsm_ctx_get_plan_mode(self._h) == _lib.PLANS_RUNTIME else "compiled"

    @plan_mode.setter
    def plan_mode(self, m: str):
        codes = {"compiled": _lib.PLANS_COMPILED, "runtime": _lib.PLANS_RUNTIME}
        if m not in codes:
            raise ValueError(f"plan mode must be one of {sorted(codes)}")
        _check(self, self._lib.qsm_ctx_set_plan_mode(self._h, codes[m]))

    @property
    def krylov_precision(self) -> str:
        """Arithmetic of iLSQR's LSQR/LSMR steps in a mixed context: "f64" (default) or
        "mixed" (float vectors and transforms, FP64 norms and recurrences)."""
        return "mixed" if self._lib.qsm_ctx_get_krylov_precision(self._h) == _lib.PRECISION_MIXED else "f64"

    @krylov_precision.setter
    def krylov_precision(self, p: str):
        _check(self, self._lib.qsm_ctx_set_krylov_precision(self._h, _prec_code(p)))

    def set_autotune(self, on: bool):
        """Autotuner of the compile-time Y/Z pass launch shapes (on by default); results
        do not depend on it."""
        _check(self, self._lib.qsm_ctx_set_autotune(self._h, 1 if on else 0))

    def force_launch_shape(self, shape: int):
        """Test hook: run every tunable pass in candidate shape 0..3, or -1 for the
        autotuner's choice."""
        _check(self, self._lib.qsm_ctx_force_launch_shape(self._h, int(shape)))

    def autotune_entries(self) -> dict:
        """Launch shapes the autotuner chose: {key: {"choice": c, "us": {candidate: us}}}."""
        out = {}
        for i in range(int(self._lib.qsm_ctx_autotune_count(self._h))):
            key = C.create_string_buffer(256)
            choice = C.c_int(0)
            cands = (C.c_int * 16)()
            us = (C.c_float * 16)()
            count = C.c_size_t(0)
            _check(self, self._lib.qsm_ctx_autotune_entry(self._h, i, key, 256, C.byref(choice), cands, us, 16,
                                                          C.byref(count)))
            n = min(int(count.value), 16)
            out[key.value.decode()] = {"choice": int(choice.value),
                                       "us": {int(cands[k]): round(float(us[k]), 2) for k in range(n)}}
        return out

    def set_input_check(self, on: bool):
        """Reject input volumes holding NaN or infinity (off by default, as in the reference)."""
        _check(self, self._lib.qsm_ctx_set_input_check(self._h, 1 if on else 0))

    def inject_alloc_failure(self, after: int):
        """Make the context's device allocation after `after` more successful ones fail
        with QSM_ERR_ALLOC (simulated on the host); negative cancels."""
        _check(self, self._lib.qsm_ctx_inject_alloc_failure(self._h, int(after)))

    def last_error(self) -> str:
        s = self._lib.qsm_last_error(self._h)
        return s.decode() if s else ""

    def kernel_launches(self) -> int:
        return int(self._lib.qsm_ctx_kernel_launches(self._h))

    def stream_handle(self) -> int:
        """The context's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        return int(self._lib.qsm_ctx_stream(self._h) or 0)

    def release_workspace(self):
        _check(self, self._lib.qsm_ctx_release_workspace(self._h))

    def tv_last_iterations(self) -> int:
        return int(self._lib.qsm_tv_last_iterations(self._h))

    def set_profiling(self, on: bool):
        """Bracket every kernel launch with CUDA events on the context's stream."""
        _check(self, self._lib.qsm_ctx_set_profiling(self._h, 1 if on else 0))

    def profile_reset(self):
        _check(self, self._lib.qsm_ctx_profile_reset(self._h))

    def profile(self) -> dict:
        """{kernel name: (launches, total_ms)} accumulated since the last reset."""
        out = {}
        n = int(self._lib.qsm_ctx_profile_count(self._h))
        buf = C.create_string_buffer(128)
        for i in range(n):
            cnt = C.c_uint64()
            ms = C.c_double()
            _check(self, self._lib.qsm_ctx_profile_entry(self._h, i, buf, 128, C.byref(cnt), C.byref(ms)))
            out[buf.value.decode()] = (int(cnt.value), float(ms.value))
        return out


def _prec_code(p: str) -> int:
    if p in ("f64", "fp64", "double"):
        return _lib.PRECISION_F64
    if p in ("mixed", "fp32", "f32"):
        return _lib.PRECISION_MIXED
    raise ValueError(f"unknown precision {p!r}")


_default = None
_default_lock = threading.Lock()


def default_context() -> Context:
    """Lazily created context on device 0 (f64)."""
    global _default
    with _default_lock:
        if _default is None:
            _default = Context(0, "f64")
        return _default


def _ctx(ctx: Optional[Context]) -> Context:
    return ctx if ctx is not None else default_context()


def _as_f64(a, grid: Grid, name: str):
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return arr


def _as_u8(a, name: str):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint8))


def _ptr_d(a: np.ndarray):
    return a.ctypes.data_as(_lib.c_double_p)


def _ptr_u8(a: np.ndarray):
    return a.ctypes.data_as(_lib.c_u8_p)


def _bdir(b):
    arr = (C.c_double * 3)(*[float(v) for v in b])
    return C.cast(arr, _lib.c_double_p), arr


def _progress(cb: Optional[Callable[[int, int], None]]):
    if cb is None:
        return _lib.PROGRESS_FN(), None

    def tramp(_user, cur, mx):
        cb(int(cur), int(mx))

    f = _lib.PROGRESS_FN(tramp)
    return f, f


def _check_len(arr: np.ndarray, grid: Grid, name: str):
    if arr.size != grid.n_total():
        # the reference's algorithm functions index out of bounds (panic) here
        raise ValueError(f"{name} has {arr.size} values, grid needs {grid.n_total()}")


from . import inversion, unwrap, bgremove, pipeline, fft, multi_echo, nifti  # noqa: E402
