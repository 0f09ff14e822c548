"""NIfTI-1 I/O — mirrors the reference's ``io`` module (src/io.rs:62-460).

Volumes are flat float64 arrays with x fastest (index x + y*nx + z*nx*ny), as the
reference returns them; ``reshape(nz, ny, nx)`` gives the (z, y, x) arrays the rest of
this package takes.  The host functions need no GPU; ``load_nifti_device`` and
``save_nifti_device`` move the voxels between the file image and device memory,
decoding or encoding them on the GPU.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _lib
from . import Context, QsmError, DimensionMismatch, _ctx, _check, _ptr_d

_ERR_CAP = 1024


@dataclass
class NiftiData:
    """io::NiftiData (src/io.rs:13-27)."""

    data: np.ndarray
    dims: Tuple[int, int, int]
    voxel_size: Tuple[float, float, float]
    affine: np.ndarray  # 16 values, row-major 4x4
    scl_slope: float
    scl_inter: float


def _raise(status: int, err):
    msg = err.value.decode(errors="replace")
    if status == 2:
        raise DimensionMismatch(status, msg)
    raise QsmError(status, msg)


def _bytes_arg(b):
    buf = np.frombuffer(bytes(b), np.uint8) if not isinstance(b, np.ndarray) else np.ascontiguousarray(b, np.uint8)
    return buf, buf.ctypes.data_as(_lib.c_u8_p), buf.size


def parse_header(b) -> "_lib.QsmNiftiHeader":
    lib = _lib.load()
    buf, p, n = _bytes_arg(b)
    h = _lib.QsmNiftiHeader()
    err = C.create_string_buffer(_ERR_CAP)
    s = lib.qsm_nifti_parse_header(p, n, C.byref(h), err, _ERR_CAP)
    if s != 0:
        _raise(s, err)
    return h


def _load(b, all_volumes: bool):
    lib = _lib.load()
    buf, p, n = _bytes_arg(b)
    h = parse_header(buf)
    count = h.nx * h.ny * h.nz * (h.nt if all_volumes else 1)
    out = np.empty(count)
    err = C.create_string_buffer(_ERR_CAP)
    s = lib.qsm_nifti_load(p, n, 1 if all_volumes else 0, _ptr_d(out), count, C.byref(h), err, _ERR_CAP)
    if s != 0:
        _raise(s, err)
    return out, h


def _data(out, h) -> NiftiData:
    return NiftiData(out, (h.nx, h.ny, h.nz), tuple(h.voxel_size), np.array(h.affine[:]), h.scl_slope, h.scl_inter)


def load_nifti(b) -> NiftiData:
    """io::load_nifti (src/io.rs:62-158): .nii or .nii.gz bytes; the first volume of 4D data."""
    out, h = _load(b, False)
    return _data(out, h)


def load_nifti_4d(b):
    """io::load_nifti_4d (src/io.rs:161-224) -> (data, (nx, ny, nz, nt), voxel_size, affine)."""
    out, h = _load(b, True)
    return out, (h.nx, h.ny, h.nz, h.nt), tuple(h.voxel_size), np.array(h.affine[:])


def _save(data, dims, voxel_size, affine, gz: bool) -> bytes:
    lib = _lib.load()
    d = np.ascontiguousarray(np.asarray(data, np.float64).ravel())
    vs = np.ascontiguousarray(np.asarray(voxel_size, np.float64))
    af = np.ascontiguousarray(np.asarray(affine, np.float64).ravel())
    nx, ny, nz = (int(v) for v in dims)
    if d.size != nx * ny * nz or vs.size != 3 or af.size != 16:
        raise ValueError("data, dims, voxel_size and affine disagree")
    need = C.c_size_t(0)
    err = C.create_string_buffer(_ERR_CAP)
    s = lib.qsm_nifti_save(_ptr_d(d), nx, ny, nz, _ptr_d(vs), _ptr_d(af), 1 if gz else 0, None, 0, C.byref(need),
                           err, _ERR_CAP)
    if s != 0:
        _raise(s, err)
    out = np.empty(need.value, np.uint8)
    got = C.c_size_t(0)
    s = lib.qsm_nifti_save(_ptr_d(d), nx, ny, nz, _ptr_d(vs), _ptr_d(af), 1 if gz else 0,
                           out.ctypes.data_as(_lib.c_u8_p), out.size, C.byref(got), err, _ERR_CAP)
    if s != 0:
        _raise(s, err)
    return out[:got.value].tobytes()


def save_nifti(data, dims, voxel_size, affine) -> bytes:
    """io::save_nifti (src/io.rs:255-338): uncompressed .nii bytes, float32 voxels."""
    return _save(data, dims, voxel_size, affine, False)


def save_nifti_gz(data, dims, voxel_size, affine) -> bytes:
    """io::save_nifti_gz (src/io.rs:340-364)."""
    return _save(data, dims, voxel_size, affine, True)


def read_nifti_dims(path) -> Tuple[int, int, int]:
    """io::read_nifti_dims (src/io.rs:366-421)."""
    lib = _lib.load()
    dims = (C.c_size_t * 3)()
    err = C.create_string_buffer(_ERR_CAP)
    s = lib.qsm_nifti_read_dims(os.fsencode(path), dims, err, _ERR_CAP)
    if s != 0:
        _raise(s, err)
    return (dims[0], dims[1], dims[2])


def read_nifti_file(path) -> NiftiData:
    """io::read_nifti_file (src/io.rs:424-431)."""
    lib = _lib.load()
    h = _lib.QsmNiftiHeader()
    err = C.create_string_buffer(_ERR_CAP)
    s = lib.qsm_nifti_read_file_header(os.fsencode(path), C.byref(h), err, _ERR_CAP)
    if s != 0:
        _raise(s, err)
    count = h.nx * h.ny * h.nz
    out = np.empty(count)
    s = lib.qsm_nifti_read_file(os.fsencode(path), 0, _ptr_d(out), count, C.byref(h), err, _ERR_CAP)
    if s != 0:
        _raise(s, err)
    return _data(out, h)


def save_nifti_to_file(path, data, dims, voxel_size, affine):
    """io::save_nifti_to_file (src/io.rs:434-452): gzip when the path ends in .nii.gz."""
    lib = _lib.load()
    d = np.ascontiguousarray(np.asarray(data, np.float64).ravel())
    vs = np.ascontiguousarray(np.asarray(voxel_size, np.float64))
    af = np.ascontiguousarray(np.asarray(affine, np.float64).ravel())
    nx, ny, nz = (int(v) for v in dims)
    if d.size != nx * ny * nz:
        raise ValueError("data and dims disagree")
    err = C.create_string_buffer(_ERR_CAP)
    s = lib.qsm_nifti_save_file(os.fsencode(path), _ptr_d(d), nx, ny, nz, _ptr_d(vs), _ptr_d(af), err, _ERR_CAP)
    if s != 0:
        _raise(s, err)


def load_nifti_device(b, d_out: int, out_len: int, all_volumes: bool = False, *, ctx: Optional[Context] = None):
    """Decode into device memory at d_out (an int pointer to out_len doubles); returns the header."""
    c = _ctx(ctx)
    buf, p, n = _bytes_arg(b)
    h = _lib.QsmNiftiHeader()
    _check(c, c._lib.qsm_nifti_load_device(c.handle, p, n, 1 if all_volumes else 0, C.c_void_p(d_out), int(out_len),
                                           C.byref(h)))
    return h


def save_nifti_device(d_data: int, dims, voxel_size, affine, gz: bool = False, *,
                      ctx: Optional[Context] = None) -> bytes:
    """save_nifti / save_nifti_gz of device data at d_data (float32 rounding on the GPU)."""
    c = _ctx(ctx)
    vs = np.ascontiguousarray(np.asarray(voxel_size, np.float64))
    af = np.ascontiguousarray(np.asarray(affine, np.float64).ravel())
    nx, ny, nz = (int(v) for v in dims)
    need = C.c_size_t(0)
    _check(c, c._lib.qsm_nifti_save_device(c.handle, C.c_void_p(d_data), nx, ny, nz, _ptr_d(vs), _ptr_d(af),
                                           1 if gz else 0, None, 0, C.byref(need)))
    out = np.empty(need.value, np.uint8)
    got = C.c_size_t(0)
    _check(c, c._lib.qsm_nifti_save_device(c.handle, C.c_void_p(d_data), nx, ny, nz, _ptr_d(vs), _ptr_d(af),
                                           1 if gz else 0, out.ctypes.data_as(_lib.c_u8_p), out.size,
                                           C.byref(got)))
    return out[:got.value].tobytes()
