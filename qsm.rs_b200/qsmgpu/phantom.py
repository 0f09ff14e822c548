"""Seeded synthetic phantoms with the shapes and value ranges of the benchmark cases.

No public dataset is used: the reference's own integration data (a private BIDS
bundle) is not available, so every input here is generated from a seed.

* ``tv_case_64``   — 64^3 at 1 mm, B0 = z: 12 random ellipsoids (semi-axes 3-12 voxels,
  chi ~ U[-0.1, 0.2] ppm) in a sphere mask of radius 28; local field =
  Re IFFT(D * FFT(chi)) + N(0, 0.01) ppm inside the mask.
* ``brain_tv_case`` — 256 x 256 x 176 at 1 mm, B0 = z: 12 ellipsoids inside a
  100 x 120 x 75-voxel ellipsoid brain mask; local field = dipole-convolved chi +
  N(0, 0.01) ppm inside the mask (the TV-ADMM throughput case).
* ``chain_case``   — 256 x 256 x 176 at 1 mm, 3 T, TE 20 ms: ellipsoid brain mask with
  semi-axes 100 x 120 x 75 voxels, ellipsoid chi phantom inside, background field from
  4 point dipoles outside the mask; wrapped phase = angle(exp(i * 2 pi * 42.58 * 3 *
  0.020 * B_ppm)).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Tuple

import numpy as np

GAMMA_MHZ_T = 42.58


def _rotation(rng) -> np.ndarray:
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def add_ellipsoids(chi: np.ndarray, rng, n: int, center_box, semi=(3.0, 12.0), value=(-0.1, 0.2)):
    """Paint n random rotated ellipsoids into chi (shape (nz, ny, nx)); later ones overwrite."""
    nz, ny, nx = chi.shape
    for _ in range(n):
        c = np.array([rng.uniform(lo, hi) for lo, hi in center_box])  # (x, y, z)
        a = rng.uniform(semi[0], semi[1], size=3)
        R = _rotation(rng)
        val = rng.uniform(value[0], value[1])
        r = float(a.max()) + 1.0
        lo = np.maximum(np.floor(c - r).astype(int), 0)
        hi = np.minimum(np.ceil(c + r).astype(int) + 1, [nx, ny, nz])
        if np.any(hi <= lo):
            continue
        z, y, x = np.meshgrid(np.arange(lo[2], hi[2]), np.arange(lo[1], hi[1]), np.arange(lo[0], hi[0]),
                              indexing="ij")
        p = np.stack([x - c[0], y - c[1], z - c[2]], axis=-1) @ R  # body coordinates
        inside = ((p / a) ** 2).sum(-1) <= 1.0
        sub = chi[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
        sub[inside] = val
    return chi


def dipole_kernel_np(shape_zyx, voxel_size=(1.0, 1.0, 1.0), bdir=(0.0, 0.0, 1.0)) -> np.ndarray:
    nz, ny, nx = shape_zyx
    kx = np.fft.fftfreq(nx, voxel_size[0])[None, None, :]
    ky = np.fft.fftfreq(ny, voxel_size[1])[None, :, None]
    kz = np.fft.fftfreq(nz, voxel_size[2])[:, None, None]
    b = np.asarray(bdir, dtype=np.float64)
    b = b / np.linalg.norm(b)
    kdb = kx * b[0] + ky * b[1] + kz * b[2]
    k2 = kx * kx + ky * ky + kz * kz
    with np.errstate(divide="ignore", invalid="ignore"):
        d = 1.0 / 3.0 - kdb * kdb / k2
    return np.where(k2 > 1e-20, d, 0.0)


def forward_field(chi: np.ndarray, voxel_size=(1.0, 1.0, 1.0), bdir=(0.0, 0.0, 1.0)) -> np.ndarray:
    D = dipole_kernel_np(chi.shape, voxel_size, bdir)
    return np.fft.ifftn(D * np.fft.fftn(chi)).real


def sphere_mask(shape_zyx, radius, center=None) -> np.ndarray:
    nz, ny, nx = shape_zyx
    cx, cy, cz = center if center is not None else ((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2)
    z, y, x = np.ogrid[:nz, :ny, :nx]
    return (((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) <= radius * radius).astype(np.uint8)


def ellipsoid_mask(shape_zyx, semi_axes_xyz) -> np.ndarray:
    nz, ny, nx = shape_zyx
    ax, ay, az = semi_axes_xyz
    z, y, x = np.ogrid[:nz, :ny, :nx]
    return ((((x - (nx - 1) / 2) / ax) ** 2 + ((y - (ny - 1) / 2) / ay) ** 2 +
             ((z - (nz - 1) / 2) / az) ** 2) <= 1.0).astype(np.uint8)


@dataclass
class TvCase:
    dims: Tuple[int, int, int]
    voxel_size: Tuple[float, float, float]
    bdir: Tuple[float, float, float]
    chi: np.ndarray
    mask: np.ndarray
    local_field: np.ndarray


def tv_case(n=(64, 64, 64), seed=0, n_ellipsoids=12, mask_radius=28.0, noise=0.01, bdir=(0.0, 0.0, 1.0),
            voxel_size=(1.0, 1.0, 1.0)) -> TvCase:
    """Ellipsoid phantom in a sphere mask; local field = dipole-convolved chi + noise in the mask."""
    nx, ny, nz = n
    rng = np.random.default_rng(seed)
    shape = (nz, ny, nx)
    chi = np.zeros(shape)
    cr = max(mask_radius - 12.0, 1.0)
    ctr = ((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2)
    box = [(ctr[0] - cr, ctr[0] + cr), (ctr[1] - cr, ctr[1] + cr), (ctr[2] - cr, ctr[2] + cr)]
    add_ellipsoids(chi, rng, n_ellipsoids, box)
    mask = sphere_mask(shape, mask_radius)
    chi *= mask
    f = forward_field(chi, voxel_size, bdir)
    f = f + rng.normal(0.0, noise, size=shape) * mask
    return TvCase((nx, ny, nz), voxel_size, bdir, chi, mask, f)


def tv_case_64(seed=0) -> TvCase:
    return tv_case((64, 64, 64), seed=seed)


def brain_tv_case(seed=0, dims=(256, 256, 176)):
    """(local_field, mask) of the TV-ADMM throughput case: 12 ellipsoids (semi-axes 3-12
    voxels, chi ~ U[-0.1, 0.2] ppm) centred within +-60/72/45 voxels of the middle, an
    ellipsoid brain mask with semi-axes 100 x 120 x 75 voxels, noise N(0, 0.01) ppm."""
    nx, ny, nz = dims
    rng = np.random.default_rng(seed)
    shape = (nz, ny, nx)
    mask = ellipsoid_mask(shape, (100.0, 120.0, 75.0))
    chi = np.zeros(shape)
    ctr = ((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2)
    box = [(ctr[0] - 60, ctr[0] + 60), (ctr[1] - 72, ctr[1] + 72), (ctr[2] - 45, ctr[2] + 45)]
    add_ellipsoids(chi, rng, 12, box)
    chi *= mask
    f = forward_field(chi) + rng.normal(0.0, 0.01, size=shape) * mask
    return np.ascontiguousarray(f), np.ascontiguousarray(mask)


@dataclass
class ChainCase:
    dims: Tuple[int, int, int]
    voxel_size: Tuple[float, float, float]
    bdir: Tuple[float, float, float]
    field_strength: float
    te: float
    chi: np.ndarray
    mask: np.ndarray
    b_total_ppm: np.ndarray
    wrapped_phase: np.ndarray

    @property
    def rad_per_ppm(self) -> float:
        return 2.0 * math.pi * GAMMA_MHZ_T * self.field_strength * self.te


def chain_case(n=(256, 256, 176), seed=0, semi_axes=(100.0, 120.0, 75.0), n_ellipsoids=30,
               field_strength=3.0, te=0.020, n_sources=4) -> ChainCase:
    """Brain-shaped ellipsoid mask, chi phantom inside, 4 point-dipole background sources outside."""
    nx, ny, nz = n
    rng = np.random.default_rng(seed)
    shape = (nz, ny, nx)
    mask = ellipsoid_mask(shape, semi_axes)
    chi = np.zeros(shape)
    ctr = ((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2)
    box = [(ctr[i] - 0.6 * semi_axes[i], ctr[i] + 0.6 * semi_axes[i]) for i in range(3)]
    add_ellipsoids(chi, rng, n_ellipsoids, box)
    chi *= mask
    local = forward_field(chi)
    # background: point dipoles (moment along z) outside the mask
    z, y, x = np.meshgrid(np.arange(nz, dtype=np.float64), np.arange(ny, dtype=np.float64),
                          np.arange(nx, dtype=np.float64), indexing="ij")
    bg = np.zeros(shape)
    for _ in range(n_sources):
        while True:
            s = np.array([rng.uniform(0, nx - 1), rng.uniform(0, ny - 1), rng.uniform(0, nz - 1)])
            q = ((s[0] - ctr[0]) / semi_axes[0]) ** 2 + ((s[1] - ctr[1]) / semi_axes[1]) ** 2 + \
                ((s[2] - ctr[2]) / semi_axes[2]) ** 2
            if q > 1.15:
                break
        dx, dy, dz = x - s[0], y - s[1], z - s[2]
        r2 = dx * dx + dy * dy + dz * dz + 1.0
        r = np.sqrt(r2)
        cos2 = dz * dz / r2
        strength = rng.uniform(2.0e3, 6.0e3)  # ppm * voxel^3
        bg += strength * (3.0 * cos2 - 1.0) / (r2 * r)
    b_total = local + bg
    case = ChainCase((nx, ny, nz), (1.0, 1.0, 1.0), (0.0, 0.0, 1.0), field_strength, te, chi, mask, b_total, None)
    phase = np.angle(np.exp(1j * case.rad_per_ppm * b_total))
    case.wrapped_phase = phase
    return case
