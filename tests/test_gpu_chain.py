"""The full reconstruction chain on one synthetic scan: wrapped phase -> laplacian_unwrap
(src/unwrap/laplacian.rs:135-161) -> ppm -> vsharp with default radii
(src/bgremove/vsharp.rs:55-199) -> tv_admm (src/inversion/tv.rs:63-97), with the error
against the float64 oracle reported at each stage.  The scan follows the structure of
the 256x256x176 benchmark case at a size the oracle finishes in seconds: an ellipsoid
susceptibility phantom inside an ellipsoid brain mask, a background from four point
dipoles outside the mask, 3 T, TE 20 ms."""
import math

import numpy as np
import pytest

from qsmgpu import Grid, inversion, unwrap, bgremove
from oracle import qsm_oracle as O

pytestmark = pytest.mark.gpu

RAD_PER_PPM = 2.0 * math.pi * 42.58 * 3.0 * 0.020


def rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def scan(grid: Grid, seed=0):
    rng = np.random.default_rng(seed)
    nz, ny, nx = grid.shape
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = ((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2)
    ax = (0.39 * nx, 0.47 * ny, 0.43 * nz)
    mask = ((i - c[0]) / ax[0]) ** 2 + ((j - c[1]) / ax[1]) ** 2 + ((k - c[2]) / ax[2]) ** 2 < 1.0
    chi = np.zeros(grid.shape)
    for _ in range(12):
        p = [c[a] + rng.uniform(-0.5, 0.5) * ax[a] for a in range(3)]
        s = rng.uniform(1.5, 5.0, 3)
        chi[((i - p[0]) / s[0]) ** 2 + ((j - p[1]) / s[1]) ** 2 + ((k - p[2]) / s[2]) ** 2 < 1] = rng.uniform(-0.1, 0.2)
    chi *= mask
    d = O.dipole_kernel(O.Grid(grid.dims, grid.voxel_size), (0, 0, 1))
    b = np.fft.ifftn(d * np.fft.fftn(chi)).real
    for _ in range(4):  # point dipoles outside the mask
        while True:
            p = [rng.uniform(0, n) for n in (nx, ny, nz)]
            if ((p[0] - c[0]) / ax[0]) ** 2 + ((p[1] - c[1]) / ax[1]) ** 2 + ((p[2] - c[2]) / ax[2]) ** 2 > 1.3:
                break
        rx, ry, rz = i - p[0], j - p[1], k - p[2]
        r2 = rx * rx + ry * ry + rz * rz + 1.0
        b += rng.uniform(5.0, 20.0) * (3 * rz * rz / r2 - 1) / r2 ** 1.5
    phase = np.angle(np.exp(1j * RAD_PER_PPM * b))
    return np.ascontiguousarray(phase), np.ascontiguousarray(mask.astype(np.uint8))


@pytest.mark.parametrize("prec,tol", [("f64", 1e-9), ("mixed", 1e-4)])
def test_unwrap_vsharp_tv_chain(request, prec, tol):
    ctx = request.getfixturevalue("ctx64" if prec == "f64" else "ctx32")
    grid = Grid.new(64, 56, 48)
    og = O.Grid(grid.dims, grid.voxel_size)
    phase, mask = scan(grid)
    # stage 1: unwrap
    uw = unwrap.laplacian_unwrap(phase, mask, grid, ctx=ctx)
    uw_ref = O.laplacian_unwrap(phase, mask, og)
    e1 = rel(uw, uw_ref)
    # stage 2: V-SHARP on the field in ppm (the oracle's own stage-1 output feeds both,
    # so each stage's error is its own)
    field = uw_ref / RAD_PER_PPM
    local, fmask = bgremove.vsharp(field, mask, grid, ctx=ctx)
    local_ref, fmask_ref = O.vsharp(field, mask, og)
    np.testing.assert_array_equal(fmask.reshape(fmask_ref.shape), fmask_ref)
    e2 = rel(local, local_ref)
    # stage 3: TV-ADMM, 60 fixed iterations
    p = inversion.TvParams(tol=0.0, max_iter=60)
    chi = inversion.tv_admm(local_ref, fmask_ref, grid, (0, 0, 1), p, ctx=ctx)
    chi_ref = O.tv_admm(local_ref, fmask_ref, og, (0, 0, 1), O.TvParams(tol=0.0, max_iter=60))
    e3 = rel(chi, chi_ref)
    print(f"\n{prec}: unwrap {e1:.2e}  vsharp {e2:.2e}  tv_admm {e3:.2e}")
    assert e1 < tol and e2 < tol and e3 < tol, (e1, e2, e3)
