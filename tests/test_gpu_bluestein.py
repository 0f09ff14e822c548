"""Axis lengths with a prime factor above 13, which the reference transforms like any other
(rustfft plans every length, src/fft.rs:66-74, and its pipeline never pads).  The GPU
engine runs them as Bluestein convolutions of a 7-smooth length m >= 2n - 1 inside the
same pass kernels.  Checked against numpy's DFT for the transform itself and against the
float64 oracle for TKD, Laplacian unwrapping, TV-ADMM and V-SHARP, including the MNI grid
182 x 218 x 182 (218 = 2 * 109)."""
import math
import os

import numpy as np
import pytest

from qsmgpu import Grid, bgremove, inversion, unwrap
from qsmgpu import fft as qfft
from oracle import qsm_oracle as O

pytestmark = pytest.mark.gpu

OBLIQUE = (math.sin(0.3) * math.cos(1.1), math.sin(0.3) * math.sin(1.1), math.cos(0.3))


def rel(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def rnd(grid, seed):
    return np.random.default_rng(seed).standard_normal(grid.shape)


FFT_SHAPES = [(17, 19, 23), (109, 4, 6), (4, 127, 6), (6, 4, 218), (218, 3, 2), (31, 37, 41), (2039, 2, 2),
              (2, 2048, 2), (3, 2, 1031), (34, 38, 46), (1, 17, 1)]


@pytest.mark.parametrize("dims", FFT_SHAPES, ids=["x".join(map(str, d)) for d in FFT_SHAPES])
def test_fft3d_bluestein_f64(ctx64, dims):
    grid = Grid.new(*dims)
    x = rnd(grid, sum(dims))
    got = qfft.fft3d_real(x, grid, ctx=ctx64)
    assert rel(got, np.fft.fftn(x)) < 1e-12, rel(got, np.fft.fftn(x))


@pytest.mark.parametrize("dims", FFT_SHAPES, ids=["x".join(map(str, d)) for d in FFT_SHAPES])
def test_fft3d_bluestein_mixed(ctx32, dims):
    grid = Grid.new(*dims)
    x = rnd(grid, sum(dims) + 1)
    got = qfft.fft3d_real(x, grid, ctx=ctx32)
    assert rel(got, np.fft.fftn(x)) < 2e-6, rel(got, np.fft.fftn(x))


def phantom(grid, bdir, seed):
    from test_gpu_rts import case
    return case(grid, bdir, seed)


@pytest.mark.parametrize("dims", [(17, 19, 23), (34, 38, 46), (29, 16, 12)])
def test_tkd_unwrap_bluestein_f64(ctx64, dims):
    grid = Grid.new(*dims, 1.0, 0.9, 1.1)
    og = O.Grid(grid.dims, grid.voxel_size)
    f, m = phantom(grid, OBLIQUE, sum(dims))
    got = inversion.tkd(f, m, grid, OBLIQUE, inversion.TkdParams(0.19), ctx=ctx64)
    assert rel(got, O.tkd(f, m, og, OBLIQUE, O.TkdParams(0.19))) < 1e-10
    ph = np.angle(np.exp(1j * 40.0 * f))
    got = unwrap.laplacian_unwrap(ph, m, grid, ctx=ctx64)
    assert rel(got, O.laplacian_unwrap(ph, m, og)) < 1e-10


@pytest.mark.parametrize("prec,tol", [("f64", 1e-9), ("mixed", 1e-4)])
@pytest.mark.parametrize("dims", [(17, 19, 23), (46, 34, 38)])
def test_tv_admm_bluestein(request, prec, tol, dims):
    ctx = request.getfixturevalue("ctx64" if prec == "f64" else "ctx32")
    grid = Grid.new(*dims)
    f, m = phantom(grid, OBLIQUE, 3 * sum(dims))
    p = inversion.TvParams(2e-4, 2e-2, 0.0, 30)
    got = inversion.tv_admm(f, m, grid, OBLIQUE, p, ctx=ctx)
    ref = O.tv_admm(f, m, O.Grid(grid.dims, grid.voxel_size), OBLIQUE, O.TvParams(2e-4, 2e-2, 0.0, 30),
                    exact_dc=True)
    assert rel(got, ref) < tol, rel(got, ref)


@pytest.fixture(scope="module")
def mni():
    from qsmgpu import phantom as ph
    grid = Grid.new(182, 218, 182)
    nz, ny, nx = grid.shape
    mask = ph.ellipsoid_mask(grid.shape, (70.0, 90.0, 65.0))
    rng = np.random.default_rng(9)
    chi = np.zeros(grid.shape)
    ctr = ((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2)
    ph.add_ellipsoids(chi, rng, 10, [(c - 40, c + 40) for c in ctr])
    chi *= mask
    f = ph.forward_field(chi) + rng.normal(0.0, 0.01, grid.shape) * mask
    O.set_fft_workers(os.cpu_count() or 1)
    yield np.ascontiguousarray(f), np.ascontiguousarray(mask), grid
    O.set_fft_workers(None)


@pytest.mark.parametrize("prec,tol", [("f64", 1e-9), ("mixed", 1e-4)])
def test_tv_admm_mni_182x218x182(request, mni, prec, tol):
    ctx = request.getfixturevalue("ctx64" if prec == "f64" else "ctx32")
    f, m, grid = mni
    got = inversion.tv_admm(f, m, grid, (0, 0, 1), inversion.TvParams(2e-4, 2e-2, 0.0, 4), ctx=ctx)
    ref = O.tv_admm(f, m, O.Grid(grid.dims, grid.voxel_size), (0, 0, 1), O.TvParams(2e-4, 2e-2, 0.0, 4))
    assert rel(got, ref) < tol, rel(got, ref)


@pytest.mark.parametrize("prec,tol", [("f64", 1e-9), ("mixed", 1e-5)])
def test_vsharp_mni_182x218x182(request, mni, prec, tol):
    ctx = request.getfixturevalue("ctx64" if prec == "f64" else "ctx32")
    f, m, grid = mni
    radii = [8.0, 3.0]
    local, fm = bgremove.vsharp_with_radii(f, m, grid, radii, 0.05, ctx=ctx)
    ref_local, ref_mask = O.vsharp_with_radii(f, m, O.Grid(grid.dims, grid.voxel_size), radii, 0.05)
    np.testing.assert_array_equal(fm.reshape(ref_mask.shape), ref_mask)
    assert rel(local, ref_local) < tol, rel(local, ref_local)
