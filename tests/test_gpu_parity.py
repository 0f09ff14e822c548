"""GPU parity: every entry point of libqsmgpu.so against the float64 oracle.

Tolerances (relative L2 error against the oracle, computed over the whole volume):
  * FP64 context   : 1e-10 for closed-form methods and transforms, 1e-9 for iterative ones;
  * mixed context  : 1e-5 for closed-form methods, 1e-4 for TV-ADMM (the project target);
  * masks (erosion, V-SHARP selection): exact equality in both precisions.
"""
import math

import numpy as np
import pytest

import qsmgpu
from qsmgpu import Grid, inversion, unwrap, bgremove, pipeline, phantom
from qsmgpu import fft as qfft
from oracle import qsm_oracle as O

pytestmark = pytest.mark.gpu

OBLIQUE = (math.sin(0.35) * math.cos(0.8), math.sin(0.35) * math.sin(0.8), math.cos(0.35))


def rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def og(grid: Grid):
    return O.Grid(grid.dims, grid.voxel_size)


def rnd(grid, seed=0):
    return np.random.default_rng(seed).standard_normal(grid.shape)


# ---------------------------------------------------------------- transforms --
FFT_SIZES = [(8, 6, 10), (16, 16, 16), (15, 9, 25), (64, 64, 64), (1, 7, 13), (22, 12, 11), (96, 100, 27),
             (176, 4, 6), (256, 2, 3), (384, 3, 2), (2, 2, 2), (4, 256, 2), (2, 4, 256), (6, 5, 384)]


@pytest.mark.parametrize("dims", FFT_SIZES)
def test_fft3d_real_matches_numpy_f64(ctx64, dims):
    grid = Grid.new(*dims)
    x = rnd(grid, 1)
    got = qfft.fft3d_real(x, grid, ctx=ctx64)
    assert rel(got.real, np.fft.fftn(x).real) < 1e-12
    assert np.linalg.norm(got - np.fft.fftn(x)) / np.linalg.norm(np.fft.fftn(x)) < 1e-12


@pytest.mark.parametrize("dims", [(8, 6, 10), (64, 64, 64), (15, 9, 25), (176, 4, 6), (4, 256, 2), (2, 4, 256), (512, 2, 2)])
def test_fft3d_real_matches_numpy_mixed(ctx32, dims):
    grid = Grid.new(*dims)
    x = rnd(grid, 2)
    got = qfft.fft3d_real(x, grid, ctx=ctx32)
    ref = np.fft.fftn(x)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 2e-6


# -------------------------------------------------------- closed-form inversion --
CF_GRIDS = [Grid.new(8, 6, 10), Grid.new(24, 20, 18, 1.0, 0.9, 1.2), Grid.new(15, 16, 9)]


@pytest.mark.parametrize("grid", CF_GRIDS, ids=lambda g: "x".join(map(str, g.dims)))
@pytest.mark.parametrize("bdir", [(0.0, 0.0, 1.0), OBLIQUE], ids=["z", "oblique"])
def test_tkd_tsvd_tikhonov_f64(ctx64, grid, bdir):
    f = rnd(grid, 3) * 0.05
    m = (np.random.default_rng(4).random(grid.shape) > 0.2).astype(np.uint8)
    for thr in (0.15, 0.19):
        p = inversion.TkdParams(thr)
        assert rel(inversion.tkd(f, m, grid, bdir, p, ctx=ctx64), O.tkd(f, m, og(grid), bdir, O.TkdParams(thr))) < 1e-10
        assert rel(inversion.tsvd(f, m, grid, bdir, p, ctx=ctx64),
                   O.tsvd(f, m, og(grid), bdir, O.TkdParams(thr))) < 1e-10
    for reg in (0, 1, 2):
        got = inversion.tikhonov(f, m, grid, bdir, inversion.TikhonovParams(0.01, reg), ctx=ctx64)
        ref = O.tikhonov(f, m, og(grid), bdir, O.TikhonovParams(0.01, reg))
        assert rel(got, ref) < 1e-10
    # masked voxels are exactly zero
    chi = inversion.tkd(f, m, grid, bdir, ctx=ctx64)
    assert np.all(chi[m == 0] == 0.0)


@pytest.mark.parametrize("bdir", [(0.0, 0.0, 1.0), OBLIQUE], ids=["z", "oblique"])
def test_tkd_tikhonov_mixed(ctx32, bdir):
    grid = Grid.new(32, 30, 28)
    f = rnd(grid, 5) * 0.05
    m = np.ones(grid.shape, np.uint8)
    assert rel(inversion.tkd(f, m, grid, bdir, ctx=ctx32), O.tkd(f, m, og(grid), bdir)) < 1e-5
    got = inversion.tikhonov(f, m, grid, bdir, inversion.TikhonovParams(0.01, 1), ctx=ctx32)
    assert rel(got, O.tikhonov(f, m, og(grid), bdir, O.TikhonovParams(0.01, 1))) < 1e-5


def test_closed_form_reference_properties(ctx64):
    """src/inversion/tkd.rs:160-224, tikhonov.rs:144-195 on the GPU."""
    grid = Grid.new(8, 8, 8)
    m = np.ones(grid.shape, np.uint8)
    assert np.abs(inversion.tkd(np.zeros(grid.shape), m, grid, ctx=ctx64)).max() < 1e-10
    m2 = m.ravel().copy()
    m2[:2] = 0
    chi = inversion.tkd(np.ones(512), m2, grid, ctx=ctx64)
    assert chi[0] == 0.0 and chi[1] == 0.0
    assert np.abs(inversion.tikhonov(np.zeros(512), m2, grid, ctx=ctx64)).max() < 1e-10


def test_dipole_forward(ctx64):
    grid = Grid.new(20, 18, 16)
    chi = rnd(grid, 6)
    ref = O.ifft3d(O.fft3d(chi) * O.dipole_kernel(og(grid), OBLIQUE)).real
    assert rel(inversion.dipole_forward(chi, grid, OBLIQUE, ctx=ctx64), ref) < 1e-10


# ------------------------------------------------------------------ TV-ADMM --
def _tv_case(n, seed, bdir=(0.0, 0.0, 1.0)):
    c = phantom.tv_case((n, n, n), seed=seed, n_ellipsoids=6, mask_radius=n * 0.4, bdir=bdir)
    return Grid.new(n, n, n), c


@pytest.mark.parametrize("bdir", [(0.0, 0.0, 1.0), OBLIQUE], ids=["z", "oblique"])
def test_tv_admm_fixed_iterations_f64(ctx64, bdir):
    grid, c = _tv_case(24, 7, bdir)
    p = inversion.TvParams(2e-4, 2e-2, 0.0, 31)  # tol = 0: a fixed 31 iterations (odd on purpose)
    got = inversion.tv_admm(c.local_field, c.mask, grid, bdir, p, ctx=ctx64)
    ref = O.tv_admm(c.local_field, c.mask, og(grid), bdir, O.TvParams(2e-4, 2e-2, 0.0, 31))
    assert rel(got, ref) < 1e-9
    assert ctx64.tv_last_iterations() == 31


def test_tv_admm_early_exit_and_progress_f64(ctx64):
    grid, c = _tv_case(20, 8)
    calls, ref_calls = [], []
    p = inversion.TvParams(1e-3, 0.1, 2e-2, 60)
    got = inversion.tv_admm(c.local_field, c.mask, grid, (0, 0, 1), p, lambda a, b: calls.append((a, b)), ctx=ctx64)
    ref, iters = O.tv_admm(c.local_field, c.mask, og(grid), (0, 0, 1), O.TvParams(1e-3, 0.1, 2e-2, 60),
                           lambda a, b: ref_calls.append((a, b)), return_iters=True)
    assert iters < 60, "case must converge early"
    assert ctx64.tv_last_iterations() == iters
    assert calls == ref_calls
    assert rel(got, ref) < 1e-9


@pytest.mark.parametrize("vs", [(0.9, 1.0, 1.2), (1.0, 0.9, 1.0), (1.0, 1.0, 0.9)])
def test_tv_admm_anisotropic_f64(ctx64, vs):
    """Anisotropic voxels on odd and even axes.  The GPU's Laplacian tables hold the exact
    DC eigenvalue 0; the reference's FFT of the taps leaves roundoff there at some voxel
    sizes, which only shifts the iterate by a constant (oracle exact_dc)."""
    for dims in ((24, 28, 16), (25, 27, 15)):
        grid = Grid.new(*dims, *vs)
        c = phantom.tv_case(dims, seed=3, n_ellipsoids=6, mask_radius=min(dims) * 0.4, bdir=OBLIQUE, voxel_size=vs)
        got = inversion.tv_admm(c.local_field, c.mask, grid, OBLIQUE, inversion.TvParams(2e-4, 2e-2, 0.0, 9),
                                ctx=ctx64)
        ref = O.tv_admm(c.local_field, c.mask, og(grid), OBLIQUE, O.TvParams(2e-4, 2e-2, 0.0, 9), exact_dc=True)
        assert rel(got, ref) < 1e-9, (dims, rel(got, ref))


def test_tv_admm_progress_at_max_iter_f64(ctx64):
    """tol > 0 but no convergence: progress stops at (max_iter, max_iter's total)
    (src/inversion/tv.rs:78-93), with the last iterate still tested."""
    grid, c = _tv_case(20, 8)
    calls, ref_calls = [], []
    p = inversion.TvParams(1e-3, 0.1, 1e-9, 6)
    inversion.tv_admm(c.local_field, c.mask, grid, (0, 0, 1), p, lambda a, b: calls.append((a, b)), ctx=ctx64)
    O.tv_admm(c.local_field, c.mask, og(grid), (0, 0, 1), O.TvParams(1e-3, 0.1, 1e-9, 6),
              lambda a, b: ref_calls.append((a, b)))
    assert calls == ref_calls == [(i + 1, 6) for i in range(6)]
    assert ctx64.tv_last_iterations() == 6


def test_tv_admm_mixed_target(ctx32):
    grid, c = _tv_case(32, 9)
    p = inversion.TvParams(2e-4, 2e-2, 0.0, 60)
    got = inversion.tv_admm(c.local_field, c.mask, grid, (0, 0, 1), p, ctx=ctx32)
    ref = O.tv_admm(c.local_field, c.mask, og(grid), (0, 0, 1), O.TvParams(2e-4, 2e-2, 0.0, 60))
    assert rel(got, ref) < 1e-4


def test_tv_admm_reference_properties(ctx64):
    """src/inversion/tv.rs:112-145: zero field -> 0, finite."""
    grid = Grid.new(8, 8, 8)
    m = np.ones(512, np.uint8)
    p = inversion.TvParams(1e-3, 0.1, 1e-2, 10)
    assert np.abs(inversion.tv_admm(np.zeros(512), m, grid, (0, 0, 1), p, ctx=ctx64)).max() < 1e-8
    out = inversion.tv_admm(np.arange(512) * 0.001, m, grid, (0, 0, 1), p, ctx=ctx64)
    assert np.all(np.isfinite(out))


# ---------------------------------------------------------------- unwrapping --
@pytest.mark.parametrize("dims", [(16, 16, 16), (20, 18, 22), (15, 12, 9)])
def test_laplacian_unwrap_f64(ctx64, dims):
    grid = Grid.new(*dims, 1.0, 1.1, 0.9)
    z, y, x = np.meshgrid(*[np.arange(n) for n in grid.shape], indexing="ij")
    true = 3.0 * np.sin(2 * np.pi * x / grid.nx) + 0.05 * (y - grid.ny / 2) ** 2 + 0.3 * z
    ph = np.angle(np.exp(1j * true))
    m = (np.random.default_rng(1).random(grid.shape) > 0.1).astype(np.uint8)
    got = unwrap.laplacian_unwrap(ph, m, grid, ctx=ctx64)
    assert rel(got, O.laplacian_unwrap(ph, m, og(grid))) < 1e-10


def test_laplacian_unwrap_mixed(ctx32):
    grid = Grid.new(32, 32, 24)
    z, y, x = np.meshgrid(*[np.arange(n) for n in grid.shape], indexing="ij")
    ph = np.angle(np.exp(1j * (0.02 * (x - 16) ** 2 + 0.3 * y)))
    m = np.ones(grid.shape, np.uint8)
    assert rel(unwrap.laplacian_unwrap(ph, m, grid, ctx=ctx32), O.laplacian_unwrap(ph, m, og(grid))) < 1e-5


# --------------------------------------------------------- background removal --
def _bg_case(grid, seed=0):
    rng = np.random.default_rng(seed)
    m = O.create_sphere_mask(og(grid), grid.nx / 2 - 0.5, grid.ny / 2 - 0.5, grid.nz / 2 - 0.5,
                             min(grid.dims) * 0.38)
    f = rng.standard_normal(grid.shape) * 0.01
    z, y, x = np.meshgrid(*[np.arange(n) for n in grid.shape], indexing="ij")
    f += 0.001 * x * y / grid.nx + 0.002 * z
    return f, m


@pytest.mark.parametrize("vs", [(1.0, 1.0, 1.0), (0.6, 0.9, 1.3)])
def test_smv_sharp_f64(ctx64, vs):
    grid = Grid.new(24, 22, 20, *vs)
    f, m = _bg_case(grid, 1)
    lo, mo = bgremove.smv(f, m, grid, 3.0, ctx=ctx64)
    lr, mr = O.smv(f, m, og(grid), 3.0)
    assert np.array_equal(mo, mr) and rel(lo, lr) < 1e-10
    lo, mo = bgremove.sharp(f, m, grid, bgremove.SharpParams(0.05, 3.0), ctx=ctx64)
    lr, mr = O.sharp(f, m, og(grid), O.SharpParams(0.05, 3.0))
    assert np.array_equal(mo, mr) and rel(lo, lr) < 1e-10


@pytest.mark.parametrize("vs", [(1.0, 1.0, 1.0), (0.8, 1.0, 1.25)])
def test_vsharp_f64(ctx64, vs):
    grid = Grid.new(28, 26, 24, *vs)
    f, m = _bg_case(grid, 2)
    calls = []
    lo, mo = bgremove.vsharp(f, m, grid, bgremove.VsharpParams(0.05, 6.0, 1.0), lambda a, b: calls.append((a, b)),
                             ctx=ctx64)
    lr, mr = O.vsharp(f, m, og(grid), O.VsharpParams(0.05, 6.0, 1.0))
    assert np.array_equal(mo, mr)
    assert rel(lo, lr) < 1e-9
    assert calls == [(i + 1, 6) for i in range(6)]


def test_vsharp_mixed_masks_exact(ctx32):
    grid = Grid.new(32, 32, 32)
    f, m = _bg_case(grid, 3)
    lo, mo = bgremove.vsharp_with_radii(f, m, grid, [2.0, 5.0, 4.0, 3.0], 0.05, ctx=ctx32)
    lr, mr = O.vsharp_with_radii(f, m, og(grid), [2.0, 5.0, 4.0, 3.0], 0.05)
    assert np.array_equal(mo, mr)
    assert rel(lo, lr) < 1e-5


def test_vsharp_reference_properties(ctx64):
    """src/bgremove/vsharp.rs:205-461: empty radii, single radius == SHARP, sorted == unsorted."""
    grid = Grid.new(8, 8, 8)
    m = np.ones(512, np.uint8)
    f = np.arange(512) * 0.001
    le, me = bgremove.vsharp_with_radii(f, m, grid, [], 0.05, ctx=ctx64)
    assert np.all(le == 0) and np.array_equal(me, m)
    l1, m1 = bgremove.vsharp_with_radii(f, m, grid, [3.0], 0.05, ctx=ctx64)
    l2, m2 = bgremove.sharp(f, m, grid, bgremove.SharpParams(0.05, 3.0), ctx=ctx64)
    assert np.abs(l1 - l2).max() < 1e-10 and np.array_equal(m1, m2)
    la, ma = bgremove.vsharp_with_radii(f, m, grid, [4.0, 3.0, 2.0], 0.05, ctx=ctx64)
    lb, mb = bgremove.vsharp_with_radii(f, m, grid, [2.0, 4.0, 3.0], 0.05, ctx=ctx64)
    assert np.array_equal(ma, mb) and np.abs(la - lb).max() < 1e-10


# ------------------------------------------------------------------ pipeline --
def test_pipeline_dispatch_and_errors(ctx64):
    grid = Grid.new(16, 16, 16)
    f = rnd(grid, 9) * 0.01
    m = np.ones(grid.shape, np.uint8)
    md = pipeline.ScanMetadata((16, 16, 16), (1.0, 1.0, 1.0), (0.02,), 3.0, (0.0, 0.0, 1.0))
    cfg = pipeline.InversionConfig(algorithm=pipeline.TKD)
    np.testing.assert_array_equal(pipeline.run_dipole_inversion(f, m, md, cfg, ctx=ctx64),
                                  inversion.tkd(f, m, grid, ctx=ctx64).ravel())
    with pytest.raises(qsmgpu.DimensionMismatch):
        pipeline.run_dipole_inversion(f.ravel()[:100], m, md, cfg, ctx=ctx64)
    for alg in (pipeline.TGV, pipeline.QSMART):
        with pytest.raises(qsmgpu.InvalidConfig):
            pipeline.run_dipole_inversion(f, m, md, pipeline.InversionConfig(algorithm=alg), ctx=ctx64)
    res = pipeline.run_bg_removal(f, m, md, pipeline.BgRemovalConfig(
        algorithm=pipeline.SHARP, sharp=bgremove.SharpParams(0.05, 3.0)), ctx=ctx64)
    lr, mr = O.sharp(f, m, og(grid), O.SharpParams(0.05, 3.0))
    assert np.array_equal(res.eroded_mask.reshape(grid.shape), mr) and rel(res.local_field_ppm, lr) < 1e-10
    with pytest.raises(qsmgpu.DimensionMismatch):
        pipeline.run_bg_removal(f.ravel()[:10], m, md, pipeline.BgRemovalConfig(), ctx=ctx64)


def test_invalid_arguments_are_errors_not_faults(ctx64):
    grid = Grid.new(2053, 4, 4)  # a prime above the Bluestein limit (2048) has no plan
    with pytest.raises(qsmgpu.QsmError) as e:
        inversion.tkd(np.zeros(grid.shape), np.ones(grid.shape, np.uint8), grid, ctx=ctx64)
    assert e.value.status == 3
    with pytest.raises(qsmgpu.QsmError):
        inversion.tkd(np.zeros(8 * 8 * 8), np.ones(512, np.uint8), Grid.new(8, 8, 8), (0, 0, float("nan")),
                      ctx=ctx64)
