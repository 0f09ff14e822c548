"""GPU parity of RTS (src/inversion/rts.rs:72-211), the pipeline's default inversion,
against the float64 oracle: FP64 context rel-L2 1e-9 with the same iteration count and
progress sequence; mixed context 1e-4 with a fixed iteration count.

The GPU's Laplacian eigenvalue tables hold the exact 0 at k = 0, so the oracle runs with
exact_dc=True.  At voxel sizes where the reference's FFT of the Laplacian taps leaves a
few ulp there, the reference's iterate differs from that by a constant over the grid
(amplified roundoff at DC); test_rts_faithful_dc_offset checks that this is all that
differs."""
import math

import numpy as np
import pytest

from qsmgpu import Grid, inversion, pipeline
from oracle import qsm_oracle as O

pytestmark = pytest.mark.gpu

OBLIQUE = (math.sin(0.35) * math.cos(0.8), math.sin(0.35) * math.sin(0.8), math.cos(0.35))


def rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def case(grid, bdir, seed):
    rng = np.random.default_rng(seed)
    nz, ny, nx = grid.shape
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = ((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2)
    mask = ((i - c[0]) / (0.4 * nx)) ** 2 + ((j - c[1]) / (0.4 * ny)) ** 2 + ((k - c[2]) / (0.4 * nz)) ** 2 < 1
    chi = np.zeros(grid.shape)
    for _ in range(6):
        p = [rng.uniform(0.3, 0.7) * s for s in (nx, ny, nz)]
        r = rng.uniform(1.5, 3.5)
        chi[(i - p[0]) ** 2 + (j - p[1]) ** 2 + (k - p[2]) ** 2 < r * r] = rng.uniform(-0.1, 0.2)
    chi *= mask
    d = O.dipole_kernel(O.Grid(grid.dims, grid.voxel_size), bdir)
    f = np.fft.ifftn(d * np.fft.fftn(chi)).real + rng.normal(0, 0.01, grid.shape) * mask
    return np.ascontiguousarray(f), np.ascontiguousarray(mask.astype(np.uint8))


@pytest.mark.parametrize("dims,vs,bdir", [((32, 28, 24), (1.0, 1.0, 1.0), (0.0, 0.0, 1.0)),
                                          ((30, 26, 22), (1.0, 1.1, 1.3), OBLIQUE),
                                          ((25, 27, 15), (0.9, 1.0, 1.2), OBLIQUE)])
def test_rts_default_params_f64(ctx64, dims, vs, bdir):
    grid = Grid.new(*dims, *vs)
    f, m = case(grid, bdir, sum(dims))
    seen, ref_seen = [], []
    got = inversion.rts(f, m, grid, bdir, progress=lambda a, b: seen.append((a, b)), ctx=ctx64)
    ref, iters = O.rts(f, m, O.Grid(grid.dims, grid.voxel_size), bdir, progress=lambda a, b: ref_seen.append((a, b)),
                       return_iters=True, exact_dc=True)
    assert rel(got, ref) < 1e-9, rel(got, ref)
    assert ctx64.tv_last_iterations() == iters
    assert seen == ref_seen


def test_rts_mixed_fixed_iterations(ctx32):
    grid = Grid.new(30, 26, 22, 1.0, 1.1, 1.3)
    f, m = case(grid, OBLIQUE, 5)
    p = inversion.RtsParams(tol=0.0, max_iter=20)
    got = inversion.rts(f, m, grid, OBLIQUE, p, ctx=ctx32)
    ref = O.rts(f, m, O.Grid(grid.dims, grid.voxel_size), OBLIQUE, O.RtsParams(tol=0.0, max_iter=20), exact_dc=True)
    assert rel(got, ref) < 1e-4, rel(got, ref)


@pytest.mark.parametrize("solver", ["tv", "rts"])
def test_faithful_dc_offset(ctx64, solver):
    """At (1, 1, 0.9) mm the reference's DC Laplacian eigenvalue is FFT roundoff (nonzero):
    the GPU result equals the faithful oracle up to a constant inside the mask, and equals
    the exact-DC oracle outright."""
    grid = Grid.new(24, 28, 16, 1.0, 1.0, 0.9)
    og = O.Grid(grid.dims, grid.voxel_size)
    f, m = case(grid, (0, 0, 1), 67)
    if solver == "tv":
        got = inversion.tv_admm(f, m, grid, (0, 0, 1), inversion.TvParams(tol=0.0, max_iter=7), ctx=ctx64)
        ref = lambda e: O.tv_admm(f, m, og, (0, 0, 1), O.TvParams(tol=0.0, max_iter=7), exact_dc=e)
    else:
        got = inversion.rts(f, m, grid, (0, 0, 1), inversion.RtsParams(tol=0.0, max_iter=7), ctx=ctx64)
        ref = lambda e: O.rts(f, m, og, (0, 0, 1), O.RtsParams(tol=0.0, max_iter=7), exact_dc=e)
    exact, faithful = ref(True), ref(False)
    assert rel(got, exact) < 1e-9, rel(got, exact)
    d = (faithful - got.reshape(faithful.shape))[m != 0]
    assert np.abs(d - d.mean()).max() < 1e-9 * np.abs(exact).max()


def test_rts_reference_tests(ctx64):
    """src/inversion/rts.rs:213-263."""
    n = 8
    grid = Grid.new(n, n, n)
    p = inversion.RtsParams(0.15, 1e5, 10.0, 1e-2, 5, 2)
    assert np.all(np.abs(inversion.rts(np.zeros((n, n, n)), np.ones((n, n, n), np.uint8), grid, (0, 0, 1), p,
                                       ctx=ctx64)) < 1e-6)
    field = (np.arange(n ** 3, dtype=np.float64) * 0.001).reshape(n, n, n)
    mask = np.ones(n ** 3, np.uint8)
    mask[0] = 0
    mask[10] = 0
    chi = inversion.rts(field, mask.reshape(n, n, n), grid, (0, 0, 1), p, ctx=ctx64)
    assert np.all(np.isfinite(chi)) and chi.ravel()[0] == 0.0 and chi.ravel()[10] == 0.0


def test_pipeline_default_is_rts(ctx64):
    """InversionConfig::default selects Rts (src/pipeline/config.rs:251)."""
    grid = Grid.new(24, 20, 18)
    f, m = case(grid, (0, 0, 1), 9)
    md = pipeline.ScanMetadata(grid.dims, grid.voxel_size)
    chi = pipeline.run_dipole_inversion(f, m, md, pipeline.InversionConfig(), ctx=ctx64)
    np.testing.assert_array_equal(chi.ravel(), inversion.rts(f, m, grid, (0, 0, 1), ctx=ctx64).ravel())
