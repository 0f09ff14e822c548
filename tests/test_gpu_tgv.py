"""GPU parity of TGV-QSM (src/inversion/tgv.rs:1045-1299) against the float32 oracle.

Both sides iterate in float; they differ in rounding (fused multiply-adds, summation
order of the mean and the convergence sums, libm sin/cos), so the comparison is a
relative-L2 bound on chi rather than bit equality: 1e-4 after 10 iterations, 2e-3 after
300 (primal-dual iterations carry rounding differences forward)."""
import math

import numpy as np
import pytest

import qsmgpu
from qsmgpu import Grid, inversion
from oracle import qsm_oracle as O

pytestmark = pytest.mark.gpu

OBLIQUE = (math.sin(0.35) * math.cos(0.8), math.sin(0.35) * math.sin(0.8), math.cos(0.35))
RAD_PER_PPM = 2.0 * math.pi * 0.020 * 3.0 * 42.5781


def rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def og(grid: Grid):
    return O.Grid(grid.dims, grid.voxel_size)


def small_case():
    n = 12
    c = 6.0
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    mask = (np.sqrt((i - c) ** 2 + (j - c) ** 2 + (k - c) ** 2) < 4.0).astype(np.uint8)
    phase = np.where(mask > 0, 0.1 * k, 0.0)
    return phase, mask


def phantom_phase(grid: Grid, b0, seed):
    """Wrapped phase of a blob phantom in an ellipsoid head mask (rad, TE 20 ms, 3 T)."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = grid.shape
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = ((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2)
    mask = ((i - c[0]) / (0.42 * nx)) ** 2 + ((j - c[1]) / (0.42 * ny)) ** 2 + ((k - c[2]) / (0.42 * nz)) ** 2 < 1
    chi = np.zeros(grid.shape)
    for _ in range(8):
        p = [rng.uniform(0.3, 0.7) * s for s in (nx, ny, nz)]
        r = rng.uniform(2.0, 4.0)
        chi[(i - p[0]) ** 2 + (j - p[1]) ** 2 + (k - p[2]) ** 2 < r * r] = rng.uniform(-0.1, 0.3)
    chi *= mask
    d = O.dipole_kernel(og(grid), b0)
    field = np.fft.ifftn(d * np.fft.fftn(chi)).real
    phase = np.angle(np.exp(1j * field * RAD_PER_PPM)) * mask
    return np.ascontiguousarray(phase), np.ascontiguousarray(mask.astype(np.uint8))


def test_tgv_reference_small_case(ctx64):
    """src/inversion/tgv.rs:1379-1437 (10 iterations, 1 erosion)."""
    phase, mask = small_case()
    grid = Grid.new(12, 12, 12)
    p = inversion.TgvParams(iterations=10, erosions=1)
    seen = []
    got = inversion.tgv_qsm(phase, mask, grid, p, (0, 0, 1), progress=lambda a, b: seen.append((a, b)), ctx=ctx64)
    ref = O.tgv_qsm(phase, mask, og(grid), O.TgvParams(iterations=10, erosions=1), (0, 0, 1))
    assert np.all(np.isfinite(got)) and np.any(np.abs(got) > 1e-20)
    # a linear ramp has a zero Laplacian inside the mask: chi stays at rounding level
    # (~1e-9 ppm), so only an absolute bound is meaningful here
    assert np.abs(got - ref).max() < 1e-6
    assert seen == [(t, 10) for t in range(10)] + [(10, 10)]


def test_tgv_small_quadratic_phase(ctx64):
    """The reference's 12^3 sphere with a quadratic phase (non-zero Laplacian)."""
    phase, mask = small_case()
    k, j, i = np.meshgrid(np.arange(12), np.arange(12), np.arange(12), indexing="ij")
    phase = np.where(mask > 0, 0.05 * ((k - 6.0) ** 2 - 0.5 * (i - 6.0) ** 2), 0.0)
    grid = Grid.new(12, 12, 12)
    got = inversion.tgv_qsm(phase, mask, grid, inversion.TgvParams(iterations=10, erosions=1), (0, 0, 1), ctx=ctx64)
    ref = O.tgv_qsm(phase, mask, og(grid), O.TgvParams(iterations=10, erosions=1), (0, 0, 1))
    assert np.abs(ref).max() > 1e-7
    assert rel(got, ref) < 1e-3, rel(got, ref)


@pytest.mark.parametrize("dims,vs,b0,iters", [((32, 28, 24), (1.0, 1.0, 1.0), (0.0, 0.0, 1.0), 300),
                                               ((30, 26, 22), (1.0, 1.1, 1.3), OBLIQUE, 250)])
def test_tgv_phantom(ctx64, dims, vs, b0, iters):
    grid = Grid.new(*dims, *vs)
    phase, mask = phantom_phase(grid, b0, seed=sum(dims))
    p = inversion.TgvParams(iterations=iters, erosions=2, tol=0.0)
    got = inversion.tgv_qsm(phase, mask, grid, p, b0, ctx=ctx64)
    ref = O.tgv_qsm(phase, mask, og(grid), O.TgvParams(iterations=iters, erosions=2, tol=0.0), b0)
    assert rel(got, ref) < 2e-3, rel(got, ref)
    assert np.all(got[ref == 0] == 0.0)


def test_tgv_convergence_and_progress(ctx32):
    """src/inversion/tgv.rs:1562-1599: zero phase with tol 1.1 stops at the first check."""
    _, mask = small_case()
    grid = Grid.new(12, 12, 12)
    seen = []
    got = inversion.tgv_qsm(np.zeros(mask.shape), mask, grid, inversion.TgvParams(iterations=1000, erosions=1, tol=1.1),
                            (0, 0, 1), progress=lambda a, b: seen.append((a, b)), ctx=ctx32)
    assert np.all(got == 0.0)
    assert seen == [(t, 1000) for t in range(101)] + [(100, 1000)]


def test_tgv_empty_mask_is_an_error(ctx64):
    grid = Grid.new(8, 8, 8)
    m = np.zeros(grid.shape, np.uint8)
    m[3:5, 3:5, 3:5] = 1  # vanishes after the erosions
    with pytest.raises(qsmgpu.QsmError):
        inversion.tgv_qsm(np.zeros(grid.shape), m, grid, inversion.TgvParams(iterations=5), (0, 0, 1), ctx=ctx64)


def test_apply_reference_known_answers(ctx64):
    """src/pipeline/referencing.rs:49-82 through the C ABI."""
    from qsmgpu import pipeline
    np.testing.assert_allclose(pipeline.apply_reference([1.0, 2.0, 3.0, 4.0], [1, 1, 1, 0], ctx=ctx64),
                               [-1.0, 0.0, 1.0, 0.0], atol=1e-10)
    assert list(pipeline.apply_reference([1.0, 2.0, 3.0], [1, 0, 1], pipeline.REFERENCE_NONE, ctx=ctx64)) == [1.0, 0.0, 3.0]
    assert list(pipeline.apply_reference([1.0, 2.0], [0, 0], ctx=ctx64)) == [0.0, 0.0]


def test_run_tgv_single_echo_and_errors(ctx64):
    """pipeline::run_tgv (src/pipeline/inversion.rs:124-157): tgv_qsm then apply_reference."""
    from qsmgpu import pipeline
    grid = Grid.new(30, 26, 22, 1.0, 1.1, 1.3)
    phase, mask = phantom_phase(grid, OBLIQUE, seed=3)
    p = inversion.TgvParams(iterations=120, erosions=2)
    md = pipeline.ScanMetadata(grid.dims, grid.voxel_size, b0_direction=OBLIQUE)
    got = pipeline.run_tgv([phase], mask, md, p, pipeline.REFERENCE_MEAN, ctx=ctx64)
    chi = inversion.tgv_qsm(phase, mask, grid, p, OBLIQUE, ctx=ctx64)
    want = O.apply_reference(chi, mask)
    assert rel(got, want) < 1e-12
    with pytest.raises(qsmgpu.InvalidConfig):
        pipeline.run_tgv([phase, phase], mask, md, p, ctx=ctx64)
    with pytest.raises(qsmgpu.DimensionMismatch):
        pipeline.run_tgv([phase.ravel()[:-1]], mask, md, p, ctx=ctx64)
