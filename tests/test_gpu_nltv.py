"""GPU parity of NLTV (src/inversion/nltv.rs:62-131) against the float64 oracle: FP64
context rel-L2 1e-9 with the same inner-step count and progress sequence, across passes
that converge early and passes that run to max_iter; mixed context at a fixed step count.

As for TV-ADMM, the oracle runs with exact_dc=True: the GPU's Laplacian tables hold the
exact DC eigenvalue 0 (the reference's FFT of the taps can leave roundoff there)."""
import math

import numpy as np
import pytest

from qsmgpu import Grid, inversion, pipeline
from oracle import qsm_oracle as O
from test_gpu_rts import case, rel

pytestmark = pytest.mark.gpu

OBLIQUE = (math.sin(0.35) * math.cos(0.8), math.sin(0.35) * math.sin(0.8), math.cos(0.35))


def og(grid):
    return O.Grid(grid.dims, grid.voxel_size)


@pytest.mark.parametrize("dims,vs,bdir,params", [
    ((32, 28, 24), (1.0, 1.0, 1.0), (0.0, 0.0, 1.0), (1e-3, 1.0, 1e-2, 30, 3)),   # 63 of 90 steps
    ((30, 26, 22), (1.0, 1.1, 1.3), OBLIQUE, (1e-3, 1.0, 2e-2, 30, 3)),            # 26 of 90
    ((25, 27, 15), (0.9, 1.0, 1.2), OBLIQUE, (2e-3, 0.5, 5e-2, 30, 3)),            # early exits
    ((25, 27, 15), (0.9, 1.0, 1.2), OBLIQUE, (1e-3, 1.0, 1e-3, 9, 3)),             # every pass to max_iter
])
def test_nltv_f64(ctx64, dims, vs, bdir, params):
    grid = Grid.new(*dims, *vs)
    f, m = case(grid, bdir, sum(dims))
    seen, ref_seen = [], []
    got = inversion.nltv(f, m, grid, bdir, inversion.NltvParams(*params), lambda a, b: seen.append((a, b)), ctx=ctx64)
    ref, steps = O.nltv(f, m, og(grid), bdir, O.NltvParams(*params), lambda a, b: ref_seen.append((a, b)),
                        return_iters=True, exact_dc=True)
    assert rel(got, ref) < 1e-9, rel(got, ref)
    assert ctx64.tv_last_iterations() == steps
    assert seen == ref_seen


@pytest.mark.parametrize("max_iter", [1, 2, 6, 7])
def test_nltv_fixed_steps_f64(ctx64, max_iter):
    """tol = 0: every pass runs max_iter steps (odd and even counts, one-step passes)."""
    grid = Grid.new(24, 20, 18)
    f, m = case(grid, OBLIQUE, 3)
    p = (1e-3, 1.0, 0.0, max_iter, 3)
    got = inversion.nltv(f, m, grid, OBLIQUE, inversion.NltvParams(*p), ctx=ctx64)
    ref = O.nltv(f, m, og(grid), OBLIQUE, O.NltvParams(*p), exact_dc=True)
    assert rel(got, ref) < 1e-9, rel(got, ref)
    assert ctx64.tv_last_iterations() == 3 * max_iter


def test_nltv_mixed(ctx32):
    """The reweighting divides by the largest weight, 1/(min |grad x| + mu 1e-6), set by the
    flattest voxel of the grid, where |grad x| ~ 1e-6 is of the order of single-precision
    error in x.  On this case Gaussian noise of 1e-7 max|x| added to x before each
    reweighting moves the float64 result by 9e-4 (rel-L2); the bound is 1e-3, and a single
    pass (no reweighting) keeps the TV-ADMM bound of 1e-4."""
    grid = Grid.new(32, 28, 24)
    f, m = case(grid, OBLIQUE, 11)
    p = (1e-3, 1.0, 0.0, 20, 3)
    got = inversion.nltv(f, m, grid, OBLIQUE, inversion.NltvParams(*p), ctx=ctx32)
    ref = O.nltv(f, m, og(grid), OBLIQUE, O.NltvParams(*p), exact_dc=True)
    assert rel(got, ref) < 1e-3, rel(got, ref)
    p1 = (1e-3, 1.0, 0.0, 20, 1)
    got = inversion.nltv(f, m, grid, OBLIQUE, inversion.NltvParams(*p1), ctx=ctx32)
    ref = O.nltv(f, m, og(grid), OBLIQUE, O.NltvParams(*p1), exact_dc=True)
    assert rel(got, ref) < 1e-4, rel(got, ref)


def test_nltv_reference_tests(ctx64):
    """src/inversion/nltv.rs:137-163: zero field -> 0; ramp -> finite."""
    n = 8
    grid = Grid.new(n, n, n)
    p = inversion.NltvParams(1e-3, 1.0, 1e-2, 10, 2)
    ones = np.ones((n, n, n), np.uint8)
    assert np.all(np.abs(inversion.nltv(np.zeros((n, n, n)), ones, grid, (0, 0, 1), p, ctx=ctx64)) < 1e-8)
    field = (np.arange(n ** 3, dtype=np.float64) * 0.001).reshape(n, n, n)
    chi = inversion.nltv(field, ones, grid, (0, 0, 1), p, ctx=ctx64)
    assert np.all(np.isfinite(chi))
    ref = O.nltv(field, ones, O.Grid.new(n, n, n), (0, 0, 1), O.NltvParams(1e-3, 1.0, 1e-2, 10, 2), exact_dc=True)
    assert rel(chi, ref) < 1e-9


@pytest.mark.parametrize("max_iter,newton_iter", [(0, 3), (5, 0)])
def test_nltv_no_steps_gives_zero(ctx64, max_iter, newton_iter):
    grid = Grid.new(12, 10, 8)
    f, m = case(grid, (0, 0, 1), 2)
    calls = []
    chi = inversion.nltv(f, m, grid, (0, 0, 1), inversion.NltvParams(1e-3, 1.0, 1e-3, max_iter, newton_iter),
                         lambda a, b: calls.append((a, b)), ctx=ctx64)
    assert np.all(chi == 0.0) and calls == []


def test_pipeline_nltv(ctx64):
    """InversionAlgorithm::Nltv (src/pipeline/inversion.rs:73-77)."""
    grid = Grid.new(24, 20, 18)
    f, m = case(grid, (0, 0, 1), 9)
    md = pipeline.ScanMetadata(grid.dims, grid.voxel_size)
    cfg = pipeline.InversionConfig(algorithm=pipeline.NLTV, nltv=inversion.NltvParams(1e-3, 1.0, 1e-3, 15, 2))
    chi = pipeline.run_dipole_inversion(f, m, md, cfg, ctx=ctx64)
    np.testing.assert_array_equal(chi.ravel(), inversion.nltv(f, m, grid, (0, 0, 1), cfg.nltv, ctx=ctx64).ravel())
