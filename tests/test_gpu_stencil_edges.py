"""TV-ADMM in mixed precision on grids that exercise the edges of the staged float
stencil: x extents whose 16-byte vectors do not fill a 32-lane row, row counts that
are not a multiple of the 8-row tile, z extents shorter than a z-chunk (down to one
plane), and x extents that are not a multiple of 4 (the unstaged kernel).  Each result
is compared with the float64 oracle at the mixed-precision tolerance and with the FP64
GPU result."""
import math

import numpy as np
import pytest

from qsmgpu import Grid, inversion
from oracle import qsm_oracle as O
from test_gpu_rts import case, rel

pytestmark = pytest.mark.gpu

OBLIQUE = (math.sin(0.35) * math.cos(0.8), math.sin(0.35) * math.sin(0.8), math.cos(0.35))


@pytest.mark.parametrize("dims", [(36, 27, 13), (100, 45, 7), (8, 9, 3), (16, 8, 1), (4, 1, 5), (132, 18, 2),
                                  (20, 11, 9), (30, 14, 6)])
def test_tv_mixed_edges(ctx32, ctx64, dims):
    grid = Grid.new(*dims, 1.0, 1.1, 0.9)
    f, m = case(grid, OBLIQUE, sum(dims))
    if m.sum() == 0:
        m[...] = 1
    p = inversion.TvParams(2e-4, 2e-2, 0.0, 12)
    got = inversion.tv_admm(f, m, grid, OBLIQUE, p, ctx=ctx32)
    f64 = inversion.tv_admm(f, m, grid, OBLIQUE, p, ctx=ctx64)
    ref = O.tv_admm(f, m, O.Grid(grid.dims, grid.voxel_size), OBLIQUE, O.TvParams(2e-4, 2e-2, 0.0, 12), exact_dc=True)
    assert rel(f64, ref) < 1e-9, rel(f64, ref)
    assert rel(got, ref) < 1e-4, rel(got, ref)


def test_tv_mixed_early_exit_near_f64_iterations(ctx32, ctx64):
    """With tol > 0 the staged stencil's FP64 convergence sums stop at (nearly) the same
    iteration as the FP64 path: single-precision iterates can move a relative change that
    sits right at tol by one iteration."""
    grid = Grid.new(44, 27, 21)
    f, m = case(grid, (0, 0, 1), 5)
    p = inversion.TvParams(1e-3, 0.1, 2e-2, 80)
    inversion.tv_admm(f, m, grid, (0, 0, 1), p, ctx=ctx64)
    n64 = ctx64.tv_last_iterations()
    inversion.tv_admm(f, m, grid, (0, 0, 1), p, ctx=ctx32)
    assert n64 < 80 and abs(ctx32.tv_last_iterations() - n64) <= 1
