"""TV-ADMM in mixed precision on grids whose axis lengths take the compile-time FFT
passes of the wide length list (5- and 7-smooth lengths from 72 to 240, used by the
TV-ADMM iteration only).  The 21 grids are a Latin arrangement of the 21 lengths, so
each length runs once as the X (r2c / c2r), once as the Y and once as the fused Z axis.
Each mixed result is compared with the FP64 GPU path, which has no compile-time plans
(runtime Stockham engine) and is pinned to the oracle by the other TV tests; two of the
grids are also compared with the float64 oracle directly."""
import math

import numpy as np
import pytest

from qsmgpu import Grid, inversion
from oracle import qsm_oracle as O
from test_gpu_rts import case, rel

pytestmark = pytest.mark.gpu

WIDE = [72, 75, 80, 81, 90, 100, 108, 112, 120, 125, 135, 144, 150, 162, 168, 180, 200, 216, 224, 225, 240]
GRIDS = [(WIDE[i], WIDE[(i + 7) % 21], WIDE[(i + 14) % 21]) for i in range(21)]
OBLIQUE = (math.sin(0.3) * math.cos(1.1), math.sin(0.3) * math.sin(1.1), math.cos(0.3))


def test_latin_arrangement_covers_every_role():
    for axis in range(3):
        assert sorted(g[axis] for g in GRIDS) == WIDE


@pytest.mark.parametrize("dims", GRIDS, ids=["x".join(map(str, d)) for d in GRIDS])
def test_tv_mixed_wide_plans_vs_fp64(ctx32, ctx64, dims):
    grid = Grid.new(*dims, 1.0, 0.9, 1.2)
    f, m = case(grid, OBLIQUE, sum(dims))
    p = inversion.TvParams(2e-4, 2e-2, 0.0, 10)
    got = inversion.tv_admm(f, m, grid, OBLIQUE, p, ctx=ctx32)
    f64 = inversion.tv_admm(f, m, grid, OBLIQUE, p, ctx=ctx64)
    assert rel(got, f64) < 1e-4, rel(got, f64)


@pytest.mark.parametrize("dims", [(75, 81, 72), (112, 90, 100)])
def test_tv_mixed_wide_plans_vs_oracle(ctx32, dims):
    grid = Grid.new(*dims)
    f, m = case(grid, (0, 0, 1), 11)
    p = inversion.TvParams(2e-4, 2e-2, 0.0, 8)
    got = inversion.tv_admm(f, m, grid, (0, 0, 1), p, ctx=ctx32)
    ref = O.tv_admm(f, m, O.Grid(grid.dims, grid.voxel_size), (0, 0, 1), O.TvParams(2e-4, 2e-2, 0.0, 8),
                    exact_dc=True)
    assert rel(got, ref) < 1e-4, rel(got, ref)
    assert np.all(got[m == 0] == 0.0)
