"""Launch shapes of the compile-time Y/Z passes (the autotuner's candidates: a persistent
grid of resident blocks, capped or not, or one block per tile; edge tiles for a narrow
column remainder).  No shape changes any arithmetic, so every one must give bit-identical
TV-ADMM results, and the autotuned default must match the oracle like every other TV path
(reference: src/inversion/tv.rs:63-97, src/inversion/admm.rs:76-145)."""
import numpy as np
import pytest

import qsmgpu
from qsmgpu import Grid, inversion
from oracle import qsm_oracle as O
from test_gpu_rts import case, rel

pytestmark = pytest.mark.gpu

# nx/2 + 1 = 65 and 129 leave one column after the 16- and 8-column tiles (edge tiles);
# 96 and 176 are compile-time lengths in the Y and fused Z roles
GRIDS = [(128, 96, 64), (256, 64, 176)]


def _solve(f, m, grid, p, shape, autotune=True):
    with qsmgpu.Context(0, "mixed") as ctx:
        ctx.set_autotune(autotune)
        ctx.force_launch_shape(shape)
        chi = inversion.tv_admm(f, m, grid, (0.0, 0.0, 1.0), p, ctx=ctx)
        return chi, ctx.autotune_entries()


@pytest.mark.parametrize("dims", GRIDS, ids=["x".join(map(str, d)) for d in GRIDS])
def test_tv_identical_across_launch_shapes(dims):
    grid = Grid.new(*dims)
    f, m = case(grid, (0.0, 0.0, 1.0), sum(dims))
    p = inversion.TvParams(2e-4, 2e-2, 0.0, 12)
    ref, _ = _solve(f, m, grid, p, 0, autotune=False)
    # edge tiles off/on, persistent grid / one block per tile, and a persistent grid
    # capped at two resident blocks per SM (bits 2-5)
    for shape in (0, 1, 2, 3, 2 << 2, (2 << 2) | 1):
        got, _ = _solve(f, m, grid, p, shape)
        assert np.array_equal(got, ref), (shape, rel(got, ref))


@pytest.mark.parametrize("dims", GRIDS, ids=["x".join(map(str, d)) for d in GRIDS])
def test_autotuned_tv_matches_oracle(dims):
    grid = Grid.new(*dims)
    f, m = case(grid, (0.0, 0.0, 1.0), sum(dims) + 1)
    p = inversion.TvParams(2e-4, 2e-2, 0.0, 8)
    got, entries = _solve(f, m, grid, p, -1)
    # the Y passes (both directions) and the fused Z pass were tuned for this grid
    tag = "x".join(map(str, dims)) + ":f32"
    keys = sorted(k for k in entries if k.endswith(tag))
    assert len(keys) == 3, entries
    for k in keys:
        e = entries[k]
        assert e["choice"] in e["us"] and len(e["us"]) >= 4, e
    ref = O.tv_admm(f, m, O.Grid(grid.dims, grid.voxel_size), (0.0, 0.0, 1.0), O.TvParams(2e-4, 2e-2, 0.0, 8))
    assert rel(got, ref) < 1e-4, rel(got, ref)


def test_force_launch_shape_rejects_unknown():
    with qsmgpu.Context(0, "mixed") as ctx:
        with pytest.raises(qsmgpu.QsmError):
            ctx.force_launch_shape(64)
