"""GPU parity of iSMV background removal (src/bgremove/ismv.rs:48-166) against the
float64 oracle: FP64 rel-L2 1e-10 with the same iteration count and progress sequence,
mixed 1e-5; eroded masks exact (the 1 - 1e-10 erosion runs in double in both
precisions)."""
import numpy as np
import pytest

from qsmgpu import Grid, bgremove, pipeline
from oracle import qsm_oracle as O
from test_gpu_cg_resharp import field_case, og, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims,vs,params", [
    ((32, 28, 24), (1.0, 1.0, 1.0), (1e-6, 50, 5.0)),    # the defaults: stops after 19
    ((30, 26, 22), (1.0, 1.1, 1.3), (1e-3, 200, 3.0)),   # stops after 21
    ((25, 27, 15), (0.9, 1.0, 1.2), (1e-2, 200, 2.5)),   # stops after 13
    ((25, 27, 15), (0.9, 1.0, 1.2), (1e-14, 12, 2.5)),   # runs to max_iter
])
def test_ismv_f64(ctx64, dims, vs, params):
    grid = Grid.new(*dims, *vs)
    f, m = field_case(grid, sum(dims))
    seen, ref_seen = [], []
    lo, mo = bgremove.ismv(f, m, grid, bgremove.IsmvParams(*params), lambda a, b: seen.append((a, b)), ctx=ctx64)
    lr, mr, _ = O.ismv(f, m, og(grid), O.IsmvParams(*params), lambda a, b: ref_seen.append((a, b)),
                       return_iters=True)
    assert np.array_equal(np.asarray(mo).ravel(), mr.ravel())
    assert rel(lo, lr) < 1e-10, rel(lo, lr)
    assert seen == ref_seen


def test_ismv_mixed(ctx32):
    grid = Grid.new(32, 28, 24)
    f, m = field_case(grid, 4)
    p = (1e-6, 50, 4.0)
    lo, mo = bgremove.ismv(f, m, grid, bgremove.IsmvParams(*p), ctx=ctx32)
    lr, mr = O.ismv(f, m, og(grid), O.IsmvParams(*p))
    assert np.array_equal(np.asarray(mo).ravel(), mr.ravel())
    assert rel(lo, lr) < 1e-5, rel(lo, lr)


def test_ismv_reference_tests(ctx64):
    """src/bgremove/ismv.rs:163-230: zero field -> 0 with a non-empty eroded mask; finite."""
    grid = Grid.new(8, 8, 8)
    ones = np.ones(grid.shape, np.uint8)
    calls = []
    local, er = bgremove.ismv(np.zeros(grid.shape), ones, grid, bgremove.IsmvParams(1e-3, 10, 2.0),
                              lambda a, b: calls.append((a, b)), ctx=ctx64)
    assert np.abs(local).max() < 1e-10 and np.asarray(er).sum() > 0
    assert calls == [(1, 10), (1, 1)]
    ramp = (np.arange(512) * 0.001).reshape(grid.shape)
    local, _ = bgremove.ismv(ramp, ones, grid, bgremove.IsmvParams(1e-3, 20, 2.0), ctx=ctx64)
    lr, _ = O.ismv(ramp, ones, og(grid), O.IsmvParams(1e-3, 20, 2.0))
    assert np.all(np.isfinite(local)) and rel(local, lr) < 1e-10
    for n_it in (0, 1, 2):
        lo, _ = bgremove.ismv(ramp, ones, grid, bgremove.IsmvParams(1e-9, n_it, 2.0), ctx=ctx64)
        lr, _ = O.ismv(ramp, ones, og(grid), O.IsmvParams(1e-9, n_it, 2.0))
        assert rel(lo, lr) < 1e-10, (n_it, rel(lo, lr))


def test_pipeline_ismv(ctx64):
    """BgRemovalAlgorithm::Ismv (src/pipeline/bg_removal.rs:55-59)."""
    grid = Grid.new(24, 20, 18)
    f, m = field_case(grid, 2)
    md = pipeline.ScanMetadata(grid.dims, grid.voxel_size)
    cfg = pipeline.BgRemovalConfig(algorithm=pipeline.ISMV, ismv=bgremove.IsmvParams(1e-4, 30, 3.0))
    r = pipeline.run_bg_removal(f, m, md, cfg, ctx=ctx64)
    lo, mo = bgremove.ismv(f, m, grid, cfg.ismv, ctx=ctx64)
    np.testing.assert_array_equal(np.asarray(r.local_field_ppm).ravel(), np.asarray(lo).ravel())
    np.testing.assert_array_equal(np.asarray(r.eroded_mask).ravel(), np.asarray(mo).ravel())
