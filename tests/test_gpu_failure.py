"""Failure paths, exercised without faulting the GPU.

* Injected allocation failure (qsm_ctx_inject_alloc_failure): the failure is simulated
  on the host, the call returns QSM_ERR_ALLOC with a message, and the same context then
  solves correctly.
* Input check (qsm_ctx_set_input_check): off by default, as in the reference, where a
  NaN in the field propagates into the result (compared with the oracle); when on, a
  NaN or infinite voxel is rejected with QSM_ERR_INVALID_ARGUMENT before any solve.
"""
import math

import numpy as np
import pytest

import qsmgpu
from qsmgpu import Grid, bgremove, inversion, unwrap
from oracle import qsm_oracle as O

pytestmark = pytest.mark.gpu

OBLIQUE = (math.sin(0.3) * math.cos(1.1), math.sin(0.3) * math.sin(1.1), math.cos(0.3))


def case(dims=(24, 20, 18), seed=0):
    from test_gpu_rts import case as c
    grid = Grid.new(*dims)
    f, m = c(grid, OBLIQUE, seed)
    return grid, f, m


@pytest.mark.parametrize("prec", ["f64", "mixed"])
@pytest.mark.parametrize("after", [0, 2, 5])
def test_injected_alloc_failure_then_recovery(prec, after):
    grid, f, m = case()
    p = inversion.TvParams(2e-4, 2e-2, 0.0, 10)
    with qsmgpu.Context(0, prec) as ctx:
        ctx.inject_alloc_failure(after)
        with pytest.raises(qsmgpu.QsmError) as e:
            inversion.tv_admm(f, m, grid, OBLIQUE, p, ctx=ctx)
        assert e.value.status == 4  # QSM_ERR_ALLOC
        assert "alloc" in str(e.value).lower()
        got = inversion.tv_admm(f, m, grid, OBLIQUE, p, ctx=ctx)
    with qsmgpu.Context(0, prec) as fresh:
        want = inversion.tv_admm(f, m, grid, OBLIQUE, p, ctx=fresh)
    np.testing.assert_array_equal(got, want)


def test_injected_alloc_failure_cancelled():
    grid, f, m = case()
    with qsmgpu.Context(0, "f64") as ctx:
        ctx.inject_alloc_failure(0)
        ctx.inject_alloc_failure(-1)
        out = inversion.tkd(f, m, grid, OBLIQUE, ctx=ctx)
        assert np.all(np.isfinite(out))


def test_nan_propagates_like_the_reference_when_unchecked(ctx64):
    grid, f, m = case(seed=3)
    f = f.copy()
    f[9, 10, 11] = np.nan
    got = inversion.tkd(f, m, grid, OBLIQUE, inversion.TkdParams(0.19), ctx=ctx64)
    ref = O.tkd(f, m, O.Grid(grid.dims, grid.voxel_size), OBLIQUE, O.TkdParams(0.19))
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    assert np.isnan(got).any()


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_input_check_rejects_non_finite_voxels(bad):
    grid, f, m = case(seed=4)
    f = f.copy()
    f[1, 2, 3] = bad
    f[5, 6, 7] = bad
    ph = np.angle(np.exp(1j * 30.0 * np.nan_to_num(f, posinf=0.0, neginf=0.0)))
    ph[0, 0, 0] = bad
    with qsmgpu.Context(0, "mixed") as ctx:
        ctx.set_input_check(True)
        calls = [lambda: inversion.tv_admm(f, m, grid, OBLIQUE, inversion.TvParams(max_iter=5), ctx=ctx),
                 lambda: inversion.tkd(f, m, grid, OBLIQUE, ctx=ctx),
                 lambda: inversion.rts(f, m, grid, OBLIQUE, ctx=ctx),
                 lambda: inversion.ilsqr(f, m, grid, OBLIQUE, ctx=ctx),
                 lambda: bgremove.vsharp(f, m, grid, ctx=ctx),
                 lambda: unwrap.laplacian_unwrap(ph, m, grid, ctx=ctx)]
        for call in calls:
            with pytest.raises(qsmgpu.QsmError) as e:
                call()
            assert e.value.status == 1 and "non-finite" in str(e.value)
        # finite input still solves on the same context
        good = np.nan_to_num(f, nan=0.0, posinf=0.0, neginf=0.0)
        out = inversion.tkd(good, m, grid, OBLIQUE, ctx=ctx)
        assert np.all(np.isfinite(out))
