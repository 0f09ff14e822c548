"""Parity at the benchmark configurations' own sizes, for the kernels the benchmark times.

* Configuration 1 exactly: TV-ADMM (src/inversion/tv.rs:63-97, src/inversion/admm.rs:76-145)
  on the 64^3 ellipsoid phantom in a radius-28 sphere, default TvParams with tol = 0 (250
  iterations), f64 and mixed, against the float64 oracle.
* The 256x256x176 throughput volume: a few TV-ADMM iterations of both precisions against
  the oracle, and the full 250-iteration mixed solve against the f64 GPU solve.
* The base list of compile-time transform lengths {64, 96, 128, 160, 176, 192, 256, 384}
  in a Latin arrangement, so that every compile-time X (r2c / c2r), Y and fused-Z pass of
  the TV-ADMM iteration runs in every role: mixed against f64, mixed with compile-time
  passes against mixed with the runtime engine only, and f64 against the oracle.
* V-SHARP (src/bgremove/vsharp.rs:88-199) on the 256x256x176 chain volume, whose per-radius
  inverse Z pass takes the compile-time operator kernel, against the oracle (masks exactly
  equal) and against the runtime engine.

Oracle runs at full size use scipy.fft with every host core."""
import math
import os

import numpy as np
import pytest

from qsmgpu import Grid, bgremove, inversion, phantom
from oracle import qsm_oracle as O

pytestmark = pytest.mark.gpu

BASE = [64, 96, 128, 160, 176, 192, 256, 384]
LATIN = [(BASE[i], BASE[(i + 3) % 8], BASE[(i + 5) % 8]) for i in range(8)]
OBLIQUE = (math.sin(0.3) * math.cos(1.1), math.sin(0.3) * math.sin(1.1), math.cos(0.3))


def rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


@pytest.fixture(scope="module")
def fast_oracle():
    O.set_fft_workers(os.cpu_count() or 1)
    yield
    O.set_fft_workers(None)


@pytest.fixture(scope="module")
def config1():
    case = phantom.tv_case_64(0)
    grid = Grid.new(64, 64, 64)
    ref = O.tv_admm(case.local_field, case.mask, O.Grid(grid.dims, grid.voxel_size), (0, 0, 1),
                    O.TvParams(2e-4, 2e-2, 0.0, 250))
    return case, grid, ref


@pytest.mark.parametrize("prec,tol", [("f64", 1e-9), ("mixed", 1e-4)])
def test_config1_tv_admm_64cubed_250_iterations(request, config1, prec, tol):
    ctx = request.getfixturevalue("ctx64" if prec == "f64" else "ctx32")
    case, grid, ref = config1
    got = inversion.tv_admm(case.local_field, case.mask, grid, (0, 0, 1), inversion.TvParams(2e-4, 2e-2, 0.0, 250),
                            ctx=ctx)
    assert ctx.tv_last_iterations() == 250
    e = rel(got, ref)
    print(f"\n{prec}: rel-L2 {e:.2e}, max-abs {np.abs(got - ref).max():.2e}")
    assert e < tol, e
    assert np.all(got[case.mask == 0] == 0.0)


@pytest.fixture(scope="module")
def brain():
    f, m = phantom.brain_tv_case(0)
    return f, m, Grid.new(256, 256, 176)


@pytest.fixture(scope="module")
def brain_oracle5(brain, fast_oracle):
    f, m, grid = brain
    return O.tv_admm(f, m, O.Grid(grid.dims, grid.voxel_size), (0, 0, 1), O.TvParams(2e-4, 2e-2, 0.0, 5))


@pytest.mark.parametrize("prec,tol", [("f64", 1e-9), ("mixed", 1e-4)])
def test_brain_256x256x176_vs_oracle(request, brain, brain_oracle5, prec, tol):
    ctx = request.getfixturevalue("ctx64" if prec == "f64" else "ctx32")
    f, m, grid = brain
    got = inversion.tv_admm(f, m, grid, (0, 0, 1), inversion.TvParams(2e-4, 2e-2, 0.0, 5), ctx=ctx)
    e = rel(got, brain_oracle5)
    print(f"\n{prec}: 5 iterations, rel-L2 {e:.2e}")
    assert e < tol, e


def test_brain_256x256x176_mixed_vs_f64_250(ctx32, ctx64, brain):
    f, m, grid = brain
    p = inversion.TvParams(2e-4, 2e-2, 0.0, 250)
    got = inversion.tv_admm(f, m, grid, (0, 0, 1), p, ctx=ctx32)
    ref = inversion.tv_admm(f, m, grid, (0, 0, 1), p, ctx=ctx64)
    e = rel(got, ref)
    print(f"\nmixed vs f64, 250 iterations: rel-L2 {e:.2e}, max-abs {np.abs(got - ref).max():.2e}")
    assert e < 1e-4, e


def test_brain_compiled_vs_runtime_passes(ctx32, brain):
    f, m, grid = brain
    p = inversion.TvParams(2e-4, 2e-2, 0.0, 20)
    got = inversion.tv_admm(f, m, grid, (0, 0, 1), p, ctx=ctx32)
    ctx32.plan_mode = "runtime"
    try:
        ref = inversion.tv_admm(f, m, grid, (0, 0, 1), p, ctx=ctx32)
    finally:
        ctx32.plan_mode = "compiled"
    assert rel(got, ref) < 1e-6, rel(got, ref)


def test_latin_base_list_covers_every_role():
    for axis in range(3):
        assert sorted(g[axis] for g in LATIN) == BASE


def _latin_case(dims):
    grid = Grid.new(*dims, 1.0, 0.9, 1.2)
    from test_gpu_rts import case
    f, m = case(grid, OBLIQUE, sum(dims))
    return grid, f, m


@pytest.mark.parametrize("dims", LATIN, ids=["x".join(map(str, d)) for d in LATIN])
def test_tv_base_list_mixed(ctx32, ctx64, dims):
    """Mixed (compile-time passes) against f64 (runtime Y/Z, compile-time X) and against
    mixed with every pass on the runtime engine."""
    grid, f, m = _latin_case(dims)
    p = inversion.TvParams(2e-4, 2e-2, 0.0, 10)
    got = inversion.tv_admm(f, m, grid, OBLIQUE, p, ctx=ctx32)
    f64 = inversion.tv_admm(f, m, grid, OBLIQUE, p, ctx=ctx64)
    assert rel(got, f64) < 1e-4, rel(got, f64)
    ctx32.plan_mode = "runtime"
    try:
        rt = inversion.tv_admm(f, m, grid, OBLIQUE, p, ctx=ctx32)
    finally:
        ctx32.plan_mode = "compiled"
    assert rel(got, rt) < 1e-6, rel(got, rt)


@pytest.mark.parametrize("dims", LATIN, ids=["x".join(map(str, d)) for d in LATIN])
def test_tv_base_list_f64_vs_oracle(ctx64, fast_oracle, dims):
    """The f64 iteration's compile-time X passes at every base length against the oracle."""
    grid, f, m = _latin_case(dims)
    got = inversion.tv_admm(f, m, grid, OBLIQUE, inversion.TvParams(2e-4, 2e-2, 0.0, 3), ctx=ctx64)
    ref = O.tv_admm(f, m, O.Grid(grid.dims, grid.voxel_size), OBLIQUE, O.TvParams(2e-4, 2e-2, 0.0, 3),
                    exact_dc=True)
    assert rel(got, ref) < 1e-9, rel(got, ref)


@pytest.fixture(scope="module")
def chain_field():
    case = phantom.chain_case()
    grid = Grid.new(*case.dims)
    og = O.Grid(grid.dims, grid.voxel_size)
    field = O.laplacian_unwrap(case.wrapped_phase, case.mask, og) / case.rad_per_ppm
    return np.ascontiguousarray(field), np.ascontiguousarray(case.mask), grid


RADII = [12.0, 6.0, 2.0]


@pytest.fixture(scope="module")
def vsharp_oracle(chain_field, fast_oracle):
    field, mask, grid = chain_field
    return O.vsharp_with_radii(field, mask, O.Grid(grid.dims, grid.voxel_size), RADII, 0.05)


@pytest.mark.parametrize("prec,tol", [("f64", 1e-9), ("mixed", 1e-5)])
def test_vsharp_256x256x176_vs_oracle(request, chain_field, vsharp_oracle, prec, tol):
    ctx = request.getfixturevalue("ctx64" if prec == "f64" else "ctx32")
    field, mask, grid = chain_field
    local, fmask = bgremove.vsharp_with_radii(field, mask, grid, RADII, 0.05, ctx=ctx)
    ref_local, ref_mask = vsharp_oracle
    np.testing.assert_array_equal(fmask.reshape(ref_mask.shape), ref_mask)
    e = rel(local, ref_local)
    print(f"\n{prec}: V-SHARP rel-L2 {e:.2e}")
    assert e < tol, e


def test_vsharp_256x256x176_compiled_vs_runtime(ctx32, chain_field):
    field, mask, grid = chain_field
    a, ma = bgremove.vsharp_with_radii(field, mask, grid, RADII, 0.05, ctx=ctx32)
    ctx32.plan_mode = "runtime"
    try:
        b, mb = bgremove.vsharp_with_radii(field, mask, grid, RADII, 0.05, ctx=ctx32)
    finally:
        ctx32.plan_mode = "compiled"
    np.testing.assert_array_equal(ma, mb)
    assert rel(a, b) < 1e-6, rel(a, b)
