"""GPU parity of conjugate gradients (src/solvers/cg.rs:34-101) with the fixed operator
A x = H^T H x + lambda x, and of RESHARP (src/bgremove/resharp.rs:58-125) built on it,
against the float64 oracle.  FP64: rel-L2 1e-9 (CG amplifies transform rounding
mildly); mixed: 1e-4.  Eroded masks: exact."""
import math

import numpy as np
import pytest
import torch

import qsmgpu
from qsmgpu import Grid, bgremove, pipeline
from oracle import qsm_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def og(grid: Grid):
    return O.Grid(grid.dims, grid.voxel_size)


def field_case(grid, seed):
    rng = np.random.default_rng(seed)
    nz, ny, nx = grid.shape
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = ((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2)
    mask = (((i - c[0]) / (0.4 * nx)) ** 2 + ((j - c[1]) / (0.4 * ny)) ** 2 + ((k - c[2]) / (0.4 * nz)) ** 2 < 1)
    bg = 0.05 * (i - c[0]) / nx + 0.02 * ((j - c[1]) / ny) ** 2
    local = np.zeros(grid.shape)
    for _ in range(5):
        p = [rng.uniform(0.3, 0.7) * s for s in (nx, ny, nz)]
        local[(i - p[0]) ** 2 + (j - p[1]) ** 2 + (k - p[2]) ** 2 < 9] += rng.uniform(-0.02, 0.02)
    f = (bg + local) * mask + rng.normal(0, 1e-3, grid.shape) * mask
    return np.ascontiguousarray(f), np.ascontiguousarray(mask.astype(np.uint8))


@pytest.mark.parametrize("dims,vs", [((24, 20, 18), (1.0, 1.0, 1.0)), ((15, 9, 25), (1.0, 1.2, 0.9))])
def test_cg_kspace_normal_f64(ctx64, dims, vs):
    grid = Grid.new(*dims, *vs)
    rng = np.random.default_rng(3)
    K = O.fft_real_kernel(O.smv_kernel(og(grid), 2.0))
    K = 1.0 - K  # an even, real multiplier (RESHARP's)
    w = (rng.random(grid.shape) < 0.7).astype(np.float64)
    b = rng.standard_normal(grid.shape)
    x0 = 0.1 * rng.standard_normal(grid.shape)
    lam, tol, it = 1e-2, 1e-8, 40
    seen = []
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).ravel()).cuda()
    dK, dw, db, dx0 = dev(K), dev(w), dev(b), dev(x0)
    dx = torch.empty_like(db)
    bgremove.cg_kspace_normal_device(ctx64, grid, dK.data_ptr(), dw.data_ptr(), lam, db.data_ptr(), dx0.data_ptr(),
                                     tol, it, dx.data_ptr(), progress=lambda a, c: seen.append(a))
    ref_seen = []
    op = lambda v: (O.apply_ht_h(K, w, v.reshape(grid.shape)) + lam * v.reshape(grid.shape)).ravel()
    ref = O.cg_solve(op, b.ravel(), x0.ravel(), tol, it, lambda a, c: ref_seen.append(a))
    assert rel(dx.cpu().numpy(), ref) < 1e-9, rel(dx.cpu().numpy(), ref)
    assert seen == ref_seen


@pytest.mark.parametrize("dims,vs,radius", [((32, 28, 24), (1.0, 1.0, 1.0), 4.0), ((30, 22, 26), (1.0, 1.1, 0.9), 3.0)])
def test_resharp_f64(ctx64, dims, vs, radius):
    grid = Grid.new(*dims, *vs)
    f, m = field_case(grid, sum(dims))
    p = bgremove.ResharpParams(radius=radius)
    seen = []
    local, em = bgremove.resharp(f, m, grid, p, progress=lambda a, b: seen.append((a, b)), ctx=ctx64)
    ref_seen = []
    rl, rm = O.resharp(f, m, og(grid), O.ResharpParams(radius=radius),
                       progress=lambda a, b: ref_seen.append((a, b)))
    np.testing.assert_array_equal(em.reshape(rm.shape), rm)
    assert rel(local, rl) < 1e-9, rel(local, rl)
    assert seen == ref_seen


def test_resharp_mixed(ctx32):
    grid = Grid.new(32, 28, 24)
    f, m = field_case(grid, 7)
    local, em = bgremove.resharp(f, m, grid, bgremove.ResharpParams(radius=4.0), ctx=ctx32)
    rl, rm = O.resharp(f, m, og(grid), O.ResharpParams(radius=4.0))
    np.testing.assert_array_equal(em.reshape(rm.shape), rm)
    assert rel(local, rl) < 1e-4, rel(local, rl)


def test_resharp_reference_tests(ctx64):
    """src/bgremove/resharp.rs:159-190."""
    n = 16
    grid = Grid.new(n, n, n)
    p = bgremove.ResharpParams(2.0, 1e-4, 1e-6, 50)
    local, _ = bgremove.resharp(np.zeros((n, n, n)), np.ones((n, n, n), np.uint8), grid, p, ctx=ctx64)
    assert np.all(np.abs(local) < 1e-8)
    field = (np.arange(n ** 3, dtype=np.float64) * 0.01).reshape(n, n, n)
    local, eroded = bgremove.resharp(field, np.ones((n, n, n), np.uint8), grid, p, ctx=ctx64)
    assert np.all(np.isfinite(local)) and eroded.sum() > 0


def test_resharp_pipeline_dispatch(ctx64):
    grid = Grid.new(24, 20, 18)
    f, m = field_case(grid, 11)
    md = pipeline.ScanMetadata(grid.dims, grid.voxel_size)
    cfg = pipeline.BgRemovalConfig(algorithm=pipeline.RESHARP)
    res = pipeline.run_bg_removal(f, m, md, cfg, ctx=ctx64)
    local, em = bgremove.resharp(f, m, grid, bgremove.ResharpParams(), ctx=ctx64)
    np.testing.assert_array_equal(res.local_field_ppm.ravel(), local.ravel())
    np.testing.assert_array_equal(res.eroded_mask.ravel(), em.ravel())
