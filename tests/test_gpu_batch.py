"""Batched TV-ADMM and TKD over volumes of uneven size and field direction (one call,
one CUDA graph per two iterations for the whole batch).  Each volume's result must equal
the single-volume call bit for bit, and the float64 oracle within the usual tolerances.
The batch follows the structure of the 32-volume benchmark case at sizes the oracle
finishes in seconds."""
import math

import numpy as np
import pytest
import torch

from qsmgpu import Grid, inversion
from oracle import qsm_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def fast_size(n):
    """Smallest 2^a 3^b 5^c >= n (src/utils/padding.rs:9)."""
    m = n
    while True:
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
        m += 1


def batch_cases(n, lo=(20, 20, 14), hi=(40, 40, 30), seed=0):
    rng = np.random.default_rng(seed)
    cases = []
    for _ in range(n):
        dims = tuple(fast_size(int(rng.integers(l, h + 1))) for l, h in zip(lo, hi))
        grid = Grid.new(*dims)
        th, ph = math.radians(rng.uniform(0, 25)), rng.uniform(0, 2 * math.pi)
        bdir = (math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th))
        nz, ny, nx = grid.shape
        k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        c = ((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2)
        mask = ((i - c[0]) / (0.4 * nx)) ** 2 + ((j - c[1]) / (0.4 * ny)) ** 2 + ((k - c[2]) / (0.4 * nz)) ** 2 < 1
        chi = np.zeros(grid.shape)
        for _ in range(5):
            p = [rng.uniform(0.3, 0.7) * s for s in (nx, ny, nz)]
            r = rng.uniform(1.5, 3.0)
            chi[(i - p[0]) ** 2 + (j - p[1]) ** 2 + (k - p[2]) ** 2 < r * r] = rng.uniform(-0.1, 0.2)
        chi *= mask
        d = O.dipole_kernel(O.Grid(grid.dims, grid.voxel_size), bdir)
        f = np.fft.ifftn(d * np.fft.fftn(chi)).real + rng.normal(0, 0.01, grid.shape) * mask
        cases.append((np.ascontiguousarray(f), np.ascontiguousarray(mask.astype(np.uint8)), grid, bdir))
    return cases


@pytest.mark.parametrize("prec,tol", [("f64", 1e-9), ("mixed", 1e-4)])
def test_tv_admm_batch_matches_single_and_oracle(request, prec, tol):
    ctx = request.getfixturevalue("ctx64" if prec == "f64" else "ctx32")
    cases = batch_cases(6, seed=1)
    p = inversion.TvParams(tol=0.0, max_iter=41)  # odd: the last iteration runs outside the graph
    seen = []
    outs, iters = inversion.tv_admm_batch(cases, p, progress=lambda a, b: seen.append((a, b)), ctx=ctx)
    assert iters == [41] * len(cases)
    assert seen[-1] == (len(cases), len(cases))
    for (f, m, g, b), chi in zip(cases, outs):
        single = inversion.tv_admm(f, m, g, b, p, ctx=ctx)
        np.testing.assert_array_equal(chi, single)
        ref = O.tv_admm(f, m, O.Grid(g.dims, g.voxel_size), b, O.TvParams(tol=0.0, max_iter=41))
        assert rel(chi, ref) < tol, rel(chi, ref)


def test_tv_admm_batch_early_exit_per_volume(ctx64):
    """With tol > 0 every volume stops at its own iteration, as a single call does."""
    cases = batch_cases(5, seed=2)
    p = inversion.TvParams(tol=2e-3, max_iter=200)
    outs, iters = inversion.tv_admm_batch(cases, p, ctx=ctx64)
    for (f, m, g, b), chi, it in zip(cases, outs, iters):
        single = inversion.tv_admm(f, m, g, b, p, ctx=ctx64)
        np.testing.assert_array_equal(chi, single)
        assert it == ctx64.tv_last_iterations()
        assert it < 200


def test_tkd_batch_device(ctx32):
    cases = batch_cases(4, seed=3)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).ravel()).cuda()
    keep, dcases = [], []
    for f, m, g, b in cases:
        df, dm = dev(f), dev(m)
        do = torch.empty_like(df)
        keep += [df, dm, do]
        dcases.append((df.data_ptr(), dm.data_ptr(), do.data_ptr(), g, b))
    p = inversion.TkdParams(0.19)
    inversion.tkd_batch_device(ctx32, dcases, p)
    for (f, m, g, b), (_, _, do, _, _), t in zip(cases, dcases, keep[2::3]):
        np.testing.assert_array_equal(t.cpu().numpy().reshape(f.shape), inversion.tkd(f, m, g, b, p, ctx=ctx32))
