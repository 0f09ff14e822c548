"""Differentiable unrolled TV-ADMM: the hand-written adjoint (vector-Jacobian product)
of K fixed TV-ADMM iterations with checkpointing, wrapped in a torch.autograd.Function,
checked against (1) a float64 torch autograd unrolling of the reference iteration
(src/inversion/tv.rs:63-97, admm.rs:76-178) on the CPU, (2) central finite differences
(h = 1e-3 relative) and (3) the float64 GPU gradient, all within 1e-3 relative for the
mixed-precision adjoint.  The larger case has the benchmark's adjoint shape
(160x192x160, K = 50, checkpoints every 10, lambda ~ logU[1e-4, 1e-2], rho fixed)."""
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


def case(dims, seed, bdir=(0.0, 0.0, 1.0)):
    rng = np.random.default_rng(seed)
    grid = Grid.new(*dims)
    nz, ny, nx = grid.shape
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = ((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2)
    mask = ((i - c[0]) / (0.4 * nx)) ** 2 + ((j - c[1]) / (0.4 * ny)) ** 2 + ((k - c[2]) / (0.4 * nz)) ** 2 < 1
    chi = np.zeros(grid.shape)
    for _ in range(8):
        p = [rng.uniform(0.3, 0.7) * s for s in (nx, ny, nz)]
        a = rng.uniform(2.0, max(3.0, min(nx, ny, nz) / 8), 3)
        chi[((i - p[0]) / a[0]) ** 2 + ((j - p[1]) / a[1]) ** 2 + ((k - p[2]) / a[2]) ** 2 < 1] = rng.uniform(-0.1, 0.2)
    chi *= mask
    d = O.dipole_kernel(O.Grid(grid.dims, grid.voxel_size), bdir)
    f = np.fft.ifftn(d * np.fft.fftn(chi)).real + rng.normal(0, 0.01, grid.shape) * mask
    return grid, np.ascontiguousarray(f), np.ascontiguousarray(mask.astype(np.uint8)), chi


class UnrolledTv(torch.autograd.Function):
    """chi_K = unrolled TV-ADMM(f, lambda) on the GPU; backward calls the library's adjoint."""

    @staticmethod
    def forward(fctx, f, lam, mask, grid, bdir, rho, K, C, qctx):
        out = torch.empty_like(f)
        inversion.tv_admm_unrolled_vjp_device(qctx, f.data_ptr(), mask.data_ptr(), grid, bdir, float(lam), rho, K, C,
                                              0, out.data_ptr())
        fctx.save_for_backward(f, mask)
        fctx.args = (float(lam), grid, bdir, rho, K, C, qctx)
        return out

    @staticmethod
    def backward(fctx, gchi):
        f, mask = fctx.saved_tensors
        lam, grid, bdir, rho, K, C, qctx = fctx.args
        chi = torch.empty_like(f)
        gf = torch.empty_like(f)
        gchi = gchi.contiguous()
        gl = inversion.tv_admm_unrolled_vjp_device(qctx, f.data_ptr(), mask.data_ptr(), grid, bdir, lam, rho, K, C,
                                                   gchi.data_ptr(), chi.data_ptr(), gf.data_ptr())
        return gf, torch.tensor(gl, dtype=torch.float64), None, None, None, None, None, None, None


def torch_unrolled_tv(f, lam, mask, grid, bdir, rho, K):
    """float64 torch restatement of K reference TV-ADMM iterations (full C2C FFTs)."""
    og = O.Grid(grid.dims, grid.voxel_size)
    d = torch.from_numpy(O.dipole_kernel(og, bdir))
    lap = torch.from_numpy(O.fft3d(O.laplacian_kernel(og, True).astype(np.complex128)).real)
    a = d * d + rho * lap
    inv_a = torch.where(a.abs() > 1e-20, 1.0 / a, torch.zeros_like(a))
    h = [1.0 / v for v in grid.voxel_size]
    fhat = torch.fft.fftn(f.to(torch.complex128)) * d * inv_a
    x = torch.zeros_like(f)
    u = [torch.zeros_like(f) for _ in range(3)]
    g = [torch.zeros_like(f) for _ in range(3)]
    t = lam / rho
    axes = (2, 1, 0)
    for _ in range(K):
        div = sum((g[c] - torch.roll(g[c], 1, axes[c])) * h[c] for c in range(3))
        x = torch.fft.ifftn(fhat - rho * torch.fft.fftn(div.to(torch.complex128)) * inv_a).real
        v = [(torch.roll(x, -1, axes[c]) - x) * h[c] + u[c] for c in range(3)]
        z = [torch.where(vc > t, vc - t, torch.where(vc < -t, vc + t, torch.zeros_like(vc))) for vc in v]
        u = [v[c] - z[c] for c in range(3)]
        g = [2.0 * z[c] - v[c] for c in range(3)]
    return x * mask


def loss_and_grads(qctx, grid, f, mask, chi_true, lam, rho, K, C, bdir=(0.0, 0.0, 1.0)):
    ft = torch.from_numpy(f.ravel()).cuda().requires_grad_(True)
    lt = torch.tensor(lam, dtype=torch.float64, requires_grad=True)
    mt = torch.from_numpy(mask.ravel()).cuda()
    chi = UnrolledTv.apply(ft, lt, mt, grid, bdir, rho, K, C, qctx)
    L = ((chi - torch.from_numpy(chi_true.ravel()).cuda()) ** 2).sum()
    L.backward()
    return float(L.detach()), ft.grad.cpu().numpy(), float(lt.grad)


def loss_only(qctx, grid, f, mask, chi_true, lam, rho, K, C, bdir=(0.0, 0.0, 1.0)):
    ft = torch.from_numpy(f.ravel()).cuda()
    mt = torch.from_numpy(mask.ravel()).cuda()
    out = torch.empty_like(ft)
    inversion.tv_admm_unrolled_vjp_device(qctx, ft.data_ptr(), mt.data_ptr(), grid, bdir, lam, rho, K, C, 0,
                                          out.data_ptr())
    return float(((out.cpu().numpy() - chi_true.ravel()) ** 2).sum())


def test_unrolled_forward_equals_tv_admm(ctx32):
    grid, f, mask, _ = case((32, 28, 24), 1)
    K = 9
    ft = torch.from_numpy(f.ravel()).cuda()
    mt = torch.from_numpy(mask.ravel()).cuda()
    out = torch.empty_like(ft)
    inversion.tv_admm_unrolled_vjp_device(ctx32, ft.data_ptr(), mt.data_ptr(), grid, (0, 0, 1), 2e-4, 2e-2, K, 4, 0,
                                          out.data_ptr())
    ref = inversion.tv_admm(f, mask, grid, (0, 0, 1), inversion.TvParams(2e-4, 2e-2, 0.0, K), ctx=ctx32)
    np.testing.assert_array_equal(out.cpu().numpy(), ref.ravel())


@pytest.mark.parametrize("prec,tol", [("f64", 1e-9), ("mixed", 1e-3)])
@pytest.mark.parametrize("K,C", [(12, 5), (7, 7), (1, 3)])
def test_vjp_matches_torch_float64_autograd(request, prec, tol, K, C):
    qctx = request.getfixturevalue("ctx64" if prec == "f64" else "ctx32")
    grid, f, mask, chi_true = case((24, 20, 18), 2)
    lam, rho = 3e-3, 2e-2
    L, gf, gl = loss_and_grads(qctx, grid, f, mask, chi_true, lam, rho, K, C)
    ft = torch.from_numpy(f).requires_grad_(True)
    lt = torch.tensor(lam, dtype=torch.float64, requires_grad=True)
    chi = torch_unrolled_tv(ft, lt, torch.from_numpy(mask.astype(np.float64)), grid, (0.0, 0.0, 1.0), rho, K)
    Lr = ((chi - torch.from_numpy(chi_true)) ** 2).sum()
    Lr.backward()
    assert abs(L - float(Lr.detach())) / float(Lr.detach()) < tol
    assert rel(gf, ft.grad.numpy()) < tol, rel(gf, ft.grad.numpy())
    if lt.grad is None:  # K = 1: the first iterate does not depend on lambda
        assert gl == 0.0
    else:
        assert abs(gl - float(lt.grad)) / abs(float(lt.grad)) < tol, (gl, float(lt.grad))


def _fd_lambda(qctx, grid, f, mask, chi_true, lam, rho, K, C, gl, tol):
    """Central difference in lambda with h = 1e-3 * lambda."""
    h = 1e-3 * lam
    fd_l = (loss_only(qctx, grid, f, mask, chi_true, lam + h, rho, K, C) -
            loss_only(qctx, grid, f, mask, chi_true, lam - h, rho, K, C)) / (2 * h)
    assert abs(gl - fd_l) / abs(fd_l) < tol, (gl, fd_l)


def _fd_field(qctx, grid, f, mask, chi_true, lam, rho, K, C, gf, tol, seed, h_rel=1e-5):
    """Directional central difference in f along a seeded direction.  The unrolled map is
    piecewise linear through the shrink, so the step must stay below the kink spacing: at
    h = 1e-3 relative the float64 torch reference's own central difference differs from
    its autograd by 1.9e-3 on the small case, at 1e-5 by 1.6e-10."""
    delta = np.random.default_rng(seed).standard_normal(f.shape)
    hf = h_rel * np.linalg.norm(f) / np.linalg.norm(delta)
    fd_f = (loss_only(qctx, grid, f + hf * delta, mask, chi_true, lam, rho, K, C) -
            loss_only(qctx, grid, f - hf * delta, mask, chi_true, lam, rho, K, C)) / (2 * hf)
    ad_f = float(np.dot(gf, delta.ravel()))
    assert abs(ad_f - fd_f) / abs(fd_f) < tol, (ad_f, fd_f)


def test_vjp_central_differences_small(ctx64):
    grid, f, mask, chi_true = case((24, 20, 18), 3)
    lam, rho, K, C = 2e-3, 2e-2, 10, 4
    _, gf, gl = loss_and_grads(ctx64, grid, f, mask, chi_true, lam, rho, K, C)
    _fd_lambda(ctx64, grid, f, mask, chi_true, lam, rho, K, C, gl, 1e-3)
    _fd_field(ctx64, grid, f, mask, chi_true, lam, rho, K, C, gf, 1e-6, 3)


def test_vjp_benchmark_shape(ctx32, ctx64):
    """160x192x160, K = 50, checkpoints every 10, lambda ~ logU[1e-4, 1e-2]: the mixed
    adjoint against central differences in lambda (h = 1e-3 relative) and against the
    float64 GPU gradient, which is itself checked by a directional difference in f."""
    rng = np.random.default_rng(4)
    lam = float(10.0 ** rng.uniform(-4, -2))
    rho, K, C = 2e-2, 50, 10
    grid, f, mask, chi_true = case((160, 192, 160), 4)
    _, gf32, gl32 = loss_and_grads(ctx32, grid, f, mask, chi_true, lam, rho, K, C)
    _fd_lambda(ctx32, grid, f, mask, chi_true, lam, rho, K, C, gl32, 1e-3)
    _, gf64, gl64 = loss_and_grads(ctx64, grid, f, mask, chi_true, lam, rho, K, C)
    _fd_field(ctx64, grid, f, mask, chi_true, lam, rho, K, C, gf64, 1e-5, 4)
    assert rel(gf32, gf64) < 1e-3, rel(gf32, gf64)
    assert abs(gl32 - gl64) / abs(gl64) < 1e-3, (gl32, gl64)
