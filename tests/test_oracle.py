"""Pin the CPU oracle against the reference's own unit tests (known answers and properties).

Every check here restates a test from astewartau/QSM.rs (file:line in each docstring);
the numeric known answers live in tests/golden/reference_known_answers.json.
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import qsm_oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_known_answers.json")))


def g(n, vs=(1.0, 1.0, 1.0)):
    return O.Grid.new(n, n, n, *vs)


def test_fftfreq_known_answers():
    """src/fft.rs:724-739."""
    for case in GOLD["fftfreq"]:
        np.testing.assert_allclose(O.fftfreq(case["n"], case["d"]), case["values"], atol=case["tol"])
        np.testing.assert_allclose(O.fftfreq(case["n"], case["d"]), np.fft.fftfreq(case["n"], case["d"]),
                                   atol=1e-15)


def test_fft_roundtrip():
    """src/fft.rs:692-721: fft -> ifft roundtrip < 1e-10."""
    x = np.arange(64, dtype=np.float64).reshape(4, 4, 4)
    np.testing.assert_allclose(O.ifft3d(O.fft3d(x)).real, x, atol=1e-10)


def test_shrink_known_answers():
    """src/inversion/tv.rs:105-110."""
    for c in GOLD["shrink"]:
        assert abs(float(O.shrink(c["x"], c["t"])) - c["value"]) < 1e-10


def test_wrap_known_answers():
    """src/unwrap/laplacian.rs:172-179."""
    for c in GOLD["wrap"]:
        assert abs(float(O.wrap(c["x_over_pi"] * math.pi)) - c["value_over_pi"] * math.pi) < 1e-10


def test_laplacian_kernel_facts():
    """src/kernels/laplacian.rs:78-98: sums to 0, centre -6, negative flips sign."""
    c = GOLD["laplacian_kernel"]
    lk = O.laplacian_kernel(g(c["n"]), False)
    assert abs(lk.sum() - c["sum"]) < c["tol"]
    assert abs(lk.ravel()[0] - c["center"]) < c["tol"]
    np.testing.assert_allclose(lk + O.laplacian_kernel(g(c["n"]), True), 0.0, atol=1e-10)


def test_smv_kernel_facts():
    """src/kernels/smv.rs:174-192."""
    a, b = GOLD["smv_kernel"]
    assert abs(O.smv_kernel(g(a["n"]), a["radius"]).sum() - a["sum"]) < a["tol"]
    assert O.smv_kernel(g(16), 2.0).ravel()[0] > 0
    assert int((O.smv_kernel(g(b["n"]), b["radius"]) > 0).sum()) == b["nonzero_count"]


def test_dipole_kernel_facts():
    """src/kernels/dipole.rs:145-185: DC = 0, range [-2/3, 1/3], point symmetry."""
    c = GOLD["dipole_kernel"]
    assert abs(O.dipole_kernel(g(c["n_dc"]), (0, 0, 1)).ravel()[0]) < c["tol"]
    d = O.dipole_kernel(g(c["n_range"]), (0, 0, 1)).ravel()
    assert np.all(d[1:] >= c["min"] - 1e-10) and np.all(d[1:] <= c["max"] + 1e-10)
    n = 8
    dd = O.dipole_kernel(g(n), (0, 0, 1))
    for i in range(1, n // 2):
        for j in range(1, n // 2):
            for k in range(1, n // 2):
                assert abs(dd[k, j, i] - dd[n - k, n - j, n - i]) < 1e-10


def test_grad_constant_and_adjoint():
    """src/utils/gradient.rs:573-621: grad(const) = 0 and <grad x, h> = <x, -div h>."""
    grid = g(4)
    gx, gy, gz = O.fgrad(np.ones(grid.shape), grid)
    assert np.abs(gx).max() < 1e-10 and np.abs(gy).max() < 1e-10 and np.abs(gz).max() < 1e-10
    idx = np.arange(64, dtype=np.float64)
    x = (idx * 0.1).reshape(grid.shape)
    hx = np.sin(idx * 0.2).reshape(grid.shape)
    hy = np.cos(idx * 0.3).reshape(grid.shape)
    hz = np.sin(idx * 0.1).reshape(grid.shape)
    gx, gy, gz = O.fgrad(x, grid)
    lhs = (gx * hx).sum() + (gy * hy).sum() + (gz * hz).sum()
    rhs = -(x * O.bdiv(hx, hy, hz, grid)).sum()
    assert abs(lhs - rhs) / (abs(lhs) + abs(rhs) + 1e-10) < GOLD["grad_div_adjoint"]["rel_tol"]


def test_tv_admm_properties():
    """src/inversion/tv.rs:112-160: zero field -> 0, finite output."""
    grid = g(8)
    p = O.TvParams(1e-3, 0.1, 1e-2, 10)
    mask = np.ones(grid.shape, np.uint8)
    assert np.abs(O.tv_admm(np.zeros(grid.shape), mask, grid, (0, 0, 1), p)).max() < 1e-8
    f = (np.arange(512) * 0.001).reshape(grid.shape)
    assert np.all(np.isfinite(O.tv_admm(f, mask, grid, (0, 0, 1), p)))


def test_tv_admm_progress_contract():
    """src/inversion/tv.rs:80-91: progress(iter+1, max) per iteration, (it, it) on convergence."""
    grid = g(8)
    f = np.sin(np.arange(512) * 0.7).reshape(grid.shape) * 0.01
    calls = []
    out, iters = O.tv_admm(f, np.ones(grid.shape, np.uint8), grid, (0, 0, 1), O.TvParams(1e-3, 0.1, 1e-1, 50),
                           lambda a, b: calls.append((a, b)), return_iters=True)
    assert calls[:iters] == [(i + 1, 50) for i in range(iters)]
    if iters < 50:
        assert calls[-1] == (iters, iters)


def test_tkd_tsvd_properties():
    """src/inversion/tkd.rs:160-224."""
    grid = g(8)
    m = np.ones(grid.shape, np.uint8)
    assert np.abs(O.tkd(np.zeros(grid.shape), m, grid, (0, 0, 1))).max() < 1e-10
    m2 = m.copy().ravel()
    m2[0] = m2[1] = 0
    chi = O.tkd(np.ones(grid.shape), m2.reshape(grid.shape), grid, (0, 0, 1)).ravel()
    assert chi[0] == 0.0 and chi[1] == 0.0
    assert np.all(np.isfinite(O.tkd((np.arange(512) * 0.01).reshape(grid.shape), m, grid, (0, 0, 1))))
    g16 = g(16)
    f = np.sin(np.arange(16 ** 3) * 0.1).reshape(g16.shape)
    m16 = np.ones(g16.shape, np.uint8)
    assert np.abs(O.tkd(f, m16, g16, (0, 0, 1)) - O.tsvd(f, m16, g16, (0, 0, 1))).sum() > 1e-10


def test_tikhonov_properties():
    """src/inversion/tikhonov.rs:144-195."""
    grid = g(8)
    m = np.ones(grid.shape, np.uint8)
    assert np.abs(O.tikhonov(np.zeros(grid.shape), m, grid, (0, 0, 1))).max() < 1e-10
    f = np.sin(np.arange(512) * 0.1).reshape(grid.shape)
    ci = O.tikhonov(f, m, grid, (0, 0, 1), O.TikhonovParams(0.01, O.REG_IDENTITY))
    cg = O.tikhonov(f, m, grid, (0, 0, 1), O.TikhonovParams(0.01, O.REG_GRADIENT))
    cl = O.tikhonov(f, m, grid, (0, 0, 1), O.TikhonovParams(0.01, O.REG_LAPLACIAN))
    assert np.abs(ci - cg).sum() > 1e-10 and np.abs(cg - cl).sum() > 1e-10


def test_laplacian_unwrap_properties():
    """src/unwrap/laplacian.rs:181-230."""
    grid = g(8)
    m = np.ones(grid.shape, np.uint8)
    u = O.laplacian_unwrap(np.ones(grid.shape), m, grid)
    assert np.abs(u - u.mean()).max() < 1e-6
    g16 = g(16)
    i = np.arange(16)
    ph = np.broadcast_to(0.5 * np.sin(2 * np.pi * i / 16)[None, None, :], g16.shape).copy()
    u = O.laplacian_unwrap(ph, np.ones(g16.shape, np.uint8), g16)
    assert np.all(np.isfinite(u)) and np.abs(ph - u).max() < 1.0
    ph = O.wrap(np.arange(512) * 0.1).reshape(grid.shape)
    assert np.all(np.isfinite(O.laplacian_unwrap(ph, m, grid)))


def test_sharp_properties():
    """src/bgremove/sharp.rs:137-170."""
    grid = g(16)
    m = np.ones(grid.shape, np.uint8)
    local, _ = O.sharp(np.zeros(grid.shape), m, grid, O.SharpParams(0.05, 2.0))
    assert np.abs(local).max() < 1e-8
    local, er = O.sharp((np.arange(16 ** 3) * 0.01).reshape(grid.shape), m, grid, O.SharpParams(0.05, 2.0))
    assert np.all(np.isfinite(local)) and er.sum() > 0


def test_vsharp_properties():
    """src/bgremove/vsharp.rs:205-461."""
    grid = g(8)
    m = np.ones(grid.shape, np.uint8)
    local, _ = O.vsharp_with_radii(np.zeros(grid.shape), m, grid, [4.0, 3.0, 2.0], 0.05)
    assert np.abs(local).max() < 1e-10
    g16 = g(16)
    m16 = np.ones(g16.shape, np.uint8)
    _, vm = O.vsharp_with_radii(np.zeros(g16.shape), m16, g16, [5.0, 4.0, 3.0, 2.0], 0.05)
    _, sm = O.sharp_core(np.zeros(g16.shape), m16, g16, 0.05, 5.0)
    assert vm.sum() >= sm.sum()
    ga = O.Grid.new(8, 8, 8, 0.5, 1.0, 2.0)
    f = (np.arange(512) * 0.001).reshape(ga.shape)
    local, fm = O.vsharp_with_radii(f, m, ga, [4.0, 3.0, 2.0], 0.05)
    assert np.all(np.isfinite(local)) and fm.sum() > 0
    # single radius == SHARP
    c = GOLD["vsharp_single_radius_equals_sharp"]
    f = (np.arange(512) * 0.001).reshape(grid.shape)
    l1, m1 = O.vsharp_with_radii(f, m, grid, [c["radius"]], c["threshold"])
    l2, m2 = O.sharp_core(f, m, grid, c["threshold"], c["radius"])
    assert np.abs(l1 - l2).max() < c["tol"] and np.array_equal(m1, m2)
    # sorted == unsorted
    s = GOLD["vsharp_sorted_equals_unsorted"]
    la, ma = O.vsharp_with_radii(f, m, grid, s["radii_sorted"], 0.05)
    lb, mb = O.vsharp_with_radii(f, m, grid, s["radii_unsorted"], 0.05)
    assert np.array_equal(ma, mb) and np.abs(la - lb).max() < 1e-10
    # empty radii -> zeros and the input mask
    le, me = O.vsharp_with_radii(f, m, grid, [], 0.05)
    assert np.all(le == 0) and np.array_equal(me, m)


def test_vsharp_radii_list():
    """src/bgremove/vsharp.rs:70-82: defaults give 12, 11, ..., 1."""
    assert O.vsharp_radii(O.VsharpParams()) == [float(r) for r in range(12, 0, -1)]


def test_cg_known_answers():
    """src/solvers/cg.rs:109-138."""
    for c in GOLD["cg"]:
        d = np.asarray(c["diag"])
        x = O.cg_solve(lambda v: v * d, c["b"], np.zeros(3), 1e-10, 100)
        np.testing.assert_allclose(x, c["x"], atol=c["tol"])


def test_next_fast_fft_size():
    """src/utils/padding.rs:9-25."""
    assert O.next_fast_fft_size(97) == 100
    assert O.next_fast_fft_size(176) == 180
    assert O.next_fast_fft_size(64) == 64


def test_nyquist_symmetrised_multiplier_matches_c2c():
    """The half-spectrum GPU path applies (M(k)+M(-k))/2; for real input this equals the
    reference's C2C multiply followed by Re() (src/fft.rs:514-540), including oblique B0
    on even-length Nyquist planes."""
    grid = O.Grid.new(8, 6, 10)
    rng = np.random.default_rng(1)
    x = rng.standard_normal(grid.shape)
    b = (math.sin(0.4), 0.2, math.cos(0.4))
    M = O.dipole_kernel(grid, b)
    ref = O.ifft3d(O.fft3d(x) * M).real
    Mm = np.roll(np.flip(M, axis=(0, 1, 2)), 1, axis=(0, 1, 2))  # M(-k)
    sym = O.ifft3d(O.fft3d(x) * 0.5 * (M + Mm)).real
    np.testing.assert_allclose(sym, ref, atol=1e-14)
    # the unsymmetrised half-spectrum product would differ
    half = np.fft.irfftn(np.fft.rfftn(x) * M[:, :, :5], s=grid.shape, axes=(0, 1, 2))
    assert np.abs(half - ref).max() > 1e-3


# ---------------------------------------------------------------------------- iLSQR --
def test_lsqr_real_diagonal():
    """src/inversion/ilsqr.rs:1357-1372: diag(1..10) x = 2*diag -> x = 2."""
    d = np.arange(1, 11, dtype=np.float64)
    x = O.lsqr_real(lambda v: v * d, lambda v: v * d, d * 2.0, 1e-10, 100)
    assert np.all(np.abs(x - 2.0) < 1e-6)


def test_norm_and_sign_known_answers():
    """src/inversion/ilsqr.rs:1374-1385: norm([3,4]) = 5; sign([-2,0,3]) = [-1,0,1]."""
    assert abs(float(np.linalg.norm([3.0, 4.0])) - 5.0) < 1e-10
    assert list(np.sign([-2.0, 0.0, 3.0])) == [-1.0, 0.0, 1.0]


def test_lsqr_complex_relres_stop():
    """src/inversion/ilsqr.rs:1387-1432: diag(1,10,100,1000), tol 1e-6 -> relres <= 10*tol."""
    d = np.array([1.0, 10.0, 100.0, 1000.0])
    b = (d * d).astype(np.complex128)
    x = O.lsqr_complex(lambda v: v * d, lambda v: v * d, b, 1e-6, 200)
    assert np.linalg.norm(x * d - b) / np.linalg.norm(b) <= 1e-5


def test_lsqr_complex_diagonal():
    """src/inversion/ilsqr.rs:1434-1465: diag(1,2,3), x = [1+i, 2+i, 3+i]."""
    d = np.array([1.0, 2.0, 3.0])
    e = np.array([1 + 1j, 2 + 1j, 3 + 1j])
    x = O.lsqr_complex(lambda v: v * d, lambda v: v * d, e * d, 1e-10, 100)
    assert np.all(np.abs(x.real - e.real) < 1e-6) and np.all(np.abs(x.imag - e.imag) < 1e-6)


def test_lsmr_identity():
    """src/inversion/ilsqr.rs:1467-1492: identity, b = [3,5,7]: finite, residual < ||b||."""
    b = np.array([3.0, 5.0, 7.0])
    x = O.lsmr(lambda v: v.copy(), lambda v: v.copy(), b, 3, 1e-6, 1e-6, 200)
    assert x.shape == (3,) and np.all(np.isfinite(x))
    assert np.linalg.norm(x - b) < np.linalg.norm(b)
    np.testing.assert_allclose(x, b, atol=1e-12)  # one iteration solves the identity exactly


def test_prctile_linear_interpolation():
    """src/inversion/ilsqr.rs:937-946 (MATLAB-style linear interpolation)."""
    v = np.sort(np.array([4.0, 1.0, 3.0, 2.0, 5.0]))
    assert O.prctile(v, 50.0) == 3.0
    assert O.prctile(v, 10.0) == 1.4
    assert O.prctile(v, 100.0) == 5.0
    assert O.prctile(np.array([7.0]), 30.0) == 7.0 and O.prctile(np.array([]), 30.0) == 0.0
    r = np.random.default_rng(0).standard_normal(1001)
    for p in (1.0, 30.0, 60.0, 99.9):
        assert abs(O.prctile(np.sort(r), p) - np.percentile(r, p)) < 1e-12


def _sphere44():
    n = 4
    mask = np.zeros((n, n, n), np.uint8)
    f = np.zeros((n, n, n))
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    r2 = (i - 1.5) ** 2 + (j - 1.5) ** 2 + (k - 1.5) ** 2
    mask[r2 < 2.5] = 1
    f[r2 < 2.5] = 5.0
    return f, mask


def test_laplacian_weights_known_properties():
    """src/inversion/ilsqr.rs:1494-1536: constant field in a 4^3 sphere, weights in [0,1],
    0 outside the mask."""
    f, mask = _sphere44()
    w = O.laplacian_weights_ilsqr(f, mask, g(4), 10.0, 90.0)
    assert np.all(np.isfinite(w)) and np.all((w >= 0) & (w <= 1))
    assert np.all(w[mask == 0] == 0.0)
    # the Laplacian of a constant is zero everywhere, so every weight is 0 (range <= 1e-10)
    assert np.all(O.ilsqr_laplacian(f, mask, g(4)) == 0.0)


def test_lap1_stencils_follow_mask():
    """src/inversion/ilsqr.rs:583-669: central / 4th-order one-sided / 2nd-order / first
    difference chosen by the mask, checked on a 1-D profile along x."""
    grid = O.Grid.new(8, 1, 1)
    x = np.arange(8, dtype=np.float64)
    f = (x ** 3).reshape(1, 1, 8)
    m = np.ones((1, 1, 8), np.uint8)
    lap = O._lap1_axis(f, m, 2, 1.0).ravel()
    # interior central difference of x^3 is 6x; the ends use the 4th-order one-sided forms
    np.testing.assert_allclose(lap[1:7], 6.0 * x[1:7])
    assert lap[0] == 2 * 0 - 5 * 1 + 4 * 8 - 27 and lap[7] == -(4 ** 3) + 4 * 125 - 5 * 216 + 2 * 343
    m2 = m.copy()
    m2[0, 0, 5] = 0  # voxel 4 loses its forward neighbour: backward 4th order
    lap2 = O._lap1_axis(f, m2, 2, 1.0).ravel()
    assert lap2[4] == -(1 ** 3) + 4 * 8 - 5 * 27 + 2 * 64
    assert grid.n_total() == 8


def test_dipole_kspace_weights_known_properties():
    """src/inversion/ilsqr.rs:1538-1559."""
    d = np.array([0.0, 0.01, 0.1, 0.3, 0.5, 0.7, 1.0, -0.5, -1.0, 0.0])
    w = O.dipole_kspace_weights_ilsqr(d, 1.0, 1.0, 90.0)
    assert np.all((w >= 0) & (w <= 1))
    assert w[0] <= 1e-10 and w[6] > 0.5 and w[8] > 0.5


def test_gradient_weights_known_properties():
    """src/inversion/ilsqr.rs:1561-1600: linear field in x, full mask."""
    n = 4
    f = np.tile(np.arange(n, dtype=np.float64), (n, n, 1))
    mask = np.ones((n, n, n), np.uint8)
    gx, gy, gz = O.fgrad_masked(f, mask, g(n))
    for comp in (gx, gy, gz):
        w = O._percentile_weights(comp, mask, 10.0, 90.0, True)
        assert np.all(np.isfinite(w)) and np.all((w >= 0) & (w <= 1))
    assert np.all(gx == 1.0) and np.all(gy == 0.0) and np.all(gz == 0.0)


def ilsqr_small_case():
    """The 8^3 sphere case of src/inversion/ilsqr.rs:1602-1681."""
    n = 8
    c = (n - 1) / 2.0
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    di, dj, dk = i - c, j - c, k - c
    r2 = di * di + dj * dj + dk * dk
    mask = (r2 < 9.0).astype(np.uint8)
    field = np.where(mask > 0, 0.01 * (dk * dk - di * di - dj * dj) / (r2 + 1.0), 0.0)
    return field, mask


def test_ilsqr_small():
    """src/inversion/ilsqr.rs:1602-1681: finite, zero outside the mask, not all zero inside."""
    field, mask = ilsqr_small_case()
    seen = []
    chi, xsa, xfs, xlsqr = O.ilsqr(field, mask, g(8), (0, 0, 1), O.IlsqrParams(0.1, 5),
                                   progress=lambda a, b: seen.append((a, b)))
    assert chi.shape == field.shape and np.all(np.isfinite(chi))
    assert np.all(chi[mask == 0] == 0.0)
    assert np.abs(chi[mask > 0]).sum() > 0.0
    assert seen == [(1, 4), (2, 4), (3, 4), (4, 4)]  # src/inversion/ilsqr.rs:1324-1343
    np.testing.assert_array_equal(chi, np.where(mask > 0, xlsqr - xsa, 0.0))


def _ilsqr_phantom():
    """24x20x18 ellipsoid-mask phantom at (1, 1.2, 0.9) mm with an oblique field."""
    rng = np.random.default_rng(5)
    nx, ny, nz = 24, 20, 18
    grid = O.Grid.new(nx, ny, nz, 1.0, 1.2, 0.9)
    bdir = (math.sin(0.35) * math.cos(0.8), math.sin(0.35) * math.sin(0.8), math.cos(0.35))
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = ((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2)
    mask = ((i - c[0]) / (0.4 * nx)) ** 2 + ((j - c[1]) / (0.4 * ny)) ** 2 + ((k - c[2]) / (0.4 * nz)) ** 2 < 1.0
    chi = np.zeros(grid.shape)
    for _ in range(6):
        p = [rng.uniform(0.3, 0.7) * s for s in (nx, ny, nz)]
        r = rng.uniform(1.5, 3.5)
        chi[((i - p[0]) ** 2 + (j - p[1]) ** 2 + (k - p[2]) ** 2) < r * r] = rng.uniform(-0.1, 0.2)
    chi *= mask
    d = O.dipole_kernel(grid, bdir)
    f = np.fft.ifftn(d * np.fft.fftn(chi)).real + rng.normal(0, 0.01, grid.shape) * mask
    return f, mask.astype(np.uint8), grid, bdir


def test_ilsqr_krylov_steps_amplify_rounding():
    """Why mixed-precision iLSQR keeps its Krylov steps in FP64.  The reference's LSQR step
    (src/inversion/ilsqr.rs:953-1030) stops at relres 0.01 or 50 iterations; on this phantom
    it runs all 50 and its iterate is far (> 10%) from the converged least-squares
    solution, so the result is the truncated Krylov iterate itself:
      * relative noise of 1e-7 (float rounding) on every FFT output moves the outputs by
        more than 1e-4, while the same noise on the input field alone moves them by ~1e-7:
        the Krylov recurrences amplify per-operation rounding about a thousandfold;
      * an outer iterative-refinement step (FP64 residual b - A x, truncated LSQR on it)
        converges towards the least-squares solution and away from the reference's iterate.
    """
    f, mask, grid, bdir = _ilsqr_phantom()
    ref = O.ilsqr(f, mask, grid, bdir, O.IlsqrParams())
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    # input perturbation: small response
    noisy = f * (1 + 1e-7 * np.random.default_rng(1).standard_normal(f.shape))
    r_in = O.ilsqr(noisy, mask, grid, bdir, O.IlsqrParams())
    assert max(rel(a, b) for a, b in zip(r_in, ref)) < 1e-6
    # per-FFT rounding-level noise: amplified by the Krylov steps
    f0, i0 = O.fft3d, O.ifft3d
    rng = np.random.default_rng(0)
    noise = lambda a: a * (1 + 1e-7 * rng.standard_normal(a.shape))
    try:
        O.fft3d = lambda a: noise(f0(a))
        O.ifft3d = lambda a: noise(i0(a))
        r_fft = O.ilsqr(f, mask, grid, bdir, O.IlsqrParams())
    finally:
        O.fft3d, O.ifft3d = f0, i0
    e = {n: rel(a, b) for n, a, b in zip(("chi", "xsa", "xfs", "xlsqr"), r_fft, ref)}
    assert e["xlsqr"] > 1e-4 and e["xsa"] > 1e-4 and e["xfs"] < 1e-6, e
    # truncated LSQR vs converged, and one refinement step
    d = O.dipole_kernel(grid, bdir)
    w = O.laplacian_weights_ilsqr(f, mask, grid)
    b = (O.fft3d((w * f).astype(np.complex128)) * d).ravel()

    def apply_a(x):
        r = O.ifft3d(d * x.reshape(grid.shape)).real
        return (O.fft3d((w * r).astype(np.complex128)) * d).ravel()

    x_ref, iters = O.lsqr_complex(apply_a, apply_a, b, 0.01, 50, return_iters=True)
    x_conv = O.lsqr_complex(apply_a, apply_a, b, 1e-12, 2000)
    assert iters == 50 and rel(x_ref, x_conv) > 0.1
    x_ref1 = x_ref + O.lsqr_complex(apply_a, apply_a, b - apply_a(x_ref), 0.01, 50)
    assert rel(x_ref1, x_ref) > 0.1 and rel(x_ref1, x_conv) < rel(x_ref, x_conv)


# ------------------------------------------------------------------------------ TGV --
def test_tgv_erode_mask():
    """src/inversion/tgv.rs:1335-1347: 5^3 all-ones mask, one erosion keeps the centre."""
    e = O.erode_mask(np.ones((5, 5, 5), np.uint8), 1)
    assert e[2, 2, 2] == 1 and e[0, 0, 0] == 0 and e.sum() == 27


def test_tgv_bounding_box():
    """src/inversion/tgv.rs:1356-1377: 3..7 cube, padding 1 -> [2, 8)."""
    m = np.zeros((10, 10, 10), np.uint8)
    m[3:7, 3:7, 3:7] = 1
    lo, hi = O.tgv_bounding_box(m, 1)
    assert lo[:2] == [2, 2] and hi[:2] == [8, 8]


def test_tgv_oblique_stencil_properties():
    """src/inversion/tgv.rs:1439-1490: sum ~0, centre = -sum(others), anisotropic case."""
    st = O.tgv_oblique_stencil((1.0, 1.0, 1.0), (0.0, 0.0, 1.0))
    assert abs(float(st.astype(np.float64).sum())) < 1e-4
    off = float(st.sum() - st[1, 1, 1])
    assert abs(float(st[1, 1, 1]) + off) < 1e-6
    st2 = O.tgv_oblique_stencil((1.0, 1.0, 2.0), (0.2, 0.3, 0.9))
    assert abs(float(st2.astype(np.float64).sum())) < 1e-4
    # centrosymmetric pairs share their coefficient
    np.testing.assert_array_equal(st2, st2[::-1, ::-1, ::-1])


def test_tgv_phase_laplacian_of_constant():
    """src/inversion/tgv.rs:1319-1333: constant phase -> Laplacian ~0 (through tgv_qsm's
    first step: a constant phase gives chi = 0)."""
    n = 8
    mask = np.ones((n, n, n), np.uint8)
    out = O.tgv_qsm(np.ones((n, n, n)), mask, O.Grid.new(n, n, n), O.TgvParams(iterations=3, erosions=1))
    assert np.all(np.abs(out) < 1e-12)


def _tgv_small_case():
    n = 12
    c = 6.0
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    mask = (np.sqrt((i - c) ** 2 + (j - c) ** 2 + (k - c) ** 2) < 4.0).astype(np.uint8)
    phase = np.where(mask > 0, 0.1 * k, 0.0)
    return phase, mask


def test_tgv_qsm_small():
    """src/inversion/tgv.rs:1379-1437: 12^3 sphere, z ramp, 10 iterations, 1 erosion."""
    phase, mask = _tgv_small_case()
    r = O.tgv_qsm(phase, mask, O.Grid.new(12, 12, 12), O.TgvParams(iterations=10, erosions=1))
    assert r.shape == (12, 12, 12) and np.all(np.isfinite(r)) and np.any(np.abs(r) > 1e-20)


def test_tgv_convergence_progress():
    """src/inversion/tgv.rs:1562-1599: zero phase, tol 1.1 -> stops at the first check
    (iteration 100); progress is 0..100 then (100, 1000)."""
    _, mask = _tgv_small_case()
    seen = []
    r = O.tgv_qsm(np.zeros(mask.shape), mask, O.Grid.new(12, 12, 12), O.TgvParams(iterations=1000, erosions=1,
                                                                                   tol=1.1),
                  progress=lambda a, b: seen.append((a, b)))
    assert seen[:101] == [(t, 1000) for t in range(101)] and seen[101:] == [(100, 1000)]
    assert np.all(r == 0.0)


def test_resharp_reference_tests():
    """src/bgremove/resharp.rs:159-190: zero field -> ~0; ramp field -> finite, eroded mask
    not empty."""
    n = 16
    grid = O.Grid.new(n, n, n)
    p = O.ResharpParams(2.0, 1e-4, 1e-6, 50)
    local, _ = O.resharp(np.zeros((n, n, n)), np.ones((n, n, n), np.uint8), grid, p)
    assert np.all(np.abs(local) < 1e-8)
    field = (np.arange(n ** 3, dtype=np.float64) * 0.01).reshape(n, n, n)
    local, eroded = O.resharp(field, np.ones((n, n, n), np.uint8), grid, p)
    assert np.all(np.isfinite(local)) and eroded.sum() > 0


def test_apply_reference_known_answers():
    """src/pipeline/referencing.rs:49-82."""
    np.testing.assert_allclose(O.apply_reference([1.0, 2.0, 3.0, 4.0], [1, 1, 1, 0]), [-1.0, 0.0, 1.0, 0.0], atol=1e-10)
    assert list(O.apply_reference([1.0, 2.0, 3.0], [1, 0, 1], "none")) == [1.0, 0.0, 3.0]
    assert list(O.apply_reference([1.0, 2.0], [0, 0])) == [0.0, 0.0]


def test_rts_reference_tests():
    """src/inversion/rts.rs:213-263: zero field -> ~0; ramp -> finite; masked voxels zero."""
    n = 8
    grid = g(n)
    p = O.RtsParams(0.15, 1e5, 10.0, 1e-2, 5, 2)
    assert np.all(np.abs(O.rts(np.zeros((n, n, n)), np.ones((n, n, n), np.uint8), grid, (0, 0, 1), p)) < 1e-6)
    field = (np.arange(n ** 3, dtype=np.float64) * 0.001).reshape(n, n, n)
    mask = np.ones(n ** 3, np.uint8)
    mask[0] = 0
    mask[10] = 0
    chi = O.rts(field, mask.reshape(n, n, n), grid, (0, 0, 1), p)
    assert np.all(np.isfinite(chi)) and chi.ravel()[0] == 0.0 and chi.ravel()[10] == 0.0


@pytest.mark.parametrize("solver", ["tv", "rts"])
def test_laplacian_dc_roundoff_is_a_constant_offset(solver):
    """src/inversion/admm.rs:159-167 and src/inversion/rts.rs:93-113 take the Laplacian's
    eigenvalues from an FFT of its taps, so at voxel sizes whose taps do not sum to exactly
    0 in floating point the DC eigenvalue is a few ulp and inv_a(0) is ~1e17.  The effect
    is confined to k = 0: the faithful iterate and the one with the exact eigenvalue 0
    differ by a constant over the grid, i.e. inside the mask."""
    grid = O.Grid.new(24, 28, 16, 1.0, 1.0, 0.9)
    lap = O.laplacian_eigenvalues(grid)
    assert lap[0, 0, 0] != 0.0 and abs(lap[0, 0, 0]) < 1e-14
    assert O.laplacian_eigenvalues(grid, exact_dc=True)[0, 0, 0] == 0.0
    rng = np.random.default_rng(5)
    mask = np.zeros(grid.shape, np.uint8)
    mask[3:13, 4:24, 4:20] = 1
    f = rng.normal(0, 0.01, grid.shape) * mask
    if solver == "tv":
        run = lambda e: O.tv_admm(f, mask, grid, (0, 0, 1), O.TvParams(2e-4, 2e-2, 0.0, 6), exact_dc=e)
    else:
        run = lambda e: O.rts(f, mask, grid, (0, 0, 1), O.RtsParams(0.15, 1e5, 10.0, 0.0, 6, 4), exact_dc=e)
    faithful, exact = run(False), run(True)
    diff = (faithful - exact)[mask != 0]
    assert abs(diff.mean()) > 1e-6 * np.abs(exact).max()  # the roundoff does move the DC term
    assert np.abs(diff - diff.mean()).max() < 1e-9 * np.abs(exact).max()
    assert np.all((faithful - exact)[mask == 0] == 0.0)


def test_nltv_reference_tests():
    """src/inversion/nltv.rs:137-177: zero field -> 0, ramp -> finite, weighted_shrink."""
    n = 8
    grid = g(n)
    p = O.NltvParams(1e-3, 1.0, 1e-2, 10, 2)
    ones = np.ones((n, n, n), np.uint8)
    assert np.all(np.abs(O.nltv(np.zeros((n, n, n)), ones, grid, (0, 0, 1), p)) < 1e-8)
    field = (np.arange(n ** 3, dtype=np.float64) * 0.001).reshape(n, n, n)
    assert np.all(np.isfinite(O.nltv(field, ones, grid, (0, 0, 1), p)))
    ws = lambda x, t, w: float(O.shrink(x, t * w))
    assert abs(ws(1.0, 0.5, 1.0) - 0.5) < 1e-10 and abs(ws(-1.0, 0.5, 1.0) + 0.5) < 1e-10
    assert abs(ws(0.3, 0.5, 1.0)) < 1e-10
    assert abs(ws(1.0, 0.5, 0.5) - 0.75) < 1e-10 and abs(ws(0.3, 0.5, 0.5) - 0.05) < 1e-10


def test_nltv_single_pass_is_weighted_tv():
    """With one outer pass the weights stay 1, so NLTV is TV-ADMM with rho = 100 lambda
    (src/inversion/nltv.rs:76-106 against src/inversion/tv.rs:63-97)."""
    grid = O.Grid.new(12, 10, 8)
    rng = np.random.default_rng(2)
    f = rng.normal(0, 0.01, grid.shape)
    m = np.ones(grid.shape, np.uint8)
    a = O.nltv(f, m, grid, (0, 0, 1), O.NltvParams(2e-3, 1.0, 0.0, 7, 1))
    b = O.tv_admm(f, m, grid, (0, 0, 1), O.TvParams(2e-3, 0.2, 0.0, 7))
    assert np.abs(a - b).max() < 1e-14


def test_nltv_progress_contract():
    """progress(k, max_iter * newton_iter) before every inner step; no (k, k) call."""
    grid = g(8)
    f = np.sin(np.arange(512) * 0.7).reshape(grid.shape) * 0.01
    calls = []
    _, k = O.nltv(f, np.ones(grid.shape, np.uint8), grid, (0, 0, 1), O.NltvParams(1e-3, 1.0, 5e-2, 20, 3),
                  lambda a, b: calls.append((a, b)), return_iters=True)
    assert calls == [(i + 1, 60) for i in range(k)] and k < 60


def _ball_mask(n, radius):
    c = n // 2
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    return (((i - c) ** 2 + (j - c) ** 2 + (k - c) ** 2) <= radius * radius).astype(np.uint8)


def test_ismv_reference_tests():
    """src/bgremove/ismv.rs:163-420: zero field; finite; interior kept; larger radius
    erodes more; linear background on a 16^3 sphere."""
    grid = g(8)
    ones = np.ones(grid.shape, np.uint8)
    local, er = O.ismv(np.zeros(grid.shape), ones, grid, O.IsmvParams(1e-3, 10, 2.0))
    assert np.abs(local).max() < 1e-10 and er.sum() > 0
    ramp = (np.arange(512) * 0.001).reshape(grid.shape)
    assert np.all(np.isfinite(O.ismv(ramp, ones, grid, O.IsmvParams(1e-3, 20, 2.0))[0]))
    g16 = g(16)
    sph = _ball_mask(16, 16 // 3)
    _, er = O.ismv(np.full(g16.shape, 0.1), sph, g16, O.IsmvParams(1e-3, 50, 1.5))
    assert 0 < er.sum() <= sph.sum()
    _, es = O.ismv(ramp, ones, grid, O.IsmvParams(1e-3, 20, 1.5))
    _, el = O.ismv(ramp, ones, grid, O.IsmvParams(1e-3, 20, 3.0))
    assert el.sum() <= es.sum()
    z = np.arange(16)[:, None, None] * 0.1 * np.ones(g16.shape)
    local, er = O.ismv(z, sph, g16, O.IsmvParams(1e-3, 50, 2.0))
    assert local.shape == g16.shape and np.all(np.isfinite(local))
    assert np.all(local[sph == 0] == 0.0)


def test_ismv_progress_contract():
    """(iter+1, max) per iteration; (iter+1, iter+1) when the change falls below tol."""
    grid = g(8)
    calls = []
    O.ismv(np.zeros(grid.shape), np.ones(grid.shape, np.uint8), grid, O.IsmvParams(1e-3, 10, 2.0),
           lambda a, b: calls.append((a, b)))
    assert calls == [(1, 10), (1, 1)]
    g16 = g(16)
    f = np.sin(np.arange(16 ** 3) * 0.01).reshape(g16.shape)
    calls = []
    _, _, it = O.ismv(f, _ball_mask(16, 6), g16, O.IsmvParams(1e-2, 200, 2.0), lambda a, b: calls.append((a, b)),
                      return_iters=True)
    assert it < 200 and calls == [(i + 1, 200) for i in range(it + 1)] + [(it + 1, it + 1)]


def test_calculate_b0_weighted_reference_tests():
    """src/utils/multi_echo.rs:1153-1263."""
    tes = [0.005, 0.010, 0.015]
    ph = [np.full(64, 200.0 * te) for te in tes]
    b0 = O.calculate_b0_weighted(ph, [np.ones(64)] * 3, tes, np.ones(64, np.uint8), O.B0W_PHASE_SNR)
    assert np.all(np.abs(b0 - 200.0 / (2 * math.pi)) < 1e-8)
    ph = [np.full(16, 100.0 * te) for te in tes]
    for wt in range(5):
        b0 = O.calculate_b0_weighted(ph, [np.full(16, 2.0)] * 3, tes, np.ones(16, np.uint8), wt)
        assert np.all(np.abs(b0 - 100.0 / (2 * math.pi)) < 1e-8)
    b0 = O.calculate_b0_weighted([np.full(8, 500 * te) for te in tes[:2]], [np.ones(8)] * 2, tes[:2],
                                 np.zeros(8, np.uint8))
    assert np.all(b0 == 0.0)
    ph = [np.full(4, 0.2 * te) for te in tes]
    assert np.all(O.calculate_b0_weighted(ph, [np.zeros(4)] * 3, tes, np.ones(4, np.uint8)) == 0.0)
    b0 = O.calculate_b0_weighted(ph, [np.zeros(4)] * 3, tes, np.ones(4, np.uint8), O.B0W_AVERAGE)
    assert np.all(np.abs(b0 - 0.2 / (2 * math.pi)) < 1e-8)


def test_multi_echo_linear_fit_reference_tests():
    """src/utils/multi_echo.rs:1267-1491."""
    tes = [0.005, 0.010, 0.015]
    f, o, r, rm = O.multi_echo_linear_fit([np.full(32, 100.0 * te) for te in tes], [np.ones(32)] * 3, tes,
                                          np.ones(32, np.uint8), False, 0.0)
    assert np.all(np.abs(f - 100.0) < 1e-6) and np.all(o == 0.0) and np.all(r < 1e-10) and np.all(rm == 1)
    tes4 = [0.005, 0.010, 0.015, 0.020]
    f, o, r, _ = O.multi_echo_linear_fit([np.full(16, 0.5 + 200.0 * te) for te in tes4], [np.ones(16)] * 4, tes4,
                                         np.ones(16, np.uint8), True, 0.0)
    assert np.all(np.abs(f - 200.0) < 1e-4) and np.all(np.abs(o - 0.5) < 1e-4) and np.all(r < 1e-8)
    f, o, r, _ = O.multi_echo_linear_fit([np.full(8, 100.0 * te) for te in tes], [np.ones(8)] * 3, tes,
                                         np.zeros(8, np.uint8), True, 0.0)
    assert np.all(f == 0) and np.all(o == 0) and np.all(r == 0)
    slopes = 50.0 * (np.arange(8) + 1.0)
    f, _, _, _ = O.multi_echo_linear_fit([slopes * te for te in tes], [np.ones(8)] * 3, tes, np.ones(8, np.uint8),
                                         False, 0.0)
    assert np.all(np.abs(f - slopes) < 1e-6)
    ph = [np.full(100, 100.0 * te) for te in tes]
    for e in range(3):
        ph[e][90:] += 2.0 if e % 2 == 0 else -2.0
    _, _, r, rm = O.multi_echo_linear_fit(ph, [np.ones(100)] * 3, tes, np.ones(100, np.uint8), False, 80.0)
    assert r[:90].max() < r[90:].min() and set(np.unique(rm)) <= {0, 1}
    for off in (False, True):
        f, _, _, _ = O.multi_echo_linear_fit([np.full(4, 100.0 * te) for te in tes], [np.zeros(4)] * 3, tes,
                                             np.ones(4, np.uint8), off, 0.0)
        assert np.all(np.isfinite(f))
    rm = O.compute_reliability_mask(np.arange(1, 11) * 0.1, np.ones(10, np.uint8), 50.0)
    assert 0 < rm.sum() < 10
    assert np.array_equal(O.compute_reliability_mask(np.zeros(5), np.ones(5, np.uint8), 50.0), np.ones(5))
