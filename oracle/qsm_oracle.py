"""CPU oracle: a float64 numpy restatement of QSM.rs's FFT-driven reconstruction path.

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA library: only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm may import it.  The product path never calls it.

Parity status
-------------
The reference (astewartau/QSM.rs, Rust) cannot be compiled here (no cargo/rustc,
crates not vendored), and it ships no golden arrays.  This restatement is pinned
against every known-answer and property test the reference's own unit tests hold
for the path (see ``tests/test_oracle.py`` and ``tests/golden/reference_known_answers.json``):
``fftfreq`` values, the Laplacian/SMV/dipole kernel facts, the grad/div adjoint
identity, ``wrap`` values, shrink values, single-radius V-SHARP == SHARP,
sorted == unsorted radii, CG identity/diagonal solves, and so on.  Array-level values
of the reference are therefore pinned only through those tests and through this
line-by-line restatement.

Conventions (same as the reference)
-----------------------------------
* Volumes are Fortran-order flat arrays, index ``i + j*nx + k*nx*ny``
  (``src/fft.rs:236-241``).  Here they are handled as C-order numpy arrays of
  shape ``(nz, ny, nx)``, which has exactly that flat layout.
* FFTs are full complex-to-complex, forward unnormalised and inverse scaled by
  1/N (``src/fft.rs:1-9,197``); numpy's ``fftn``/``ifftn`` use the same definition.
  rustfft 6.4.1 (the reference's third-party FFT, pinned in ``Cargo.lock``) is
  replaced by numpy's pocketfft; both compute the same DFT to rounding.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

PI = math.pi


# ---------------------------------------------------------------------------
# Grid (src/grid.rs:9-44)
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class Grid:
    """Volume dims (nx, ny, nz) and voxel size in mm (src/grid.rs:9-13)."""

    dims: Tuple[int, int, int]
    voxel_size: Tuple[float, float, float] = (1.0, 1.0, 1.0)

    @staticmethod
    def new(nx, ny, nz, vsx=1.0, vsy=1.0, vsz=1.0) -> "Grid":
        return Grid((int(nx), int(ny), int(nz)), (float(vsx), float(vsy), float(vsz)))

    @property
    def nx(self):
        return self.dims[0]

    @property
    def ny(self):
        return self.dims[1]

    @property
    def nz(self):
        return self.dims[2]

    def n_total(self) -> int:  # src/grid.rs:41
        return self.dims[0] * self.dims[1] * self.dims[2]

    @property
    def shape(self):
        """numpy shape (nz, ny, nx) whose C order is the reference's Fortran order."""
        return (self.dims[2], self.dims[1], self.dims[0])


def _vol(a, grid: Grid, dtype=np.float64):
    return np.asarray(a, dtype=dtype).reshape(grid.shape)


# ---------------------------------------------------------------------------
# FFT helpers (src/fft.rs)
# ---------------------------------------------------------------------------
def fftfreq(n: int, d: float) -> np.ndarray:
    """numpy-style frequencies (src/fft.rs:544-566); even n maps index n/2 to -n/2."""
    val = 1.0 / (n * d)
    out = np.zeros(n)
    if n % 2 == 0:
        for i in range(n // 2):
            out[i] = i * val
        for i in range(n // 2, n):
            out[i] = float(i - n) * val
    else:
        for i in range((n - 1) // 2 + 1):
            out[i] = i * val
        for i in range((n + 1) // 2, n):
            out[i] = float(i - n) * val
    return out


_FFT_WORKERS = None


def set_fft_workers(n: Optional[int]) -> None:
    """Use scipy.fft with n threads for the 3D transforms (the reference's Rayon axis
    passes, src/fft.rs:423-479); None restores single-threaded numpy.  Same DFT."""
    global _FFT_WORKERS
    _FFT_WORKERS = n


def fft3d(a: np.ndarray) -> np.ndarray:
    """Forward unnormalised 3D C2C FFT (src/fft.rs:97-141, 412)."""
    if _FFT_WORKERS:
        import scipy.fft
        return scipy.fft.fftn(a, workers=_FFT_WORKERS)
    return np.fft.fftn(a)


def ifft3d(a: np.ndarray) -> np.ndarray:
    """Inverse 3D C2C FFT with 1/N (src/fft.rs:157-209, 485)."""
    if _FFT_WORKERS:
        import scipy.fft
        return scipy.fft.ifftn(a, workers=_FFT_WORKERS)
    return np.fft.ifftn(a)


def fft_real_kernel(kernel: np.ndarray) -> np.ndarray:
    """Re(FFT(kernel)) (src/fft.rs:514-520)."""
    return fft3d(kernel.astype(np.complex128)).real


def apply_real_kernel(x: np.ndarray, kernel_fft: np.ndarray) -> np.ndarray:
    """Re(IFFT(FFT(x) * kernel_fft)) (src/fft.rs:526-540)."""
    return ifft3d(fft3d(x.astype(np.complex128)) * kernel_fft).real


# ---------------------------------------------------------------------------
# k-space kernels (src/kernels/)
# ---------------------------------------------------------------------------
def dipole_kernel(grid: Grid, bdir) -> np.ndarray:
    """D(k) = 1/3 - (k.b)^2/|k|^2, DC -> 0 when |k|^2 <= 1e-20 (src/kernels/dipole.rs:24-72)."""
    nx, ny, nz = grid.dims
    vsx, vsy, vsz = grid.voxel_size
    kx = fftfreq(nx, vsx)[None, None, :]
    ky = fftfreq(ny, vsy)[None, :, None]
    kz = fftfreq(nz, vsz)[:, None, None]
    bx, by, bz = (float(b) for b in bdir)
    bnorm = math.sqrt(bx * bx + by * by + bz * bz)
    bx, by, bz = bx / bnorm, by / bnorm, bz / bnorm
    kdotb = kx * bx + ky * by + kz * bz
    k2 = kx * kx + ky * ky + kz * kz
    with np.errstate(divide="ignore", invalid="ignore"):
        d = (1.0 / 3.0) - (kdotb * kdotb) / k2
    return np.where(k2 > 1e-20, d, 0.0)


def laplacian_kernel(grid: Grid, negative: bool) -> np.ndarray:
    """7-point Laplacian placed at wrap positions (src/kernels/laplacian.rs:20-61)."""
    nx, ny, nz = grid.dims
    vsx, vsy, vsz = grid.voxel_size
    hx, hy, hz = 1.0 / (vsx * vsx), 1.0 / (vsy * vsy), 1.0 / (vsz * vsz)
    center = -2.0 * (hx + hy + hz)
    sign = -1.0 if negative else 1.0
    flat = np.zeros(nx * ny * nz)
    flat[0] = sign * center
    if nx > 1:
        flat[1] = sign * hx
        flat[nx - 1] = sign * hx
    if ny > 1:
        flat[nx] = sign * hy
        flat[(ny - 1) * nx] = sign * hy
    if nz > 1:
        flat[nx * ny] = sign * hz
        flat[(nz - 1) * nx * ny] = sign * hz
    return flat.reshape(grid.shape)


def smv_kernel(grid: Grid, radius: float) -> np.ndarray:
    """Normalised binary sphere at wrap-centred coordinates (src/kernels/smv.rs:19-67)."""
    nx, ny, nz = grid.dims
    vsx, vsy, vsz = grid.voxel_size

    def coords(n, vs):
        i = np.arange(n)
        return np.where(i <= n // 2, i, i - n).astype(np.float64) * vs

    dx = coords(nx, vsx)[None, None, :]
    dy = coords(ny, vsy)[None, :, None]
    dz = coords(nz, vsz)[:, None, None]
    dist_sq = dx * dx + dy * dy + dz * dz
    s = (dist_sq <= radius * radius).astype(np.float64)
    count = s.sum()
    if count > 0:
        s *= 1.0 / count
    return s


def erode_mask_smv(mask: np.ndarray, smv_kernel_fft: np.ndarray, delta: float) -> np.ndarray:
    """Keep voxels where Re(IFFT(FFT(mask)*S)) > delta (src/kernels/smv.rs:79-105)."""
    conv = ifft3d(fft3d(mask.astype(np.complex128)) * smv_kernel_fft)
    return (conv.real > delta).astype(np.uint8)


# ---------------------------------------------------------------------------
# Gradient / divergence, periodic f64 (src/utils/gradient.rs:121-205)
# ---------------------------------------------------------------------------
def fgrad(x: np.ndarray, grid: Grid):
    """Forward differences with periodic BC, scaled by 1/vs (src/utils/gradient.rs:121-165)."""
    vsx, vsy, vsz = grid.voxel_size
    hx, hy, hz = 1.0 / vsx, 1.0 / vsy, 1.0 / vsz
    gx = (np.roll(x, -1, axis=2) - x) * hx
    gy = (np.roll(x, -1, axis=1) - x) * hy
    gz = (np.roll(x, -1, axis=0) - x) * hz
    return gx, gy, gz


def bdiv(gx, gy, gz, grid: Grid) -> np.ndarray:
    """Backward divergence, periodic (= -grad^T) (src/utils/gradient.rs:170-205)."""
    vsx, vsy, vsz = grid.voxel_size
    hx, hy, hz = 1.0 / vsx, 1.0 / vsy, 1.0 / vsz
    return ((gx - np.roll(gx, 1, axis=2)) * hx
            + (gy - np.roll(gy, 1, axis=1)) * hy
            + (gz - np.roll(gz, 1, axis=0)) * hz)


# ---------------------------------------------------------------------------
# Small utilities (src/utils/mod.rs, src/utils/mask.rs)
# ---------------------------------------------------------------------------
def shrink(x, t):
    """Soft threshold (src/utils/mod.rs:44-56)."""
    x = np.asarray(x, dtype=np.float64)
    return np.where(x > t, x - t, np.where(x < -t, x + t, 0.0))


def relative_change(x, x_prev) -> float:
    """||x - x_prev|| / (||x|| + 1e-20) (src/utils/mod.rs:69-77)."""
    d = (x - x_prev).ravel()
    xr = x.ravel()
    return math.sqrt(float(np.dot(d, d))) / (math.sqrt(float(np.dot(xr, xr))) + 1e-20)


def apply_mask_zero(data: np.ndarray, mask: np.ndarray) -> np.ndarray:
    """Zero where mask == 0 (src/utils/mask.rs:47-53)."""
    return np.where(mask != 0, data, 0.0)


def create_sphere_mask(grid: Grid, cx, cy, cz, radius) -> np.ndarray:
    """Binary sphere in voxel coordinates (src/utils/mask.rs:20-44)."""
    nx, ny, nz = grid.dims
    i = np.arange(nx)[None, None, :] - cx
    j = np.arange(ny)[None, :, None] - cy
    k = np.arange(nz)[:, None, None] - cz
    return ((i * i + j * j + k * k) <= radius * radius).astype(np.uint8)


def next_fast_fft_size(size: int) -> int:
    """Smallest n >= size with only 2/3/5 factors (src/utils/padding.rs:9-25)."""
    n = size
    while True:
        m = n
        for p in (2, 3, 5):
            while m % p == 0:
                m //= p
        if m == 1:
            return n
        n += 1


# ---------------------------------------------------------------------------
# Dipole inversion: TKD / TSVD / Tikhonov / TV-ADMM
# ---------------------------------------------------------------------------
@dataclass
class TkdParams:  # src/inversion/tkd.rs:23-32
    threshold: float = 0.15


def tkd(local_field, mask, grid: Grid, bdir, params: TkdParams = TkdParams()) -> np.ndarray:
    """Truncated k-space division (src/inversion/tkd.rs:48-99)."""
    d = dipole_kernel(grid, bdir)
    t = params.threshold
    inv_t = 1.0 / t
    with np.errstate(divide="ignore"):
        inv_d = np.where(np.abs(d) <= t, np.where(d >= 0.0, inv_t, -inv_t), 1.0 / d)
    f = _vol(local_field, grid)
    chi = ifft3d(fft3d(f.astype(np.complex128)) * inv_d).real
    return apply_mask_zero(chi, _vol(mask, grid, np.uint8))


def tsvd(local_field, mask, grid: Grid, bdir, params: TkdParams = TkdParams()) -> np.ndarray:
    """Truncated SVD variant: |D| <= t -> 0 (src/inversion/tkd.rs:105-153)."""
    d = dipole_kernel(grid, bdir)
    t = params.threshold
    with np.errstate(divide="ignore"):
        inv_d = np.where(np.abs(d) <= t, 0.0, 1.0 / d)
    f = _vol(local_field, grid)
    chi = ifft3d(fft3d(f.astype(np.complex128)) * inv_d).real
    return apply_mask_zero(chi, _vol(mask, grid, np.uint8))


REG_IDENTITY, REG_GRADIENT, REG_LAPLACIAN = 0, 1, 2


@dataclass
class TikhonovParams:  # src/inversion/tikhonov.rs:38-49
    lambda_: float = 0.01
    reg: int = REG_IDENTITY


def tikhonov(local_field, mask, grid: Grid, bdir, params: TikhonovParams = TikhonovParams()) -> np.ndarray:
    """D/(D^2 + lambda*Gamma) with Gamma in {1, L, L^2} (src/inversion/tikhonov.rs:62-138)."""
    d = dipole_kernel(grid, bdir)
    if params.reg == REG_IDENTITY:
        gamma = np.ones(grid.shape)
    elif params.reg == REG_GRADIENT:
        gamma = fft_real_kernel(laplacian_kernel(grid, True))
    else:
        lr = fft_real_kernel(laplacian_kernel(grid, False))
        gamma = lr * lr
    denom = d * d + params.lambda_ * gamma
    with np.errstate(divide="ignore", invalid="ignore"):
        inv_d = np.where(np.abs(denom) > 1e-20, d / denom, 0.0)
    f = _vol(local_field, grid)
    chi = ifft3d(fft3d(f.astype(np.complex128)) * inv_d).real
    return apply_mask_zero(chi, _vol(mask, grid, np.uint8))


@dataclass
class TvParams:  # src/inversion/tv.rs:23-43
    lambda_: float = 2e-4
    rho: float = 2e-2
    tol: float = 1e-3
    max_iter: int = 250


def prepare_admm_spectral(local_field, grid: Grid, bdir, rho):
    """(inv_a, f_hat) (src/inversion/admm.rs:150-178)."""
    d = dipole_kernel(grid, bdir)
    lap = fft3d(laplacian_kernel(grid, True).astype(np.complex128)).real
    a = d * d + rho * lap
    with np.errstate(divide="ignore"):
        inv_a = np.where(np.abs(a) > 1e-20, 1.0 / a, 0.0)
    f_hat = fft3d(_vol(local_field, grid).astype(np.complex128)) * d * inv_a
    return inv_a, f_hat


def tv_admm(local_field, mask, grid: Grid, bdir, params: TvParams = TvParams(),
            progress: Optional[Callable[[int, int], None]] = None, return_iters=False):
    """TV-ADMM dipole inversion (src/inversion/tv.rs:63-97, src/inversion/admm.rs:76-145).

    State starts at x = u = g = 0.  Each iteration: div = bdiv(g); x = Re IFFT(f_hat -
    rho*FFT(div)*inv_a); stop if relative_change(x, x_prev) < tol (checked before the
    z/u update, admm.rs:117); then v = grad x + u, z = shrink(v, lambda/rho), u = v - z,
    g = 2z - v.
    """
    inv_a, f_hat = prepare_admm_spectral(local_field, grid, bdir, params.rho)
    shape = grid.shape
    x = np.zeros(shape)
    ux = np.zeros(shape); uy = np.zeros(shape); uz = np.zeros(shape)
    gx = np.zeros(shape); gy = np.zeros(shape); gz = np.zeros(shape)
    lam_over_rho = params.lambda_ / params.rho
    iters = 0
    for it in range(params.max_iter):
        if progress is not None:
            progress(it + 1, params.max_iter)
        x_prev = x
        div = bdiv(gx, gy, gz, grid)
        work = fft3d(div.astype(np.complex128))
        work = f_hat - params.rho * work * inv_a
        x = ifft3d(work).real
        iters = it + 1
        if relative_change(x, x_prev) < params.tol:
            if progress is not None:
                progress(it + 1, it + 1)
            break
        ggx, ggy, ggz = fgrad(x, grid)
        vx, vy, vz = ggx + ux, ggy + uy, ggz + uz
        zx, zy, zz = shrink(vx, lam_over_rho), shrink(vy, lam_over_rho), shrink(vz, lam_over_rho)
        ux, uy, uz = vx - zx, vy - zy, vz - zz
        gx, gy, gz = 2.0 * zx - vx, 2.0 * zy - vy, 2.0 * zz - vz
    out = apply_mask_zero(x, _vol(mask, grid, np.uint8))
    return (out, iters) if return_iters else out


# ---------------------------------------------------------------------------
# Laplacian phase unwrapping (src/unwrap/laplacian.rs)
# ---------------------------------------------------------------------------
def wrap(x):
    """Wrap to [-pi, pi] with a truncated fmod like Rust's % (src/unwrap/laplacian.rs:21-30)."""
    y = np.fmod(np.asarray(x, dtype=np.float64), 2.0 * PI)
    y = np.where(y > PI, y - 2.0 * PI, np.where(y < -PI, y + 2.0 * PI, y))
    return y


def wrapped_laplacian_periodic(phase: np.ndarray, grid: Grid) -> np.ndarray:
    """Sum of wrapped second differences, periodic (src/unwrap/laplacian.rs:34-78)."""
    vsx, vsy, vsz = grid.voxel_size
    dx2, dy2, dz2 = 1.0 / (vsx * vsx), 1.0 / (vsy * vsy), 1.0 / (vsz * vsz)
    u = phase
    lap_x = (wrap(np.roll(u, -1, 2) - u) - wrap(u - np.roll(u, 1, 2))) * dx2
    lap_y = (wrap(np.roll(u, -1, 1) - u) - wrap(u - np.roll(u, 1, 1))) * dy2
    lap_z = (wrap(np.roll(u, -1, 0) - u) - wrap(u - np.roll(u, 1, 0))) * dz2
    return lap_x + lap_y + lap_z


def poisson_eigenvalues(grid: Grid) -> np.ndarray:
    """lambda(k) = sum 2(cos 2 pi f - 1)/h^2 (src/unwrap/laplacian.rs:91-105)."""
    nx, ny, nz = grid.dims
    vsx, vsy, vsz = grid.voxel_size

    def lam(n, vs):
        i = np.arange(n, dtype=np.float64)
        f = np.where(np.arange(n) <= n // 2, i / n, (i - n) / n)
        return 2.0 * (np.cos(2.0 * PI * f) - 1.0) * (1.0 / (vs * vs))

    return (lam(nx, vsx)[None, None, :] + lam(ny, vsy)[None, :, None]) + lam(nz, vsz)[:, None, None]


def solve_poisson_fft(f: np.ndarray, grid: Grid) -> np.ndarray:
    """FFT Poisson solve, DC -> 0 when |lambda| <= 1e-20 (src/unwrap/laplacian.rs:81-121)."""
    lam = poisson_eigenvalues(grid)
    F = fft3d(f.astype(np.complex128))
    with np.errstate(divide="ignore", invalid="ignore"):
        F = np.where(np.abs(lam) > 1e-20, F / lam, 0.0)
    return ifft3d(F).real


def laplacian_unwrap(phase, mask, grid: Grid) -> np.ndarray:
    """Laplacian unwrapping (src/unwrap/laplacian.rs:135-161)."""
    ph = _vol(phase, grid)
    m = _vol(mask, grid, np.uint8)
    d2u = wrapped_laplacian_periodic(ph, grid)
    d2u = np.where(m != 0, d2u, 0.0)
    un = solve_poisson_fft(d2u, grid)
    return np.where(m != 0, un, 0.0)


# ---------------------------------------------------------------------------
# Background removal: SMV / SHARP / V-SHARP (src/bgremove/)
# ---------------------------------------------------------------------------
SMV_DELTA = 1.0 - 1e-10                  # src/bgremove/smv.rs:44
SHARP_DELTA = 1.0 - math.sqrt(1e-7)      # src/bgremove/sharp.rs:79, vsharp.rs:129


def smv(field_, mask, grid: Grid, radius: float):
    """local = field - SMV(field) inside the SMV-eroded mask (src/bgremove/smv.rs:31-59)."""
    f = _vol(field_, grid)
    m = _vol(mask, grid, np.uint8)
    s_fft = fft_real_kernel(smv_kernel(grid, radius))
    eroded = erode_mask_smv(m, s_fft, SMV_DELTA)
    smv_field = apply_real_kernel(f, s_fft)
    local = np.where(eroded == 1, f - smv_field, 0.0)
    return local, eroded


@dataclass
class SharpParams:  # src/bgremove/sharp.rs:22-37
    threshold: float = 0.05
    radius: float = 6.0


def sharp_core(field_, mask, grid: Grid, threshold: float, radius: float):
    """SHARP (src/bgremove/sharp.rs:64-131)."""
    f = _vol(field_, grid)
    m = _vol(mask, grid, np.uint8)
    s_fft = fft_real_kernel(smv_kernel(grid, radius))
    eroded = erode_mask_smv(m, s_fft, SHARP_DELTA)
    oms = 1.0 - s_fft
    F = fft3d(f.astype(np.complex128)) * oms
    g = ifft3d(F)
    g = np.where(eroded == 0, 0.0, g)
    G = fft3d(g)
    with np.errstate(divide="ignore", invalid="ignore"):
        G = np.where(np.abs(oms) < threshold, 0.0, G / oms)
    out = ifft3d(G)
    local = np.where(eroded == 1, out.real, 0.0)
    return local, eroded


def sharp(field_, mask, grid: Grid, params: SharpParams = SharpParams()):
    """src/bgremove/sharp.rs:51-58."""
    return sharp_core(field_, mask, grid, params.threshold, params.radius)


@dataclass
class VsharpParams:  # src/bgremove/vsharp.rs:22-40
    threshold: float = 0.05
    max_radius: float = 12.0
    min_radius: float = 1.0


def vsharp_radii(params: VsharpParams) -> List[float]:
    """Descending radii max, max-step, ... >= step (src/bgremove/vsharp.rs:70-82)."""
    radii = []
    r = params.max_radius
    step = params.min_radius
    while r >= step:
        radii.append(r)
        r -= step
    if not radii:
        radii.append(params.max_radius)
    return radii


def vsharp_with_radii(field_, mask, grid: Grid, radii: Sequence[float], threshold: float,
                      progress: Optional[Callable[[int, int], None]] = None):
    """Multi-radius first-hit V-SHARP, deconvolved with the largest kernel (src/bgremove/vsharp.rs:88-199)."""
    f = _vol(field_, grid)
    m = _vol(mask, grid, np.uint8)
    if len(radii) == 0:
        return np.zeros(grid.shape), m.copy()
    if len(radii) == 1:
        if progress is not None:
            progress(1, 1)
        return sharp_core(f, m, grid, threshold, radii[0])
    sorted_radii = sorted(radii, reverse=True)
    field_fft = fft3d(f.astype(np.complex128))
    processed = np.zeros(grid.shape, dtype=bool)
    local = np.zeros(grid.shape)
    final_mask = np.zeros(grid.shape, dtype=np.uint8)
    inv_kernel = None
    for idx, radius in enumerate(sorted_radii):
        if progress is not None:
            progress(idx + 1, len(sorted_radii))
        s_fft = fft_real_kernel(smv_kernel(grid, radius))
        if inv_kernel is None:
            oms = 1.0 - s_fft
            with np.errstate(divide="ignore"):
                inv_kernel = np.where(np.abs(oms) < threshold, 0.0, 1.0 / oms)
        eroded = erode_mask_smv(m, s_fft, SHARP_DELTA)
        filtered = ifft3d(field_fft * (1.0 - s_fft)).real
        sel = (eroded == 1) & (~processed)
        local = np.where(sel, filtered, local)
        processed |= sel
        final_mask[sel] = 1
    out = ifft3d(fft3d(local.astype(np.complex128)) * inv_kernel).real
    local = np.where(final_mask == 1, out, 0.0)
    return local, final_mask


def vsharp(field_, mask, grid: Grid, params: VsharpParams = VsharpParams(), progress=None):
    """src/bgremove/vsharp.rs:55-63."""
    return vsharp_with_radii(field_, mask, grid, vsharp_radii(params), params.threshold, progress)


# ---------------------------------------------------------------------------
# Conjugate gradient (src/solvers/cg.rs:34-101)
# ---------------------------------------------------------------------------
def cg_solve(a_op, b, x0, tol, max_iter, progress=None):
    """CG on a closure operator; |p.Ap| < 1e-20 breaks; stop when ||r|| < tol*||b||."""
    b = np.asarray(b, dtype=np.float64).ravel()
    x = np.asarray(x0, dtype=np.float64).ravel().copy()
    r = b - a_op(x)
    p = r.copy()
    rsold = float(np.dot(r, r))
    b_norm = math.sqrt(float(np.dot(b, b)))
    for it in range(max_iter):
        if progress is not None:
            progress(it, max_iter)
        ap = a_op(p)
        pap = float(np.dot(p, ap))
        if abs(pap) < 1e-20:
            break
        alpha = rsold / pap
        x = x + alpha * p
        r = r - alpha * ap
        rsnew = float(np.dot(r, r))
        if math.sqrt(rsnew) < tol * b_norm:
            break
        beta = rsnew / rsold
        p = r + beta * p
        rsold = rsnew
    return x
