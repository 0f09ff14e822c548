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


def laplacian_eigenvalues(grid: Grid, exact_dc: bool = False) -> np.ndarray:
    """Re FFT(laplacian_kernel(negative=True)) as src/inversion/admm.rs:159-163 and
    src/inversion/rts.rs:93-99 compute it.  The DC bin is the floating-point sum of the
    seven taps: exactly 0 for some voxel sizes and a few ulp (e.g. 4.4e-16 at
    (1, 1, 0.9)) for others, depending on the FFT's summation order.  A nonzero value
    there defeats the |a| > 1e-20 guard of the ADMM inverse, so inv_a(0) becomes ~1e17
    and the iterate picks up a constant offset made of amplified roundoff.
    exact_dc=True stores the exact eigenvalue 0 there, which makes the guard fire as
    intended; the GPU tables hold that value."""
    lap = fft3d(laplacian_kernel(grid, True).astype(np.complex128)).real
    if exact_dc:
        lap[0, 0, 0] = 0.0
    return lap


def prepare_admm_spectral(local_field, grid: Grid, bdir, rho, exact_dc: bool = False):
    """(inv_a, f_hat) (src/inversion/admm.rs:150-178)."""
    d = dipole_kernel(grid, bdir)
    lap = laplacian_eigenvalues(grid, exact_dc)
    a = d * d + rho * lap
    with np.errstate(divide="ignore"):
        inv_a = np.where(np.abs(a) > 1e-20, 1.0 / a, 0.0)
    f_hat = fft3d(_vol(local_field, grid).astype(np.complex128)) * d * inv_a
    return inv_a, f_hat


def tv_admm(local_field, mask, grid: Grid, bdir, params: TvParams = TvParams(),
            progress: Optional[Callable[[int, int], None]] = None, return_iters=False, exact_dc=False):
    """TV-ADMM dipole inversion (src/inversion/tv.rs:63-97, src/inversion/admm.rs:76-145).

    State starts at x = u = g = 0.  Each iteration: div = bdiv(g); x = Re IFFT(f_hat -
    rho*FFT(div)*inv_a); stop if relative_change(x, x_prev) < tol (checked before the
    z/u update, admm.rs:117); then v = grad x + u, z = shrink(v, lambda/rho), u = v - z,
    g = 2z - v.  exact_dc: see laplacian_eigenvalues.
    """
    inv_a, f_hat = prepare_admm_spectral(local_field, grid, bdir, params.rho, exact_dc)
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


# ---------------------------------------------------------------------------
# iLSQR (src/inversion/ilsqr.rs)
# ---------------------------------------------------------------------------
@dataclass
class IlsqrParams:  # src/inversion/ilsqr.rs:20-34
    tol: float = 0.01
    max_iter: int = 50


def lsqr_real(apply_a, apply_at, b, tol, max_iter):
    """Real LSQR, relative-residual stop (src/inversion/ilsqr.rs:62-148)."""
    u = np.array(b, dtype=np.float64)
    beta = float(np.linalg.norm(u))
    if beta > 0:
        u = u * (1.0 / beta)
    v = apply_at(u)
    alpha = float(np.linalg.norm(v))
    if alpha > 0:
        v = v * (1.0 / alpha)
    w = v.copy()
    x = np.zeros_like(v)
    phi_bar, rho_bar, bnorm = beta, alpha, beta
    for _ in range(max_iter):
        u_new = apply_a(v) - alpha * u
        beta = float(np.linalg.norm(u_new))
        if beta > 0:
            u_new = u_new * (1.0 / beta)
        u = u_new
        v_new = apply_at(u) - beta * v
        alpha = float(np.linalg.norm(v_new))
        if alpha > 0:
            v_new = v_new * (1.0 / alpha)
        v = v_new
        rho = math.sqrt(rho_bar * rho_bar + beta * beta)
        c, s = rho_bar / rho, beta / rho
        theta = s * alpha
        rho_bar = -c * alpha
        phi = c * phi_bar
        phi_bar *= s
        t1, t2 = phi / rho, -theta / rho
        x = x + t1 * w
        w = v + t2 * w
        if phi_bar / (bnorm + 1e-20) < tol:
            break
    return x


def lsqr_complex(apply_a, apply_ah, b, tol, max_iter, return_iters=False):
    """Complex LSQR stopping on ||r||/||b|| <= tol (src/inversion/ilsqr.rs:177-321)."""
    u = np.array(b, dtype=np.complex128)
    beta = float(np.linalg.norm(u))
    if beta > 0:
        u = u * (1.0 / beta)
    v = apply_ah(u)
    alpha = float(np.linalg.norm(v))
    if alpha > 0:
        v = v * (1.0 / alpha)
    w = v.copy()
    x = np.zeros_like(v)
    phi_bar, rho_bar, bnorm = beta, alpha, beta
    it_done = 0
    if alpha * beta == 0.0:
        return (x, 0) if return_iters else x
    for it in range(max_iter):
        u_new = apply_a(v) - alpha * u
        beta = float(np.linalg.norm(u_new))
        if beta > 0:
            u_new = u_new * (1.0 / beta)
        u = u_new
        v_new = apply_ah(u) - beta * v
        alpha = float(np.linalg.norm(v_new))
        if alpha > 0:
            v_new = v_new * (1.0 / alpha)
        v = v_new
        rho = math.sqrt(rho_bar * rho_bar + beta * beta)
        c, s = rho_bar / rho, beta / rho
        theta = s * alpha
        rho_bar = -c * alpha
        phi = c * phi_bar
        phi_bar *= s
        t1, t2 = phi / rho, -theta / rho
        x = x + t1 * w
        w = v + t2 * w
        it_done = it + 1
        if phi_bar / (bnorm + 1e-20) <= tol:
            break
    return (x, it_done) if return_iters else x


def lsmr(apply_a, apply_at, b, n, atol, btol, max_iter, return_iters=False):
    """LSMR, undamped, Fong & Saunders tests 1-3 with conlim 1e8 (src/inversion/ilsqr.rs:344-517)."""
    u = np.array(b, dtype=np.float64)
    beta = float(np.linalg.norm(u))
    if beta > 0:
        u = u * (1.0 / beta)
    v = apply_at(u)
    alpha = float(np.linalg.norm(v))
    if alpha > 0:
        v = v * (1.0 / alpha)
    alpha_bar, zeta_bar = alpha, alpha * beta
    rho, rho_bar, c_bar, s_bar = 1.0, 1.0, 1.0, 0.0
    h = v.copy()
    h_bar = np.zeros(n)
    x = np.zeros(n)
    normb, betadd, betad, rhodold, tautildeold, thetatilde, zeta, d = beta, beta, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0
    norm_a2 = alpha * alpha
    maxrbar, minrbar = 0.0, 1e100
    ctol = 1.0 / 1e8
    it_done = 0
    if alpha * beta == 0.0:
        return (x, 0) if return_iters else x
    for it in range(max_iter):
        u_new = apply_a(v) - alpha * u
        beta = float(np.linalg.norm(u_new))
        if beta > 0:
            u_new = u_new * (1.0 / beta)
        u = u_new
        v_new = apply_at(u) - beta * v
        alpha = float(np.linalg.norm(v_new))
        if alpha > 0:
            v_new = v_new * (1.0 / alpha)
        v = v_new
        rho_old = rho
        rho = math.sqrt(alpha_bar * alpha_bar + beta * beta)
        c, s = alpha_bar / rho, beta / rho
        theta_new = s * alpha
        alpha_bar = c * alpha
        rho_bar_old, zeta_old = rho_bar, zeta
        theta_bar = s_bar * rho
        rho_temp = c_bar * rho
        rho_bar = math.sqrt(rho_temp * rho_temp + theta_new * theta_new)
        c_bar, s_bar = rho_temp / rho_bar, theta_new / rho_bar
        zeta = c_bar * zeta_bar
        zeta_bar *= -s_bar
        h_bar = h - (theta_bar * rho / (rho_old * rho_bar_old)) * h_bar
        x = x + (zeta / (rho * rho_bar)) * h_bar
        h = v - (theta_new / rho) * h
        betaacute = betadd
        betahat = c * betaacute
        betadd = -s * betaacute
        thetatildeold = thetatilde
        rhotildeold = math.sqrt(rhodold * rhodold + theta_bar * theta_bar)
        ctildeold, stildeold = rhodold / rhotildeold, theta_bar / rhotildeold
        thetatilde = stildeold * rho_bar
        rhodold = ctildeold * rho_bar
        betad = -stildeold * betad + ctildeold * betahat
        tautildeold = (zeta_old - thetatildeold * tautildeold) / rhotildeold
        taud = (zeta - thetatilde * tautildeold) / rhodold
        normr = math.sqrt(d + (betad - taud) ** 2 + betadd * betadd)
        norm_a2 += beta * beta
        norm_a = math.sqrt(norm_a2)
        norm_a2 += alpha * alpha
        maxrbar = max(maxrbar, rho_bar_old)
        if it > 0:
            minrbar = min(minrbar, rho_bar_old)
        cond_a = max(maxrbar, rho_temp) / min(minrbar, rho_temp)
        norm_ar = abs(zeta_bar)
        normx = float(np.linalg.norm(x))
        test1 = normr / (normb + 1e-20)
        test2 = norm_ar / ((norm_a * normr) + 1e-20)
        test3 = 1.0 / (cond_a + 1e-20)
        rtol = btol + atol * norm_a * normx / (normb + 1e-20)
        it_done = it + 1
        if test3 <= ctol or test2 <= atol or test1 <= rtol:
            break
    return (x, it_done) if return_iters else x


def prctile(sorted_vals, p):
    """Linear-interpolation percentile of a sorted array (src/inversion/ilsqr.rs:937-946)."""
    n = len(sorted_vals)
    if n == 0:
        return 0.0
    if n == 1:
        return float(sorted_vals[0])
    h = (p / 100.0) * (n - 1)
    lo = int(math.floor(h))
    hi = min(lo + 1, n - 1)
    frac = h - lo
    return float(sorted_vals[lo] + frac * (sorted_vals[hi] - sorted_vals[lo]))


def _lap1_axis(f, m, axis, h):
    """Mask-adaptive second difference along one axis (src/inversion/ilsqr.rs:571-669)."""
    n = f.shape[axis]
    fm = np.moveaxis(f, axis, -1)
    mm = np.moveaxis(m, axis, -1)
    out = np.zeros_like(fm)
    for c in range(n):
        # stencil selector: interior -> 2*mask[+1] + mask[-1]; first -> 2; last -> 1
        if 1 <= c <= n - 2:
            sel = 2 * mm[..., c + 1].astype(np.int64) + mm[..., c - 1].astype(np.int64)
        else:
            sel = np.full(fm.shape[:-1], 2 if c == 0 else (1 if c == n - 1 else 0), dtype=np.int64)
        val = np.zeros(fm.shape[:-1])
        central = sel == 3
        if central.any():
            val = np.where(central, fm[..., c - 1] - 2.0 * fm[..., c] + fm[..., c + 1] if 1 <= c <= n - 2 else 0.0, val)
        fwd = sel == 2
        if fwd.any() and c + 1 < n:
            o4 = (c + 3 < n)
            m2 = mm[..., c + 2] != 0 if c + 2 < n else np.zeros(fm.shape[:-1], bool)
            m3 = mm[..., c + 3] != 0 if c + 3 < n else np.zeros(fm.shape[:-1], bool)
            v4 = (2.0 * fm[..., c] - 5.0 * fm[..., c + 1] + 4.0 * fm[..., c + 2] - fm[..., c + 3]) if o4 else 0.0
            v2 = (fm[..., c] - 2.0 * fm[..., c + 1] + fm[..., c + 2]) if c + 2 < n else 0.0
            v1 = fm[..., c + 1] - fm[..., c]
            fv = np.where(o4 & m2 & m3, v4, np.where((c + 2 < n) & m2, v2, v1))
            val = np.where(fwd, fv, val)
        bwd = sel == 1
        if bwd.any() and c - 1 >= 0:
            m2 = mm[..., c - 2] != 0 if c - 2 >= 0 else np.zeros(fm.shape[:-1], bool)
            m3 = mm[..., c - 3] != 0 if c - 3 >= 0 else np.zeros(fm.shape[:-1], bool)
            v4 = (-fm[..., c - 3] + 4.0 * fm[..., c - 2] - 5.0 * fm[..., c - 1] + 2.0 * fm[..., c]) if c - 3 >= 0 else 0.0
            v2 = (fm[..., c - 2] - 2.0 * fm[..., c - 1] + fm[..., c]) if c - 2 >= 0 else 0.0
            v1 = fm[..., c - 1] - fm[..., c]
            bv = np.where((c - 3 >= 0) & m3 & m2, v4, np.where((c - 2 >= 0) & m2, v2, v1))
            val = np.where(bwd, bv, val)
        out[..., c] = val
    return np.moveaxis(out, -1, axis) * h


def ilsqr_laplacian(f, mask, grid: Grid):
    """Mask-adaptive Laplacian, zero outside the mask (src/inversion/ilsqr.rs:528-566)."""
    vsx, vsy, vsz = grid.voxel_size
    m = (mask != 0)
    lap = np.zeros(grid.shape)
    lap += _lap1_axis(f, mask, 2, 1.0 / (vsx * vsx))
    lap += _lap1_axis(f, mask, 1, 1.0 / (vsy * vsy))
    lap += _lap1_axis(f, mask, 0, 1.0 / (vsz * vsz))
    return np.where(m, lap, 0.0)


def _percentile_weights(vals, mask, pmin, pmax, extra_mask_multiply=False):
    sel = np.sort(vals[mask != 0])
    w = np.zeros(vals.shape)
    if sel.size == 0:
        return w
    tmin, tmax = prctile(sel, pmin), prctile(sel, pmax)
    rng = tmax - tmin
    inner = np.where(rng > 1e-10, (tmax - vals) / (rng if rng != 0 else 1.0), 0.0)
    ww = np.where(vals < tmin, 1.0, np.where(vals > tmax, 0.0, inner))
    if extra_mask_multiply:
        ww = ww * mask.astype(np.float64)
    return np.where(mask != 0, ww, 0.0)


def laplacian_weights_ilsqr(f, mask, grid: Grid, pmin=60.0, pmax=99.9):
    """Equation 7 weights (src/inversion/ilsqr.rs:672-719)."""
    return _percentile_weights(ilsqr_laplacian(f, mask, grid), mask, pmin, pmax)


def dipole_kspace_weights_ilsqr(d, n_exp=0.001, pa=1.0, pb=30.0):
    """|D|^n normalised by percentiles over all values (src/inversion/ilsqr.rs:724-760)."""
    w = np.abs(d) ** n_exp
    vals = np.sort(w.ravel())
    lo, hi = prctile(vals, pa), prctile(vals, pb)
    rng = hi - lo
    if rng > 1e-20:
        w = (w - lo) / rng
    return np.clip(w, 0.0, 1.0)


def fgrad_masked(f, mask, grid: Grid):
    """Mask-adaptive forward/backward gradient (src/inversion/ilsqr.rs:767-823)."""
    vsx, vsy, vsz = grid.voxel_size
    m = mask != 0
    out = []
    for axis, h in ((2, 1.0 / vsx), (1, 1.0 / vsy), (0, 1.0 / vsz)):
        n = f.shape[axis]
        fp = np.roll(f, -1, axis)
        fmn = np.roll(f, 1, axis)
        mp = np.roll(m, -1, axis)
        mmn = np.roll(m, 1, axis)
        idx = np.arange(n).reshape([-1 if a == axis else 1 for a in range(3)])
        can_f = (idx < n - 1) & mp
        can_b = (idx > 0) & mmn
        g = np.where(can_f, h * (fp - f), np.where(can_b, h * (f - fmn), 0.0))
        out.append(np.where(m, g, 0.0))
    return tuple(out)


def lsqr_step(f, mask, grid: Grid, d):
    """Step 1 (src/inversion/ilsqr.rs:953-1030)."""
    w = laplacian_weights_ilsqr(f, mask, grid)
    b = fft3d((w * f).astype(np.complex128)) * d

    def apply_a(x):
        x3 = x.reshape(grid.shape)
        r = ifft3d(d * x3).real
        return (fft3d((w * r).astype(np.complex128)) * d).ravel()

    x = lsqr_complex(apply_a, apply_a, b.ravel(), 0.01, 50)
    xi = ifft3d(x.reshape(grid.shape))
    return np.where(mask != 0, xi.real, 0.0)


def fastqsm_step(f, mask, grid: Grid, d):
    """Step 2 (src/inversion/ilsqr.rs:1037-1167)."""
    F = fft3d(f.astype(np.complex128))
    x = F * np.sign(d)
    wfs = dipole_kspace_weights_ilsqr(d)
    h = fft_real_kernel(smv_kernel(grid, 3.0))
    filt = wfs + h * (1.0 - wfs)
    xf = ifft3d(x * wfs + x * h * (1.0 - wfs))
    xf = np.where(mask != 0, xf.real, 0.0).astype(np.complex128)
    xf = fft3d(xf)
    xf2 = ifft3d(xf * wfs + xf * h * (1.0 - wfs))
    x_fs = np.where(mask != 0, xf2.real, 0.0)
    t0 = 1.0 / 8.0
    with np.errstate(divide="ignore"):
        inv_d = np.where(np.abs(d) < t0, np.sign(d) / t0, 1.0 / d)
    # Rust f64::signum(0.0) = 1.0 (src/inversion/ilsqr.rs:1129)
    inv_d = np.where((np.abs(d) < t0) & (d == 0.0), np.copysign(1.0, d) / t0, inv_d)
    x_tkd = np.where(mask != 0, ifft3d(F * inv_d).real, 0.0)
    n_all = float(f.size)
    s_fs, s_tkd = float(x_fs.sum()), float(x_tkd.sum())
    s_fs2, s_ft = float((x_fs * x_fs).sum()), float((x_fs * x_tkd).sum())
    det = s_fs2 * n_all - s_fs * s_fs
    if abs(det) > 1e-20:
        a = (n_all * s_ft - s_fs * s_tkd) / det
        bb = (s_fs2 * s_tkd - s_fs * s_ft) / det
    else:
        a, bb = 1.0, 0.0
    del filt
    return np.where(mask != 0, a * x_fs + bb, 0.0)


def susceptibility_artifacts_step(x0, xfs, mask, grid: Grid, d, tol, maxit):
    """Step 3 (src/inversion/ilsqr.rs:1174-1289)."""
    gx, gy, gz = fgrad_masked(xfs, mask, grid)
    wx = _percentile_weights(gx, mask, 50.0, 70.0, True)
    wy = _percentile_weights(gy, mask, 50.0, 70.0, True)
    wz = _percentile_weights(gz, mask, 50.0, 70.0, True)
    mic = (np.abs(d) < 0.1).astype(np.float64)
    dx, dy, dz = fgrad(x0, grid)
    b = np.concatenate([(wx * dx).ravel(), (wy * dy).ravel(), (wz * dz).ravel()])
    n = x0.size

    def apply_a(xin):
        xr = ifft3d(fft3d(xin.reshape(grid.shape).astype(np.complex128)) * mic).real
        ax, ay, az = fgrad(xr, grid)
        return np.concatenate([(wx * ax).ravel(), (wy * ay).ravel(), (wz * az).ravel()])

    def apply_at(yin):
        yx, yy, yz = (yin[i * n:(i + 1) * n].reshape(grid.shape) for i in range(3))
        dv = bdiv(wx * yx, wy * yy, wz * yz, grid)
        return ifft3d(fft3d((-dv).astype(np.complex128)) * mic).real.ravel()

    xsa = lsmr(apply_a, apply_at, b, n, tol, tol, maxit)
    return np.where(mask.ravel() != 0, xsa, 0.0).reshape(grid.shape)


def ilsqr(field_, mask, grid: Grid, bdir, params: IlsqrParams = IlsqrParams(), progress=None):
    """iLSQR: (chi, xsa, xfs, xlsqr) (src/inversion/ilsqr.rs:1307-1351)."""
    f = _vol(field_, grid)
    m = _vol(mask, grid, np.uint8)
    d = dipole_kernel(grid, bdir)
    if progress:
        progress(1, 4)
    xlsqr = lsqr_step(f, m, grid, d)
    if progress:
        progress(2, 4)
    xfs = fastqsm_step(f, m, grid, d)
    if progress:
        progress(3, 4)
    xsa = susceptibility_artifacts_step(xlsqr, xfs, m, grid, d, params.tol, params.max_iter)
    if progress:
        progress(4, 4)
    chi = np.where(m != 0, xlsqr - xsa, 0.0)
    return chi, xsa, xfs, xlsqr


# ---------------------------------------------------------------------------
# TGV-QSM (src/inversion/tgv.rs), single precision like the reference
# ---------------------------------------------------------------------------
F32 = np.float32


@dataclass
class TgvParams:  # src/inversion/tgv.rs:39-76
    alpha1: float = 0.0005
    alpha0: float = 0.0015
    iterations: int = 1000
    erosions: int = 3
    step_size: float = 3.0
    fieldstrength: float = 3.0
    te: float = 0.020
    tol: float = 1e-5


def erode_mask(mask: np.ndarray, iterations: int = 1) -> np.ndarray:
    """6-connected erosion, boundary voxels removed (src/utils/mask.rs:59-92)."""
    cur = (np.asarray(mask) != 0).astype(np.uint8)
    for _ in range(iterations):
        keep = cur.copy()
        inner = np.zeros_like(cur, dtype=bool)
        inner[1:-1, 1:-1, 1:-1] = True
        nb = np.ones_like(cur, dtype=bool)
        for ax in range(3):
            for sh in (1, -1):
                nb &= np.roll(cur, sh, axis=ax) != 0
        keep[(cur != 0) & ~(inner & nb)] = 0
        cur = keep
    return cur


def tgv_bounding_box(mask: np.ndarray, padding: int):
    """BoundingBox::from_mask (src/inversion/tgv.rs:110-144): (lo, hi) per axis in (x, y, z)."""
    nz, ny, nx = mask.shape
    idx = np.nonzero(mask)
    if len(idx[0]) == 0:
        lo = [nx, ny, nz]
        hi = [0, 0, 0]
    else:
        lo = [int(idx[2].min()), int(idx[1].min()), int(idx[0].min())]
        hi = [int(idx[2].max()), int(idx[1].max()), int(idx[0].max())]
    dims = (nx, ny, nz)
    lo = [max(v - padding, 0) for v in lo]
    hi = [min(v + padding + 1, d) for v, d in zip(hi, dims)]
    return lo, hi


def _dst_sin_table(n):
    """src/inversion/tgv.rs:481-491."""
    scale = math.pi / (n + 1.0)
    j = np.arange(n, dtype=np.float64) + 1.0
    return np.sin(np.outer(j, j) * scale)


def _dst3d(a, s):
    """Separable DST-I along x, y, z (src/inversion/tgv.rs:494-540); a is (z, y, x)."""
    a = np.einsum("zyj,jk->zyk", a, s)
    a = np.einsum("zjx,jk->zkx", a, s)
    return np.einsum("jyx,jk->kyx", a, s)


def _jacobi_pinv_solve(g, h):
    """solve_symmetric_pseudoinverse (src/inversion/tgv.rs:558-654): cyclic Jacobi, then
    eigenvalues below 1e-10 * max |lambda| dropped."""
    n = len(h)
    a = [list(map(float, row)) for row in g]
    v = [[1.0 if i == j else 0.0 for j in range(n)] for i in range(n)]
    for _ in range(100):
        max_off = 0.0
        for i in range(n):
            for j in range(i + 1, n):
                max_off = max(max_off, abs(a[i][j]))
        if max_off < 1e-15:
            break
        for p in range(n):
            for q in range(p + 1, n):
                if abs(a[p][q]) < 1e-15:
                    continue
                app, aqq, apq = a[p][p], a[q][q], a[p][q]
                tau = (aqq - app) / (2.0 * apq)
                t = 1.0 / (tau + math.sqrt(1.0 + tau * tau)) if tau >= 0.0 else -1.0 / (-tau + math.sqrt(1.0 + tau * tau))
                c = 1.0 / math.sqrt(1.0 + t * t)
                s = t * c
                for i in range(n):
                    if i == p or i == q:
                        continue
                    aip, aiq = a[i][p], a[i][q]
                    a[i][p] = c * aip - s * aiq
                    a[p][i] = a[i][p]
                    a[i][q] = s * aip + c * aiq
                    a[q][i] = a[i][q]
                a[p][p] = c * c * app - 2.0 * c * s * apq + s * s * aqq
                a[q][q] = s * s * app + 2.0 * c * s * apq + c * c * aqq
                a[p][q] = 0.0
                a[q][p] = 0.0
                for i in range(n):
                    vip, viq = v[i][p], v[i][q]
                    v[i][p] = c * vip - s * viq
                    v[i][q] = s * vip + c * viq
    ev = [a[i][i] for i in range(n)]
    thr = 1e-10 * max(abs(e) for e in ev)
    vth = [sum(v[j][i] * h[j] for j in range(n)) for i in range(n)]
    vth = [vth[i] / ev[i] if abs(ev[i]) > thr else 0.0 for i in range(n)]
    return [sum(v[i][j] * vth[j] for j in range(n)) for i in range(n)]


def tgv_oblique_stencil(res, b0):
    """compute_oblique_stencil (src/inversion/tgv.rs:272-479): least-squares fit of 13
    centrosymmetric stencil pairs to the dipole field on a 64^3 grid through DST-I
    Poisson solves, resolution-weighted, centre = -sum(others).  Returns st[di][dj][dk]
    as float32."""
    n, mid = 64, 32
    dx, dy, dz = (float(F32(r)) for r in res)
    bf = [F32(c) for c in b0]
    bn = math.sqrt(float(bf[0] * bf[0] + bf[1] * bf[1] + bf[2] * bf[2]))  # f32 sum, f64 sqrt
    bd = (float(bf[0]) / bn, float(bf[1]) / bn, float(bf[2]) / bn)
    z, y, x = np.meshgrid(np.arange(n) - mid, np.arange(n) - mid, np.arange(n) - mid, indexing="ij")
    x, y, z = x.astype(np.float64), y.astype(np.float64), z.astype(np.float64)
    r = np.sqrt(x * x + y * y + z * z)
    valid = r >= 4.0
    with np.errstate(invalid="ignore", divide="ignore"):
        xz = (bd[0] * x + bd[1] * y + bd[2] * z) / r
        kappa = (3.0 * xz * xz - 1.0) / (4.0 * math.pi * r * r * r)
    c2 = (2.0 * np.sin(math.pi * (np.arange(n) + 1.0) / (2.0 * (n + 1.0)))) ** 2
    lam = c2[None, None, :] + c2[None, :, None] + c2[:, None, None]
    s = _dst_sin_table(n)
    iscale = (2.0 / (n + 1.0)) ** 3
    pos = [(di, dj, dk) for dk in (-1, 0, 1) for dj in (-1, 0, 1) for di in (-1, 0, 1) if (di, dj, dk) != (0, 0, 0)]
    rows = []
    for p in range(13):
        di, dj, dk = pos[p]
        delta = np.zeros((n, n, n))
        delta[mid + dk, mid + dj, mid + di] = 1.0
        delta[mid - dk, mid - dj, mid - di] += 1.0
        delta[mid, mid, mid] = -2.0
        fd = _dst3d(delta, s) / -lam
        rows.append(_dst3d(fd, s)[valid] * iscale)
    dv = kappa[valid]
    g = [[float(np.dot(rows[i], rows[j])) for j in range(13)] for i in range(13)]
    h = [float(np.dot(rows[i], dv)) for i in range(13)]
    yv = _jacobi_pinv_solve(g, h)
    st = np.zeros((3, 3, 3), dtype=F32)
    for p in range(13):
        di, dj, dk = pos[p]
        st[di + 1, dj + 1, dk + 1] = F32(yv[p])
        di2, dj2, dk2 = pos[25 - p]
        st[di2 + 1, dj2 + 1, dk2 + 1] = F32(yv[p])
    for dk in (-1, 0, 1):
        for dj in (-1, 0, 1):
            for di in (-1, 0, 1):
                if (di, dj, dk) == (0, 0, 0):
                    continue
                i2, j2, k2 = di * di, dj * dj, dk * dk
                w = (i2 / (dx * dx) + j2 / (dy * dy) + k2 / (dz * dz)) / (i2 + j2 + k2)
                st[di + 1, dj + 1, dk + 1] = F32(st[di + 1, dj + 1, dk + 1] * F32(w))
    total = F32(0.0)
    for dk in range(3):
        for dj in range(3):
            for di in range(3):
                if not (di == 1 and dj == 1 and dk == 1):
                    total = F32(total + st[di, dj, dk])
    st[1, 1, 1] = -total
    return st


def _tgv_lap_neumann(a, mask, h2):
    """apply_laplacian_inplace (src/inversion/tgv.rs:780-824): Neumann BC, 0 outside the mask."""
    hx2, hy2, hz2 = h2
    two = F32(2.0)

    def nb(axis, sh):
        b = np.roll(a, sh, axis=axis)
        edge = [slice(None)] * 3
        edge[axis] = 0 if sh == 1 else -1
        b[tuple(edge)] = a[tuple(edge)]
        return b

    out = (hx2 * (nb(2, 1) - two * a + nb(2, -1)) + hy2 * (nb(1, 1) - two * a + nb(1, -1))
           + hz2 * (nb(0, 1) - two * a + nb(0, -1)))
    return np.where(mask != 0, out, F32(0)).astype(F32)


def _tgv_apply_stencil(x, st, mask):
    """apply_stencil (src/inversion/tgv.rs:667-713): 27-point, 0 outside the mask and on the
    sub-volume's faces; summed in dk, dj, di order."""
    nz, ny, nx = x.shape
    out = np.zeros_like(x)
    if nz < 3 or ny < 3 or nx < 3:
        return out
    acc = np.zeros((nz - 2, ny - 2, nx - 2), dtype=F32)
    for dk in range(3):
        for dj in range(3):
            for di in range(3):
                acc = (acc + st[di, dj, dk] * x[dk:nz - 2 + dk, dj:ny - 2 + dj, di:nx - 2 + di]).astype(F32)
    out[1:-1, 1:-1, 1:-1] = acc
    return np.where(mask != 0, out, F32(0)).astype(F32)


def _fgrad_f32(x, h):
    """fgrad_inplace_f32 (src/utils/gradient.rs:222-257): forward differences, 0 on the last slice."""
    out = []
    for axis, hh in ((2, h[0]), (1, h[1]), (0, h[2])):
        g = np.zeros_like(x)
        sl = [slice(None)] * 3
        sp = [slice(None)] * 3
        sl[axis] = slice(0, -1)
        sp[axis] = slice(1, None)
        g[tuple(sl)] = (x[tuple(sp)] - x[tuple(sl)]) * hh
        out.append(g)
    return out


def _bwd(a, axis):
    """a[i-1] along axis with 0 for i = 0."""
    b = np.zeros_like(a)
    sl = [slice(None)] * 3
    sp = [slice(None)] * 3
    sl[axis] = slice(1, None)
    sp[axis] = slice(0, -1)
    b[tuple(sl)] = a[tuple(sp)]
    return b


def _symgrad_f32(wx, wy, wz, h):
    """symgrad_inplace_f32 (src/utils/gradient.rs:300-372)."""
    half = F32(0.5)
    dxx, dyx, dzx = _fgrad_f32(wx, h)  # d/dx, d/dy, d/dz of wx
    dxy, dyy, dzy = _fgrad_f32(wy, h)
    dxz, dyz, dzz = _fgrad_f32(wz, h)
    sxx = dxx
    sxy = (dxy * half + dyx * half).astype(F32)
    sxz = (dxz * half + dzx * half).astype(F32)
    syy = dyy
    syz = (dyz * half + dzy * half).astype(F32)
    szz = dzz
    return sxx, sxy, sxz, syy, syz, szz


def _symdiv_f32(sxx, sxy, sxz, syy, syz, szz, h):
    """symdiv_inplace_f32 (src/utils/gradient.rs:380-432): backward differences, zero BC."""
    hx, hy, hz = h

    def row(a, b, c):
        return ((a - _bwd(a, 2)) * hx + (b - _bwd(b, 1)) * hy + (c - _bwd(c, 0)) * hz).astype(F32)

    return row(sxx, sxy, sxz), row(sxy, syy, syz), row(sxz, syz, szz)


def _bdiv_masked_f32(gx, gy, gz, mask, h):
    """bdiv_masked_inplace_f32 (src/utils/gradient.rs:497-565)."""
    m = (mask != 0).astype(F32)
    hx, hy, hz = h
    tx = m * gx * hx - _bwd(m, 2) * _bwd(gx, 2) * hx
    ty = m * gy * hy - _bwd(m, 1) * _bwd(gy, 1) * hy
    tz = m * gz * hz - _bwd(m, 0) * _bwd(gz, 0) * hz
    return np.where(mask != 0, (tx + ty + tz), F32(0)).astype(F32)


def tgv_qsm(phase, mask, grid: Grid, params: TgvParams = TgvParams(), b0=(0.0, 0.0, 1.0), progress=None):
    """tgv_qsm (src/inversion/tgv.rs:1045-1299) in float32."""
    ph = _vol(phase, grid).astype(F32)
    m_in = _vol(mask, grid, np.uint8)
    vs = tuple(F32(v) for v in grid.voxel_size)
    b0f = tuple(F32(v) for v in b0)
    me = m_in.copy()
    for _ in range(params.erosions):
        me = erode_mask(me, 1)
    m0 = erode_mask(me, 1)
    lo, hi = tgv_bounding_box(m0, 2)
    sl = (slice(lo[2], hi[2]), slice(lo[1], hi[1]), slice(lo[0], hi[0]))
    phs, m0s, mes = ph[sl], m0[sl], me[sl]
    hx2, hy2, hz2 = (F32(1.0) / (v * v) for v in vs)
    h = tuple(F32(1.0) / v for v in vs)
    # compute_phase_laplacian (tgv.rs:716-738) with the clamped 7-point Laplacian (:741-777)
    sp, cp = np.sin(phs).astype(F32), np.cos(phs).astype(F32)
    centre = F32(-2.0) * (hx2 + hy2 + hz2)

    def lap_clamped(a):
        def nb(axis, sh):
            b = np.roll(a, sh, axis=axis)
            edge = [slice(None)] * 3
            edge[axis] = 0 if sh == 1 else -1
            b[tuple(edge)] = a[tuple(edge)]
            return b
        return (centre * a + hx2 * (nb(2, 1) + nb(2, -1)) + hy2 * (nb(1, 1) + nb(1, -1))
                + hz2 * (nb(0, 1) + nb(0, -1))).astype(F32)

    lphi = np.where(m0s != 0, lap_clamped(sp) * cp - lap_clamped(cp) * sp, F32(0)).astype(F32)
    cnt = int((m0s != 0).sum())
    if cnt > 0:
        s = F32(0.0)
        for v in lphi[m0s != 0]:
            s = F32(s + v)
        mean = F32(s / F32(cnt))
        lphi = np.where(m0s != 0, lphi - mean, lphi).astype(F32)
    st = tgv_oblique_stencil(vs, b0f)
    gns = F32(4.0) * (F32(1.0) / (vs[0] * vs[0]) + F32(1.0) / (vs[1] * vs[1]) + F32(1.0) / (vs[2] * vs[2]))
    gn = F32(np.sqrt(gns))
    wave = F32(0.0)
    for v in st.ravel():  # [[[f32; 3]; 3]; 3] flattened with the last index fastest
        wave = F32(wave + abs(v))
    ns = _tgv_operator_norm_sqr(gn, gns, wave)
    tau = F32(F32(1.0) / F32(np.sqrt(ns)))
    sigma = tau
    sstep, tstep = F32(sigma * F32(params.step_size)), F32(tau * F32(params.step_size))
    a0, a1 = F32(params.alpha0), F32(params.alpha1)
    shp = lphi.shape
    z = lambda: np.zeros(shp, F32)
    chi, chi_, chi_prev, phi, phi_ = z(), z(), z(), z(), z()
    w = [z(), z(), z()]
    w_ = [z(), z(), z()]
    eta = z()
    p = [z(), z(), z()]
    q = [z() for _ in range(6)]
    in0, inm = m0s != 0, mes != 0
    final_iter = params.iterations
    for it in range(params.iterations):
        if progress:
            progress(it, params.iterations)
        if it > 0 and it % 100 == 0:
            d = F32(0.0)
            nrm = F32(0.0)
            for a, b in zip(chi[in0], chi_prev[in0]):
                dd = F32(a - b)
                d = F32(d + dd * dd)
                nrm = F32(nrm + a * a)
            rc = F32(np.sqrt(d / nrm)) if nrm > 1e-10 else F32(1.0)
            if rc < F32(params.tol):
                final_iter = it
                break
            chi_prev = chi.copy()
        t1 = _tgv_lap_neumann(phi_, m0s, (hx2, hy2, hz2))
        t2 = _tgv_apply_stencil(chi_, st, m0s)
        eta = np.where(in0, eta + sigma * (-t1 + t2 - lphi), eta).astype(F32)
        g = _fgrad_f32(chi_, h)
        s0 = np.where(in0, sstep, F32(0)).astype(F32)
        s1 = np.where(inm, sstep, F32(0)).astype(F32)
        upd = in0 | inm
        for c in range(3):
            p[c] = np.where(upd, p[c] + (s0 * g[c] - s1 * w_[c]), p[c]).astype(F32)
        nrm3 = np.sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]).astype(F32)
        with np.errstate(divide="ignore", invalid="ignore"):
            sc = np.where(upd & (nrm3 > a1), a1 / nrm3, F32(1.0)).astype(F32)
        for c in range(3):
            p[c] = np.where(upd & (nrm3 > a1), p[c] * sc, p[c]).astype(F32)
        sg = _symgrad_f32(w_[0], w_[1], w_[2], h)
        for c in range(6):
            q[c] = np.where(in0, q[c] + sstep * sg[c], q[c]).astype(F32)
        fro = np.sqrt(q[0] * q[0] + q[3] * q[3] + q[5] * q[5]
                      + F32(2.0) * (q[1] * q[1] + q[2] * q[2] + q[4] * q[4])).astype(F32)
        with np.errstate(divide="ignore", invalid="ignore"):
            sc = np.where(in0 & (fro > a0), a0 / fro, F32(1.0)).astype(F32)
        for c in range(6):
            q[c] = np.where(in0 & (fro > a0), q[c] * sc, q[c]).astype(F32)
        phi, phi_ = phi_, phi
        chi, chi_ = chi_, chi
        w, w_ = w_, w
        t1 = np.where(in0, eta, F32(0)).astype(F32)
        t2 = _tgv_lap_neumann(t1, m0s, (hx2, hy2, hz2))
        den = (F32(1.0) + np.where(inm, tau, F32(0))).astype(F32)
        phi = ((phi_ + tau * t2) / den).astype(F32)
        t1 = _bdiv_masked_f32(p[0], p[1], p[2], m0s, h)
        t2 = _tgv_apply_stencil(np.where(in0, eta, F32(0)).astype(F32), st, m0s)
        chi = (chi_ + tstep * (t1 - t2)).astype(F32)
        qm = [np.where(in0, qc, F32(0)).astype(F32) for qc in q]
        dq = _symdiv_f32(*qm, h)
        w = [np.where(inm, w_[c] + tstep * (p[c] + dq[c]), w_[c]).astype(F32) for c in range(3)]
        phi_ = (F32(2.0) * phi - phi_).astype(F32)
        chi_ = (F32(2.0) * chi - chi_).astype(F32)
        w_ = [(F32(2.0) * w[c] - w_[c]).astype(F32) for c in range(3)]
    if progress:
        progress(final_iter, params.iterations)
    gamma = F32(42.5781)
    scale = F32(F32(1.0) / (F32(2.0) * F32(math.pi) * F32(params.te) * F32(params.fieldstrength) * gamma))
    out = np.zeros(grid.shape, dtype=F32)
    out[sl] = np.where(inm, chi * scale, F32(0))
    return out.astype(np.float64)


def _tgv_operator_norm_sqr(g, g2, w):
    """compute_operator_norm_sqr (src/inversion/tgv.rs:839-876): 20 power iterations in f32."""
    g4, g2w, g2w2, g21 = F32(g2 * g2), F32(g2 * w), F32(g2 + w * w), F32(g2 + F32(1.0))
    v = [F32(1.0)] * 3
    for _ in range(20):
        y0 = F32(g4 * v[0] + g2w * v[1])
        y1 = F32(g2w * v[0] + g2w2 * v[1] + g * v[2])
        y2 = F32(g * v[1] + g21 * v[2])
        nrm = F32(np.sqrt(F32(y0 * y0 + y1 * y1 + y2 * y2)))
        if nrm < 1e-10:
            break
        v = [F32(y0 / nrm), F32(y1 / nrm), F32(y2 / nrm)]
    y0 = F32(g4 * v[0] + g2w * v[1])
    y1 = F32(g2w * v[0] + g2w2 * v[1] + g * v[2])
    y2 = F32(g * v[1] + g21 * v[2])
    return F32(v[0] * y0 + v[1] * y1 + v[2] * y2)


# ---------------------------------------------------------------------------
# RESHARP (src/bgremove/resharp.rs) on CG (src/solvers/cg.rs)
# ---------------------------------------------------------------------------
@dataclass
class ResharpParams:  # src/bgremove/resharp.rs:22-45
    radius: float = 6.0
    tik_reg: float = 1e-4
    tol: float = 1e-6
    max_iter: int = 30


def apply_ht_h(dker, w, x):
    """Re IFFT(DKER * FFT(w * IFFT(DKER * FFT(x)))) with the complex intermediate kept
    (src/bgremove/resharp.rs:133-153)."""
    t = ifft3d(fft3d(x.astype(np.complex128)) * dker) * w
    return ifft3d(fft3d(t) * dker).real


def resharp(field_, mask, grid: Grid, params: ResharpParams = ResharpParams(), progress=None):
    """src/bgremove/resharp.rs:58-125 -> (local_field, eroded_mask)."""
    f = _vol(field_, grid)
    m = _vol(mask, grid, np.uint8)
    s_fft = fft_real_kernel(smv_kernel(grid, params.radius))
    dker = 1.0 - s_fft
    eroded = erode_mask_smv(m, s_fft, 1.0 - math.sqrt(1e-7))
    w = eroded.astype(np.float64)
    b = apply_ht_h(dker, w, f)
    lam = params.tik_reg
    x = cg_solve(lambda v: (apply_ht_h(dker, w, v.reshape(grid.shape)) + lam * v.reshape(grid.shape)).ravel(),
                 b.ravel(), np.zeros(f.size), params.tol, params.max_iter, progress)
    return np.where(eroded.ravel() == 1, x, 0.0).reshape(grid.shape), eroded


def apply_reference(chi, mask, method="mean"):
    """src/pipeline/referencing.rs:12-43: Mean subtracts the masked mean; zero outside."""
    x = np.asarray(chi, dtype=np.float64)
    m = np.asarray(mask) > 0
    mu = float(x[m].sum()) / int(m.sum()) if (method == "mean" and m.any()) else 0.0
    return np.where(m, x - mu, 0.0)


# ---------------------------------------------------------------------------
# RTS (src/inversion/rts.rs)
# ---------------------------------------------------------------------------
@dataclass
class RtsParams:  # src/inversion/rts.rs:22-51
    delta: float = 0.15
    mu: float = 1e5
    rho: float = 10.0
    tol: float = 1e-2
    max_iter: int = 20
    lsmr_iter: int = 4


def rts(local_field, mask, grid: Grid, bdir, params: RtsParams = RtsParams(), progress=None, return_iters=False,
        exact_dc=False):
    """src/inversion/rts.rs:72-211: k-space refinement in the well-conditioned region, then
    ADMM (admm.rs:76-145) with inv_a = rho/(M + rho L), unit divergence factor, shrink
    threshold 1/rho, first convergence test against the step-1 estimate.  exact_dc: see
    laplacian_eigenvalues."""
    d = dipole_kernel(grid, bdir)
    lap = laplacian_eigenvalues(grid, exact_dc)
    well = np.abs(d) > params.delta
    m_mask = np.where(well, params.mu, 0.0)
    a = m_mask + params.rho * lap
    with np.errstate(divide="ignore"):
        inv_a = np.where(np.abs(a) > 1e-20, params.rho / a, 0.0)
    F = fft3d(_vol(local_field, grid).astype(np.complex128))
    chi = np.where(well, F * d / (d * d + 1e-6), 0.0)
    for _ in range(params.lsmr_iter):
        res = F - chi * d
        chi = np.where(well, chi + res * d / (d * d + 1e-6), chi)
    m = _vol(mask, grid, np.uint8)
    x = np.where(m != 0, ifft3d(chi).real, 0.0)
    X = fft3d(x.astype(np.complex128))
    f_hat = np.where((np.abs(m_mask) > 1e-20) & (np.abs(inv_a) > 1e-20), X * (m_mask / params.rho) * inv_a, 0.0)
    z = np.zeros(grid.shape)
    ux, uy, uz, gx, gy, gz = z.copy(), z.copy(), z.copy(), z.copy(), z.copy(), z.copy()
    t = 1.0 / params.rho
    iters = 0
    for it in range(params.max_iter):
        if progress is not None:
            progress(it + 1, params.max_iter)
        x_prev = x
        div = bdiv(gx, gy, gz, grid)
        x = ifft3d(f_hat - 1.0 * fft3d(div.astype(np.complex128)) * inv_a).real
        iters = it + 1
        if relative_change(x, x_prev) < params.tol:
            if progress is not None:
                progress(it + 1, it + 1)
            break
        ggx, ggy, ggz = fgrad(x, grid)
        vx, vy, vz = ggx + ux, ggy + uy, ggz + uz
        zx, zy, zz = shrink(vx, t), shrink(vy, t), shrink(vz, t)
        ux, uy, uz = vx - zx, vy - zy, vz - zz
        gx, gy, gz = 2.0 * zx - vx, 2.0 * zy - vy, 2.0 * zz - vz
    out = apply_mask_zero(x, m)
    return (out, iters) if return_iters else out


# ---------------------------------------------------------------------------
# NLTV (src/inversion/nltv.rs)
# ---------------------------------------------------------------------------
@dataclass
class NltvParams:  # src/inversion/nltv.rs:24-48
    lambda_: float = 1e-3
    mu: float = 1.0
    tol: float = 1e-3
    max_iter: int = 250
    newton_iter: int = 10


def nltv(local_field, mask, grid: Grid, bdir, params: NltvParams = NltvParams(), progress=None,
         return_iters=False, exact_dc=False):
    """src/inversion/nltv.rs:62-131 over the shared ADMM step (src/inversion/admm.rs:76-145).

    rho = 100 lambda.  newton_iter outer passes, each an inner ADMM loop of at most
    max_iter steps with the weighted shrink shrink(v, (lambda/rho) w_i) (src/utils/mod.rs:57-59)
    and the usual relative-change exit.  x, x_prev, u and g carry over between passes,
    except that after each pass g is overwritten with grad x (nltv.rs:114) and the weights
    become 1/(|grad x| + mu 1e-6), divided by their maximum when that exceeds 1.
    progress(k, max_iter * newton_iter) is called before every inner step with a running k.
    """
    rho = 100.0 * params.lambda_
    inv_a, f_hat = prepare_admm_spectral(local_field, grid, bdir, rho, exact_dc)
    shape = grid.shape
    x = np.zeros(shape)
    ux = np.zeros(shape); uy = np.zeros(shape); uz = np.zeros(shape)
    gx = np.zeros(shape); gy = np.zeros(shape); gz = np.zeros(shape)
    w = np.ones(shape)
    total = params.max_iter * params.newton_iter
    cur = 0
    t = params.lambda_ / rho
    for _ in range(params.newton_iter):
        for _ in range(params.max_iter):
            cur += 1
            if progress is not None:
                progress(cur, total)
            x_prev = x
            div = bdiv(gx, gy, gz, grid)
            x = ifft3d(f_hat - rho * fft3d(div.astype(np.complex128)) * inv_a).real
            if relative_change(x, x_prev) < params.tol:
                break
            ggx, ggy, ggz = fgrad(x, grid)
            vx, vy, vz = ggx + ux, ggy + uy, ggz + uz
            tw = t * w
            zx, zy, zz = shrink(vx, tw), shrink(vy, tw), shrink(vz, tw)
            ux, uy, uz = vx - zx, vy - zy, vz - zz
            gx, gy, gz = 2.0 * zx - vx, 2.0 * zy - vy, 2.0 * zz - vz
        gx, gy, gz = fgrad(x, grid)
        w = 1.0 / (np.sqrt(gx * gx + gy * gy + gz * gz) + params.mu * 1e-6)
        wmax = float(w.max(initial=0.0))
        if wmax > 1.0:
            w = w / wmax
    out = apply_mask_zero(x, _vol(mask, grid, np.uint8))
    return (out, cur) if return_iters else out


# ---------------------------------------------------------------------------
# iSMV (src/bgremove/ismv.rs)
# ---------------------------------------------------------------------------
@dataclass
class IsmvParams:  # src/bgremove/ismv.rs:19-34
    tol: float = 1e-6
    max_iter: int = 50
    radius: float = 5.0


def ismv(field_, mask, grid: Grid, params: IsmvParams = IsmvParams(), progress=None, return_iters=False):
    """src/bgremove/ismv.rs:48-157: erode with the SMV kernel at 1 - 1e-10, then
    f <- eroded * Re IFFT(F(f) * FFT(S)) + (mask - eroded) * field until the change
    ||f0 - f|| <= tol * ||eroded * field|| (tested at the top of each iteration, f0 the
    previous f, initially eroded * field).  Returns (mask * (field - f), eroded)."""
    s = smv_kernel(grid, params.radius)
    s_fft = fft3d(s.astype(np.complex128))  # complex, as the iteration uses it (ismv.rs:80-85)
    m = _vol(mask, grid, np.uint8)
    eroded = erode_mask_smv(m, fft_real_kernel(s), 1.0 - 1e-10).astype(np.float64)
    m0 = (m != 0).astype(np.float64)
    fld = _vol(field_, grid)
    bc = fld * (m0 - eroded)
    f = fld.copy()
    f0 = fld * eroded
    nr = math.sqrt(float(np.dot(f0.ravel(), f0.ravel())))
    eps = params.tol * nr
    done = 0
    for it in range(params.max_iter):
        if progress is not None:
            progress(it + 1, params.max_iter)
        if nr <= eps:
            if progress is not None:
                progress(it + 1, it + 1)
            break
        f = eroded * ifft3d(fft3d(f.astype(np.complex128)) * s_fft).real + bc
        d = (f0 - f).ravel()
        nr = math.sqrt(float(np.dot(d, d)))
        f0 = f
        done = it + 1
    local = np.where(m != 0, fld - f, 0.0)
    out = (local, (eroded > 0.5).astype(np.uint8))
    return out + (done,) if return_iters else out


# ---------------------------------------------------------------------------
# Multi-echo field mapping (src/utils/multi_echo.rs)
# ---------------------------------------------------------------------------
B0W_PHASE_SNR, B0W_PHASE_VAR, B0W_AVERAGE, B0W_TES, B0W_MAG = range(5)  # B0WeightType, multi_echo.rs:78-91


def calculate_b0_weighted(phases, mags, tes, mask, weight_type=B0W_PHASE_SNR):
    """B0 in Hz = (1/2pi) sum_e (phase_e/TE_e) w_e / sum_e w_e over mask != 0, 0 where
    sum w <= 1e-10 (src/utils/multi_echo.rs:450-506).  Echo loop in the reference's
    order, so the float64 result is the reference's bit for bit."""
    phases = [np.asarray(p, np.float64).ravel() for p in phases]
    mags = [np.asarray(m, np.float64).ravel() for m in mags]
    m = np.asarray(mask).ravel()
    ws_ = np.zeros_like(phases[0])
    w_sum = np.zeros_like(phases[0])
    for e, te in enumerate(tes):
        mag = mags[e]
        if weight_type == B0W_PHASE_SNR:
            w = mag * te
        elif weight_type == B0W_PHASE_VAR:
            w = mag * mag * te * te
        elif weight_type == B0W_AVERAGE:
            w = np.ones_like(mag)
        elif weight_type == B0W_TES:
            w = np.full_like(mag, te)
        else:
            w = mag
        ws_ = ws_ + (phases[e] / te) * w
        w_sum = w_sum + w
    scale = 1.0 / (2.0 * math.pi)
    with np.errstate(divide="ignore", invalid="ignore"):
        b0 = scale * ws_ / w_sum
    return np.where((m != 0) & (w_sum > 1e-10), b0, 0.0)


def compute_reliability_mask(fit_residual, mask, threshold_percentile):
    """src/utils/multi_echo.rs:771-804: threshold = the floor(p/100 * count)-th smallest
    (clamped) of the residuals with mask > 0, r > 0 and finite; reliable where
    mask > 0 and r < threshold; the mask itself when no residual qualifies."""
    r = np.asarray(fit_residual, np.float64).ravel()
    m = np.asarray(mask).ravel()
    sel = (m > 0) & (r > 0.0) & np.isfinite(r)
    vals = np.sort(r[sel])
    if vals.size == 0:
        return m.astype(np.uint8).copy()
    idx = int((threshold_percentile / 100.0) * vals.size)
    thr = vals[min(idx, vals.size - 1)]
    return ((m > 0) & (r < thr)).astype(np.uint8)


def multi_echo_linear_fit(phases, mags, tes, mask, estimate_offset=True, reliability_threshold_percentile=90.0):
    """Magnitude-weighted linear fit phase = offset + slope * TE per voxel
    (src/utils/multi_echo.rs:631-768): (field rad/s, phase_offset, fit_residual,
    reliability_mask).  Echo sums in the reference's order (float64 bit for bit)."""
    phases = [np.asarray(p, np.float64).ravel() for p in phases]
    mags = [np.asarray(w, np.float64).ravel() for w in mags]
    m = np.asarray(mask).ravel()
    n_e = len(phases)
    zero = np.zeros_like(phases[0])
    field, offset, resid = zero.copy(), zero.copy(), zero.copy()
    on = m != 0
    with np.errstate(divide="ignore", invalid="ignore"):
        if estimate_offset:
            sw, swt, swp = zero.copy(), zero.copy(), zero.copy()
            for e in range(n_e):
                w = mags[e]
                sw = sw + w
                swt = swt + w * tes[e]
                swp = swp + w * phases[e]
            ok = on & ~(sw < 1e-10)
            te_mean = swt / sw
            ph_mean = swp / sw
            sxx, sxy = zero.copy(), zero.copy()
            for e in range(n_e):
                w = mags[e]
                tc = tes[e] - te_mean
                pc = phases[e] - ph_mean
                sxx = sxx + w * tc * tc
                sxy = sxy + w * tc * pc
            ok = ok & (sxx > 1e-10)
            slope = sxy / sxx
            icpt = ph_mean - slope * te_mean
            srr = zero.copy()
            for e in range(n_e):
                w = mags[e]
                d = phases[e] - (icpt + slope * tes[e])
                srr = srr + w * d * d
            field = np.where(ok, slope, 0.0)
            offset = np.where(ok, icpt, 0.0)
            resid = np.where(ok, srr / sw * n_e, 0.0)
        else:
            stp, stt, sw = zero.copy(), zero.copy(), zero.copy()
            for e in range(n_e):
                w = mags[e]
                stp = stp + w * tes[e] * phases[e]
                stt = stt + w * tes[e] * tes[e]
                sw = sw + w
            ok = on & (stt > 1e-10)
            slope = stp / stt
            srr = zero.copy()
            for e in range(n_e):
                w = mags[e]
                d = phases[e] - slope * tes[e]
                srr = srr + w * d * d
            field = np.where(ok, slope, 0.0)
            resid = np.where(ok & (sw > 1e-10), srr / sw * n_e, 0.0)
    if reliability_threshold_percentile > 0.0:
        rel_mask = compute_reliability_mask(resid, m, reliability_threshold_percentile)
    else:
        rel_mask = m.astype(np.uint8).copy()
    return field, offset, resid, rel_mask


# ---------------------------------------------------------------------------
# NIfTI-1 (src/io.rs; decoding restated from the `nifti` crate 0.17.0 the reference calls)
# ---------------------------------------------------------------------------
NIFTI_DTYPES = {2: "u1", 4: "i2", 8: "i4", 16: "f4", 64: "f8", 256: "i1", 512: "u2", 768: "u4", 1024: "i8",
                1280: "u8"}


def nifti_save_bytes(data, dims, voxel_size, affine) -> bytes:
    """save_nifti (src/io.rs:255-338): 348-byte header + 4 zero bytes + float32 LE voxels."""
    import struct
    nx, ny, nz = dims
    h = bytearray(348)
    struct.pack_into("<i", h, 0, 348)
    struct.pack_into("<8h", h, 40, 3, nx, ny, nz, 1, 1, 1, 1)
    struct.pack_into("<hh", h, 70, 16, 32)
    struct.pack_into("<8f", h, 76, 1.0, voxel_size[0], voxel_size[1], voxel_size[2], 1.0, 1.0, 1.0, 1.0)
    struct.pack_into("<fff", h, 108, 352.0, 1.0, 0.0)
    struct.pack_into("<h", h, 254, 1)
    struct.pack_into("<12f", h, 280, *[float(a) for a in list(affine)[:12]])
    h[344:348] = b"n+1\0"
    return bytes(h) + b"\0\0\0\0" + np.asarray(data, np.float64).astype("<f4").tobytes()


def nifti_load(raw: bytes, all_volumes=False):
    """load_nifti / load_nifti_4d (src/io.rs:62-224): header fields either byte order,
    voxels from vox_offset cast to float64 and, when scl_slope != 0, raw * slope + inter;
    x fastest; first volume unless all_volumes.  Returns a dict."""
    import gzip as _gz
    import struct
    if len(raw) >= 2 and raw[0] == 0x1F and raw[1] == 0x8B:
        raw = _gz.decompress(raw)
    if len(raw) < 348:
        raise ValueError("header too short")
    e = "<" if struct.unpack_from("<i", raw, 0)[0] == 348 else ">"
    if struct.unpack_from(e + "i", raw, 0)[0] != 348 or raw[344:348] != b"n+1\0":
        raise ValueError("not a NIfTI-1 single file")
    dim = struct.unpack_from(e + "8h", raw, 40)
    if dim[0] < 3:
        raise ValueError("Expected at least 3D volume")
    dt = struct.unpack_from(e + "h", raw, 70)[0]
    pix = struct.unpack_from(e + "8f", raw, 76)
    vo = int(struct.unpack_from(e + "f", raw, 108)[0])
    vo = 352 if vo < 348 else vo
    slope, inter = struct.unpack_from(e + "ff", raw, 112)
    sform = struct.unpack_from(e + "h", raw, 254)[0]
    nx, ny, nz = dim[1], dim[2], dim[3]
    nt = dim[4] if dim[0] >= 4 else 1
    count = nx * ny * nz * (nt if all_volumes else 1)
    vals = np.frombuffer(raw, np.dtype(NIFTI_DTYPES[dt]).newbyteorder(e), count, vo).astype(np.float64)
    if slope != 0.0:
        vals = vals * np.float64(slope) + np.float64(inter)
    if sform > 0:
        aff = list(np.float64(v) for v in struct.unpack_from(e + "12f", raw, 280)) + [0.0, 0.0, 0.0, 1.0]
    else:
        aff = [pix[1], 0, 0, 0, 0, pix[2], 0, 0, 0, 0, pix[3], 0, 0, 0, 0, 1.0]
    return {"data": vals, "dims": (nx, ny, nz, nt), "voxel_size": (float(pix[1]), float(pix[2]), float(pix[3])),
            "affine": np.array(aff, np.float64), "scl_slope": 1.0 if slope == 0.0 else float(slope),
            "scl_inter": float(inter), "datatype": dt}


def nifti_craft(data, dims4, datatype, big_endian=False, slope=0.0, inter=0.0, voxel_size=(1.0, 1.0, 1.0),
                sform=None, ndim=None) -> bytes:
    """A NIfTI-1 single-file image with any stored datatype and byte order (test input)."""
    import struct
    e = ">" if big_endian else "<"
    nx, ny, nz, nt = dims4
    nd = ndim if ndim is not None else (4 if nt > 1 else 3)
    h = bytearray(348)
    struct.pack_into(e + "i", h, 0, 348)
    struct.pack_into(e + "8h", h, 40, nd, nx, ny, nz, nt, 1, 1, 1)
    struct.pack_into(e + "hh", h, 70, datatype, 8 * np.dtype(NIFTI_DTYPES[datatype]).itemsize)
    struct.pack_into(e + "8f", h, 76, 1.0, *voxel_size, 1.0, 1.0, 1.0, 1.0)
    struct.pack_into(e + "fff", h, 108, 352.0, slope, inter)
    if sform is not None:
        struct.pack_into(e + "h", h, 254, 1)
        struct.pack_into(e + "12f", h, 280, *sform)
    h[344:348] = b"n+1\0"
    vals = np.asarray(data).astype(np.dtype(NIFTI_DTYPES[datatype]).newbyteorder(e))
    return bytes(h) + b"\0\0\0\0" + vals.tobytes()
