// iLSQR dipole inversion (src/inversion/ilsqr.rs:1307-1351) -> (chi, xsa, xfs, xlsqr).
//
// Step 1, lsqr_step (ilsqr.rs:953-1030).  Laplacian weights w (mask-adaptive stencil,
//   thresholds at the 60th / 99.9th percentile by exact radix selection), b = D*FFT(w*f),
//   then complex LSQR (ilsqr.rs:177-321, relative-residual stop) on k-space vectors with
//   A = A^H = D*FFT(w*Re IFFT(D*x)).  The vectors are full complex spectra: D is not
//   symmetric under k -> -k on even-length Nyquist planes and the reference iterates on
//   the whole complex vector.  One application of A is five passes,
//     Z inv (pre: *s*D) -> Y inv -> X [inv, w*Re/N, fwd] -> Y fwd -> Z fwd (post: *D - c*old)
//   where s is the deferred 1/beta or 1/alpha of the input vector and the Z fwd pass
//   also accumulates the FP64 norm of its output.  The block that finishes that pass
//   last completes the norm and runs the scalar recurrence on the device, so one LSQR
//   iteration (two applications and the x/w update) is 11 launches without a host
//   synchronisation, replayed as a CUDA graph.
// Step 2, fastqsm_step (ilsqr.rs:1037-1167).  F = FFT(f); k-space weights |D|^0.001
//   normalised by the 1st/30th percentiles of all values; the SMV (r = 3) kernel
//   spectrum; Eq. 9/11 filtering chains with the masked real part taken in the fused X
//   pass between inverse and forward transforms; TKD (t0 = 1/8, sign(+0) = +1) and the
//   2x2 least-squares fit over all voxels (FP64 sums).
// Step 3, susceptibility_artifacts_step (ilsqr.rs:1174-1289).  Gradient weights from
//   the mask-adaptive gradient of xfs (percentiles 50 / 70 per component); LSMR
//   (ilsqr.rs:344-517) on real vectors.  Its k-space mask mic = |D| < 0.1 acts through
//   Re IFFT(FFT(x)*mic), which equals a half-spectrum transform with the multiplier
//   (mic(k) + mic(-k))/2; periodic gradient / divergence stencils carry the weights,
//   the axpy terms and the FP64 norms.
// Step 4: chi = mask * (xlsqr - xsa).
#include "functors.cuh"
#include "select.h"
#include "solvers.h"

#include <algorithm>
#include <cmath>

namespace qsm {

namespace {

// ===================================================================== setup ==
// Mask-adaptive second difference along one axis at linear index l (coordinate c of
// n, stride s), src/inversion/ilsqr.rs:583-669.  The stencil selector is
// 2*m[l+s] + m[l-s] in u8 arithmetic inside, forward (2) at c = 0 and backward (1) at
// c = n-1.
__device__ double lap1(const double* __restrict__ f, const uint8_t* __restrict__ m, long long l, int c, int n,
                       long long s) {
  int sel;
  if (c >= 1 && c <= n - 2) sel = (uint8_t)(2u * m[l + s] + m[l - s]);
  else sel = (c == 0) ? 2 : (c == n - 1 ? 1 : 0);
  if (sel == 3) return f[l - s] - 2.0 * f[l] + f[l + s];
  if (sel == 2) {
    if (c + 3 < n && m[l + 2 * s] != 0 && m[l + 3 * s] != 0)
      return 2.0 * f[l] - 5.0 * f[l + s] + 4.0 * f[l + 2 * s] - f[l + 3 * s];
    if (c + 2 < n && m[l + 2 * s] != 0) return f[l] - 2.0 * f[l + s] + f[l + 2 * s];
    return f[l + s] - f[l];
  }
  if (sel == 1) {
    if (c >= 3 && m[l - 3 * s] != 0 && m[l - 2 * s] != 0)
      return -f[l - 3 * s] + 4.0 * f[l - 2 * s] - 5.0 * f[l - s] + 2.0 * f[l];
    if (c >= 2 && m[l - 2 * s] != 0) return f[l - 2 * s] - 2.0 * f[l - s] + f[l];
    return f[l - s] - f[l];
  }
  return 0.0;
}

// compute_laplacian, src/inversion/ilsqr.rs:528-566 (0 outside the mask)
__global__ void k_ilsqr_lap(const double* __restrict__ f, const uint8_t* __restrict__ m, int nx, int ny, int nz,
                            double hx, double hy, double hz, double* __restrict__ lap) {
  const long long N = (long long)nx * ny * nz, sxy = (long long)nx * ny;
  for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += (long long)gridDim.x * blockDim.x) {
    double v = 0.0;
    if (m[l] != 0) {
      const int i = (int)(l % nx);
      const int j = (int)((l / nx) % ny);
      const int k = (int)(l / sxy);
      v += hx * lap1(f, m, l, i, nx, 1);
      v += hy * lap1(f, m, l, j, ny, nx);
      v += hz * lap1(f, m, l, k, nz, sxy);
    }
    lap[l] = v;
  }
}

// Percentile weight of one value (src/inversion/ilsqr.rs:703-716, 882-897): 1 below
// tmin, 0 above tmax, linear in between when the range exceeds 1e-10.
__device__ __forceinline__ double pct_weight(double v, double tmin, double tmax) {
  const double range = tmax - tmin;
  if (v < tmin) return 1.0;
  if (v > tmax) return 0.0;
  if (range > 1e-10) return (tmax - v) / range;
  return 0.0;
}

template <typename T>
__global__ void k_lap_weights(long long N, const double* __restrict__ lap, const uint8_t* __restrict__ m,
                              double tmin, double tmax, T* __restrict__ w) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    w[i] = m[i] != 0 ? (T)pct_weight(lap[i], tmin, tmax) : T(0);
}

// fgrad_masked, src/inversion/ilsqr.rs:767-823: forward difference when the forward
// neighbour is inside the axis and the mask, else backward, else 0; 0 outside the mask.
template <typename T>
__global__ void k_fgrad_masked(const T* __restrict__ f, const uint8_t* __restrict__ m, int nx, int ny, int nz,
                               double hx, double hy, double hz, double* __restrict__ g) {
  const long long N = (long long)nx * ny * nz, sxy = (long long)nx * ny;
  for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += (long long)gridDim.x * blockDim.x) {
    double gx = 0.0, gy = 0.0, gz = 0.0;
    if (m[l] != 0) {
      const int i = (int)(l % nx);
      const int j = (int)((l / nx) % ny);
      const int k = (int)(l / sxy);
      const double fl = (double)f[l];
      if (i < nx - 1 && m[l + 1] != 0) gx = hx * ((double)f[l + 1] - fl);
      else if (i > 0 && m[l - 1] != 0) gx = hx * (fl - (double)f[l - 1]);
      if (j < ny - 1 && m[l + nx] != 0) gy = hy * ((double)f[l + nx] - fl);
      else if (j > 0 && m[l - nx] != 0) gy = hy * (fl - (double)f[l - nx]);
      if (k < nz - 1 && m[l + sxy] != 0) gz = hz * ((double)f[l + sxy] - fl);
      else if (k > 0 && m[l - sxy] != 0) gz = hz * (fl - (double)f[l - sxy]);
    }
    g[l] = gx;
    g[N + l] = gy;
    g[2 * N + l] = gz;
  }
}

// gradient_weights_component, src/inversion/ilsqr.rs:854-900 (times mask[i] as f64)
template <typename T>
__global__ void k_grad_weights(long long N, const double* __restrict__ g, const uint8_t* __restrict__ m, double tx0,
                               double tx1, double ty0, double ty1, double tz0, double tz1, T* __restrict__ w) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const uint8_t mi = m[i];
    if (mi == 0) {
      w[i] = T(0);
      w[N + i] = T(0);
      w[2 * N + i] = T(0);
      continue;
    }
    const double mv = (double)mi;
    w[i] = (T)(pct_weight(g[i], tx0, tx1) * mv);
    w[N + i] = (T)(pct_weight(g[N + i], ty0, ty1) * mv);
    w[2 * N + i] = (T)(pct_weight(g[2 * N + i], tz0, tz1) * mv);
  }
}

// |D(k)|^n_exp over the full spectrum in natural order (src/inversion/ilsqr.rs:735-737)
__global__ void k_dipole_pow(KSpace K, int nx, int ny, int nz, double n_exp, double* __restrict__ out) {
  const long long N = (long long)nx * ny * nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(i % nx);
    const int iy = (int)((i / nx) % ny);
    const int iz = (int)(i / ((long long)nx * ny));
    const double d = K.dipole(__ldg(K.fx + ix), __ldg(K.fy + iy), __ldg(K.fz + iz));
    out[i] = pow(fabs(d), n_exp);
  }
}

// ==================================================== loaders, stores, mids ==
template <typename T> struct LoadSpecRow {  // full-spectrum row element
  const cplx_t<T>* s;
  int pitch;
  __device__ __forceinline__ cplx_t<T> operator()(int row, int e) const { return s[(long long)row * pitch + e]; }
};
template <typename T> struct StoreSpecRow {
  cplx_t<T>* s;
  int pitch;
  __device__ __forceinline__ void operator()(int row, int e, cplx_t<T> v) { s[(long long)row * pitch + e] = v; }
  __device__ __forceinline__ void finish() {}
};
// real image value (optionally times a second real array) as a complex row element
template <typename Tin, typename T> struct LoadRealProduct {
  const Tin* a;
  const T* b;  // may be null
  int nx;
  __device__ __forceinline__ cplx_t<T> operator()(int row, int e) const {
    const long long i = (long long)row * nx + e;
    double v = (double)a[i];
    if (b != nullptr) v = (double)b[i] * v;
    return mk<cplx_t<T>>((T)v, T(0));
  }
};
// SMV sphere image (src/kernels/smv.rs:19-67) as a complex row element
struct SphereImg {
  int nx, ny, nz;
  double vsx, vsy, vsz, r2, norm;
};
__device__ __forceinline__ double sphere_coord(int i, int n, double vs) { return (double)((i <= n / 2) ? i : i - n) * vs; }
template <typename T> struct LoadSphereC {
  SphereImg s;
  __device__ __forceinline__ cplx_t<T> operator()(int row, int e) const {
    const int j = row % s.ny, k = row / s.ny;
    const double dx = sphere_coord(e, s.nx, s.vsx), dy = sphere_coord(j, s.ny, s.vsy), dz = sphere_coord(k, s.nz, s.vsz);
    const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    return mk<cplx_t<T>>((T)(d2 <= s.r2 ? s.norm : 0.0), T(0));
  }
};
SphereImg sphere_img(const GridDims& d, double radius) {
  SphereImg s{d.nx, d.ny, d.nz, d.vsx, d.vsy, d.vsz, radius * radius, 0.0};
  auto axis = [&](int n, double vs) {
    std::vector<double> v;
    for (int i = 0; i < n; ++i) {
      const double c = (double)((i <= n / 2) ? i : i - n) * vs;
      if (c * c <= s.r2) v.push_back(c);
    }
    return v;
  };
  const std::vector<double> ax = axis(d.nx, d.vsx), ay = axis(d.ny, d.vsy), az = axis(d.nz, d.vsz);
  double count = 0.0;
  for (double dz : az)
    for (double dy : ay)
      for (double dx : ax) {
        volatile double a = dx * dx;
        volatile double b = dy * dy;
        volatile double c = dz * dz;
        volatile double ab = a + b;
        volatile double d2 = ab + c;
        if (d2 <= s.r2) count += 1.0;
      }
  s.norm = count > 0.0 ? 1.0 / count : 0.0;
  return s;
}

// w * Re(v)/N as a real row element (lsqr_step's apply_a, ilsqr.rs:1000-1003)
template <typename T> struct MidWeightRe {
  const T* w;
  int nx;
  T invn;
  __device__ __forceinline__ cplx_t<T> operator()(cplx_t<T> v, int row, int e) const {
    return mk<cplx_t<T>>(w[(long long)row * nx + e] * (v.x * invn), T(0));
  }
};
// mask ? Re(v)/N : 0 as a real row element (fastqsm_step, ilsqr.rs:1093-1100)
template <typename T> struct MidMaskRe {
  const uint8_t* m;
  int nx;
  T invn;
  __device__ __forceinline__ cplx_t<T> operator()(cplx_t<T> v, int row, int e) const {
    return mk<cplx_t<T>>(m[(long long)row * nx + e] != 0 ? v.x * invn : T(0), T(0));
  }
};
// out[i] = mask ? Re(v)/N : 0
template <typename T, typename Tout> struct StoreMaskRe {
  Tout* out;
  const uint8_t* m;
  int nx;
  T invn;
  __device__ __forceinline__ void operator()(int row, int e, cplx_t<T> v) {
    const long long i = (long long)row * nx + e;
    out[i] = m[i] != 0 ? (Tout)(v.x * invn) : Tout(0);
  }
  __device__ __forceinline__ void finish() {}
};

// ====================================================================== LSQR ==
struct LsqrState {
  int done;   // every later kernel returns at once
  int stop;   // convergence seen by the rotation; committed after the x/w update
  int iters;  // completed iterations
  unsigned counter;
  double alpha, beta;
  double su, sv;  // deferred scales of u and v: 1/beta and 1/alpha (1 when zero)
  double rho_bar, phi_bar, bnorm, t1, t2, tol;
};

__device__ __forceinline__ double dip(const KSpace& K, int ix, int iy, int iz) {
  return K.dipole(__ldg(K.fx + ix), __ldg(K.fy + iy), __ldg(K.fz + iz));
}

// pre: (x * s) * D(k), s = the input vector's deferred scale
template <typename T> struct OpScaleD {
  using C = cplx_t<T>;
  KSpace K;
  const double* s;
  // the dipole evaluation runs over a staged tile (k_pass_yz_st_op): inside the first
  // stage's direct loads it lengthened their latency chain (309 against 256 us in float)
  static constexpr bool kStagedPre = true;
  __device__ __forceinline__ C pre(C v, int ix, int iy, int iz, long long) const {
    return cscale(cscale(v, (T)*s), (T)dip(K, ix, iy, iz));
  }
  __device__ __forceinline__ C post(C v, int, int, int, long long) const { return v; }
};

// Z forward epilogue of an A application.  mode 0: u = A v - alpha*u (then beta);
// 1: v = A u - beta*v (then alpha and the rotation); 2: b (then beta = ||b||);
// 3: v = A^H u (then alpha; alpha*beta = 0 ends the solve with x = 0).
template <typename T> struct OpLsqrOut {
  using C = cplx_t<T>;
  KSpace K;
  const C* old;
  LsqrState* st;
  int mode;
  // the compile-time pass stages `old` through shared memory (k_pass_yz_dx_old)
  static constexpr bool kReadsOld = true;
  struct Scalars {
    double coef, sc;
  };
  __device__ __forceinline__ C pre(C v, int, int, int, long long) const { return v; }
  __device__ __forceinline__ C post(C v, int ix, int iy, int iz, long long idx, double& acc) const {
    C r = cscale(v, (T)dip(K, ix, iy, iz));
    if (mode <= 1) {
      const double coef = mode == 0 ? -st->alpha : -st->beta;
      const double sc = mode == 0 ? st->su : st->sv;
      const C o = cscale(old[idx], (T)sc);
      r = cadd(r, cscale(o, (T)coef));
    }
    acc += (double)r.x * (double)r.x + (double)r.y * (double)r.y;
    return r;
  }
  __device__ __forceinline__ const C* old_src() const { return mode <= 1 ? old : nullptr; }
  __device__ __forceinline__ Scalars scalars() const {
    if (mode > 1) return Scalars{0.0, 0.0};
    return Scalars{mode == 0 ? -st->alpha : -st->beta, mode == 0 ? st->su : st->sv};
  }
  // post() with the old value and the scalars already in hand (same arithmetic)
  __device__ __forceinline__ C post_old(C v, int ix, int iy, int iz, C oldv, const Scalars& s, double& acc) const {
    C r = cscale(v, (T)dip(K, ix, iy, iz));
    if (mode <= 1) {
      const C o = cscale(oldv, (T)s.sc);
      r = cadd(r, cscale(o, (T)s.coef));
    }
    acc += (double)r.x * (double)r.x + (double)r.y * (double)r.y;
    return r;
  }
  __device__ void last(double total) const {
    const double nrm = sqrt(total);
    if (mode == 0 || mode == 2) {
      st->beta = nrm;
      st->su = nrm > 0.0 ? 1.0 / nrm : 1.0;
      if (mode == 2) {
        st->bnorm = nrm;
        st->phi_bar = nrm;
      }
      return;
    }
    st->alpha = nrm;
    st->sv = nrm > 0.0 ? 1.0 / nrm : 1.0;
    if (mode == 3) {
      st->rho_bar = nrm;
      if (nrm * st->beta == 0.0) st->done = 1;
      return;
    }
    // Givens rotation and step lengths, src/inversion/ilsqr.rs:261-290
    const double alpha = nrm, beta = st->beta;
    const double rho = sqrt(st->rho_bar * st->rho_bar + beta * beta);
    const double c = st->rho_bar / rho;
    const double s = beta / rho;
    const double theta = s * alpha;
    st->rho_bar = -c * alpha;
    const double phi = c * st->phi_bar;
    st->phi_bar *= s;
    st->t1 = phi / rho;
    st->t2 = -theta / rho;
    st->iters += 1;
    if (st->phi_bar / (st->bnorm + 1e-20) <= st->tol) st->stop = 1;
  }
};

template <typename T>
__global__ void k_lsqr_init_w(long long n, const cplx_t<T>* __restrict__ v, cplx_t<T>* __restrict__ w,
                              const LsqrState* st) {
  if (st->done) return;
  const T sv = (T)st->sv;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    w[i] = cscale(v[i], sv);
}

// x += t1*w; w = v + t2*w (src/inversion/ilsqr.rs:285-290); the last block commits a
// convergence stop.
template <typename T>
__global__ void k_lsqr_update(long long n, cplx_t<T>* __restrict__ x, cplx_t<T>* __restrict__ w,
                              const cplx_t<T>* __restrict__ v, LsqrState* st, double* partials) {
  if (st->done) return;
  const T t1 = (T)st->t1, t2 = (T)st->t2, sv = (T)st->sv;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const cplx_t<T> wi = w[i];
    x[i] = cadd(x[i], cscale(wi, t1));
    w[i] = cadd(cscale(v[i], sv), cscale(wi, t2));
  }
  double z[1] = {0.0};
  if (grid_sum_last<1>(z, partials, &st->counter) && threadIdx.x == 0 && st->stop) st->done = 1;
}

// ============================================================ FastQSM ops ==
// Eq. 9/11 filter x*wfs + x*h*(1 - wfs) with wfs = clamp((|D|^n - lo)/(hi - lo)),
// src/inversion/ilsqr.rs:739-757, 1080-1088
template <typename T> struct FsFilter {
  using C = cplx_t<T>;
  KSpace K;
  const cplx_t<T>* h;  // SMV kernel spectrum (real part used)
  double n_exp, lo, range;
  __device__ __forceinline__ C apply(C x, int ix, int iy, int iz, long long idx) const {
    double w = pow(fabs(dip(K, ix, iy, iz)), n_exp);
    if (range > 1e-20) w = (w - lo) / range;
    w = fmin(fmax(w, 0.0), 1.0);
    const T wt = (T)w, hh = h[idx].x;
    return cadd(cscale(x, wt), cscale(cscale(x, hh), T(1) - wt));
  }
};
// pre of the first inverse Z pass: x = F*sign(D) (ilsqr.rs:1057-1060), then the filter
template <typename T> struct OpFsFirst {
  using C = cplx_t<T>;
  FsFilter<T> F;
  __device__ __forceinline__ C pre(C v, int ix, int iy, int iz, long long idx) const {
    const double d = dip(F.K, ix, iy, iz);
    const T sg = d > 0.0 ? T(1) : (d < 0.0 ? T(-1) : T(0));
    return F.apply(cscale(v, sg), ix, iy, iz, idx);
  }
  __device__ __forceinline__ C post(C v, int, int, int, long long) const { return v; }
};
template <typename T> struct OpFsMid {
  using C = cplx_t<T>;
  FsFilter<T> F;
  __device__ __forceinline__ C mid(C v, int ix, int iy, int iz, long long idx) const {
    return F.apply(v, ix, iy, iz, idx);
  }
};
// pre: F * inv_d with inv_d = signum(D)/t0 where |D| < t0, else 1/D (ilsqr.rs:1118-1126)
template <typename T> struct OpTkdInv {
  using C = cplx_t<T>;
  KSpace K;
  double t0;
  __device__ __forceinline__ C pre(C v, int ix, int iy, int iz, long long) const {
    const double d = dip(K, ix, iy, iz);
    const double inv = fabs(d) < t0 ? copysign(1.0, d) / t0 : 1.0 / d;
    return cscale(v, (T)inv);
  }
  __device__ __forceinline__ C post(C v, int, int, int, long long) const { return v; }
};

// sums of xfs, xtkd, xfs^2, xfs*xtkd over all voxels (ilsqr.rs:1141-1146)
template <typename T>
__global__ void k_fs_sums(long long N, const T* __restrict__ a, const T* __restrict__ b, double* partials,
                          unsigned* counter, double* out) {
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const double x = (double)a[i], y = (double)b[i];
    s[0] += x;
    s[1] += y;
    s[2] += x * x;
    s[3] += x * y;
  }
  if (grid_sum_last<4>(s, partials, counter) && threadIdx.x == 0)
    for (int k = 0; k < 4; ++k) out[k] = s[k];
}

template <typename T>
__global__ void k_fs_final(long long N, const T* __restrict__ xfs, const uint8_t* __restrict__ m, double a, double b,
                           T* __restrict__ out, double* __restrict__ out64) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const double v = m[i] != 0 ? a * (double)xfs[i] + b : 0.0;
    out[i] = (T)v;
    if (out64) out64[i] = v;
  }
}

// ====================================================================== LSMR ==
struct LsmrState {
  int done;
  int iters;
  unsigned counter;
  int pad;
  double alpha, beta, su, sv;
  double alpha_bar, zeta_bar, rho, rho_bar, c_bar, s_bar, zeta;
  double normb, betadd, betad, rhodold, tautildeold, thetatilde;
  double norm_a2, maxrbar, minrbar;
  double atol, btol;
  double c_hbar, c_x, c_h;  // update coefficients of this iteration
  double normr, norm_a, cond_a, norm_ar;
};

// mic(k) = |D(k)| < 0.1 symmetrised over k -> -k (ilsqr.rs:1192-1194)
template <typename T> struct OpMic {
  using C = cplx_t<T>;
  KSpace K;
  __device__ __forceinline__ C mid(C v, int ix, int iy, int iz, long long) const {
    const double m = K.sym(ix, iy, iz, [&](double kx, double ky, double kz, int, int, int) {
      return fabs(K.dipole(kx, ky, kz)) < 0.1 ? 1.0 : 0.0;
    });
    return cscale(v, (T)m);
  }
};

template <typename T> struct LoadScaled {  // x * s (s = deferred scale in the state)
  const T* p;
  const double* s;
  int nx;
  __device__ __forceinline__ T operator()(int row, int e) const { return p[(long long)row * nx + e] * (T)*s; }
};
template <typename T> struct StoreScaledReal {
  T* out;
  int nx;
  T invn;
  __device__ __forceinline__ void operator()(int row, int e, T v) { out[(long long)row * nx + e] = v * invn; }
  __device__ __forceinline__ void finish() {}
};

// v = Re IFFT(...)/N - beta*v (ilsqr.rs:1260-1276 then :425-427), with ||v||^2; the
// last block runs the LSMR recurrences (ilsqr.rs:433-492).  init: v = A^T u only.
template <typename T> struct StoreLsmrV {
  T* v;
  int nx;
  T invn;
  LsmrState* st;
  double* partials;
  int init;
  double acc;
  __device__ __forceinline__ void operator()(int row, int e, T val) {
    const long long i = (long long)row * nx + e;
    T r = val * invn;
    if (!init) r = r + (T)(-st->beta) * (v[i] * (T)st->sv);
    v[i] = r;
    acc += (double)r * (double)r;
  }
  __device__ void finish() {
    double a[1] = {acc};
    if (!grid_sum_last<1>(a, partials, &st->counter)) return;
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    if (tid != 0) return;
    const double alpha = sqrt(a[0]);
    st->alpha = alpha;
    st->sv = alpha > 0.0 ? 1.0 / alpha : 1.0;
    if (init) {
      st->alpha_bar = alpha;
      st->zeta_bar = alpha * st->beta;
      st->norm_a2 = alpha * alpha;
      if (alpha * st->beta == 0.0) st->done = 1;
      return;
    }
    const double beta = st->beta;
    const double rho_old = st->rho;
    const double rho = sqrt(st->alpha_bar * st->alpha_bar + beta * beta);
    const double c = st->alpha_bar / rho;
    const double s = beta / rho;
    const double theta_new = s * alpha;
    st->alpha_bar = c * alpha;
    const double rho_bar_old = st->rho_bar;
    const double zeta_old = st->zeta;
    const double theta_bar = st->s_bar * rho;
    const double rho_temp = st->c_bar * rho;
    const double rho_bar = sqrt(rho_temp * rho_temp + theta_new * theta_new);
    st->c_bar = rho_temp / rho_bar;
    st->s_bar = theta_new / rho_bar;
    const double zeta = st->c_bar * st->zeta_bar;
    st->zeta_bar *= -st->s_bar;
    st->c_hbar = theta_bar * rho / (rho_old * rho_bar_old);
    st->c_x = zeta / (rho * rho_bar);
    st->c_h = theta_new / rho;
    st->rho = rho;
    st->rho_bar = rho_bar;
    st->zeta = zeta;
    // ||r|| estimate (undamped), ilsqr.rs:452-471
    const double betaacute = st->betadd;
    const double betahat = c * betaacute;
    st->betadd = -s * betaacute;
    const double thetatildeold = st->thetatilde;
    const double rhotildeold = sqrt(st->rhodold * st->rhodold + theta_bar * theta_bar);
    const double ctildeold = st->rhodold / rhotildeold;
    const double stildeold = theta_bar / rhotildeold;
    st->thetatilde = stildeold * rho_bar;
    st->rhodold = ctildeold * rho_bar;
    st->betad = -stildeold * st->betad + ctildeold * betahat;
    st->tautildeold = (zeta_old - thetatildeold * st->tautildeold) / rhotildeold;
    const double taud = (zeta - st->thetatilde * st->tautildeold) / st->rhodold;
    const double bd = st->betad - taud;
    st->normr = sqrt(0.0 + bd * bd + st->betadd * st->betadd);
    // ||A|| and cond(A), ilsqr.rs:474-484
    st->norm_a2 += beta * beta;
    st->norm_a = sqrt(st->norm_a2);
    st->norm_a2 += alpha * alpha;
    st->maxrbar = fmax(st->maxrbar, rho_bar_old);
    if (st->iters > 0) st->minrbar = fmin(st->minrbar, rho_bar_old);
    st->cond_a = fmax(st->maxrbar, rho_temp) / fmin(st->minrbar, rho_temp);
    st->norm_ar = fabs(st->zeta_bar);
  }
};

// u = w * fgrad(x) - alpha*u (ilsqr.rs:1226-1238, then :420-421), periodic forward
// differences; accumulates ||u||^2.  init: u = w * fgrad(x0) = b (no subtraction).
template <typename Tin, typename T>
__global__ void k_lsmr_grad(int nx, int ny, int nz, T hx, T hy, T hz, const Tin* __restrict__ x,
                            const T* __restrict__ w, T* __restrict__ u, LsmrState* st, double* partials, int init) {
  if (st->done) return;
  const long long N = (long long)nx * ny * nz, sxy = (long long)nx * ny;
  const T coef = init ? T(0) : (T)(-st->alpha);
  const T su = (T)st->su;
  double acc[1] = {0.0};
  for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += (long long)gridDim.x * blockDim.x) {
    const unsigned r = (unsigned)l / (unsigned)nx;  // N < 2^32 (checked by the host)
    const int i = (int)((unsigned)l - r * (unsigned)nx);
    const int j = (int)(r % (unsigned)ny);
    const int k = (int)(r / (unsigned)ny);
    const long long lx = i + 1 < nx ? l + 1 : l + 1 - nx;
    const long long ly = j + 1 < ny ? l + nx : l + nx - sxy;
    const long long lz = k + 1 < nz ? l + sxy : l + sxy - N;
    const T xl = (T)x[l];
    const T g[3] = {((T)x[lx] - xl) * hx, ((T)x[ly] - xl) * hy, ((T)x[lz] - xl) * hz};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T r = w[c * N + l] * g[c];
      if (!init) r = r + coef * (u[c * N + l] * su);
      u[c * N + l] = r;
      acc[0] += (double)r * (double)r;
    }
  }
  if (grid_sum_last<1>(acc, partials, &st->counter) && threadIdx.x == 0) {
    const double beta = sqrt(acc[0]);
    st->beta = beta;
    st->su = beta > 0.0 ? 1.0 / beta : 1.0;
    if (init) {
      st->normb = beta;
      st->betadd = beta;
    }
  }
}

// q = -bdiv(w * u) (ilsqr.rs:1248-1258), periodic backward differences
template <typename T>
__global__ void k_lsmr_div(int nx, int ny, int nz, T hx, T hy, T hz, const T* __restrict__ w,
                           const T* __restrict__ u, T* __restrict__ q, const LsmrState* st) {
  if (st->done) return;
  const long long N = (long long)nx * ny * nz, sxy = (long long)nx * ny;
  const T su = (T)st->su;
  auto wy = [&](int c, long long l) { return w[c * N + l] * (u[c * N + l] * su); };
  for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += (long long)gridDim.x * blockDim.x) {
    const unsigned r = (unsigned)l / (unsigned)nx;
    const int i = (int)((unsigned)l - r * (unsigned)nx);
    const int j = (int)(r % (unsigned)ny);
    const int k = (int)(r / (unsigned)ny);
    const long long lx = i > 0 ? l - 1 : l - 1 + nx;
    const long long ly = j > 0 ? l - nx : l - nx + sxy;
    const long long lz = k > 0 ? l - sxy : l - sxy + N;
    const T div = (wy(0, l) - wy(0, lx)) * hx + (wy(1, l) - wy(1, ly)) * hy + (wy(2, l) - wy(2, lz)) * hz;
    q[l] = -div;
  }
}

template <typename T>
__global__ void k_lsmr_init(long long N, const T* __restrict__ v, T* __restrict__ h, T* __restrict__ hbar,
                            T* __restrict__ x, const LsmrState* st) {
  const T sv = (T)st->sv;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    h[i] = v[i] * sv;
    hbar[i] = T(0);
    x[i] = T(0);
  }
}

// h_bar = h - c1*h_bar; x += c2*h_bar; h = v - c3*h (ilsqr.rs:445-449), then ||x|| and
// the stopping tests (ilsqr.rs:487-510) in the last block.
template <typename T>
__global__ void k_lsmr_update(long long N, T* __restrict__ h, T* __restrict__ hbar, T* __restrict__ x,
                              const T* __restrict__ v, LsmrState* st, double* partials) {
  if (st->done) return;
  const T c1 = (T)st->c_hbar, c2 = (T)st->c_x, c3 = (T)st->c_h, sv = (T)st->sv;
  double acc[1] = {0.0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const T hb = h[i] - c1 * hbar[i];
    hbar[i] = hb;
    const T xi = x[i] + c2 * hb;
    x[i] = xi;
    h[i] = v[i] * sv - c3 * h[i];
    acc[0] += (double)xi * (double)xi;
  }
  if (grid_sum_last<1>(acc, partials, &st->counter) && threadIdx.x == 0) {
    const double normx = sqrt(acc[0]);
    const double test1 = st->normr / (st->normb + 1e-20);
    const double test2 = st->norm_ar / ((st->norm_a * st->normr) + 1e-20);
    const double test3 = 1.0 / (st->cond_a + 1e-20);
    const double rtol = st->btol + st->atol * st->norm_a * normx / (st->normb + 1e-20);
    st->iters += 1;
    if (test3 <= 1.0 / 1e8 || test2 <= st->atol || test1 <= rtol) st->done = 1;
  }
}

template <typename T>
__global__ void k_ilsqr_out(long long N, const double* __restrict__ xlsqr, const T* __restrict__ xsa,
                            const uint8_t* __restrict__ m, double* __restrict__ chi, double* __restrict__ xsa_out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const bool in = m[i] != 0;
    const double s = in ? (double)xsa[i] : 0.0;
    chi[i] = in ? xlsqr[i] - s : 0.0;
    if (xsa_out) xsa_out[i] = s;
  }
}

// Replay `one` (a fixed sequence of launches that all return once *done is set) up to
// `iters` times: as a CUDA graph of one iteration polled every 8 launches, or eagerly
// while profiling.  Returns the number of iterations the device counted.
template <class One>
void run_iterations(qsm_ctx* ctx, size_t iters, const int* d_done, One one) {
  if (iters == 0) return;
  int h_done = 0;
  auto poll = [&]() {
    d2h(ctx, &h_done, d_done, sizeof(int));
    sync(ctx);
    return h_done != 0;
  };
  if (ctx->profiling) {
    for (size_t it = 0; it < iters; ++it) {
      one();
      if ((it + 1) % 8 == 0 && poll()) return;
    }
    return;
  }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const uint64_t l0 = ctx->launches;
  QSM_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  try {
    one();
  } catch (...) {
    cudaStreamEndCapture(ctx->stream, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  QSM_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
  const uint64_t per = ctx->launches - l0;
  ctx->launches = l0;
  cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) throw QsmError(QSM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
  try {
    for (size_t it = 0; it < iters; ++it) {
      QSM_CUDA(cudaGraphLaunch(exec, ctx->stream));
      ctx->launches += per;
      if ((it + 1) % 8 == 0 && it + 1 < iters && poll()) break;
    }
  } catch (...) {
    cudaGraphExecDestroy(exec);
    throw;
  }
  cudaGraphExecDestroy(exec);
}

}  // namespace

// T: arithmetic of the Krylov steps (LSQR, step 1; LSMR, step 3) and of their vectors;
// TD: arithmetic of the direct step 2 (fastQSM filtering, TKD, the fit).  An FP64 context
// runs both in double; a mixed context runs step 2 in float and the Krylov steps in
// double unless its Krylov precision is set to mixed: the reference stops LSQR after 50
// iterations short of its tolerance, so its result is the truncated Krylov iterate, and
// float rounding in the operator is amplified about a thousandfold there.
template <typename T, typename TD>
void ilsqr_impl(qsm_ctx* ctx, const GridDims& d, const double* f, const uint8_t* mask, const double bdir[3],
                const qsm_ilsqr_params& p, qsm_progress_fn progress, void* user, double* chi, double* xsa_out,
                double* xfs_out, double* xlsqr_out) {
  using C = cplx_t<T>;
  using CD = cplx_t<TD>;
  const long long N = d.n;
  const char* pre = sizeof(T) == 4 ? "il32." : "il64.";
  auto nm = [&](const char* s) { return std::string(pre) + s; };
  const char* pre_d = sizeof(TD) == 4 ? "il32." : "il64.";
  auto nmd = [&](const char* s) { return std::string(pre_d) + s; };
  auto report = [&](size_t k) {
    if (progress) progress(user, k, 4);
  };
  double* xlsqr = xlsqr_out ? xlsqr_out : ws<double>(ctx, nm("xlsqr"), (size_t)N);
  const long long count = count_selected(ctx, mask, N);
  if (count == 0) {
    // every weight and every masked output is zero (the reference returns zeros)
    for (double* o : {chi, xsa_out, xfs_out, xlsqr_out})
      if (o) QSM_CUDA(cudaMemsetAsync(o, 0, sizeof(double) * N, ctx->stream));
    for (size_t k = 1; k <= 4; ++k) report(k);
    sync(ctx);
    return;
  }
  Fft3<T> ff = make_fft3_full<T>(ctx, d);
  Fft3<T> fh = make_fft3<T>(ctx, d);
  KSpace K = make_kspace(ctx, d, bdir);
  const long long NF = ff.g.hsize();
  const T invn = (T)(1.0 / (double)N);
  double* partials = ws<double>(ctx, nm("partials"), (size_t)kMaxPersistentBlocks * 4);
  unsigned* counter = ws<unsigned>(ctx, nm("counter"), 1);
  QSM_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), ctx->stream));
  C* t = ws<C>(ctx, nm("t"), (size_t)NF);
  C* ub = ws<C>(ctx, nm("u"), (size_t)NF);
  C* vb = ws<C>(ctx, nm("v"), (size_t)NF);
  C* wb = ws<C>(ctx, nm("w"), (size_t)NF);
  C* xb = ws<C>(ctx, nm("x"), (size_t)NF);
  for (C* b : {t, ub, vb, wb, xb}) QSM_CUDA(cudaMemsetAsync(b, 0, sizeof(C) * NF, ctx->stream));
  double* dwork = ws<double>(ctx, nm("dwork"), (size_t)(3 * N));
  const double hx2 = 1.0 / (d.vsx * d.vsx), hy2 = 1.0 / (d.vsy * d.vsy), hz2 = 1.0 / (d.vsz * d.vsz);

  // ------------------------------------------------------------- step 1 --
  report(1);
  T* wl = ws<T>(ctx, nm("wlap"), (size_t)N);
  {
    LaunchScope ls(ctx, "ilsqr_lap");
    k_ilsqr_lap<<<grid1d(N), 256, 0, ctx->stream>>>(f, mask, d.nx, d.ny, d.nz, hx2, hy2, hz2, dwork);
    ls.done();
  }
  {
    const std::vector<double> th = percentiles(ctx, dwork, mask, N, count, {60.0, 99.9});
    LaunchScope ls(ctx, "ilsqr_lap_weights");
    k_lap_weights<T><<<grid1d(N), 256, 0, ctx->stream>>>(N, dwork, mask, th[0], th[1], wl);
    ls.done();
  }
  LsqrState* lst = ws<LsqrState>(ctx, nm("lsqr"), 1);
  {
    LsqrState init{};
    init.tol = 0.01;  // tol_lsqr, ilsqr.rs:966
    h2d(ctx, lst, &init, sizeof(init));
  }
  const int* ldone = &lst->done;
  // b = D * FFT(w*f) -> u, beta = ||b||
  run_x_full<T, -1, 0>(ctx, ff, LoadRealProduct<double, T>{f, wl, d.nx}, MidId<T>{}, StoreSpecRow<T>{t, ff.g.pitch},
                       nullptr, "fft_x_c2c");
  run_yz<T, -1, 1>(ctx, ff, t, t, OpId<T>{}, nullptr);
  run_yz_acc<T, -1, 2, true>(ctx, ff, t, ub, OpLsqrOut<T>{K, nullptr, lst, 2}, partials, counter, nullptr, "fft_z_lsqr");
  // y = A(s*x) written to dst with the given epilogue mode
  auto apply_a = [&](const C* x, const double* s, C* dst, const C* old, int mode) {
    // compile-time staged pass (a direct-fetch first stage with the dipole scale in its
    // loads ran 309 against 256 us at 384x384x256 in float, 619 against 450 us in double)
    run_yz<T, +1, 2, true>(ctx, ff, x, t, OpScaleD<T>{K, s}, ldone);
    run_yz<T, +1, 1>(ctx, ff, t, t, OpId<T>{}, ldone);
    run_x_full<T, +1, -1, true>(ctx, ff, LoadSpecRow<T>{t, ff.g.pitch}, MidWeightRe<T>{wl, d.nx, invn},
                          StoreSpecRow<T>{t, ff.g.pitch}, ldone, "fft_x_lsqr");
    run_yz<T, -1, 1>(ctx, ff, t, t, OpId<T>{}, ldone);
    run_yz_acc<T, -1, 2, true>(ctx, ff, t, dst, OpLsqrOut<T>{K, old, lst, mode}, partials, counter, ldone, "fft_z_lsqr");
  };
  // v = A^H u, alpha; w = v
  apply_a(ub, &lst->su, vb, nullptr, 3);
  {
    LaunchScope ls(ctx, "lsqr_init");
    k_lsqr_init_w<T><<<grid1d(NF), 256, 0, ctx->stream>>>(NF, vb, wb, lst);
    ls.done();
  }
  const unsigned ugrid = grid1d(NF);
  run_iterations(ctx, 50, ldone, [&]() {  // maxit_lsqr, ilsqr.rs:967
    apply_a(vb, &lst->sv, ub, ub, 0);
    apply_a(ub, &lst->su, vb, vb, 1);
    LaunchScope ls(ctx, "lsqr_update");
    k_lsqr_update<T><<<ugrid, 256, 0, ctx->stream>>>(NF, xb, wb, vb, lst, partials);
    ls.done();
  });
  // xlsqr = mask * Re IFFT(x)
  run_yz<T, +1, 2>(ctx, ff, xb, t, OpId<T>{}, nullptr);
  run_yz<T, +1, 1>(ctx, ff, t, t, OpId<T>{}, nullptr);
  run_x_full<T, +1, 0>(ctx, ff, LoadSpecRow<T>{t, ff.g.pitch}, MidId<T>{}, StoreMaskRe<T, double>{xlsqr, mask, d.nx, invn},
                       nullptr, "fft_x_c2c");

  // ------------------------------------------------------------- step 2 --
  report(2);
  // step 2 runs in TD; with TD == T its buffers are step 1's (same names, same sizes)
  Fft3<TD> ffd = make_fft3_full<TD>(ctx, d);
  const TD invnd = (TD)(1.0 / (double)N);
  CD* Fb = ws<CD>(ctx, nmd("v"), (size_t)NF);  // FFT(f)
  CD* hs = ws<CD>(ctx, nmd("u"), (size_t)NF);  // SMV kernel spectrum
  CD* td = ws<CD>(ctx, nmd("t"), (size_t)NF);
  run_x_full<TD, -1, 0>(ctx, ffd, LoadRealProduct<double, TD>{f, nullptr, d.nx}, MidId<TD>{},
                       StoreSpecRow<TD>{Fb, ffd.g.pitch}, nullptr, "fft_x_c2c");
  run_yz<TD, -1, 1>(ctx, ffd, Fb, Fb, OpId<TD>{}, nullptr);
  run_yz<TD, -1, 2>(ctx, ffd, Fb, Fb, OpId<TD>{}, nullptr);
  run_x_full<TD, -1, 0>(ctx, ffd, LoadSphereC<TD>{sphere_img(d, 3.0)}, MidId<TD>{}, StoreSpecRow<TD>{hs, ffd.g.pitch},
                       nullptr, "fft_x_c2c");
  run_yz<TD, -1, 1>(ctx, ffd, hs, hs, OpId<TD>{}, nullptr);
  run_yz<TD, -1, 2>(ctx, ffd, hs, hs, OpId<TD>{}, nullptr);
  FsFilter<TD> filt{K, hs, 0.001, 0.0, 0.0};
  {
    LaunchScope ls(ctx, "ilsqr_dipole_pow");
    k_dipole_pow<<<grid1d(N), 256, 0, ctx->stream>>>(K, d.nx, d.ny, d.nz, 0.001, dwork);
    ls.done();
    const std::vector<double> th = percentiles(ctx, dwork, nullptr, N, N, {1.0, 30.0});
    filt.lo = th[0];
    filt.range = th[1] - th[0];
  }
  TD* xfs_raw = ws<TD>(ctx, nmd("xfs_raw"), (size_t)N);
  TD* xtkd = ws<TD>(ctx, nmd("xtkd"), (size_t)N);
  TD* xfs = ws<TD>(ctx, nmd("xfs"), (size_t)N);
  run_yz<TD, +1, 2>(ctx, ffd, Fb, td, OpFsFirst<TD>{filt}, nullptr);
  run_yz<TD, +1, 1>(ctx, ffd, td, td, OpId<TD>{}, nullptr);
  run_x_full<TD, +1, -1>(ctx, ffd, LoadSpecRow<TD>{td, ffd.g.pitch}, MidMaskRe<TD>{mask, d.nx, invnd},
                        StoreSpecRow<TD>{td, ffd.g.pitch}, nullptr, "fft_x_fastqsm");
  run_yz<TD, -1, 1>(ctx, ffd, td, td, OpId<TD>{}, nullptr);
  run_z_fused<TD>(ctx, ffd, td, td, OpFsMid<TD>{filt}, nullptr);
  run_yz<TD, +1, 1>(ctx, ffd, td, td, OpId<TD>{}, nullptr);
  run_x_full<TD, +1, 0>(ctx, ffd, LoadSpecRow<TD>{td, ffd.g.pitch}, MidId<TD>{}, StoreMaskRe<TD, TD>{xfs_raw, mask, d.nx, invnd},
                       nullptr, "fft_x_c2c");
  run_yz<TD, +1, 2>(ctx, ffd, Fb, td, OpTkdInv<TD>{K, 1.0 / 8.0}, nullptr);
  run_yz<TD, +1, 1>(ctx, ffd, td, td, OpId<TD>{}, nullptr);
  run_x_full<TD, +1, 0>(ctx, ffd, LoadSpecRow<TD>{td, ffd.g.pitch}, MidId<TD>{}, StoreMaskRe<TD, TD>{xtkd, mask, d.nx, invnd},
                       nullptr, "fft_x_c2c");
  {
    double* sums = ws<double>(ctx, nmd("sums"), 4);
    LaunchScope ls(ctx, "fastqsm_sums");
    k_fs_sums<TD><<<grid1d(N), 256, 0, ctx->stream>>>(N, xfs_raw, xtkd, partials, counter, sums);
    ls.done();
    double s[4];
    d2h(ctx, s, sums, sizeof(s));
    sync(ctx);
    const double n_all = (double)N;
    const double det = s[2] * n_all - s[0] * s[0];
    double a = 1.0, b = 0.0;
    if (std::fabs(det) > 1e-20) {
      a = (n_all * s[3] - s[0] * s[1]) / det;
      b = (s[2] * s[1] - s[0] * s[3]) / det;
    }
    LaunchScope ls2(ctx, "fastqsm_final");
    k_fs_final<TD><<<grid1d(N), 256, 0, ctx->stream>>>(N, xfs_raw, mask, a, b, xfs, xfs_out);
    ls2.done();
  }

  // ------------------------------------------------------------- step 3 --
  report(3);
  T* wg = ws<T>(ctx, nm("wgrad"), (size_t)(3 * N));
  {
    LaunchScope ls(ctx, "ilsqr_fgrad_masked");
    k_fgrad_masked<TD><<<grid1d(N), 256, 0, ctx->stream>>>(xfs, mask, d.nx, d.ny, d.nz, 1.0 / d.vsx, 1.0 / d.vsy,
                                                          1.0 / d.vsz, dwork);
    ls.done();
    const std::vector<double> tx = percentiles(ctx, dwork, mask, N, count, {50.0, 70.0});
    const std::vector<double> ty = percentiles(ctx, dwork + N, mask, N, count, {50.0, 70.0});
    const std::vector<double> tz = percentiles(ctx, dwork + 2 * N, mask, N, count, {50.0, 70.0});
    LaunchScope ls2(ctx, "ilsqr_grad_weights");
    k_grad_weights<T><<<grid1d(N), 256, 0, ctx->stream>>>(N, dwork, mask, tx[0], tx[1], ty[0], ty[1], tz[0], tz[1], wg);
    ls2.done();
  }
  LsmrState* mst = ws<LsmrState>(ctx, nm("lsmr"), 1);
  {
    LsmrState init{};
    init.rho = 1.0;
    init.rho_bar = 1.0;
    init.c_bar = 1.0;
    init.rhodold = 1.0;
    init.minrbar = 1e100;
    init.atol = p.tol;
    init.btol = p.tol;
    h2d(ctx, mst, &init, sizeof(init));
  }
  const int* mdone = &mst->done;
  // N-length LSMR vectors reuse the idle LSQR buffers (each holds 2*NF >= 2N reals)
  T* vv = reinterpret_cast<T*>(vb);
  T* hh = reinterpret_cast<T*>(wb);
  T* hbar = reinterpret_cast<T*>(xb);
  T* rq = reinterpret_cast<T*>(t);  // r / q image
  T* u3 = ws<T>(ctx, nm("lsmr_u"), (size_t)(3 * N));
  T* xx = ws<T>(ctx, nm("lsmr_x"), (size_t)N);
  C* spec = ws<C>(ctx, nm("lsmr_spec"), (size_t)fh.g.hsize());
  QSM_CUDA(cudaMemsetAsync(spec, 0, sizeof(C) * fh.g.hsize(), ctx->stream));
  const T hx = (T)(1.0 / d.vsx), hy = (T)(1.0 / d.vsy), hz = (T)(1.0 / d.vsz);
  auto mic_chain = [&](const auto& load, const auto& store) {
    run_x_r2c<T>(ctx, fh, spec, load, mdone);
    run_yz<T, -1, 1>(ctx, fh, spec, spec, OpId<T>{}, mdone);
    run_z_fused<T>(ctx, fh, spec, spec, OpMic<T>{K}, mdone);
    run_yz<T, +1, 1>(ctx, fh, spec, spec, OpId<T>{}, mdone);
    run_x_c2r<T>(ctx, fh, spec, store, mdone);
  };
  auto at_u = [&](int init) {  // v = A^T u (- beta v)
    {
      LaunchScope ls(ctx, "lsmr_div");
      k_lsmr_div<T><<<grid1d(N), 256, 0, ctx->stream>>>(d.nx, d.ny, d.nz, hx, hy, hz, wg, u3, rq, mst);
      ls.done();
    }
    mic_chain(LoadCast<T, T>{rq, d.nx}, StoreLsmrV<T>{vv, d.nx, invn, mst, partials, init, 0.0});
  };
  {
    LaunchScope ls(ctx, "lsmr_grad");
    k_lsmr_grad<double, T><<<grid1d(N), 256, 0, ctx->stream>>>(d.nx, d.ny, d.nz, hx, hy, hz, xlsqr, wg, u3, mst,
                                                                partials, 1);
    ls.done();
  }
  at_u(1);
  {
    LaunchScope ls(ctx, "lsmr_init");
    k_lsmr_init<T><<<grid1d(N), 256, 0, ctx->stream>>>(N, vv, hh, hbar, xx, mst);
    ls.done();
  }
  run_iterations(ctx, p.max_iter, mdone, [&]() {
    mic_chain(LoadScaled<T>{vv, &mst->sv, d.nx}, StoreScaledReal<T>{rq, d.nx, invn});
    {
      LaunchScope ls(ctx, "lsmr_grad");
      k_lsmr_grad<T, T><<<grid1d(N), 256, 0, ctx->stream>>>(d.nx, d.ny, d.nz, hx, hy, hz, rq, wg, u3, mst, partials, 0);
      ls.done();
    }
    at_u(0);
    LaunchScope ls(ctx, "lsmr_update");
    k_lsmr_update<T><<<grid1d(N), 256, 0, ctx->stream>>>(N, hh, hbar, xx, vv, mst, partials);
    ls.done();
  });

  // ------------------------------------------------------------- step 4 --
  {
    LaunchScope ls(ctx, "ilsqr_out");
    k_ilsqr_out<T><<<grid1d(N), 256, 0, ctx->stream>>>(N, xlsqr, xx, mask, chi, xsa_out);
    ls.done();
  }
  sync(ctx);
  report(4);
}

// ---------------------------------------------------- the LSQR operator alone ----
// Contiguous complex double rows (nx values) <-> full-spectrum rows (pitch values).
template <typename T>
__global__ void k_rows_to_pitch(long long nrows, int nx, int pitch, const double2* __restrict__ in,
                                cplx_t<T>* __restrict__ out) {
  const long long total = nrows * pitch;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long row = i / pitch;
    const int e = (int)(i - row * pitch);
    cplx_t<T> v = mk<cplx_t<T>>(T(0), T(0));
    if (e < nx) {
      const double2 a = in[row * nx + e];
      v = mk<cplx_t<T>>((T)a.x, (T)a.y);
    }
    out[i] = v;
  }
}
template <typename T>
__global__ void k_pitch_to_rows(long long nrows, int nx, int pitch, const cplx_t<T>* __restrict__ in,
                                double2* __restrict__ out) {
  const long long total = nrows * nx;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long row = i / nx;
    const cplx_t<T> v = in[row * pitch + (i - row * nx)];
    out[i] = make_double2((double)v.x, (double)v.y);
  }
}
template <typename T>
__global__ void k_cast_real(long long n, const double* __restrict__ in, T* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (T)in[i];
}

// y = D * FFT(w * Re(IFFT(D * x))): one application of lsqr_step's operator
// (src/inversion/ilsqr.rs:988-1010) with the five passes of the solver's own loop.
template <typename T>
void lsqr_operator_impl(qsm_ctx* ctx, const GridDims& d, const double bdir[3], const double* w, const double2* x,
                        double2* y) {
  using C = cplx_t<T>;
  const std::string pre = sizeof(T) == 4 ? "ilop32." : "ilop64.";
  Fft3<T> ff = make_fft3_full<T>(ctx, d);
  KSpace K = make_kspace(ctx, d, bdir);
  const long long N = d.n, NF = ff.g.hsize(), nrows = (long long)d.ny * d.nz;
  C* xin = ws<C>(ctx, pre + "x", (size_t)NF);
  C* t = ws<C>(ctx, pre + "t", (size_t)NF);
  C* yo = ws<C>(ctx, pre + "y", (size_t)NF);
  T* wl = ws<T>(ctx, pre + "w", (size_t)N);
  LsqrState* st = ws<LsqrState>(ctx, pre + "state", 1);
  double* partials = ws<double>(ctx, pre + "partials", (size_t)kMaxPersistentBlocks * 4);
  unsigned* counter = ws<unsigned>(ctx, pre + "counter", 1);
  LsqrState init{};
  init.su = 1.0;
  init.sv = 1.0;
  h2d(ctx, st, &init, sizeof(init));
  QSM_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), ctx->stream));
  {
    LaunchScope ls(ctx, "ilsqr_op_pack");
    k_rows_to_pitch<T><<<grid1d(NF), 256, 0, ctx->stream>>>(nrows, d.nx, ff.g.pitch, x, xin);
    ls.done();
    LaunchScope ls2(ctx, "ilsqr_op_weights");
    k_cast_real<T><<<grid1d(N), 256, 0, ctx->stream>>>(N, w, wl);
    ls2.done();
  }
  const T invn = (T)(1.0 / (double)N);
  run_yz<T, +1, 2>(ctx, ff, xin, t, OpScaleD<T>{K, &st->su}, nullptr);
  run_yz<T, +1, 1>(ctx, ff, t, t, OpId<T>{}, nullptr);
  run_x_full<T, +1, -1, true>(ctx, ff, LoadSpecRow<T>{t, ff.g.pitch}, MidWeightRe<T>{wl, d.nx, invn},
                              StoreSpecRow<T>{t, ff.g.pitch}, nullptr, "fft_x_lsqr");
  run_yz<T, -1, 1>(ctx, ff, t, t, OpId<T>{}, nullptr);
  run_yz_acc<T, -1, 2, true>(ctx, ff, t, yo, OpLsqrOut<T>{K, nullptr, st, 2}, partials, counter, nullptr,
                             "fft_z_lsqr");
  {
    LaunchScope ls(ctx, "ilsqr_op_unpack");
    k_pitch_to_rows<T><<<grid1d(nrows * d.nx), 256, 0, ctx->stream>>>(nrows, d.nx, ff.g.pitch, yo, y);
    ls.done();
  }
  sync(ctx);
}

void ilsqr_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                  const qsm_ilsqr_params* p, qsm_progress_fn progress, void* user, double* chi, double* xsa,
                  double* xfs, double* xlsqr) {
  GridDims d = check_grid(grid);
  check_ptr(f, "local_field");
  check_ptr(m, "mask");
  check_ptr(chi, "out_chi");
  check_ptr(p, "params");
  check_bdir(bdir);
  if (std::isnan(p->tol)) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "tol is NaN");
  check_volume_finite(ctx, f, d.n, "local_field");
  if (d.nx < 2 || d.ny < 2 || d.nz < 2)
    throw QsmError(QSM_ERR_UNSUPPORTED_SIZE, "iLSQR needs every axis length >= 2 (one-sided stencils)");
  if (d.n >= (1LL << 32)) throw QsmError(QSM_ERR_UNSUPPORTED_SIZE, "iLSQR volumes hold fewer than 2^32 voxels");
  if (ctx->precision != QSM_PRECISION_MIXED)
    ilsqr_impl<double, double>(ctx, d, f, m, bdir, *p, progress, user, chi, xsa, xfs, xlsqr);
  else if (ctx->krylov_precision == QSM_PRECISION_MIXED)
    ilsqr_impl<float, float>(ctx, d, f, m, bdir, *p, progress, user, chi, xsa, xfs, xlsqr);
  else
    ilsqr_impl<double, float>(ctx, d, f, m, bdir, *p, progress, user, chi, xsa, xfs, xlsqr);
}

}  // namespace qsm

using namespace qsm;

extern "C" {

void qsm_ilsqr_params_default(qsm_ilsqr_params* p) {
  if (!p) return;
  p->tol = 0.01;  // IlsqrParams::default, src/inversion/ilsqr.rs:27-34
  p->max_iter = 50;
}

qsm_status qsm_ilsqr_device(qsm_ctx* ctx, const double* d_local_field, const uint8_t* d_mask, const qsm_grid* grid,
                            const double bdir[3], const qsm_ilsqr_params* params, qsm_progress_fn progress, void* user,
                            double* d_out_chi, double* d_out_xsa, double* d_out_xfs, double* d_out_xlsqr) {
  return guarded(ctx, [&] {
    ilsqr_device(ctx, d_local_field, d_mask, grid, bdir, params, progress, user, d_out_chi, d_out_xsa, d_out_xfs,
                 d_out_xlsqr);
  });
}

qsm_status qsm_ilsqr_lsqr_operator_device(qsm_ctx* ctx, const qsm_grid* grid, const double bdir[3],
                                          const double* d_weights, const double* d_x, double* d_y) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_bdir(bdir);
    check_ptr(d_weights, "weights");
    check_ptr(d_x, "x");
    check_ptr(d_y, "y");
    if ((reinterpret_cast<uintptr_t>(d_x) | reinterpret_cast<uintptr_t>(d_y)) % 16 != 0)
      throw QsmError(QSM_ERR_INVALID_ARGUMENT, "complex vectors must be 16-byte aligned");
    const double2* x = reinterpret_cast<const double2*>(d_x);
    double2* y = reinterpret_cast<double2*>(d_y);
    if (ctx->precision == QSM_PRECISION_MIXED) lsqr_operator_impl<float>(ctx, d, bdir, d_weights, x, y);
    else lsqr_operator_impl<double>(ctx, d, bdir, d_weights, x, y);
  });
}

qsm_status qsm_ilsqr(qsm_ctx* ctx, const double* local_field, const uint8_t* mask, const qsm_grid* grid,
                     const double bdir[3], const qsm_ilsqr_params* params, qsm_progress_fn progress, void* user,
                     double* out_chi, double* out_xsa, double* out_xfs, double* out_xlsqr) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_ptr(local_field, "local_field");
    check_ptr(mask, "mask");
    check_ptr(out_chi, "out_chi");
    const size_t N = (size_t)d.n;
    double* extra[3] = {nullptr, nullptr, nullptr};
    double* hout[3] = {out_xsa, out_xfs, out_xlsqr};
    const char* names[3] = {"io.xsa", "io.xfs", "io.xlsqr"};
    for (int i = 0; i < 3; ++i)
      if (hout[i]) extra[i] = reinterpret_cast<double*>(ws_get(ctx, names[i], N * sizeof(double)));
    with_host_io(ctx, d.n, local_field, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
      ilsqr_device(ctx, f, m, grid, bdir, params, progress, user, o, extra[0], extra[1], extra[2]);
      for (int i = 0; i < 3; ++i)
        if (hout[i]) d2h(ctx, hout[i], extra[i], N * sizeof(double));
    });
  });
}

}  // extern "C"
