// Laplacian phase unwrapping and SMV-family background removal (SMV, SHARP,
// V-SHARP) on the GPU, plus the pipeline dispatcher run_bg_removal.
//
// Mask erosion decides "SMV(mask) > delta" with delta within ~1e-8 of a rational
// count/total for realistic kernels, so the mask convolution always runs in double
// (FP64 transform error ~1e-15) whatever the context precision; field filtering runs
// in the working precision.
#include "functors.cuh"
#include "solvers.h"

#include <algorithm>
#include <cstring>

namespace qsm {

__device__ __forceinline__ double wrap_pi(double x) {
  // src/unwrap/laplacian.rs:21-30 (Rust % on f64 is the truncated fmod)
  const double two_pi = 2.0 * kPi;
  double y = fmod(x, two_pi);
  if (y > kPi) y -= two_pi;
  else if (y < -kPi) y += two_pi;
  return y;
}

// Wrapped 7-point Laplacian (periodic), masked, evaluated in double on the fly as
// the X-pass input (src/unwrap/laplacian.rs:34-78, 146-149).
template <typename T> struct LoadWrappedLap {
  const double* ph;
  const uint8_t* mask;
  int nx, ny, nz;
  double dx2, dy2, dz2;
  __device__ __forceinline__ T operator()(int row, int e) const {
    const long long sy = nx, sz = (long long)nx * ny;
    const long long i = (long long)row * nx + e;
    if (mask[i] == 0) return T(0);
    const int j = row % ny, k = row / ny;
    const long long ip = (e + 1 < nx) ? i + 1 : i - (nx - 1);
    const long long im = (e > 0) ? i - 1 : i + (nx - 1);
    const long long jp = (j + 1 < ny) ? i + sy : i - (ny - 1) * sy;
    const long long jm = (j > 0) ? i - sy : i + (ny - 1) * sy;
    const long long kp = (k + 1 < nz) ? i + sz : i - (long long)(nz - 1) * sz;
    const long long km = (k > 0) ? i - sz : i + (long long)(nz - 1) * sz;
    const double u = ph[i];
    const double lx = (wrap_pi(ph[ip] - u) - wrap_pi(u - ph[im])) * dx2;
    const double ly = (wrap_pi(ph[jp] - u) - wrap_pi(u - ph[jm])) * dy2;
    const double lz = (wrap_pi(ph[kp] - u) - wrap_pi(u - ph[km])) * dz2;
    return (T)(lx + ly + lz);
  }
};

// Poisson solve multiplier 1/lambda, 0 where |lambda| <= 1e-20 (src/unwrap/laplacian.rs:91-117)
template <typename T> struct OpPoisson {
  using C = cplx_t<T>;
  KSpace K;
  __device__ __forceinline__ C mid(C v, int ix, int iy, int iz, long long) const {
    const double lam = K.poisson(ix, iy, iz);
    if (fabs(lam) > 1e-20) return cscale(v, (T)(1.0 / lam));
    return mk<C>(T(0), T(0));
  }
};

// Normalised binary sphere at wrap-centred coordinates (src/kernels/smv.rs:19-67).
// The inclusion test is evaluated without FMA contraction so that it matches the
// reference's dx*dx + dy*dy + dz*dz <= r^2 exactly.
struct SphereGeom {
  int nx, ny, nz;
  double vsx, vsy, vsz, r2, norm;
};
__host__ __device__ __forceinline__ double sph_coord(int i, int n, double vs) {
  const int c = (i <= n / 2) ? i : i - n;
  return (double)c * vs;
}
__device__ __forceinline__ bool sph_inside(const SphereGeom& s, int i, int j, int k) {
  const double dx = sph_coord(i, s.nx, s.vsx), dy = sph_coord(j, s.ny, s.vsy), dz = sph_coord(k, s.nz, s.vsz);
  const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  return d2 <= s.r2;
}
struct LoadSphere {
  SphereGeom s;
  __device__ __forceinline__ double operator()(int row, int e) const {
    const int j = row % s.ny, k = row / s.ny;
    return sph_inside(s, e, j, k) ? s.norm : 0.0;
  }
};

SphereGeom sphere_geom(const GridDims& d, double radius) {
  SphereGeom s;
  s.nx = d.nx;
  s.ny = d.ny;
  s.nz = d.nz;
  s.vsx = d.vsx;
  s.vsy = d.vsy;
  s.vsz = d.vsz;
  s.r2 = radius * radius;
  // count the sphere's voxels on the host over the per-axis candidates
  auto axis = [&](int n, double vs) {
    std::vector<double> v;
    for (int i = 0; i < n; ++i) {
      const double c = sph_coord(i, n, vs);
      if (c * c <= s.r2) v.push_back(c);
    }
    return v;
  };
  std::vector<double> ax = axis(d.nx, d.vsx), ay = axis(d.ny, d.vsy), az = axis(d.nz, d.vsz);
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

// pre/post multiply by Re(S) from a double spectrum (the SMV kernel transform)
template <typename T> struct OpMulS {
  using C = cplx_t<T>;
  const double2* S;
  int one_minus;  // 1: multiply by (1 - S), 0: by S
  __device__ __forceinline__ T m(long long idx) const {
    const double s = S[idx].x;
    return (T)(one_minus ? 1.0 - s : s);
  }
  __device__ __forceinline__ C pre(C v, int, int, int, long long idx) const { return cscale(v, m(idx)); }
  __device__ __forceinline__ C post(C v, int, int, int, long long) const { return v; }
  __device__ __forceinline__ C mid(C v, int, int, int, long long idx) const { return cscale(v, m(idx)); }
};

// SHARP deconvolution: |1 - S| < thr -> 0, else X / (1 - S) (src/bgremove/sharp.rs:111-119,
// vsharp.rs:147-156)
template <typename T> struct OpDeconvS {
  using C = cplx_t<T>;
  const double2* S;
  double thr;
  __device__ __forceinline__ C mid(C v, int, int, int, long long idx) const {
    const double oms = 1.0 - S[idx].x;
    if (fabs(oms) < thr) return mk<C>(T(0), T(0));
    return cscale(v, (T)(1.0 / oms));
  }
};

// eroded = (v/N > delta) (src/kernels/smv.rs:100-104)
struct StoreThreshold {
  uint8_t* out;
  int nx;
  double scale, delta;
  __device__ __forceinline__ void operator()(int row, int e, double v) {
    out[(long long)row * nx + e] = (v * scale > delta) ? 1 : 0;
  }
  __device__ __forceinline__ void finish() {}
};

// V-SHARP first-hit selection (src/bgremove/vsharp.rs:168-176)
template <typename T> struct StoreSelect {
  const uint8_t* eroded;
  uint8_t* final_mask;
  T* local;
  int nx;
  T scale;
  __device__ __forceinline__ void operator()(int row, int e, T v) {
    const long long i = (long long)row * nx + e;
    if (eroded[i] == 1 && final_mask[i] == 0) {
      local[i] = v * scale;
      final_mask[i] = 1;
    }
  }
  __device__ __forceinline__ void finish() {}
};

// SMV: local = eroded == 1 ? field - SMV(field) : 0 (src/bgremove/smv.rs:50-56)
template <typename T> struct StoreSmvLocal {
  const double* field;
  const uint8_t* eroded;
  double* out;
  int nx;
  T scale;
  __device__ __forceinline__ void operator()(int row, int e, T v) {
    const long long i = (long long)row * nx + e;
    out[i] = eroded[i] == 1 ? field[i] - (double)(v * scale) : 0.0;
  }
  __device__ __forceinline__ void finish() {}
};

// ------------------------------------------------------------ shared steps --
// Full forward transform (spectrum only) of a loaded real volume.
template <typename T, class Load>
void forward3(qsm_ctx* ctx, const Fft3<T>& f, const Load& ld, cplx_t<T>* dst) {
  run_x_r2c<T>(ctx, f, dst, ld, nullptr);
  run_yz<T, -1, 1>(ctx, f, dst, dst, OpId<T>{}, nullptr);
  run_yz<T, -1, 2>(ctx, f, dst, dst, OpId<T>{}, nullptr);
}

// S = FFT(smv_kernel(r)) in double (src/kernels/smv.rs:19-67 + src/fft.rs:514-520)
void smv_spectrum(qsm_ctx* ctx, const Fft3<double>& f64, const GridDims& d, double radius, double2* S) {
  forward3<double>(ctx, f64, LoadSphere{sphere_geom(d, radius)}, S);
}

// eroded = IFFT(Fm * S) > delta, all in double
void erode_smv(qsm_ctx* ctx, const Fft3<double>& f64, const GridDims& d, const double2* Fm, const double2* S,
               double delta, uint8_t* eroded) {
  double2* tmp = ws<double2>(ctx, "bg.tmp64", (size_t)f64.g.hsize());
  run_yz<double, +1, 2>(ctx, f64, Fm, tmp, OpMulS<double>{S, 0}, nullptr);
  run_yz<double, +1, 1>(ctx, f64, tmp, tmp, OpId<double>{}, nullptr);
  run_x_c2r<double>(ctx, f64, tmp, StoreThreshold{eroded, d.nx, 1.0 / (double)d.n, delta}, nullptr);
}

// 1 - sqrt(1e-7), src/bgremove/sharp.rs:79 and vsharp.rs:129
double sharp_delta() { return 1.0 - std::sqrt(1e-7); }

// SHARP core (src/bgremove/sharp.rs:64-131)
template <typename T>
void sharp_impl(qsm_ctx* ctx, const GridDims& d, const double* field, const uint8_t* mask, double threshold,
                double radius, double* out_local, uint8_t* out_mask) {
  using C = cplx_t<T>;
  Fft3<double> f64 = make_fft3<double>(ctx, d);
  Fft3<T> f = make_fft3<T>(ctx, d);
  const size_t H = (size_t)f.g.hsize();
  double2* S = ws<double2>(ctx, "bg.S", H);
  double2* Fm = ws<double2>(ctx, "bg.Fm", H);
  C* spec = ws<C>(ctx, "spec", H);
  T* g = ws<T>(ctx, "bg.img", (size_t)d.n);
  smv_spectrum(ctx, f64, d, radius, S);
  forward3<double>(ctx, f64, LoadCast<uint8_t, double>{mask, d.nx}, Fm);
  erode_smv(ctx, f64, d, Fm, S, sharp_delta(), out_mask);
  const T scale = (T)(1.0 / (double)d.n);
  // high-pass, mask
  run_x_r2c<T>(ctx, f, spec, LoadCast<double, T>{field, d.nx}, nullptr);
  run_yz<T, -1, 1>(ctx, f, spec, spec, OpId<T>{}, nullptr);
  run_z_fused<T>(ctx, f, spec, spec, OpMulS<T>{S, 1}, nullptr);
  run_yz<T, +1, 1>(ctx, f, spec, spec, OpId<T>{}, nullptr);
  run_x_c2r<T>(ctx, f, spec, StoreMaskEqOne<T>{g, out_mask, d.nx, scale}, nullptr);
  // deconvolve, mask
  run_x_r2c<T>(ctx, f, spec, LoadCast<T, T>{g, d.nx}, nullptr);
  run_yz<T, -1, 1>(ctx, f, spec, spec, OpId<T>{}, nullptr);
  run_z_fused<T>(ctx, f, spec, spec, OpDeconvS<T>{S, threshold}, nullptr);
  run_yz<T, +1, 1>(ctx, f, spec, spec, OpId<T>{}, nullptr);
  run_x_c2r<T>(ctx, f, spec, StoreMaskedF64<T>{out_local, out_mask, d.nx, scale}, nullptr);
}

// V-SHARP (src/bgremove/vsharp.rs:88-199), radii already sorted descending, >= 2
template <typename T>
void vsharp_impl(qsm_ctx* ctx, const GridDims& d, const double* field, const uint8_t* mask,
                 const std::vector<double>& radii, double threshold, qsm_progress_fn progress, void* user,
                 double* out_local, uint8_t* out_mask) {
  using C = cplx_t<T>;
  Fft3<double> f64 = make_fft3<double>(ctx, d);
  Fft3<T> f = make_fft3<T>(ctx, d);
  const size_t H = (size_t)f.g.hsize();
  const size_t N = (size_t)d.n;
  double2* S0 = ws<double2>(ctx, "bg.S0", H);
  double2* S = ws<double2>(ctx, "bg.S", H);
  double2* Fm = ws<double2>(ctx, "bg.Fm", H);
  C* Ff = ws<C>(ctx, "bg.Ff", H);
  C* tmp = ws<C>(ctx, "bg.tmpT", H);
  uint8_t* eroded = ws<uint8_t>(ctx, "bg.eroded", N);
  T* local = ws<T>(ctx, "bg.img", N);
  QSM_CUDA(cudaMemsetAsync(out_mask, 0, N, ctx->stream));
  QSM_CUDA(cudaMemsetAsync(local, 0, N * sizeof(T), ctx->stream));
  forward3<double>(ctx, f64, LoadCast<uint8_t, double>{mask, d.nx}, Fm);
  forward3<T>(ctx, f, LoadCast<double, T>{field, d.nx}, Ff);
  const T scale = (T)(1.0 / (double)d.n);
  const double delta = sharp_delta();
  for (size_t idx = 0; idx < radii.size(); ++idx) {
    if (progress) progress(user, idx + 1, radii.size());
    double2* Sr = (idx == 0) ? S0 : S;
    smv_spectrum(ctx, f64, d, radii[idx], Sr);
    erode_smv(ctx, f64, d, Fm, Sr, delta, eroded);
    run_yz<T, +1, 2, true>(ctx, f, Ff, tmp, OpMulS<T>{Sr, 1}, nullptr);
    run_yz<T, +1, 1>(ctx, f, tmp, tmp, OpId<T>{}, nullptr);
    run_x_c2r<T>(ctx, f, tmp, StoreSelect<T>{eroded, out_mask, local, d.nx, scale}, nullptr);
  }
  // deconvolution with the largest kernel's inverse
  C* spec = ws<C>(ctx, "spec", H);
  run_x_r2c<T>(ctx, f, spec, LoadCast<T, T>{local, d.nx}, nullptr);
  run_yz<T, -1, 1>(ctx, f, spec, spec, OpId<T>{}, nullptr);
  run_z_fused<T>(ctx, f, spec, spec, OpDeconvS<T>{S0, threshold}, nullptr);
  run_yz<T, +1, 1>(ctx, f, spec, spec, OpId<T>{}, nullptr);
  run_x_c2r<T>(ctx, f, spec, StoreMaskedF64<T>{out_local, out_mask, d.nx, scale}, nullptr);
}

// SMV (src/bgremove/smv.rs:31-59)
template <typename T>
void smv_impl(qsm_ctx* ctx, const GridDims& d, const double* field, const uint8_t* mask, double radius,
              double* out_local, uint8_t* out_mask) {
  using C = cplx_t<T>;
  Fft3<double> f64 = make_fft3<double>(ctx, d);
  Fft3<T> f = make_fft3<T>(ctx, d);
  const size_t H = (size_t)f.g.hsize();
  double2* S = ws<double2>(ctx, "bg.S", H);
  double2* Fm = ws<double2>(ctx, "bg.Fm", H);
  C* spec = ws<C>(ctx, "spec", H);
  smv_spectrum(ctx, f64, d, radius, S);
  forward3<double>(ctx, f64, LoadCast<uint8_t, double>{mask, d.nx}, Fm);
  erode_smv(ctx, f64, d, Fm, S, 1.0 - 1e-10, out_mask);
  run_x_r2c<T>(ctx, f, spec, LoadCast<double, T>{field, d.nx}, nullptr);
  run_yz<T, -1, 1>(ctx, f, spec, spec, OpId<T>{}, nullptr);
  run_z_fused<T>(ctx, f, spec, spec, OpMulS<T>{S, 0}, nullptr);
  run_yz<T, +1, 1>(ctx, f, spec, spec, OpId<T>{}, nullptr);
  run_x_c2r<T>(ctx, f, spec, StoreSmvLocal<T>{field, out_mask, out_local, d.nx, (T)(1.0 / (double)d.n)}, nullptr);
}

// ------------------------------------------------------------------ iSMV --
// src/bgremove/ismv.rs:48-157.  Device state: iterations done, the change norm and its
// tolerance; the iteration whose top-of-loop test stops the loop (0: none).
struct IsmvState {
  int done;
  int k;  // iterations completed
  unsigned counter;
  int stop_at;
  double nr, eps;
};

// f_0 = field; nr_0 = ||eroded * field||, eps = tol * nr_0 (ismv.rs:106-120); a zero
// norm stops the loop at its first test
template <typename T>
__global__ void k_ismv_init(long long N, const double* __restrict__ field, const uint8_t* __restrict__ eroded,
                            double tol, size_t max_iter, T* __restrict__ f, IsmvState* st, double* partials) {
  double acc[1] = {0.0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const double v = field[i];
    f[i] = (T)v;
    const double e = v * (double)eroded[i];
    acc[0] += e * e;
  }
  if (grid_sum_last<1>(acc, partials, &st->counter) && threadIdx.x == 0) {
    const double nr = sqrt(acc[0]);
    st->nr = nr;
    st->eps = tol * nr;
    st->k = 0;
    st->stop_at = 0;
    st->done = 0;
    if (max_iter > 0 && nr <= tol * nr) {
      st->done = 1;
      st->stop_at = 1;
    }
  }
}

// f_k = eroded * Re IFFT(F(f_{k-1}) S) + (m0 - eroded) field, FP64 sum of (f0 - f_k)^2
// with f0 = eroded * field at k = 1 and f_{k-1} after (ismv.rs:127-155); the last block
// stores the norm and runs the next iteration's top-of-loop test.
template <typename T> struct StoreIsmv {
  T* out;
  const T* prev;  // f_{k-1}, or null at k = 1
  const double* field;
  const uint8_t* mask;
  const uint8_t* eroded;
  int nx;
  T scale;
  IsmvState* st;
  double* partials;
  int max_iter;
  double acc[1];
  __device__ __forceinline__ void operator()(int row, int e, T v) {
    const long long i = (long long)row * nx + e;
    const double er = (double)eroded[i];
    const double fld = field[i];
    const double m0 = mask[i] != 0 ? 1.0 : 0.0;
    const T fn = (T)(er * (double)(v * scale) + fld * (m0 - er));
    out[i] = fn;
    const double f0 = prev ? (double)prev[i] : fld * er;
    const double dd = f0 - (double)fn;
    acc[0] += dd * dd;
  }
  __device__ void finish() {
    if (!grid_sum_last<1>(acc, partials, &st->counter)) return;
    if (threadIdx.x + blockDim.x * threadIdx.y != 0) return;
    const double nr = sqrt(acc[0]);
    st->nr = nr;
    const int k = st->k + 1;
    st->k = k;
    if (k < max_iter && nr <= st->eps) {
      st->done = 1;
      st->stop_at = k + 1;
    }
  }
};

// local = mask ? field - f : 0 (ismv.rs:158-164)
template <typename T>
__global__ void k_ismv_out(long long N, const double* __restrict__ field, const uint8_t* __restrict__ mask,
                           const T* __restrict__ f, double* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    out[i] = mask[i] != 0 ? field[i] - (double)f[i] : 0.0;
}

template <typename T>
__global__ void k_re_spectrum(long long H, const double2* __restrict__ S, T* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < H; i += (long long)gridDim.x * blockDim.x)
    out[i] = (T)S[i].x;
}

template <typename T> struct OpMulRe {
  using C = cplx_t<T>;
  const T* m;
  __device__ __forceinline__ C mid(C v, int, int, int, long long idx) const { return cscale(v, m[idx]); }
};

template <typename T> struct LoadVol {
  const T* p;
  int nx;
  __device__ __forceinline__ T operator()(int row, int e) const { return p[(long long)row * nx + e]; }
};

template <typename T>
void ismv_impl(qsm_ctx* ctx, const GridDims& d, const double* field, const uint8_t* mask,
               const qsm_ismv_params& p, qsm_progress_fn progress, void* user, double* out_local,
               uint8_t* out_mask) {
  using C = cplx_t<T>;
  Fft3<double> f64 = make_fft3<double>(ctx, d);
  Fft3<T> f = make_fft3<T>(ctx, d);
  const size_t H = (size_t)f.g.hsize();
  const long long N = d.n;
  const std::string pre = sizeof(T) == 4 ? "ismv32." : "ismv64.";
  double2* S = ws<double2>(ctx, "bg.S", H);
  double2* Fm = ws<double2>(ctx, "bg.Fm", H);
  T* Sr = ws<T>(ctx, pre + "Sr", H);
  C* spec = ws<C>(ctx, pre + "spec", H);
  T* fb[2] = {ws<T>(ctx, pre + "f0", (size_t)N), ws<T>(ctx, pre + "f1", (size_t)N)};
  IsmvState* st = ws<IsmvState>(ctx, pre + "state", 1);
  double* partials = ws<double>(ctx, pre + "partials", (size_t)kMaxPersistentBlocks);
  QSM_CUDA(cudaMemsetAsync(st, 0, sizeof(IsmvState), ctx->stream));
  smv_spectrum(ctx, f64, d, p.radius, S);
  forward3<double>(ctx, f64, LoadCast<uint8_t, double>{mask, d.nx}, Fm);
  erode_smv(ctx, f64, d, Fm, S, 1.0 - 1e-10, out_mask);  // ismv.rs:166-169
  {
    LaunchScope ls(ctx, "ismv_init");
    k_re_spectrum<T><<<grid1d((long long)H), 256, 0, ctx->stream>>>((long long)H, S, Sr);
    k_ismv_init<T><<<grid1d(N), 256, 0, ctx->stream>>>(N, field, out_mask, p.tol, p.max_iter, fb[0], st, partials);
    ls.done();
  }
  const int* done = &st->done;
  const bool use_m = zm_tile_width<T>(d.nz, f.pz.m, f.pz.T) > 0;
  const T scale = (T)(1.0 / (double)N);
  const int maxi = (int)std::min<size_t>(p.max_iter, (size_t)1 << 30);
  // iteration k reads fb[(k-1) % 2] and writes fb[k % 2]
  auto iter = [&](int k) {
    const T* in = fb[(k - 1) % 2];
    StoreIsmv<T> store{fb[k % 2], k == 1 ? nullptr : in, field, mask, out_mask, d.nx, scale, st, partials, maxi,
                       {0.0}};
    run_x_r2c<T>(ctx, f, spec, LoadVol<T>{in, d.nx}, done);
    run_yz<T, -1, 1>(ctx, f, spec, spec, OpId<T>{}, done);
    if (use_m) run_z_fused_m<T>(ctx, f, spec, spec, Sr, done);
    else run_z_fused<T>(ctx, f, spec, spec, OpMulRe<T>{Sr}, done);
    run_yz<T, +1, 1>(ctx, f, spec, spec, OpId<T>{}, done);
    run_x_c2r<T>(ctx, f, spec, store, done);
  };
  IsmvState hs{};
  size_t reported = 0;
  auto poll = [&]() {
    d2h(ctx, &hs, st, sizeof(hs));
    sync(ctx);
    const size_t through = hs.stop_at ? (size_t)hs.stop_at : (size_t)hs.k;
    if (progress)
      for (; reported < through; ++reported) progress(user, reported + 1, p.max_iter);
    return hs.done != 0;
  };
  const bool watch = progress != nullptr || p.tol > 0.0;
  bool stopped = false;
  if (maxi >= 1) {
    iter(1);
    if (maxi >= 2) {
      if (ctx->profiling) {
        for (int k = 2; k <= maxi && !stopped; ++k) {
          iter(k);
          if (watch && k % 8 == 0) stopped = poll();
        }
      } else {
        cudaGraph_t graph = nullptr;
        const uint64_t l0 = ctx->launches;
        QSM_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        try {
          iter(2);
          iter(3);
        } catch (...) {
          cudaStreamEndCapture(ctx->stream, &graph);
          if (graph) cudaGraphDestroy(graph);
          throw;
        }
        QSM_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
        const uint64_t per = ctx->launches - l0;
        ctx->launches = l0;
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess)
          throw QsmError(QSM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
        try {
          const int pairs = (maxi - 1) / 2;
          for (int q = 0; q < pairs && !stopped; ++q) {
            QSM_CUDA(cudaGraphLaunch(exec, ctx->stream));
            ctx->launches += per;
            if (watch && (q + 1) % 4 == 0) stopped = poll();
          }
          if (!stopped && (maxi - 1) % 2 == 1) iter(maxi);
        } catch (...) {
          cudaGraphExecDestroy(exec);
          throw;
        }
        cudaGraphExecDestroy(exec);
      }
    }
  }
  poll();
  const int kdone = hs.k;
  {
    LaunchScope ls(ctx, "ismv_out");
    k_ismv_out<T><<<grid1d(N), 256, 0, ctx->stream>>>(N, field, mask, fb[kdone % 2], out_local);
    ls.done();
  }
  sync(ctx);
  if (progress) {
    const size_t through = hs.stop_at ? (size_t)hs.stop_at : p.max_iter;
    for (; reported < through; ++reported) progress(user, reported + 1, p.max_iter);
    if (hs.stop_at) progress(user, (size_t)hs.stop_at, (size_t)hs.stop_at);
  }
}

template <typename T>
void unwrap_impl(qsm_ctx* ctx, const GridDims& d, const double* phase, const uint8_t* mask, double* out) {
  using C = cplx_t<T>;
  Fft3<T> f = make_fft3<T>(ctx, d);
  KSpace K = make_kspace(ctx, d, nullptr);
  C* spec = ws<C>(ctx, "spec", (size_t)f.g.hsize());
  LoadWrappedLap<T> ld{phase, mask, d.nx, d.ny, d.nz, 1.0 / (d.vsx * d.vsx), 1.0 / (d.vsy * d.vsy),
                       1.0 / (d.vsz * d.vsz)};
  run_x_r2c<T>(ctx, f, spec, ld, nullptr);
  run_yz<T, -1, 1>(ctx, f, spec, spec, OpId<T>{}, nullptr);
  run_z_fused<T>(ctx, f, spec, spec, OpPoisson<T>{K}, nullptr);
  run_yz<T, +1, 1>(ctx, f, spec, spec, OpId<T>{}, nullptr);
  run_x_c2r<T>(ctx, f, spec, StoreMaskedF64<T>{out, mask, d.nx, (T)(1.0 / (double)d.n)}, nullptr);
}

void check_io(const void* a, const void* m, const void* o) {
  check_ptr(a, "input");
  check_ptr(m, "mask");
  check_ptr(o, "output");
}

void unwrap_device(qsm_ctx* ctx, const double* ph, const uint8_t* m, const qsm_grid* grid, double* out) {
  GridDims d = check_grid(grid);
  check_io(ph, m, out);
  check_volume_finite(ctx, ph, d.n, "phase");
  if (ctx->precision == QSM_PRECISION_MIXED) unwrap_impl<float>(ctx, d, ph, m, out);
  else unwrap_impl<double>(ctx, d, ph, m, out);
}

void smv_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const GridDims& d, double radius, double* ol,
                uint8_t* om) {
  check_finite(radius, "radius");
  check_volume_finite(ctx, f, d.n, "field");
  if (ctx->precision == QSM_PRECISION_MIXED) smv_impl<float>(ctx, d, f, m, radius, ol, om);
  else smv_impl<double>(ctx, d, f, m, radius, ol, om);
}

void ismv_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const GridDims& d, const qsm_ismv_params* p,
                 qsm_progress_fn progress, void* user, double* ol, uint8_t* om) {
  check_ptr(p, "params");
  check_finite(p->radius, "radius");
  if (std::isnan(p->tol)) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "tol is NaN");
  check_volume_finite(ctx, f, d.n, "field");
  if (ctx->precision == QSM_PRECISION_MIXED) ismv_impl<float>(ctx, d, f, m, *p, progress, user, ol, om);
  else ismv_impl<double>(ctx, d, f, m, *p, progress, user, ol, om);
}

void sharp_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const GridDims& d, double thr, double radius,
                  double* ol, uint8_t* om) {
  check_finite(thr, "threshold");
  check_finite(radius, "radius");
  check_volume_finite(ctx, f, d.n, "field");
  if (ctx->precision == QSM_PRECISION_MIXED) sharp_impl<float>(ctx, d, f, m, thr, radius, ol, om);
  else sharp_impl<double>(ctx, d, f, m, thr, radius, ol, om);
}

void vsharp_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const GridDims& d, const double* radii,
                   size_t n_radii, double thr, qsm_progress_fn progress, void* user, double* ol, uint8_t* om) {
  check_finite(thr, "threshold");
  if (n_radii > 0) check_ptr(radii, "radii");
  std::vector<double> r(radii, radii + n_radii);
  for (double v : r) check_finite(v, "radius");
  check_volume_finite(ctx, f, d.n, "field");
  const size_t N = (size_t)d.n;
  if (r.empty()) {  // src/bgremove/vsharp.rs:98-100
    QSM_CUDA(cudaMemsetAsync(ol, 0, N * sizeof(double), ctx->stream));
    QSM_CUDA(cudaMemcpyAsync(om, m, N, cudaMemcpyDeviceToDevice, ctx->stream));
    return;
  }
  if (r.size() == 1) {  // src/bgremove/vsharp.rs:102-108
    if (progress) progress(user, 1, 1);
    sharp_device(ctx, f, m, d, thr, r[0], ol, om);
    return;
  }
  std::stable_sort(r.begin(), r.end(), [](double a, double b) { return a > b; });
  if (ctx->precision == QSM_PRECISION_MIXED) vsharp_impl<float>(ctx, d, f, m, r, thr, progress, user, ol, om);
  else vsharp_impl<double>(ctx, d, f, m, r, thr, progress, user, ol, om);
}

// radii list of VsharpParams (src/bgremove/vsharp.rs:70-82)
std::vector<double> vsharp_radii(const qsm_vsharp_params& p) {
  std::vector<double> radii;
  double r = p.max_radius;
  const double step = p.min_radius;
  if (step > 0.0) {
    while (r >= step) {
      radii.push_back(r);
      r -= step;
    }
  } else if (step <= 0.0 && r >= step) {
    throw QsmError(QSM_ERR_INVALID_ARGUMENT, "min_radius must be > 0 (the radius list would never end)");
  }
  if (radii.empty()) radii.push_back(p.max_radius);
  return radii;
}

// host staging for the two-output functions
template <class Run>
void with_host_io2(qsm_ctx* ctx, const GridDims& d, const double* h_in, const uint8_t* h_mask, double* h_out,
                   uint8_t* h_mask_out, Run run) {
  const size_t N = (size_t)d.n;
  double* din = ws<double>(ctx, "io.in", N);
  uint8_t* dm = ws<uint8_t>(ctx, "io.mask", N);
  double* dout = ws<double>(ctx, "io.out", N);
  uint8_t* dmo = ws<uint8_t>(ctx, "io.mask_out", N);
  h2d(ctx, din, h_in, N * sizeof(double));
  h2d(ctx, dm, h_mask, N);
  run(din, dm, dout, dmo);
  d2h(ctx, h_out, dout, N * sizeof(double));
  d2h(ctx, h_mask_out, dmo, N);
  sync(ctx);
}

}  // namespace qsm

using namespace qsm;

extern "C" {

qsm_status qsm_laplacian_unwrap_device(qsm_ctx* ctx, const double* d_phase, const uint8_t* d_mask,
                                       const qsm_grid* grid, double* d_out) {
  return guarded(ctx, [&] {
    unwrap_device(ctx, d_phase, d_mask, grid, d_out);
    sync(ctx);
  });
}

qsm_status qsm_laplacian_unwrap(qsm_ctx* ctx, const double* phase, const uint8_t* mask, const qsm_grid* grid,
                                double* out) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_io(phase, mask, out);
    const size_t N = (size_t)d.n;
    double* din = ws<double>(ctx, "io.in", N);
    uint8_t* dm = ws<uint8_t>(ctx, "io.mask", N);
    double* dout = ws<double>(ctx, "io.out", N);
    h2d(ctx, din, phase, N * sizeof(double));
    h2d(ctx, dm, mask, N);
    unwrap_device(ctx, din, dm, grid, dout);
    d2h(ctx, out, dout, N * sizeof(double));
    sync(ctx);
  });
}

qsm_status qsm_smv(qsm_ctx* ctx, const double* field, const uint8_t* mask, const qsm_grid* grid, double radius,
                   double* out_local, uint8_t* out_mask) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_io(field, mask, out_local);
    check_ptr(out_mask, "out_mask");
    with_host_io2(ctx, d, field, mask, out_local, out_mask,
                  [&](const double* f, const uint8_t* m, double* o, uint8_t* om) {
                    smv_device(ctx, f, m, d, radius, o, om);
                  });
  });
}

qsm_status qsm_sharp(qsm_ctx* ctx, const double* field, const uint8_t* mask, const qsm_grid* grid,
                     const qsm_sharp_params* p, double* out_local, uint8_t* out_mask) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_io(field, mask, out_local);
    check_ptr(out_mask, "out_mask");
    check_ptr(p, "params");
    with_host_io2(ctx, d, field, mask, out_local, out_mask,
                  [&](const double* f, const uint8_t* m, double* o, uint8_t* om) {
                    sharp_device(ctx, f, m, d, p->threshold, p->radius, o, om);
                  });
  });
}

qsm_status qsm_vsharp_with_radii_device(qsm_ctx* ctx, const double* d_field, const uint8_t* d_mask,
                                        const qsm_grid* grid, const double* radii, size_t n_radii, double threshold,
                                        qsm_progress_fn progress, void* user, double* d_out_local,
                                        uint8_t* d_out_mask) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_io(d_field, d_mask, d_out_local);
    check_ptr(d_out_mask, "out_mask");
    vsharp_device(ctx, d_field, d_mask, d, radii, n_radii, threshold, progress, user, d_out_local, d_out_mask);
    sync(ctx);
  });
}

qsm_status qsm_vsharp_with_radii(qsm_ctx* ctx, const double* field, const uint8_t* mask, const qsm_grid* grid,
                                 const double* radii, size_t n_radii, double threshold, qsm_progress_fn progress,
                                 void* user, double* out_local, uint8_t* out_mask) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_io(field, mask, out_local);
    check_ptr(out_mask, "out_mask");
    with_host_io2(ctx, d, field, mask, out_local, out_mask,
                  [&](const double* f, const uint8_t* m, double* o, uint8_t* om) {
                    vsharp_device(ctx, f, m, d, radii, n_radii, threshold, progress, user, o, om);
                  });
  });
}

qsm_status qsm_vsharp(qsm_ctx* ctx, const double* field, const uint8_t* mask, const qsm_grid* grid,
                      const qsm_vsharp_params* p, qsm_progress_fn progress, void* user, double* out_local,
                      uint8_t* out_mask) {
  return guarded(ctx, [&] {
    check_ptr(p, "params");
    std::vector<double> radii = vsharp_radii(*p);
    GridDims d = check_grid(grid);
    check_io(field, mask, out_local);
    check_ptr(out_mask, "out_mask");
    with_host_io2(ctx, d, field, mask, out_local, out_mask,
                  [&](const double* f, const uint8_t* m, double* o, uint8_t* om) {
                    vsharp_device(ctx, f, m, d, radii.data(), radii.size(), p->threshold, progress, user, o, om);
                  });
  });
}

void qsm_ismv_params_default(qsm_ismv_params* p) {
  if (!p) return;
  // IsmvParams::default, src/bgremove/ismv.rs:31-35
  p->tol = 1e-6;
  p->max_iter = 50;
  p->radius = 5.0;
}

qsm_status qsm_ismv_device(qsm_ctx* ctx, const double* d_field, const uint8_t* d_mask, const qsm_grid* grid,
                           const qsm_ismv_params* params, qsm_progress_fn progress, void* user, double* d_out_local,
                           uint8_t* d_out_mask) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_io(d_field, d_mask, d_out_local);
    check_ptr(d_out_mask, "out_mask");
    ismv_device(ctx, d_field, d_mask, d, params, progress, user, d_out_local, d_out_mask);
    sync(ctx);
  });
}

qsm_status qsm_ismv(qsm_ctx* ctx, const double* field, const uint8_t* mask, const qsm_grid* grid,
                    const qsm_ismv_params* params, qsm_progress_fn progress, void* user, double* out_local,
                    uint8_t* out_mask) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_io(field, mask, out_local);
    check_ptr(out_mask, "out_mask");
    with_host_io2(ctx, d, field, mask, out_local, out_mask,
                  [&](const double* f, const uint8_t* m, double* o, uint8_t* om) {
                    ismv_device(ctx, f, m, d, params, progress, user, o, om);
                  });
  });
}

void qsm_bg_removal_config_default(qsm_bg_removal_config* c) {
  if (!c) return;
  c->algorithm = QSM_BG_VSHARP;
  qsm_vsharp_params_default(&c->vsharp);
  qsm_sharp_params_default(&c->sharp);
  qsm_resharp_params_default(&c->resharp);
  qsm_ismv_params_default(&c->ismv);
}

qsm_status qsm_run_bg_removal(qsm_ctx* ctx, const double* field_ppm, size_t len, const uint8_t* mask,
                              const qsm_scan_metadata* md, const qsm_bg_removal_config* cfg,
                              qsm_progress_fn progress, void* user, double* out_local, uint8_t* out_mask) {
  return guarded(ctx, [&] {
    check_ptr(md, "metadata");
    check_ptr(cfg, "config");
    qsm_grid g{md->nx, md->ny, md->nz, md->vsx, md->vsy, md->vsz};
    const size_t n = md->nx * md->ny * md->nz;
    if (len != n)
      throw QsmError(QSM_ERR_DIMENSION_MISMATCH,
                     "dimension mismatch: expected " + std::to_string(n) + ", got " + std::to_string(len));
    GridDims d = check_grid(&g);
    check_io(field_ppm, mask, out_local);
    check_ptr(out_mask, "out_mask");
    switch (cfg->algorithm) {
      case QSM_BG_VSHARP: {
        std::vector<double> radii = vsharp_radii(cfg->vsharp);
        with_host_io2(ctx, d, field_ppm, mask, out_local, out_mask,
                      [&](const double* f, const uint8_t* m, double* o, uint8_t* om) {
                        vsharp_device(ctx, f, m, d, radii.data(), radii.size(), cfg->vsharp.threshold, progress,
                                      user, o, om);
                      });
        break;
      }
      case QSM_BG_RESHARP:
        with_host_io2(ctx, d, field_ppm, mask, out_local, out_mask,
                      [&](const double* f, const uint8_t* m, double* o, uint8_t* om) {
                        resharp_device(ctx, f, m, d, &cfg->resharp, progress, user, o, om);
                      });
        break;
      case QSM_BG_ISMV:
        with_host_io2(ctx, d, field_ppm, mask, out_local, out_mask,
                      [&](const double* f, const uint8_t* m, double* o, uint8_t* om) {
                        ismv_device(ctx, f, m, d, &cfg->ismv, progress, user, o, om);
                      });
        break;
      case QSM_BG_SHARP:
        with_host_io2(ctx, d, field_ppm, mask, out_local, out_mask,
                      [&](const double* f, const uint8_t* m, double* o, uint8_t* om) {
                        sharp_device(ctx, f, m, d, cfg->sharp.threshold, cfg->sharp.radius, o, om);
                      });
        break;
      default:
        throw QsmError(QSM_ERR_INVALID_CONFIG, "invalid config: background removal algorithm " +
                                                   std::to_string(cfg->algorithm) + " is not provided by this library");
    }
  });
}

}  // extern "C"
