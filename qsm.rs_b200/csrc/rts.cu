// Rapid two-step (RTS) dipole inversion (src/inversion/rts.rs:72-211), the pipeline's
// default inversion (src/pipeline/config.rs:251).
//
// Step 1 (rts.rs:121-159) is a pointwise k-space refinement: chi_hat = F(f) * c(D) with
// c_0 = D/(D^2 + 1e-6) and c_{k+1} = c_k + (1 - c_k D) D/(D^2 + 1e-6) for |D| > delta, 0
// elsewhere, so lsmr_iter refinements collapse into one multiplier evaluated in double;
// x_1 = mask * Re IFFT(F(f) * c).
// Step 2 (rts.rs:164-208) is the ADMM of admm.rs:76-145 with the multiplier
// inv_a = rho / (M + rho L) (M = mu where |D| > delta), the right-hand side
// F(x_1) * (M / rho) * inv_a, a unit divergence factor and the shrink threshold 1/rho.
// Its first convergence test compares against x_1; the TV-ADMM kernels carry that
// starting iterate in x_0 = x0 - y_0 (the first update itself always sees zeros).
// Every multiplier is symmetrised over k -> -k, which reproduces the reference's
// complex-to-complex transform followed by the real part.
#include "tv_shared.cuh"

namespace qsm {

namespace {

__device__ __forceinline__ double rts_refine(double d, double delta, int iters) {
  if (!(fabs(d) > delta)) return 0.0;
  const double r = d / (d * d + 1e-6);
  double c = r;
  for (int k = 0; k < iters; ++k) c = c + (1.0 - c * d) * r;
  return c;
}

// inv_a = rho / (M + rho L), 0 where |a| <= 1e-20 (rts.rs:106-113)
__device__ __forceinline__ double rts_inv_a(const KSpace& K, double d, int ix, int iy, int iz, double delta, double mu,
                                            double rho, double* m_out) {
  const double m = fabs(d) > delta ? mu : 0.0;
  const double a = m + rho * K.lapneg(ix, iy, iz);
  *m_out = m;
  return fabs(a) > 1e-20 ? rho / a : 0.0;
}

template <typename T> struct OpRtsStep1 {
  using C = cplx_t<T>;
  KSpace K;
  double delta;
  int iters;
  __device__ __forceinline__ C mid(C v, int ix, int iy, int iz, long long) const {
    const KSpace& k = K;
    const double m = K.sym(ix, iy, iz, [&](double kx, double ky, double kz, int, int, int) {
      return rts_refine(k.dipole(kx, ky, kz), delta, iters);
    });
    return cscale(v, (T)m);
  }
};

// F(x_1) * (M / rho) * inv_a (rts.rs:173-178)
template <typename T> struct OpRtsRhs {
  using C = cplx_t<T>;
  KSpace K;
  double delta, mu, rho;
  __device__ __forceinline__ C mid(C v, int ix, int iy, int iz, long long) const {
    const KSpace& k = K;
    const double m = K.sym(ix, iy, iz, [&](double kx, double ky, double kz, int a, int b, int c) {
      double mm = 0.0;
      const double ia = rts_inv_a(k, k.dipole(kx, ky, kz), a, b, c, delta, mu, rho, &mm);
      return (mm / rho) * ia;
    });
    return cscale(v, (T)m);
  }
};

// per-iteration multiplier sym(inv_a) as a real half-spectrum array
template <typename T>
__global__ void k_rts_mult(Geom g, KSpace K, double delta, double mu, double rho, T* __restrict__ out) {
  const long long H = g.hsize();
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < H; i += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(i % g.pitch);
    const long long r = i / g.pitch;
    const int iy = (int)(r % g.ny);
    const int iz = (int)(r / g.ny);
    double m = 0.0;
    if (ix < g.nxh) {
      const KSpace& k = K;
      m = K.sym(ix, iy, iz, [&](double kx, double ky, double kz, int a, int b, int c) {
        double mm = 0.0;
        return rts_inv_a(k, k.dipole(kx, ky, kz), a, b, c, delta, mu, rho, &mm);
      });
    }
    out[i] = (T)m;
  }
}

// in-kernel form of the same multiplier (very long z axes)
template <typename T> struct OpRtsMul {
  using C = cplx_t<T>;
  KSpace K;
  double delta, mu, rho;
  __device__ __forceinline__ C mid(C v, int ix, int iy, int iz, long long) const {
    const KSpace& k = K;
    const double m = K.sym(ix, iy, iz, [&](double kx, double ky, double kz, int a, int b, int c) {
      double mm = 0.0;
      return rts_inv_a(k, k.dipole(kx, ky, kz), a, b, c, delta, mu, rho, &mm);
    });
    return cscale(v, (T)m);
  }
};

template <typename T>
__global__ void k_sub(long long N, const T* __restrict__ a, const T* __restrict__ b, T* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    out[i] = a[i] - b[i];
}

template <typename T> struct StoreMaskedT {
  T* out;
  const uint8_t* mask;
  int nx;
  T scale;
  __device__ __forceinline__ void operator()(int row, int e, T v) {
    const long long i = (long long)row * nx + e;
    out[i] = mask[i] != 0 ? v * scale : T(0);
  }
  __device__ __forceinline__ void finish() {}
};

}  // namespace

template <typename T>
void rts_impl(qsm_ctx* ctx, const GridDims& d, const double* f, const uint8_t* mask, const double bdir[3],
              const qsm_rts_params& p, qsm_progress_fn progress, void* user, double* out) {
  const std::string pre = sizeof(T) == 4 ? "rts32." : "rts64.";
  TvState* st = ws<TvState>(ctx, pre + "state", 1);
  TvVol<T> v;
  tv_alloc<T>(ctx, v, pre, d, bdir, 1.0, 1.0 / p.rho, st, mask, out);
  const KSpace K = make_kspace(ctx, d, bdir);
  T* x1 = ws<T>(ctx, pre + "x1", (size_t)d.n);
  // step 1: x_1 = mask * Re IFFT(F(f) * c(D))
  run_x_r2c<T>(ctx, v.f, v.spec, LoadCast<double, T>{f, d.nx}, nullptr);
  run_yz<T, -1, 1>(ctx, v.f, v.spec, v.spec, OpId<T>{}, nullptr);
  run_z_fused<T>(ctx, v.f, v.spec, v.spec, OpRtsStep1<T>{K, p.delta, (int)p.lsmr_iter}, nullptr);
  run_yz<T, +1, 1>(ctx, v.f, v.spec, v.spec, OpId<T>{}, nullptr);
  run_x_c2r<T>(ctx, v.f, v.spec, StoreMaskedT<T>{x1, mask, d.nx, v.scale}, nullptr);
  // x0 = Re IFFT(F(x_1) * (M / rho) * inv_a)
  run_x_r2c<T>(ctx, v.f, v.spec, LoadCast<T, T>{x1, d.nx}, nullptr);
  run_yz<T, -1, 1>(ctx, v.f, v.spec, v.spec, OpId<T>{}, nullptr);
  run_z_fused<T>(ctx, v.f, v.spec, v.spec, OpRtsRhs<T>{K, p.delta, p.mu, p.rho}, nullptr);
  run_yz<T, +1, 1>(ctx, v.f, v.spec, v.spec, OpId<T>{}, nullptr);
  run_x_c2r<T>(ctx, v.f, v.spec, StoreReal<T>{v.x0, d.nx, v.scale}, nullptr);
  tv_init_state<T>(ctx, v, p.tol);
  {
    // x_0 = x_1 for the first convergence test: y_0 = x0 - x_1
    LaunchScope ls(ctx, "rts_setup");
    k_sub<T><<<grid1d(d.n), 256, 0, ctx->stream>>>(d.n, v.x0, x1, v.yb[0]);
    k_rts_mult<T><<<grid1d(v.f.g.hsize()), 256, 0, ctx->stream>>>(v.f.g, K, p.delta, p.mu, p.rho, v.mult);
    ls.done();
  }
  if (!v.use_mult) throw QsmError(QSM_ERR_UNSUPPORTED_SIZE, "z axis too long for the RTS multiplier tiles");
  ctx->tv_last_iters = tv_run<T>(ctx, v, p.max_iter, p.tol, progress, user);
}

void rts_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                const qsm_rts_params* p, qsm_progress_fn progress, void* user, double* out) {
  GridDims d = check_grid(grid);
  check_ptr(f, "local_field");
  check_ptr(m, "mask");
  check_ptr(out, "out");
  check_ptr(p, "params");
  check_bdir(bdir);
  check_volume_finite(ctx, f, d.n, "local_field");
  check_finite(p->delta, "delta");
  check_finite(p->mu, "mu");
  check_finite(p->rho, "rho");
  if (std::isnan(p->tol)) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "tol is NaN");
  if (ctx->precision == QSM_PRECISION_MIXED) rts_impl<float>(ctx, d, f, m, bdir, *p, progress, user, out);
  else rts_impl<double>(ctx, d, f, m, bdir, *p, progress, user, out);
}

}  // namespace qsm

using namespace qsm;

extern "C" {

void qsm_rts_params_default(qsm_rts_params* p) {
  if (!p) return;
  // RtsParams::default, src/inversion/rts.rs:40-51
  p->delta = 0.15;
  p->mu = 1e5;
  p->rho = 10.0;
  p->tol = 1e-2;
  p->max_iter = 20;
  p->lsmr_iter = 4;
}

qsm_status qsm_rts_device(qsm_ctx* ctx, const double* d_local_field, const uint8_t* d_mask, const qsm_grid* grid,
                          const double bdir[3], const qsm_rts_params* params, qsm_progress_fn progress, void* user,
                          double* d_out_chi) {
  return guarded(ctx, [&] {
    rts_device(ctx, d_local_field, d_mask, grid, bdir, params, progress, user, d_out_chi);
    sync(ctx);
  });
}

qsm_status qsm_rts(qsm_ctx* ctx, const double* local_field, const uint8_t* mask, const qsm_grid* grid,
                   const double bdir[3], const qsm_rts_params* params, qsm_progress_fn progress, void* user,
                   double* out_chi) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_ptr(local_field, "local_field");
    check_ptr(mask, "mask");
    check_ptr(out_chi, "out_chi");
    with_host_io(ctx, d.n, local_field, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
      rts_device(ctx, f, m, grid, bdir, params, progress, user, o);
    });
  });
}

}  // extern "C"
