// Nonlinear TV (NLTV) dipole inversion (src/inversion/nltv.rs:62-131): newton_iter
// passes of the TV-ADMM iteration (src/inversion/admm.rs:76-145, rho = 100 lambda) with
// the weighted shrink shrink(v, (lambda/rho) w_i).  Between passes the weights become
// w = 1/(|grad x| + mu 1e-6), divided by their maximum when that exceeds 1, and the
// ADMM state carries over except g, which is overwritten with grad x (nltv.rs:114).
//
// Each pass runs on the TV-ADMM kernels (x_j = x0 - y_j, the fused convergence test +
// weighted z/u update + divergence, the FFT chain with rho * sym(inv_a)), on the device
// state's done flag and CUDA graphs of two iterations.  A pass's first step after a
// reweighting takes its divergence from g = grad x (k_nltv_lapdiv) and updates no u.
// Per pass the host reads the device state once: it needs the iteration count for
// progress and to tell which parity buffers hold the pass's last x and u.
#include "tv_shared.cuh"

#include <cmath>
#include <cstring>

namespace qsm {

namespace {

// w = 1/(|grad x| + mu_eps) with x = x0 - y, forward differences, periodic
// (src/utils/gradient.rs:21-63, nltv.rs:114-119); *wmax = max w (positive doubles order
// like their bit patterns, so an integer atomicMax on the bits is exact).
template <typename T>
__global__ void k_nltv_weights(int nx, int ny, int nz, double hx, double hy, double hz, double mu_eps,
                               const T* __restrict__ x0, const T* __restrict__ y, T* __restrict__ w,
                               unsigned long long* __restrict__ wmax) {
  const long long N = (long long)nx * ny * nz;
  const long long sz = (long long)nx * ny;
  double m = 0.0;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % nx);
    const long long r = c / nx;
    const int j = (int)(r % ny);
    const int k = (int)(r / ny);
    const long long cx = c - i + (i + 1 < nx ? i + 1 : 0);
    const long long cy = c + ((j + 1 < ny ? j + 1 : 0) - j) * (long long)nx;
    const long long cz = c + ((k + 1 < nz ? k + 1 : 0) - k) * sz;
    const double xc = (double)(x0[c] - y[c]);
    const double gx = ((double)(x0[cx] - y[cx]) - xc) * hx;
    const double gy = ((double)(x0[cy] - y[cy]) - xc) * hy;
    const double gz = ((double)(x0[cz] - y[cz]) - xc) * hz;
    const double wv = 1.0 / (sqrt(gx * gx + gy * gy + gz * gz) + mu_eps);
    w[c] = (T)wv;
    m = fmax(m, wv);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(wmax, (unsigned long long)__double_as_longlong(m));
}

// w /= max w when max w > 1 (nltv.rs:122-128)
template <typename T>
__global__ void k_nltv_normalise(long long N, const unsigned long long* __restrict__ wmax, T* __restrict__ w) {
  const double m = __longlong_as_double((long long)*wmax);
  if (!(m > 1.0)) return;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x)
    w[c] = (T)((double)w[c] / m);
}

// div = bdiv(grad x), x = x0 - y, periodic (src/utils/gradient.rs:21-108): the first
// step of a pass after a reweighting, whose g is grad x.
template <typename T>
__global__ void k_nltv_lapdiv(int nx, int ny, int nz, T hx, T hy, T hz, const T* __restrict__ x0,
                              const T* __restrict__ y, T* __restrict__ div) {
  const long long N = (long long)nx * ny * nz;
  const long long sz = (long long)nx * ny;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % nx);
    const long long r = c / nx;
    const int j = (int)(r % ny);
    const int k = (int)(r / ny);
    const long long row = c - i;
    const long long xp = row + (i + 1 < nx ? i + 1 : 0), xm = row + (i > 0 ? i - 1 : nx - 1);
    const long long yp = c + ((j + 1 < ny ? j + 1 : 0) - j) * (long long)nx;
    const long long ym = c + ((j > 0 ? j - 1 : ny - 1) - j) * (long long)nx;
    const long long zp = c + ((k + 1 < nz ? k + 1 : 0) - k) * sz;
    const long long zm = c + ((k > 0 ? k - 1 : nz - 1) - k) * sz;
    const T xc = x0[c] - y[c];
    const T gx = ((x0[xp] - y[xp]) - xc) * hx, gxm = (xc - (x0[xm] - y[xm])) * hx;
    const T gy = ((x0[yp] - y[yp]) - xc) * hy, gym = (xc - (x0[ym] - y[ym])) * hy;
    const T gz = ((x0[zp] - y[zp]) - xc) * hz, gzm = (xc - (x0[zm] - y[zm])) * hz;
    div[c] = (gx - gxm) * hx + (gy - gym) * hy + (gz - gzm) * hz;
  }
}

template <typename T> __global__ void k_fill(long long N, T v, T* __restrict__ out) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x)
    out[c] = v;
}

}  // namespace

template <typename T>
void nltv_impl(qsm_ctx* ctx, const GridDims& d, const double* f, const uint8_t* mask, const double bdir[3],
               const qsm_nltv_params& p, qsm_progress_fn progress, void* user, double* out) {
  const std::string pre = sizeof(T) == 4 ? "nltv32." : "nltv64.";
  const long long N = d.n;
  TvState* st = ws<TvState>(ctx, pre + "state", 1);
  T* w = ws<T>(ctx, pre + "w", (size_t)N);
  unsigned long long* wmax = ws<unsigned long long>(ctx, pre + "wmax", 1);
  const double rho = 100.0 * p.lambda;  // nltv.rs:76
  const qsm_tv_params tp{p.lambda, rho, p.tol, p.max_iter};
  TvVol<T> v;
  tv_setup<T>(ctx, v, pre, d, f, mask, bdir, tp, st, out);
  v.w = w;
  {
    LaunchScope ls(ctx, "nltv_fill");
    k_fill<T><<<grid1d(N), 256, 0, ctx->stream>>>(N, T(1), w);
    ls.done();
  }
  const size_t max_iter = p.max_iter;
  const size_t total = max_iter * p.newton_iter;
  const bool watch = (progress != nullptr) || (p.tol > 0.0);
  size_t cur = 0;       // inner steps of finished passes
  size_t reported = 0;  // progress calls delivered
  size_t last_y = 0;    // parity buffer holding the latest y
  TvState hs{};
  auto read_state = [&]() {
    QSM_CUDA(cudaMemcpyAsync(&hs, st, sizeof(TvState), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
  };
  auto poll = [&]() {
    read_state();
    const size_t done_now = std::min(max_iter, hs.done ? (size_t)hs.conv_iter : (size_t)(hs.k - 1));
    if (progress)
      for (; reported < cur + done_now; ++reported) progress(user, reported + 1, total);
    return hs.done != 0;
  };
  for (size_t pass = 0; pass < p.newton_iter && max_iter > 0; ++pass) {
    size_t first = 1;
    if (pass > 0) {
      // the pass's first step: g = grad x_last (y_last placed in yb[0], u in ub[1] below)
      TvState init{};
      init.k = 2;
      init.tol = p.tol;
      QSM_CUDA(cudaMemcpyAsync(st, &init, sizeof(TvState), cudaMemcpyHostToDevice, ctx->stream));
      {
        LaunchScope ls(ctx, "nltv_lapdiv");
        k_nltv_lapdiv<T><<<grid1d(N), 256, 0, ctx->stream>>>(d.nx, d.ny, d.nz, v.hx, v.hy, v.hz, v.x0, v.yb[0], v.div);
        ls.done();
      }
      tv_fft(ctx, v, 1);
      first = 2;
    }
    tv_iterate(ctx, v, first, max_iter, watch, poll, tv_poll_launches(progress));
    // the step after the last iteration tests x_max and, when that does not converge,
    // makes the reference's last z/u update (skipped on the device once done)
    tv_step_launch(ctx, v, (int)((max_iter + 1) % 2), 0);
    read_state();
    const bool conv = hs.done != 0;
    const size_t c = conv ? (size_t)hs.conv_iter : max_iter;
    cur += c;
    if (progress)
      for (; reported < cur; ++reported) progress(user, reported + 1, total);
    last_y = c % 2;
    if (pass + 1 == p.newton_iter) break;
    // u after the last update the reference made: written by the step of iteration c
    // when the pass converged at c, else by the step after max_iter
    const size_t u_idx = conv ? c % 2 : (c + 1) % 2;
    QSM_CUDA(cudaMemsetAsync(wmax, 0, sizeof(unsigned long long), ctx->stream));
    {
      LaunchScope ls(ctx, "nltv_weights");
      k_nltv_weights<T><<<grid1d(N), 256, 0, ctx->stream>>>(d.nx, d.ny, d.nz, 1.0 / d.vsx, 1.0 / d.vsy, 1.0 / d.vsz,
                                                            p.mu * 1e-6, v.x0, v.yb[last_y], w, wmax);
      k_nltv_normalise<T><<<grid1d(N), 256, 0, ctx->stream>>>(N, wmax, w);
      ls.done();
    }
    if (last_y != 0)
      QSM_CUDA(cudaMemcpyAsync(v.yb[0], v.yb[1], sizeof(T) * N, cudaMemcpyDeviceToDevice, ctx->stream));
    if (u_idx != 1)
      QSM_CUDA(cudaMemcpyAsync(v.ub[1], v.ub[0], sizeof(T) * 3 * N, cudaMemcpyDeviceToDevice, ctx->stream));
    last_y = 0;
  }
  tv_out_launch(ctx, v, last_y);
  sync(ctx);
  ctx->tv_last_iters = cur;
}

void nltv_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                 const qsm_nltv_params* p, qsm_progress_fn progress, void* user, double* out) {
  GridDims d = check_grid(grid);
  check_ptr(f, "local_field");
  check_ptr(m, "mask");
  check_ptr(out, "out");
  check_ptr(p, "params");
  check_bdir(bdir);
  check_volume_finite(ctx, f, d.n, "local_field");
  check_finite(p->lambda, "lambda");
  check_finite(p->mu, "mu");
  if (std::isnan(p->tol)) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "tol is NaN");
  if (ctx->precision == QSM_PRECISION_MIXED) nltv_impl<float>(ctx, d, f, m, bdir, *p, progress, user, out);
  else nltv_impl<double>(ctx, d, f, m, bdir, *p, progress, user, out);
}

}  // namespace qsm

using namespace qsm;

extern "C" {

void qsm_nltv_params_default(qsm_nltv_params* p) {
  if (!p) return;
  // NltvParams::default, src/inversion/nltv.rs:38-48
  p->lambda = 1e-3;
  p->mu = 1.0;
  p->tol = 1e-3;
  p->max_iter = 250;
  p->newton_iter = 10;
}

qsm_status qsm_nltv_device(qsm_ctx* ctx, const double* d_local_field, const uint8_t* d_mask, const qsm_grid* grid,
                           const double bdir[3], const qsm_nltv_params* params, qsm_progress_fn progress, void* user,
                           double* d_out_chi) {
  return guarded(ctx, [&] {
    nltv_device(ctx, d_local_field, d_mask, grid, bdir, params, progress, user, d_out_chi);
    sync(ctx);
  });
}

qsm_status qsm_nltv(qsm_ctx* ctx, const double* local_field, const uint8_t* mask, const qsm_grid* grid,
                    const double bdir[3], const qsm_nltv_params* params, qsm_progress_fn progress, void* user,
                    double* out_chi) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_ptr(local_field, "local_field");
    check_ptr(mask, "mask");
    check_ptr(out_chi, "out_chi");
    with_host_io(ctx, d.n, local_field, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
      nltv_device(ctx, f, m, grid, bdir, params, progress, user, o);
    });
  });
}

}  // extern "C"
