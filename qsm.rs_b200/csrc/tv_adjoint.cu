// Unrolled TV-ADMM with its adjoint (vector-Jacobian product) for K fixed iterations:
// chi_K = M x_K, and given dL/dchi_K the gradients dL/df (local field) and dL/dlambda.
// The reference has no derivative; the forward pass is exactly tv_admm with tol = 0 and
// max_iter = K (src/inversion/tv.rs:63-97), computed by the same kernels.
//
// Forward iteration j (x_0 = u_0 = g_0 = 0):
//   x_j = A f - B bdiv(g_{j-1}),  A = Re IFFT(sym(D inv_a) FFT .),  B = rho Re IFFT(sym(inv_a) FFT .)
//   U_j: v_j = grad x_j + u_{j-1}, z_j = shrink(v_j, t), u_j = v_j - z_j, g_j = 2 z_j - v_j, t = lambda/rho.
// A and B are real symmetric k-space multipliers, hence self-adjoint, and bdiv = -grad^T
// (periodic).  Reverse sweep, j = K .. 1, with vbar_K = 0:
//   xbar_j = M gbar_out [j = K] - bdiv(vbar_j);   s += xbar_j
//   w = B xbar_j;   gbar_{j-1} = grad w
//   U_{j-1} (j >= 2): ubar = vbar_j, zbar = -ubar + 2 gbar, a = [|v_{j-1}| > t],
//            vbar_{j-1} = ubar - gbar + a zbar,  tbar += sum a (-sign v_{j-1}) zbar
//   dL/df = A s,   dL/dlambda = tbar / rho.
// The states (y_j, u_{j-1}) are checkpointed every C iterations in the forward pass and
// recomputed one segment at a time in the reverse sweep, so memory is (K/C + C) states.
#include "tv_shared.cuh"

namespace qsm {

namespace {

// xbar_j (first: mask * gbar_out; else -bdiv(vbar) with periodic backward differences)
// as the real input of the X r2c pass; also accumulates s += xbar_j.  Each (row, e) is
// loaded exactly once by k_x_r2c.
template <typename T> struct LoadAdjX {
  const double* gout;
  const uint8_t* mask;
  const T* vbar;
  T* s;
  int nx, ny, nz;
  T hx, hy, hz;
  int first;
  __device__ __forceinline__ T operator()(int row, int e) const {
    const long long N = (long long)nx * ny * nz, sxy = (long long)nx * ny;
    const long long idx = (long long)row * nx + e;
    T xb;
    if (first) {
      xb = mask[idx] != 0 ? (T)gout[idx] : T(0);
    } else {
      const int j = row % ny, k = row / ny;
      const long long xm = e > 0 ? idx - 1 : idx - 1 + nx;
      const long long ym = j > 0 ? idx - nx : idx - nx + sxy;
      const long long zm = k > 0 ? idx - sxy : idx - sxy + N;
      const T div = (vbar[idx] - vbar[xm]) * hx + (vbar[N + idx] - vbar[N + ym]) * hy +
                    (vbar[2 * N + idx] - vbar[2 * N + zm]) * hz;
      xb = -div;
    }
    s[idx] += xb;
    return xb;
  }
};

// Adjoint of U_{j-1}: reads x_{j-1} = x0 - y, u_{j-2} = u, ubar = vbar_j (null: zero) and
// w = B xbar_j (gbar = grad w); writes vbar_{j-1}; FP64 sum of the lambda sensitivity
// added to *tbar by the last block.
template <typename T>
__global__ void __launch_bounds__(256)
    k_tv_adj_update(int nx, int ny, int nz, T hx, T hy, T hz, T thr, const T* __restrict__ x0,
                    const T* __restrict__ y, const T* __restrict__ u, const T* __restrict__ ubar,
                    const T* __restrict__ w, T* __restrict__ vbar, double* partials, unsigned* counter,
                    double* tbar) {
  const long long N = (long long)nx * ny * nz, sxy = (long long)nx * ny;
  double acc[1] = {0.0};
  for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += (long long)gridDim.x * blockDim.x) {
    const unsigned r = (unsigned)l / (unsigned)nx;  // N < 2^32 (checked by the host)
    const int i = (int)((unsigned)l - r * (unsigned)nx);
    const int j = (int)(r % (unsigned)ny);
    const int k = (int)(r / (unsigned)ny);
    const long long nb[3] = {i + 1 < nx ? l + 1 : l + 1 - nx, j + 1 < ny ? l + nx : l + nx - sxy,
                             k + 1 < nz ? l + sxy : l + sxy - N};
    const T h[3] = {hx, hy, hz};
    const T xl = x0[l] - y[l], wl = w[l];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T v = (x0[nb[c]] - y[nb[c]] - xl) * h[c] + u[c * N + l];
      const T gb = (w[nb[c]] - wl) * h[c];
      const T ub = ubar ? ubar[c * N + l] : T(0);
      const T zb = -ub + T(2) * gb;
      const bool act = v > thr || v < -thr;
      vbar[c * N + l] = ub - gb + (act ? zb : T(0));
      if (act) acc[0] += (double)(v > T(0) ? -zb : zb);
    }
  }
  if (grid_sum_last<1>(acc, partials, counter) && threadIdx.x == 0) *tbar += acc[0];
}

template <typename T>
__global__ void k_copy(long long n, const T* __restrict__ a, T* __restrict__ b) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = a[i];
}

template <typename T>
__global__ void k_accumulate_neg_bdiv(int nx, int ny, int nz, T hx, T hy, T hz, const T* __restrict__ vbar,
                                      T* __restrict__ s) {
  const long long N = (long long)nx * ny * nz, sxy = (long long)nx * ny;
  for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += (long long)gridDim.x * blockDim.x) {
    const unsigned r = (unsigned)l / (unsigned)nx;
    const int i = (int)((unsigned)l - r * (unsigned)nx);
    const int j = (int)(r % (unsigned)ny);
    const int k = (int)(r / (unsigned)ny);
    const long long xm = i > 0 ? l - 1 : l - 1 + nx;
    const long long ym = j > 0 ? l - nx : l - nx + sxy;
    const long long zm = k > 0 ? l - sxy : l - sxy + N;
    const T div = (vbar[l] - vbar[xm]) * hx + (vbar[N + l] - vbar[N + ym]) * hy + (vbar[2 * N + l] - vbar[2 * N + zm]) * hz;
    s[l] -= div;
  }
}

}  // namespace

template <typename T>
void tv_unrolled_impl(qsm_ctx* ctx, const GridDims& d, const double* f, const uint8_t* mask, const double bdir[3],
                      double lambda, double rho, size_t K, size_t C, const double* gout, double* chi,
                      double* grad_f, double* grad_lambda) {
  using Cx = cplx_t<T>;
  const long long N = d.n;
  const std::string pre = sizeof(T) == 4 ? "tvu32." : "tvu64.";
  auto nm = [&](const char* s) { return pre + s; };
  qsm_tv_params p{lambda, rho, 0.0, K};
  TvState* st = ws<TvState>(ctx, nm("state"), 1);
  TvVol<T> v;
  tv_setup<T>(ctx, v, pre, d, f, mask, bdir, p, st, chi);
  const size_t nck = (K + C - 1) / C;  // checkpoints at iterations 0, C, 2C, ... < K
  T* ck_y = ws<T>(ctx, nm("ck_y"), (size_t)N * nck);
  T* ck_u = ws<T>(ctx, nm("ck_u"), (size_t)(3 * N) * nck);
  const unsigned g = grid1d(N);
  auto copy = [&](const T* a, T* b, long long n) {
    LaunchScope ls(ctx, "tv_adj_copy");
    k_copy<T><<<grid1d(n), 256, 0, ctx->stream>>>(n, a, b);
    ls.done();
  };
  // state after iteration i: y_i in yb[i % 2], u_{i-1} in ub[i % 2]
  for (size_t i = 1; i <= K; ++i) {
    if ((i - 1) % C == 0) {
      const size_t c = (i - 1) / C;
      copy(v.yb[(i - 1) % 2], ck_y + (size_t)N * c, N);
      copy(v.ub[(i - 1) % 2], ck_u + (size_t)(3 * N) * c, 3 * N);
    }
    tv_iter(ctx, v, (int)(i % 2));
  }
  tv_out_launch(ctx, v, K);  // chi_K = M x_K
  if (gout == nullptr) {
    sync(ctx);
    return;
  }
  // ---------------------------------------------------------------- reverse --
  T* seg_y = ws<T>(ctx, nm("seg_y"), (size_t)N * C);
  T* seg_u = ws<T>(ctx, nm("seg_u"), (size_t)(3 * N) * C);
  T* vb[2] = {ws<T>(ctx, nm("vbar0"), (size_t)(3 * N)), ws<T>(ctx, nm("vbar1"), (size_t)(3 * N))};
  T* w = ws<T>(ctx, nm("w"), (size_t)N);
  T* s = ws<T>(ctx, nm("s"), (size_t)N);
  // names distinct from tv_setup's buffers: growing a workspace reallocates it
  double* partials = ws<double>(ctx, nm("adj_partials"), (size_t)kMaxPersistentBlocks);
  unsigned* counter = ws<unsigned>(ctx, nm("adj_counter"), 1);
  double* tbar = ws<double>(ctx, nm("adj_tbar"), 1);
  QSM_CUDA(cudaMemsetAsync(s, 0, sizeof(T) * N, ctx->stream));
  QSM_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), ctx->stream));
  QSM_CUDA(cudaMemsetAsync(tbar, 0, sizeof(double), ctx->stream));
  int cur = 0;           // vb[cur] holds vbar_j for the step about to run
  bool have_vbar = false;  // false: vbar_K = 0
  size_t j = K;
  for (size_t cseg = nck; cseg-- > 0;) {
    const size_t c = cseg * C;
    const size_t hi = std::min(c + C, K);  // states S_c .. S_{hi-1}
    // restore S_c into the parity slots of iteration c and recompute S_{c+1} .. S_{hi-1}
    copy(ck_y + (size_t)N * cseg, v.yb[c % 2], N);
    copy(ck_u + (size_t)(3 * N) * cseg, v.ub[c % 2], 3 * N);
    copy(v.yb[c % 2], seg_y, N);
    copy(v.ub[c % 2], seg_u, 3 * N);
    for (size_t i = c + 1; i < hi; ++i) {
      tv_iter(ctx, v, (int)(i % 2));
      copy(v.yb[i % 2], seg_y + (size_t)N * (i - c), N);
      copy(v.ub[i % 2], seg_u + (size_t)(3 * N) * (i - c), 3 * N);
    }
    // reverse steps j with j - 1 in [max(c, 1), hi - 1]
    for (; j >= 2 && j - 1 >= c; --j) {
      const size_t i = j - 1;
      // w = B xbar_j (and s += xbar_j in the loader)
      LoadAdjX<T> ld{gout, mask, have_vbar ? vb[cur] : nullptr, s, d.nx, d.ny, d.nz, v.hx, v.hy, v.hz,
                     j == K ? 1 : 0};
      if (!have_vbar && j != K) throw QsmError(QSM_ERR_CUDA, "adjoint sweep out of order");
      run_x_r2c<T>(ctx, v.f, v.spec, ld, nullptr);
      run_yz<T, -1, 1>(ctx, v.f, v.spec, v.spec, OpId<T>{}, nullptr);
      if (v.use_mult) run_z_fused_m<T>(ctx, v.f, v.spec, v.spec, v.mult, nullptr);
      else run_z_fused<T>(ctx, v.f, v.spec, v.spec, v.mul, nullptr);
      run_yz<T, +1, 1>(ctx, v.f, v.spec, v.spec, OpId<T>{}, nullptr);
      run_x_c2r<T>(ctx, v.f, v.spec, StoreReal<T>{w, d.nx, v.scale}, nullptr);
      // adjoint of U_i from S_i = (y_i, u_{i-1})
      LaunchScope ls(ctx, "tv_adj_update");
      k_tv_adj_update<T><<<g, 256, 0, ctx->stream>>>(d.nx, d.ny, d.nz, v.hx, v.hy, v.hz, v.thr, v.x0,
                                                     seg_y + (size_t)N * (i - c), seg_u + (size_t)(3 * N) * (i - c),
                                                     have_vbar ? vb[cur] : nullptr, w, vb[1 - cur], partials, counter,
                                                     tbar);
      ls.done();
      cur = 1 - cur;
      have_vbar = true;
    }
  }
  // j = 1: xbar_1 only feeds s (g_0 is constant)
  if (K == 1) {
    LoadAdjX<T> ld{gout, mask, nullptr, s, d.nx, d.ny, d.nz, v.hx, v.hy, v.hz, 1};
    run_x_r2c<T>(ctx, v.f, v.spec, ld, nullptr);  // spectrum unused: the loader accumulates s
  } else {
    LaunchScope ls(ctx, "tv_adj_accumulate");
    k_accumulate_neg_bdiv<T><<<g, 256, 0, ctx->stream>>>(d.nx, d.ny, d.nz, v.hx, v.hy, v.hz, vb[cur], s);
    ls.done();
  }
  // dL/df = A s (the x0 operator), dL/dlambda = tbar / rho
  const KSpace K64 = make_kspace(ctx, d, bdir);
  run_x_r2c<T>(ctx, v.f, v.spec, LoadCast<T, T>{s, d.nx}, nullptr);
  run_yz<T, -1, 1>(ctx, v.f, v.spec, v.spec, OpId<T>{}, nullptr);
  run_z_fused<T>(ctx, v.f, v.spec, v.spec, OpAdmmRhs<T>{K64, rho}, nullptr);
  run_yz<T, +1, 1>(ctx, v.f, v.spec, v.spec, OpId<T>{}, nullptr);
  run_x_c2r<T>(ctx, v.f, v.spec, StoreMaskedF64<T>{grad_f, nullptr, d.nx, v.scale}, nullptr);
  double tb = 0.0;
  d2h(ctx, &tb, tbar, sizeof(double));
  sync(ctx);
  if (grad_lambda) *grad_lambda = tb / rho;
  (void)sizeof(Cx);
}

void tv_unrolled_device(qsm_ctx* ctx, const double* f, const uint8_t* mask, const qsm_grid* grid,
                        const double bdir[3], double lambda, double rho, size_t K, size_t C, const double* gout,
                        double* chi, double* grad_f, double* grad_lambda) {
  GridDims d = check_grid(grid);
  check_ptr(f, "local_field");
  check_ptr(mask, "mask");
  check_ptr(chi, "out_chi");
  check_bdir(bdir);
  check_finite(lambda, "lambda");
  check_finite(rho, "rho");
  check_volume_finite(ctx, f, d.n, "local_field");
  if (K == 0) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "iterations must be >= 1");
  if (C == 0) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "checkpoint_every must be >= 1");
  if (d.n >= (1LL << 32)) throw QsmError(QSM_ERR_UNSUPPORTED_SIZE, "volumes hold fewer than 2^32 voxels");
  if (gout) check_ptr(grad_f, "out_grad_field");
  if (ctx->precision == QSM_PRECISION_MIXED)
    tv_unrolled_impl<float>(ctx, d, f, mask, bdir, lambda, rho, K, C, gout, chi, grad_f, grad_lambda);
  else tv_unrolled_impl<double>(ctx, d, f, mask, bdir, lambda, rho, K, C, gout, chi, grad_f, grad_lambda);
}

}  // namespace qsm

using namespace qsm;

extern "C" qsm_status qsm_tv_admm_unrolled_vjp_device(qsm_ctx* ctx, const double* d_local_field,
                                                      const uint8_t* d_mask, const qsm_grid* grid,
                                                      const double bdir[3], double lambda, double rho,
                                                      size_t iterations, size_t checkpoint_every,
                                                      const double* d_grad_chi, double* d_out_chi,
                                                      double* d_out_grad_field, double* out_grad_lambda) {
  return guarded(ctx, [&] {
    tv_unrolled_device(ctx, d_local_field, d_mask, grid, bdir, lambda, rho, iterations, checkpoint_every, d_grad_chi,
                       d_out_chi, d_out_grad_field, out_grad_lambda);
  });
}
