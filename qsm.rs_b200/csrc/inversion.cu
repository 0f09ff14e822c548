// Dipole inversion on the GPU: TV-ADMM, TKD, TSVD, Tikhonov and the forward dipole
// model, plus the pipeline dispatcher run_dipole_inversion.
//
// Each closed-form method is one five-pass transform chain with its k-space
// multiplier evaluated in the fused z pass:
//   X r2c (f64 field -> working precision) -> Y fwd -> Z fwd*M*inv -> Y inv
//   -> X c2r (1/N, mask, write f64).
// TV-ADMM adds one fused stencil per iteration; see tv_admm_impl.
#include "functors.cuh"

#include <algorithm>
#include <cstring>

namespace qsm {

// ------------------------------------------------------------- multipliers --
// TKD: |D| <= t -> sign(D)/t with sign(0) = +, else 1/D  (src/inversion/tkd.rs:62-72)
// TSVD: |D| <= t -> 0, else 1/D                             (src/inversion/tkd.rs:117-124)
template <typename T> struct OpTkd {
  using C = cplx_t<T>;
  KSpace K;
  double t;
  int tsvd;
  __device__ __forceinline__ C mid(C v, int ix, int iy, int iz, long long) const {
    const double th = t;
    const int zero_mode = tsvd;
    const double m = K.sym(ix, iy, iz, [&](double kx, double ky, double kz, int, int, int) {
      const double d = K.dipole(kx, ky, kz);
      if (fabs(d) <= th) return zero_mode ? 0.0 : (d >= 0.0 ? 1.0 / th : -1.0 / th);
      return 1.0 / d;
    });
    return cscale(v, (T)m);
  }
};

// Tikhonov: D / (D^2 + lambda*Gamma), Gamma in {1, Lneg, Lpos^2}; |denom| <= 1e-20 -> 0
// (src/inversion/tikhonov.rs:71-115)
template <typename T> struct OpTikhonov {
  using C = cplx_t<T>;
  KSpace K;
  double lambda;
  int reg;
  __device__ __forceinline__ C mid(C v, int ix, int iy, int iz, long long) const {
    const double lam = lambda;
    const int r = reg;
    const KSpace& k = K;
    const double m = K.sym(ix, iy, iz, [&](double kx, double ky, double kz, int a, int b, int c) {
      const double d = k.dipole(kx, ky, kz);
      double gam = 1.0;
      if (r == 1) gam = k.lapneg(a, b, c);
      else if (r == 2) {
        const double lp = -k.lapneg(a, b, c);
        gam = lp * lp;
      }
      const double den = d * d + lam * gam;
      return fabs(den) > 1e-20 ? d / den : 0.0;
    });
    return cscale(v, (T)m);
  }
};

// Forward dipole model multiplier D (src/fft.rs:214-233)
template <typename T> struct OpDipole {
  using C = cplx_t<T>;
  KSpace K;
  __device__ __forceinline__ C mid(C v, int ix, int iy, int iz, long long) const {
    const KSpace& k = K;
    const double m =
        K.sym(ix, iy, iz, [&](double kx, double ky, double kz, int, int, int) { return k.dipole(kx, ky, kz); });
    return cscale(v, (T)m);
  }
};

// ADMM spectral operators (src/inversion/admm.rs:150-178):
//   inv_a = 1/(D^2 + rho*Lneg) (0 when |a| <= 1e-20),  f_hat = F(f) * D * inv_a.
__device__ __forceinline__ double admm_inv_a(const KSpace& K, double kx, double ky, double kz, int ix, int iy, int iz,
                                             double rho) {
  const double d = K.dipole(kx, ky, kz);
  const double a = d * d + rho * K.lapneg(ix, iy, iz);
  return fabs(a) > 1e-20 ? 1.0 / a : 0.0;
}

// Z-forward post-op writing f_hat = F(f) * sym(D * inv_a)
template <typename T> struct OpAdmmRhs {
  using C = cplx_t<T>;
  KSpace K;
  double rho;
  __device__ __forceinline__ C pre(C v, int, int, int, long long) const { return v; }
  __device__ __forceinline__ C post(C v, int ix, int iy, int iz, long long) const {
    const KSpace& k = K;
    const double r = rho;
    const double m = K.sym(ix, iy, iz, [&](double kx, double ky, double kz, int a, int b, int c) {
      return k.dipole(kx, ky, kz) * admm_inv_a(k, kx, ky, kz, a, b, c, r);
    });
    return cscale(v, (T)m);
  }
};

// x-subproblem in k-space: X = f_hat - rho * F(div) * sym(inv_a)  (admm.rs:105-108)
template <typename T> struct OpAdmmSolve {
  using C = cplx_t<T>;
  KSpace K;
  double rho;
  const C* fhat;
  __device__ __forceinline__ C mid(C v, int ix, int iy, int iz, long long idx) const {
    const KSpace& k = K;
    const double r = rho;
    const double ia = K.sym(ix, iy, iz, [&](double kx, double ky, double kz, int a, int b, int c) {
      return admm_inv_a(k, kx, ky, kz, a, b, c, r);
    });
    const T m = (T)(r * ia);
    const C fh = fhat[idx];
    return mk<C>(fh.x - m * v.x, fh.y - m * v.y);
  }
};

// ------------------------------------------------------------- TV stencil --
// The z-subproblem + dual update of iteration i-1 fused with the divergence of
// iteration i (src/inversion/admm.rs:97, 120-142; src/utils/gradient.rs:21-108):
//   v = grad(x) + u, z = shrink(v, lambda/rho), u' = v - z, g = 2z - v, div = bdiv(g).
// g at the three backward neighbours is recomputed from x and u there, so u is
// read from one buffer and written to another (no in-place race).
template <typename T>
__global__ void k_tv_stencil(int nx, int ny, int nz, T hx, T hy, T hz, T thr, const T* __restrict__ x,
                             const T* __restrict__ ui, T* __restrict__ uo, T* __restrict__ div,
                             const int* __restrict__ done) {
  if (done != nullptr && *done) return;
  const long long N = (long long)nx * ny * nz;
  const T* uxi = ui;
  const T* uyi = ui + N;
  const T* uzi = ui + 2 * N;
  T* uxo = uo;
  T* uyo = uo + N;
  T* uzo = uo + 2 * N;
  const long long sy = nx, sz = (long long)nx * ny;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % nx);
    const long long r = idx / nx;
    const int j = (int)(r % ny);
    const int k = (int)(r / ny);
    const long long ip = (i + 1 < nx) ? idx + 1 : idx - (nx - 1);
    const long long im = (i > 0) ? idx - 1 : idx + (nx - 1);
    const long long jp = (j + 1 < ny) ? idx + sy : idx - (ny - 1) * sy;
    const long long jm = (j > 0) ? idx - sy : idx + (ny - 1) * sy;
    const long long kp = (k + 1 < nz) ? idx + sz : idx - (long long)(nz - 1) * sz;
    const long long km = (k > 0) ? idx - sz : idx + (long long)(nz - 1) * sz;
    const T x0 = x[idx];
    // centre
    const T vx = (x[ip] - x0) * hx + uxi[idx];
    const T vy = (x[jp] - x0) * hy + uyi[idx];
    const T vz = (x[kp] - x0) * hz + uzi[idx];
    const T zx = shrink(vx, thr), zy = shrink(vy, thr), zz = shrink(vz, thr);
    uxo[idx] = vx - zx;
    uyo[idx] = vy - zy;
    uzo[idx] = vz - zz;
    const T gx = T(2) * zx - vx, gy = T(2) * zy - vy, gz = T(2) * zz - vz;
    // backward neighbours: only the component along the neighbour's axis is needed
    const T vxm = (x0 - x[im]) * hx + uxi[im];
    const T vym = (x0 - x[jm]) * hy + uyi[jm];
    const T vzm = (x0 - x[km]) * hz + uzi[km];
    const T gxm = T(2) * shrink(vxm, thr) - vxm;
    const T gym = T(2) * shrink(vym, thr) - vym;
    const T gzm = T(2) * shrink(vzm, thr) - vzm;
    div[idx] = (gx - gxm) * hx + (gy - gym) * hy + (gz - gzm) * hz;
  }
}

struct TvState {
  int done;
  int iters;
  unsigned int counter;
  int pad;
  double tol;
  double rc;
};

// X inverse store for TV: x_new = v/N written over x_prev while accumulating
// ||x_new - x_prev||^2 and ||x_new||^2 in double; the last block reduces the
// per-block partials in a fixed order and applies the convergence test
// relative_change(x, x_prev) < tol (src/utils/mod.rs:69-77, admm.rs:117).
template <typename T> struct StoreTvX {
  T* x;
  int nx;
  T scale;
  double2* partials;
  TvState* st;
  double sd, sx;
  __device__ __forceinline__ void operator()(int row, int e, T v) {
    const long long i = (long long)row * nx + e;
    const T xn = v * scale;
    const T xo = x[i];
    const double d = (double)xn - (double)xo;
    sd += d * d;
    sx += (double)xn * (double)xn;
    x[i] = xn;
  }
  __device__ __forceinline__ void finish() {
    __shared__ int am_last;
    double a = sd, b = sx;
    block_sum2(a, b);
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int nth = blockDim.x * blockDim.y;
    if (tid == 0) {
      partials[blockIdx.x] = make_double2(a, b);
      __threadfence();
      const unsigned prev = atomicAdd(&st->counter, 1u);
      am_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (am_last) {
      __threadfence();
      double pa = 0.0, pb = 0.0;
      for (int i = tid; i < (int)gridDim.x; i += nth) {
        const double2 p = __ldcg(&partials[i]);
        pa += p.x;
        pb += p.y;
      }
      block_sum2(pa, pb);
      if (tid == 0) {
        const double rc = sqrt(pa) / (sqrt(pb) + 1e-20);
        st->rc = rc;
        st->iters += 1;
        if (rc < st->tol) st->done = 1;
        st->counter = 0u;
      }
    }
  }
};

template <typename T>
__global__ void k_mask_out(long long N, const T* __restrict__ x, const uint8_t* __restrict__ mask,
                           double* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    out[i] = mask[i] != 0 ? (double)x[i] : 0.0;
}

inline unsigned grid1d(long long n, int block = 256) {
  long long b = (n + block - 1) / block;
  long long cap = 148LL * 16;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

// --------------------------------------------------------------- closed form --
template <typename T, class Op>
void closed_form_chain(qsm_ctx* ctx, const GridDims& d, const double* d_in, const uint8_t* d_mask, const Op& op,
                       double* d_out) {
  using C = cplx_t<T>;
  Fft3<T> f = make_fft3<T>(ctx, d);
  C* spec = ws<C>(ctx, "spec", (size_t)f.g.hsize());
  run_x_r2c<T>(ctx, f, spec, LoadCast<double, T>{d_in, d.nx}, nullptr);
  run_yz<T, -1, 1>(ctx, f, spec, spec, OpId<T>{}, nullptr);
  run_z_fused<T>(ctx, f, spec, spec, op, nullptr);
  run_yz<T, +1, 1>(ctx, f, spec, spec, OpId<T>{}, nullptr);
  run_x_c2r<T>(ctx, f, spec, StoreMaskedF64<T>{d_out, d_mask, d.nx, (T)(1.0 / (double)d.n)}, nullptr);
}

template <class OpF, class OpD>
void closed_form(qsm_ctx* ctx, const GridDims& d, const double* d_in, const uint8_t* d_mask, const OpF& opf,
                 const OpD& opd, double* d_out) {
  if (ctx->precision == QSM_PRECISION_MIXED) closed_form_chain<float>(ctx, d, d_in, d_mask, opf, d_out);
  else closed_form_chain<double>(ctx, d, d_in, d_mask, opd, d_out);
}

void check_bdir(const double bdir[3]) {
  check_ptr(bdir, "bdir");
  for (int i = 0; i < 3; ++i) check_finite(bdir[i], "bdir");
}

void tkd_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                const qsm_tkd_params* p, double* out, int tsvd) {
  GridDims d = check_grid(grid);
  check_ptr(f, "local_field");
  check_ptr(m, "mask");
  check_ptr(out, "out");
  check_ptr(p, "params");
  check_bdir(bdir);
  check_finite(p->threshold, "threshold");
  KSpace K = make_kspace(ctx, d, bdir);
  closed_form(ctx, d, f, m, OpTkd<float>{K, p->threshold, tsvd}, OpTkd<double>{K, p->threshold, tsvd}, out);
}

void tikhonov_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                     const qsm_tikhonov_params* p, double* out) {
  GridDims d = check_grid(grid);
  check_ptr(f, "local_field");
  check_ptr(m, "mask");
  check_ptr(out, "out");
  check_ptr(p, "params");
  check_bdir(bdir);
  check_finite(p->lambda, "lambda");
  if (p->reg < 0 || p->reg > 2) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "unknown regularization");
  KSpace K = make_kspace(ctx, d, bdir);
  closed_form(ctx, d, f, m, OpTikhonov<float>{K, p->lambda, p->reg}, OpTikhonov<double>{K, p->lambda, p->reg}, out);
}

// ------------------------------------------------------------------ TV-ADMM --
template <typename T>
void tv_admm_impl(qsm_ctx* ctx, const GridDims& d, const double* d_f, const uint8_t* d_mask, const double bdir[3],
                  const qsm_tv_params& p, qsm_progress_fn progress, void* user, double* d_out) {
  using C = cplx_t<T>;
  Fft3<T> f = make_fft3<T>(ctx, d);
  KSpace K = make_kspace(ctx, d, bdir);
  const long long N = d.n;
  const long long H = f.g.hsize();
  const char* pre = sizeof(T) == 4 ? "tv32." : "tv64.";
  auto nm = [&](const char* s) { return std::string(pre) + s; };
  T* x = ws<T>(ctx, nm("x"), (size_t)N);
  T* u0 = ws<T>(ctx, nm("u0"), (size_t)(3 * N));
  T* u1 = ws<T>(ctx, nm("u1"), (size_t)(3 * N));
  T* div = ws<T>(ctx, nm("div"), (size_t)N);
  C* spec = ws<C>(ctx, nm("spec"), (size_t)H);
  C* fhat = ws<C>(ctx, nm("fhat"), (size_t)H);
  const long long nblk = x_blocks(f);
  double2* partials = ws<double2>(ctx, nm("partials"), (size_t)nblk);
  TvState* st = ws<TvState>(ctx, nm("state"), 1);
  int* done = &st->done;

  QSM_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * N, ctx->stream));
  QSM_CUDA(cudaMemsetAsync(u0, 0, sizeof(T) * 3 * N, ctx->stream));
  TvState init{};
  init.tol = p.tol;
  QSM_CUDA(cudaMemcpyAsync(st, &init, sizeof(TvState), cudaMemcpyHostToDevice, ctx->stream));

  // f_hat = F(f) * sym(D * inv_a)
  run_x_r2c<T>(ctx, f, spec, LoadCast<double, T>{d_f, d.nx}, nullptr);
  run_yz<T, -1, 1>(ctx, f, spec, spec, OpId<T>{}, nullptr);
  run_yz<T, -1, 2>(ctx, f, spec, fhat, OpAdmmRhs<T>{K, p.rho}, nullptr);

  const T hx = (T)(1.0 / d.vsx), hy = (T)(1.0 / d.vsy), hz = (T)(1.0 / d.vsz);
  const T thr = (T)(p.lambda / p.rho);
  const T scale = (T)(1.0 / (double)N);
  const unsigned sgrid = grid1d(N);
  auto one_iter = [&](const T* ui, T* uo) {
    LaunchScope ls(ctx, "tv_stencil");
    k_tv_stencil<T><<<sgrid, 256, 0, ctx->stream>>>(d.nx, d.ny, d.nz, hx, hy, hz, thr, x, ui, uo, div, done);
    ls.done();
    run_x_r2c<T>(ctx, f, spec, LoadCast<T, T>{div, d.nx}, done);
    run_yz<T, -1, 1>(ctx, f, spec, spec, OpId<T>{}, done);
    run_z_fused<T>(ctx, f, spec, spec, OpAdmmSolve<T>{K, p.rho, fhat}, done);
    run_yz<T, +1, 1>(ctx, f, spec, spec, OpId<T>{}, done);
    run_x_c2r<T>(ctx, f, spec, StoreTvX<T>{x, d.nx, scale, partials, st, 0.0, 0.0}, done);
  };

  if (ctx->profiling) {
    // eager launches so that every kernel is timed individually
    for (size_t it = 0; it < p.max_iter; ++it) {
      if (it % 2 == 0) one_iter(u0, u1);
      else one_iter(u1, u0);
    }
    TvState hs{};
    QSM_CUDA(cudaMemcpyAsync(&hs, st, sizeof(TvState), cudaMemcpyDeviceToHost, ctx->stream));
    {
      LaunchScope ls(ctx, "mask_out");
      k_mask_out<T><<<grid1d(N), 256, 0, ctx->stream>>>(N, x, d_mask, d_out);
      ls.done();
    }
    sync(ctx);
    if (progress) {
      for (int i = 0; i < hs.iters; ++i) progress(user, (size_t)i + 1, p.max_iter);
      if (hs.done) progress(user, (size_t)hs.iters, (size_t)hs.iters);
    }
    ctx->tv_last_iters = (size_t)hs.iters;
    return;
  }
  // Two iterations (u0 -> u1 -> u0) captured as one graph; an odd tail runs eagerly.
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const uint64_t l0 = ctx->launches;
  QSM_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  try {
    one_iter(u0, u1);
    one_iter(u1, u0);
  } catch (...) {
    cudaStreamEndCapture(ctx->stream, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  QSM_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
  const uint64_t per_pair = ctx->launches - l0;
  ctx->launches = l0;
  cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) throw QsmError(QSM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));

  const size_t max_iter = p.max_iter;
  const size_t pairs = max_iter / 2;
  const bool watch = (progress != nullptr) || (p.tol > 0.0);
  const size_t chunk = 16;  // graph launches between host checks when watching
  size_t reported = 0;
  TvState hs{};
  bool converged = false;
  try {
    size_t launched_pairs = 0;
    while (launched_pairs < pairs && !converged) {
      const size_t todo = watch ? std::min(chunk, pairs - launched_pairs) : (pairs - launched_pairs);
      for (size_t c = 0; c < todo; ++c) {
        QSM_CUDA(cudaGraphLaunch(exec, ctx->stream));
        ctx->launches += per_pair;
      }
      launched_pairs += todo;
      if (watch) {
        QSM_CUDA(cudaMemcpyAsync(&hs, st, sizeof(TvState), cudaMemcpyDeviceToHost, ctx->stream));
        sync(ctx);
        if (progress)
          for (; reported < (size_t)hs.iters; ++reported) progress(user, reported + 1, max_iter);
        if (hs.done) converged = true;
      }
    }
    if (!converged && (max_iter % 2 == 1)) one_iter(u0, u1);  // after an even count u lives in u0
  } catch (...) {
    cudaGraphExecDestroy(exec);
    throw;
  }
  cudaGraphExecDestroy(exec);

  QSM_CUDA(cudaMemcpyAsync(&hs, st, sizeof(TvState), cudaMemcpyDeviceToHost, ctx->stream));
  {
    LaunchScope ls(ctx, "mask_out");
    k_mask_out<T><<<grid1d(N), 256, 0, ctx->stream>>>(N, x, d_mask, d_out);
    ls.done();
  }
  sync(ctx);
  if (progress) {
    for (; reported < (size_t)hs.iters; ++reported) progress(user, reported + 1, max_iter);
    if (hs.done) progress(user, (size_t)hs.iters, (size_t)hs.iters);
  }
  ctx->tv_last_iters = (size_t)hs.iters;
}

void tv_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
               const qsm_tv_params* p, qsm_progress_fn progress, void* user, double* out) {
  GridDims d = check_grid(grid);
  check_ptr(f, "local_field");
  check_ptr(m, "mask");
  check_ptr(out, "out");
  check_ptr(p, "params");
  check_bdir(bdir);
  check_finite(p->lambda, "lambda");
  check_finite(p->rho, "rho");
  if (std::isnan(p->tol)) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "tol is NaN");
  if (ctx->precision == QSM_PRECISION_MIXED) tv_admm_impl<float>(ctx, d, f, m, bdir, *p, progress, user, out);
  else tv_admm_impl<double>(ctx, d, f, m, bdir, *p, progress, user, out);
}

// Host-pointer wrapper: stage inputs on the device, run, copy back.
template <class Run>
void with_host_io(qsm_ctx* ctx, const GridDims& d, const double* h_in, const uint8_t* h_mask, double* h_out,
                  Run run) {
  const size_t N = (size_t)d.n;
  double* din = ws<double>(ctx, "io.in", N);
  uint8_t* dm = h_mask ? ws<uint8_t>(ctx, "io.mask", N) : nullptr;
  double* dout = ws<double>(ctx, "io.out", N);
  h2d(ctx, din, h_in, N * sizeof(double));
  if (h_mask) h2d(ctx, dm, h_mask, N);
  run(din, dm, dout);
  d2h(ctx, h_out, dout, N * sizeof(double));
  sync(ctx);
}

template <typename T>
void fft3d_real_impl(qsm_ctx* ctx, const GridDims& d, const double* h_in, double* h_out) {
  using C = cplx_t<T>;
  Fft3<T> f = make_fft3<T>(ctx, d);
  const size_t N = (size_t)d.n;
  double* din = ws<double>(ctx, "io.in", N);
  C* spec = ws<C>(ctx, "spec", (size_t)f.g.hsize());
  h2d(ctx, din, h_in, N * sizeof(double));
  run_x_r2c<T>(ctx, f, spec, LoadCast<double, T>{din, d.nx}, nullptr);
  run_yz<T, -1, 1>(ctx, f, spec, spec, OpId<T>{}, nullptr);
  run_yz<T, -1, 2>(ctx, f, spec, spec, OpId<T>{}, nullptr);
  std::vector<C> half((size_t)f.g.hsize());
  d2h(ctx, half.data(), spec, half.size() * sizeof(C));
  sync(ctx);
  // expand with Hermitian symmetry X(k) = conj(X(-k)) to the full C2C layout
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        C v;
        if (i < f.g.nxh) {
          v = half[(size_t)i + (size_t)f.g.pitch * ((size_t)j + (size_t)ny * k)];
        } else {
          const int mi = nx - i, mj = (ny - j) % ny, mk2 = (nz - k) % nz;
          C w = half[(size_t)mi + (size_t)f.g.pitch * ((size_t)mj + (size_t)ny * mk2)];
          v = w;
          v.y = -w.y;
        }
        const size_t o = 2 * ((size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k));
        h_out[o] = (double)v.x;
        h_out[o + 1] = (double)v.y;
      }
}

}  // namespace qsm

using namespace qsm;

extern "C" {

qsm_status qsm_tv_admm_device(qsm_ctx* ctx, const double* d_local_field, const uint8_t* d_mask, const qsm_grid* grid,
                              const double bdir[3], const qsm_tv_params* params, qsm_progress_fn progress, void* user,
                              double* d_out_chi) {
  return guarded(ctx, [&] {
    tv_device(ctx, d_local_field, d_mask, grid, bdir, params, progress, user, d_out_chi);
    sync(ctx);
  });
}

qsm_status qsm_tv_admm(qsm_ctx* ctx, const double* local_field, const uint8_t* mask, const qsm_grid* grid,
                       const double bdir[3], const qsm_tv_params* params, qsm_progress_fn progress, void* user,
                       double* out_chi) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_ptr(local_field, "local_field");
    check_ptr(mask, "mask");
    check_ptr(out_chi, "out_chi");
    with_host_io(ctx, d, local_field, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
      tv_device(ctx, f, m, grid, bdir, params, progress, user, o);
    });
  });
}

size_t qsm_tv_last_iterations(const qsm_ctx* ctx) { return ctx ? ctx->tv_last_iters : 0; }

qsm_status qsm_tkd_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                          const qsm_tkd_params* p, double* out) {
  return guarded(ctx, [&] {
    tkd_device(ctx, f, m, grid, bdir, p, out, 0);
    sync(ctx);
  });
}
qsm_status qsm_tkd(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                   const qsm_tkd_params* p, double* out) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_ptr(f, "local_field");
    check_ptr(m, "mask");
    check_ptr(out, "out_chi");
    with_host_io(ctx, d, f, m, out, [&](const double* df, const uint8_t* dm, double* o) {
      tkd_device(ctx, df, dm, grid, bdir, p, o, 0);
    });
  });
}
qsm_status qsm_tsvd_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                           const qsm_tkd_params* p, double* out) {
  return guarded(ctx, [&] {
    tkd_device(ctx, f, m, grid, bdir, p, out, 1);
    sync(ctx);
  });
}
qsm_status qsm_tsvd(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                    const qsm_tkd_params* p, double* out) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_ptr(f, "local_field");
    check_ptr(m, "mask");
    check_ptr(out, "out_chi");
    with_host_io(ctx, d, f, m, out, [&](const double* df, const uint8_t* dm, double* o) {
      tkd_device(ctx, df, dm, grid, bdir, p, o, 1);
    });
  });
}
qsm_status qsm_tikhonov_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid,
                               const double bdir[3], const qsm_tikhonov_params* p, double* out) {
  return guarded(ctx, [&] {
    tikhonov_device(ctx, f, m, grid, bdir, p, out);
    sync(ctx);
  });
}
qsm_status qsm_tikhonov(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                        const qsm_tikhonov_params* p, double* out) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_ptr(f, "local_field");
    check_ptr(m, "mask");
    check_ptr(out, "out_chi");
    with_host_io(ctx, d, f, m, out, [&](const double* df, const uint8_t* dm, double* o) {
      tikhonov_device(ctx, df, dm, grid, bdir, p, o);
    });
  });
}

qsm_status qsm_dipole_forward(qsm_ctx* ctx, const double* chi, const qsm_grid* grid, const double bdir[3],
                              double* out_field) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_ptr(chi, "chi");
    check_ptr(out_field, "out_field");
    check_bdir(bdir);
    KSpace K = make_kspace(ctx, d, bdir);
    with_host_io(ctx, d, chi, nullptr, out_field, [&](const double* df, const uint8_t*, double* o) {
      closed_form(ctx, d, df, nullptr, OpDipole<float>{K}, OpDipole<double>{K}, o);
    });
  });
}

qsm_status qsm_fft3d_real(qsm_ctx* ctx, const double* in, const qsm_grid* grid, double* out_complex) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_ptr(in, "in");
    check_ptr(out_complex, "out");
    if (ctx->precision == QSM_PRECISION_MIXED) fft3d_real_impl<float>(ctx, d, in, out_complex);
    else fft3d_real_impl<double>(ctx, d, in, out_complex);
  });
}

void qsm_inversion_config_default(qsm_inversion_config* c) {
  if (!c) return;
  c->algorithm = QSM_INV_RTS;  // InversionConfig::default, src/pipeline/config.rs:251
  qsm_tkd_params_default(&c->tkd);
  qsm_tkd_params_default(&c->tsvd);
  qsm_tikhonov_params_default(&c->tikhonov);
  qsm_tv_params_default(&c->tv);
}

qsm_status qsm_run_dipole_inversion(qsm_ctx* ctx, const double* local_field_ppm, size_t len, const uint8_t* mask,
                                    const qsm_scan_metadata* md, const qsm_inversion_config* cfg,
                                    qsm_progress_fn progress, void* user, double* out_chi) {
  return guarded(ctx, [&] {
    check_ptr(md, "metadata");
    check_ptr(cfg, "config");
    qsm_grid g{md->nx, md->ny, md->nz, md->vsx, md->vsy, md->vsz};
    const size_t n = md->nx * md->ny * md->nz;
    if (len != n)
      throw QsmError(QSM_ERR_DIMENSION_MISMATCH,
                     "dimension mismatch: expected " + std::to_string(n) + ", got " + std::to_string(len));
    GridDims d = check_grid(&g);
    check_ptr(local_field_ppm, "local_field_ppm");
    check_ptr(mask, "mask");
    check_ptr(out_chi, "out_chi");
    const double* b = md->b0_direction;
    switch (cfg->algorithm) {
      case QSM_INV_TKD:
        with_host_io(ctx, d, local_field_ppm, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
          tkd_device(ctx, f, m, &g, b, &cfg->tkd, o, 0);
        });
        break;
      case QSM_INV_TSVD:
        with_host_io(ctx, d, local_field_ppm, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
          tkd_device(ctx, f, m, &g, b, &cfg->tsvd, o, 1);
        });
        break;
      case QSM_INV_TIKHONOV:
        with_host_io(ctx, d, local_field_ppm, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
          tikhonov_device(ctx, f, m, &g, b, &cfg->tikhonov, o);
        });
        break;
      case QSM_INV_TV:
        with_host_io(ctx, d, local_field_ppm, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
          tv_device(ctx, f, m, &g, b, &cfg->tv, progress, user, o);
        });
        break;
      case QSM_INV_TGV:
        throw QsmError(QSM_ERR_INVALID_CONFIG, "invalid config: Tgv should use run_tgv or run_qsmart");
      case QSM_INV_QSMART:
        throw QsmError(QSM_ERR_INVALID_CONFIG, "invalid config: Qsmart should use run_tgv or run_qsmart");
      default:
        throw QsmError(QSM_ERR_INVALID_CONFIG, "invalid config: algorithm " + std::to_string(cfg->algorithm) +
                                                   " is not provided by this library");
    }
  });
}

}  // extern "C"
