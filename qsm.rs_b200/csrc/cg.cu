// Conjugate gradients (src/solvers/cg.rs:34-101) on the GPU, for the operator family
//   A x = H^T H x + lambda x,   H x = w * Re IFFT(K * FFT(x))
// with a real, even k-space multiplier K and a real image-space weight w.  This is the
// normal operator of RESHARP (src/bgremove/resharp.rs:97-153: K = 1 - S, w = eroded
// mask), which is built on it here, and of any masked convolution least-squares
// problem.  The reference's cg_solve takes the operator as a closure; closures cannot
// cross the C ABI, so the operator is fixed and its pieces are the arguments.
//
// One iteration is three launches groups with no host synchronisation:
//   A p   : two half-spectrum filter chains (X r2c, Y, Z * K, Y, X c2r); the second
//           chain's store adds lambda*p, writes Ap and accumulates p.Ap in FP64; its
//           last block stops on |p.Ap| < 1e-20 or sets alpha = rsold / p.Ap
//   update: x += alpha p, r -= alpha Ap, ||r||^2 in FP64; the last block stops on
//           ||r|| < tol ||b|| or sets beta
//   p     : p = r + beta p
// replayed as a CUDA graph of one iteration, polled every 8 iterations.
#include "functors.cuh"
#include "solvers.h"

#include <algorithm>
#include <cmath>

namespace qsm {

// helpers defined in bgremove.cu
void smv_spectrum(qsm_ctx* ctx, const Fft3<double>& f64, const GridDims& d, double radius, double2* S);
void erode_smv(qsm_ctx* ctx, const Fft3<double>& f64, const GridDims& d, const double2* Fm, const double2* S,
               double delta, uint8_t* eroded);
double sharp_delta();

namespace {

struct CgState {
  int done;
  int started;  // iterations begun (the reference's progress calls)
  unsigned counter;
  int pad;
  double rsold, alpha, beta, bnorm, tol;
};

// multiplier array pointwise op for the in-kernel Z pass (long axes)
template <typename T> struct OpMulArr {
  using C = cplx_t<T>;
  const T* m;
  __device__ __forceinline__ C mid(C v, int, int, int, long long idx) const { return cscale(v, m[idx]); }
};

template <typename T> struct LoadImg {
  const T* p;
  int nx;
  __device__ __forceinline__ T operator()(int row, int e) const { return p[(long long)row * nx + e]; }
};

// out = w * v / N (w null: 1)
template <typename T> struct StoreWeighted {
  T* out;
  const T* w;
  int nx;
  T invn;
  __device__ __forceinline__ void operator()(int row, int e, T v) {
    const long long i = (long long)row * nx + e;
    const T y = v * invn;
    out[i] = w ? w[i] * y : y;
  }
  __device__ __forceinline__ void finish() {}
};

// Second chain of A x: (H^T H x)[i] + lambda x[i] (src/bgremove/resharp.rs:102-107).
// mode 0: r = b - A x0, p = r, FP64 sums of r^2 and b^2 -> rsold, ||b||
// mode 1: Ap = A p, FP64 sum of p.Ap -> the step length, or the |p.Ap| < 1e-20 stop
template <typename T> struct StoreCgA {
  T* out;        // r (mode 0) or Ap (mode 1)
  T* p_out;      // mode 0: p
  const T* x;    // x0 (may be null) or p
  const T* b;    // mode 0
  int nx;
  T invn, lambda;
  int mode;
  CgState* st;
  double* partials;
  double acc[2];
  __device__ __forceinline__ void operator()(int row, int e, T v) {
    const long long i = (long long)row * nx + e;
    const T xi = x ? x[i] : T(0);
    const T ax = v * invn + lambda * xi;
    if (mode == 0) {
      const T r = b[i] - ax;
      out[i] = r;
      p_out[i] = r;
      acc[0] += (double)r * (double)r;
      acc[1] += (double)b[i] * (double)b[i];
    } else {
      out[i] = ax;
      acc[0] += (double)xi * (double)ax;
    }
  }
  __device__ void finish() {
    if (!grid_sum_last<2>(acc, partials, &st->counter)) return;
    if (threadIdx.x + blockDim.x * threadIdx.y != 0) return;
    if (mode == 0) {
      st->rsold = acc[0];
      st->bnorm = sqrt(acc[1]);
      return;
    }
    st->started += 1;
    const double pap = acc[0];
    if (fabs(pap) < 1e-20) {
      st->done = 1;
      return;
    }
    st->alpha = st->rsold / pap;
  }
};

// x += alpha p; r -= alpha Ap; ||r||^2 (src/solvers/cg.rs:76-90)
template <typename T>
__global__ void k_cg_update(long long N, T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p,
                            const T* __restrict__ ap, CgState* st, double* partials) {
  if (st->done) return;
  const T alpha = (T)st->alpha;
  double acc[1] = {0.0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    const T ri = r[i] - alpha * ap[i];
    r[i] = ri;
    acc[0] += (double)ri * (double)ri;
  }
  if (grid_sum_last<1>(acc, partials, &st->counter) && threadIdx.x == 0) {
    const double rsnew = acc[0];
    if (sqrt(rsnew) < st->tol * st->bnorm) {
      st->done = 1;
      return;
    }
    st->beta = rsnew / st->rsold;
    st->rsold = rsnew;
  }
}

template <typename T>
__global__ void k_cg_p(long long N, T* __restrict__ p, const T* __restrict__ r, const CgState* st) {
  if (st->done) return;
  const T beta = (T)st->beta;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    p[i] = r[i] + beta * p[i];
}

// Symmetrised half-spectrum multiplier (K(k) + K(-k))/2 from a full spectrum in natural
// order; 0 in the padding columns.
template <typename T>
__global__ void k_half_from_full(Geom g, const double* __restrict__ K, T* __restrict__ out) {
  const long long H = g.hsize();
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < H; i += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(i % g.pitch);
    const long long rr = i / g.pitch;
    const int iy = (int)(rr % g.ny), iz = (int)(rr / g.ny);
    double v = 0.0;
    if (ix < g.nxh) {
      const int jx = ix == 0 ? 0 : g.nx - ix, jy = iy == 0 ? 0 : g.ny - iy, jz = iz == 0 ? 0 : g.nz - iz;
      const long long a = ix + (long long)g.nx * (iy + (long long)g.ny * iz);
      const long long b = jx + (long long)g.nx * (jy + (long long)g.ny * jz);
      v = 0.5 * (K[a] + K[b]);
    }
    out[i] = (T)v;
  }
}

// 1 - Re(S) on the half spectrum (RESHARP's DKER, src/bgremove/resharp.rs:71-72)
template <typename T>
__global__ void k_one_minus_re(long long H, const double2* __restrict__ S, T* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < H; i += (long long)gridDim.x * blockDim.x)
    out[i] = (T)(1.0 - S[i].x);
}

template <typename Tin, typename Tout>
__global__ void k_convert(long long N, const Tin* __restrict__ in, Tout* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    out[i] = in ? (Tout)in[i] : Tout(0);
}

template <typename T>
__global__ void k_masked_out(long long N, const T* __restrict__ x, const uint8_t* __restrict__ m,
                             double* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    out[i] = (m == nullptr || m[i] == 1) ? (double)x[i] : 0.0;
}

// y = Re IFFT(K * FFT(x)) then the store functor
template <typename T, class Load, class Store>
void k_filter(qsm_ctx* ctx, const Fft3<T>& f, cplx_t<T>* spec, const T* Kh, bool use_m, const Load& ld,
              const Store& st, const int* done) {
  run_x_r2c<T>(ctx, f, spec, ld, done);
  run_yz<T, -1, 1>(ctx, f, spec, spec, OpId<T>{}, done);
  if (use_m) run_z_fused_m<T>(ctx, f, spec, spec, Kh, done);
  else run_z_fused<T>(ctx, f, spec, spec, OpMulArr<T>{Kh}, done);
  run_yz<T, +1, 1>(ctx, f, spec, spec, OpId<T>{}, done);
  run_x_c2r<T>(ctx, f, spec, st, done);
}

}  // namespace

// CG on device vectors of working precision T (b, x0, w in T; Kh half-spectrum T).
// x0 may be null (zero start); w may be null (weight 1).  Returns the iterations begun.
template <typename T>
size_t cg_normal_impl(qsm_ctx* ctx, const GridDims& d, const T* Kh, const T* w, double lambda, const T* b,
                      const T* x0, double tol, size_t max_iter, qsm_progress_fn progress, void* user, T* x) {
  using C = cplx_t<T>;
  Fft3<T> f = make_fft3<T>(ctx, d);
  const long long N = d.n;
  const char* pre = sizeof(T) == 4 ? "cg32." : "cg64.";
  auto nm = [&](const char* s) { return std::string(pre) + s; };
  T* r = ws<T>(ctx, nm("r"), (size_t)N);
  T* p = ws<T>(ctx, nm("p"), (size_t)N);
  T* ap = ws<T>(ctx, nm("ap"), (size_t)N);
  T* t = ws<T>(ctx, nm("t"), (size_t)N);
  C* spec = ws<C>(ctx, nm("spec"), (size_t)f.g.hsize());
  double* partials = ws<double>(ctx, nm("partials"), (size_t)kMaxPersistentBlocks * 2);
  CgState* st = ws<CgState>(ctx, nm("state"), 1);
  {
    CgState s0{};
    s0.tol = tol;
    h2d(ctx, st, &s0, sizeof(s0));
  }
  const int* done = &st->done;
  const bool use_m = zm_tile_width<T>(d.nz, f.pz.m, f.pz.T) > 0;
  const T invn = (T)(1.0 / (double)N);
  const T lam = (T)lambda;
  // x = x0
  {
    LaunchScope ls(ctx, "cg_init");
    k_convert<T, T><<<grid1d(N), 256, 0, ctx->stream>>>(N, x0, x);
    ls.done();
  }
  auto apply_a = [&](const T* in, const StoreCgA<T>& store) {
    k_filter<T>(ctx, f, spec, Kh, use_m, LoadImg<T>{in, d.nx}, StoreWeighted<T>{t, w, d.nx, invn}, done);
    k_filter<T>(ctx, f, spec, Kh, use_m, LoadImg<T>{t, d.nx}, store, done);
  };
  // r = b - A x0; p = r (src/solvers/cg.rs:50-60)
  apply_a(x, StoreCgA<T>{r, p, x, b, d.nx, invn, lam, 0, st, partials, {0.0, 0.0}});
  const unsigned g = grid1d(N);
  auto one = [&]() {
    apply_a(p, StoreCgA<T>{ap, nullptr, p, nullptr, d.nx, invn, lam, 1, st, partials, {0.0, 0.0}});
    {
      LaunchScope ls(ctx, "cg_update");
      k_cg_update<T><<<g, 256, 0, ctx->stream>>>(N, x, r, p, ap, st, partials);
      ls.done();
    }
    LaunchScope ls(ctx, "cg_p");
    k_cg_p<T><<<g, 256, 0, ctx->stream>>>(N, p, r, st);
    ls.done();
  };
  CgState hs{};
  size_t reported = 0;
  auto poll = [&]() {
    d2h(ctx, &hs, st, sizeof(hs));
    sync(ctx);
    if (progress)
      for (; reported < (size_t)hs.started; ++reported) progress(user, reported, max_iter);
    return hs.done != 0;
  };
  if (max_iter > 0) {
    if (ctx->profiling) {
      for (size_t it = 0; it < max_iter; ++it) {
        one();
        if ((it + 1) % 8 == 0 && poll()) break;
      }
    } else {
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
      const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) throw QsmError(QSM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
      try {
        for (size_t it = 0; it < max_iter; ++it) {
          QSM_CUDA(cudaGraphLaunch(exec, ctx->stream));
          ctx->launches += per;
          if ((it + 1) % 8 == 0 && it + 1 < max_iter && poll()) break;
        }
      } catch (...) {
        cudaGraphExecDestroy(exec);
        throw;
      }
      cudaGraphExecDestroy(exec);
    }
  }
  poll();
  return (size_t)hs.started;
}

// ------------------------------------------------------------------ RESHARP --
// src/bgremove/resharp.rs:58-125
template <typename T>
void resharp_impl(qsm_ctx* ctx, const GridDims& d, const double* field, const uint8_t* mask,
                  const qsm_resharp_params& p, qsm_progress_fn progress, void* user, double* out_local,
                  uint8_t* out_mask) {
  using C = cplx_t<T>;
  Fft3<double> f64 = make_fft3<double>(ctx, d);
  Fft3<T> f = make_fft3<T>(ctx, d);
  const long long N = d.n;
  const size_t H = (size_t)f.g.hsize();
  double2* S = ws<double2>(ctx, "bg.S", H);
  double2* Fm = ws<double2>(ctx, "bg.Fm", H);
  smv_spectrum(ctx, f64, d, p.radius, S);
  run_x_r2c<double>(ctx, f64, Fm, LoadCast<uint8_t, double>{mask, d.nx}, nullptr);
  run_yz<double, -1, 1>(ctx, f64, Fm, Fm, OpId<double>{}, nullptr);
  run_yz<double, -1, 2>(ctx, f64, Fm, Fm, OpId<double>{}, nullptr);
  erode_smv(ctx, f64, d, Fm, S, sharp_delta(), out_mask);
  const char* pre = sizeof(T) == 4 ? "rs32." : "rs64.";
  auto nm = [&](const char* s) { return std::string(pre) + s; };
  T* Kh = ws<T>(ctx, nm("dker"), H);
  T* w = ws<T>(ctx, nm("w"), (size_t)N);
  T* fld = ws<T>(ctx, nm("field"), (size_t)N);
  T* b = ws<T>(ctx, nm("b"), (size_t)N);
  T* t = ws<T>(ctx, nm("t"), (size_t)N);
  T* x = ws<T>(ctx, nm("x"), (size_t)N);
  C* spec = ws<C>(ctx, nm("spec"), H);
  {
    LaunchScope ls(ctx, "resharp_setup");
    k_one_minus_re<T><<<grid1d((long long)H), 256, 0, ctx->stream>>>((long long)H, S, Kh);
    k_convert<uint8_t, T><<<grid1d(N), 256, 0, ctx->stream>>>(N, out_mask, w);
    k_convert<double, T><<<grid1d(N), 256, 0, ctx->stream>>>(N, field, fld);
    ls.done();
  }
  // b = H^T H field (resharp.rs:84-85)
  const bool use_m = zm_tile_width<T>(d.nz, f.pz.m, f.pz.T) > 0;
  const T invn = (T)(1.0 / (double)N);
  k_filter<T>(ctx, f, spec, Kh, use_m, LoadImg<T>{fld, d.nx}, StoreWeighted<T>{t, w, d.nx, invn}, nullptr);
  k_filter<T>(ctx, f, spec, Kh, use_m, LoadImg<T>{t, d.nx}, StoreWeighted<T>{b, nullptr, d.nx, invn}, nullptr);
  cg_normal_impl<T>(ctx, d, Kh, w, p.tik_reg, b, nullptr, p.tol, p.max_iter, progress, user, x);
  LaunchScope ls(ctx, "resharp_out");
  k_masked_out<T><<<grid1d(N), 256, 0, ctx->stream>>>(N, x, out_mask, out_local);
  ls.done();
  sync(ctx);
}

void resharp_device(qsm_ctx* ctx, const double* field, const uint8_t* mask, const GridDims& d,
                    const qsm_resharp_params* p, qsm_progress_fn progress, void* user, double* out_local,
                    uint8_t* out_mask) {
  check_ptr(field, "field");
  check_ptr(mask, "mask");
  check_ptr(out_local, "out_local");
  check_ptr(out_mask, "out_mask");
  check_ptr(p, "params");
  check_finite(p->radius, "radius");
  check_volume_finite(ctx, field, d.n, "field");
  check_finite(p->tik_reg, "tik_reg");
  if (std::isnan(p->tol)) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "tol is NaN");
  if (ctx->precision == QSM_PRECISION_MIXED)
    resharp_impl<float>(ctx, d, field, mask, *p, progress, user, out_local, out_mask);
  else resharp_impl<double>(ctx, d, field, mask, *p, progress, user, out_local, out_mask);
}

// Generic entry: double inputs, converted to the working precision.
template <typename T>
void cg_generic(qsm_ctx* ctx, const GridDims& d, const double* K, const double* w, double lambda, const double* b,
                const double* x0, double tol, size_t max_iter, qsm_progress_fn progress, void* user, double* x_out) {
  Fft3<T> f = make_fft3<T>(ctx, d);
  const long long N = d.n;
  const size_t H = (size_t)f.g.hsize();
  const char* pre = sizeof(T) == 4 ? "cgg32." : "cgg64.";
  auto nm = [&](const char* s) { return std::string(pre) + s; };
  T* Kh = ws<T>(ctx, nm("K"), H);
  T* wt = w ? ws<T>(ctx, nm("w"), (size_t)N) : nullptr;
  T* bt = ws<T>(ctx, nm("b"), (size_t)N);
  T* x0t = x0 ? ws<T>(ctx, nm("x0"), (size_t)N) : nullptr;
  T* xt = ws<T>(ctx, nm("x"), (size_t)N);
  {
    LaunchScope ls(ctx, "cg_setup");
    k_half_from_full<T><<<grid1d((long long)H), 256, 0, ctx->stream>>>(f.g, K, Kh);
    if (w) k_convert<double, T><<<grid1d(N), 256, 0, ctx->stream>>>(N, w, wt);
    k_convert<double, T><<<grid1d(N), 256, 0, ctx->stream>>>(N, b, bt);
    if (x0) k_convert<double, T><<<grid1d(N), 256, 0, ctx->stream>>>(N, x0, x0t);
    ls.done();
  }
  cg_normal_impl<T>(ctx, d, Kh, wt, lambda, bt, x0t, tol, max_iter, progress, user, xt);
  LaunchScope ls(ctx, "cg_out");
  k_masked_out<T><<<grid1d(N), 256, 0, ctx->stream>>>(N, xt, nullptr, x_out);
  ls.done();
  sync(ctx);
}

void cg_kspace_normal_device(qsm_ctx* ctx, const qsm_grid* grid, const double* K, const double* w, double lambda,
                             const double* b, const double* x0, double tol, size_t max_iter,
                             qsm_progress_fn progress, void* user, double* x) {
  GridDims d = check_grid(grid);
  check_ptr(K, "kernel_spectrum");
  check_ptr(b, "b");
  check_ptr(x, "x");
  check_finite(lambda, "lambda");
  if (std::isnan(tol)) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "tol is NaN");
  if (ctx->precision == QSM_PRECISION_MIXED)
    cg_generic<float>(ctx, d, K, w, lambda, b, x0, tol, max_iter, progress, user, x);
  else cg_generic<double>(ctx, d, K, w, lambda, b, x0, tol, max_iter, progress, user, x);
}

}  // namespace qsm

using namespace qsm;

extern "C" {

void qsm_resharp_params_default(qsm_resharp_params* p) {
  if (!p) return;
  p->radius = 6.0;  // ResharpParams::default, src/bgremove/resharp.rs:35-44
  p->tik_reg = 1e-4;
  p->tol = 1e-6;
  p->max_iter = 30;
}

qsm_status qsm_resharp_device(qsm_ctx* ctx, const double* d_field, const uint8_t* d_mask, const qsm_grid* grid,
                              const qsm_resharp_params* params, qsm_progress_fn progress, void* user,
                              double* d_out_local, uint8_t* d_out_mask) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    resharp_device(ctx, d_field, d_mask, d, params, progress, user, d_out_local, d_out_mask);
  });
}

qsm_status qsm_resharp(qsm_ctx* ctx, const double* field, const uint8_t* mask, const qsm_grid* grid,
                       const qsm_resharp_params* params, qsm_progress_fn progress, void* user, double* out_local,
                       uint8_t* out_mask) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_ptr(field, "field");
    check_ptr(mask, "mask");
    check_ptr(out_local, "out_local");
    check_ptr(out_mask, "out_mask");
    const size_t N = (size_t)d.n;
    double* din = ws<double>(ctx, "io.in", N);
    uint8_t* dm = ws<uint8_t>(ctx, "io.mask", N);
    double* dout = ws<double>(ctx, "io.out", N);
    uint8_t* dmo = ws<uint8_t>(ctx, "io.mask_out", N);
    h2d(ctx, din, field, N * sizeof(double));
    h2d(ctx, dm, mask, N);
    resharp_device(ctx, din, dm, d, params, progress, user, dout, dmo);
    d2h(ctx, out_local, dout, N * sizeof(double));
    d2h(ctx, out_mask, dmo, N);
    sync(ctx);
  });
}

qsm_status qsm_cg_kspace_normal_device(qsm_ctx* ctx, const qsm_grid* grid, const double* d_kernel_spectrum,
                                       const double* d_weight, double lambda, const double* d_b, const double* d_x0,
                                       double tol, size_t max_iter, qsm_progress_fn progress, void* user,
                                       double* d_x) {
  return guarded(ctx, [&] {
    cg_kspace_normal_device(ctx, grid, d_kernel_spectrum, d_weight, lambda, d_b, d_x0, tol, max_iter, progress, user,
                            d_x);
  });
}

}  // extern "C"
