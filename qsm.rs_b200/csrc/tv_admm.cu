// TV-ADMM dipole inversion (src/inversion/tv.rs:63-97, src/inversion/admm.rs:76-178).
//
// The reference iteration is
//   div = bdiv(g); x = Re IFFT(f_hat - rho*FFT(div)*inv_a); stop if relchange(x) < tol;
//   v = grad x + u; z = shrink(v, lambda/rho); u = v - z; g = 2z - v.
// Because the x-update is linear, x_i = x0 - y_i with x0 = Re IFFT(f_hat) (computed
// once) and y_i = Re IFFT(rho*inv_a*FFT(div_i)).  One iteration is six kernels:
//
//   k_tv_step   : convergence test of the previous iterate (FP64 sums of
//                 (x_{i-1}-x_{i-2})^2 and x_{i-1}^2, last-block reduction) fused with the
//                 z/u update and the divergence (reads x0, y, u; writes u', div)
//   X r2c (div) -> Y fwd -> Z fwd * rho*sym(inv_a) * Z inv -> Y inv -> X c2r (y_i)
//
// so the inverse X pass is a plain store.  A device-side state (iteration counter,
// done flag) lets every kernel of a converged solve return immediately, so two
// iterations are captured once as a CUDA graph and replayed without host syncs.
#include "tv_shared.cuh"

#include <algorithm>
#include <cmath>

namespace qsm {

template <typename T>
void tv_admm_impl(qsm_ctx* ctx, const GridDims& d, const double* d_f, const uint8_t* d_mask, const double bdir[3],
                  const qsm_tv_params& p, qsm_progress_fn progress, void* user, double* d_out) {
  const char* pre = sizeof(T) == 4 ? "tv32." : "tv64.";
  TvState* st = ws<TvState>(ctx, std::string(pre) + "state", 1);
  TvVol<T> v;
  tv_setup<T>(ctx, v, pre, d, d_f, d_mask, bdir, p, st, d_out);

  ctx->tv_last_iters = tv_run<T>(ctx, v, p.max_iter, p.tol, progress, user);
}

// Batched TV-ADMM: every volume keeps its own buffers, grid, field direction and
// device state; one CUDA graph holds two iterations of every volume as parallel
// branches on up to 8 streams (volumes placed longest-first on the least-loaded
// stream), so small volumes run side by side and one graph launch advances the whole
// batch.  Converged volumes' kernels return at once.  progress(k, n) reports the
// number of finished volumes.
template <typename T>
void tv_admm_batch_impl(qsm_ctx* ctx, const qsm_volume* vols, size_t n, const qsm_tv_params& p,
                        qsm_progress_fn progress, void* user, size_t* out_iters) {
  const char* pre = sizeof(T) == 4 ? "tvb32." : "tvb64.";
  TvState* states = ws<TvState>(ctx, std::string(pre) + "states", n);
  std::vector<TvVol<T>> V(n);
  for (size_t b = 0; b < n; ++b) {
    const GridDims d = check_grid(&vols[b].grid);
    tv_setup<T>(ctx, V[b], std::string(pre) + std::to_string(b) + ".", d, vols[b].local_field, vols[b].mask,
                vols[b].bdir, p, states + b, vols[b].out_chi);
  }
  // longest-processing-time placement on K branch streams (cost ~ N log N)
  const int K = (int)std::min<size_t>(n, 8);
  std::vector<size_t> order(n);
  for (size_t b = 0; b < n; ++b) order[b] = b;
  auto cost = [&](size_t b) { return (double)V[b].d.n * std::log2((double)V[b].d.n + 2.0); };
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return cost(a) > cost(b); });
  std::vector<int> lane(n, 0);
  std::vector<double> load(K, 0.0);
  for (size_t b : order) {
    const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    lane[b] = k;
    load[k] += cost(b);
  }
  std::vector<cudaStream_t> streams(K, nullptr);
  std::vector<cudaEvent_t> joins(K, nullptr);
  cudaEvent_t fork = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t s0 = ctx->stream;
  auto cleanup = [&]() {
    ctx->stream = s0;
    if (exec) cudaGraphExecDestroy(exec);
    for (auto& e : joins)
      if (e) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    for (auto& s : streams)
      if (s) cudaStreamDestroy(s);
  };
  try {
    QSM_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    for (int k = 0; k < K; ++k) {
      QSM_CUDA(cudaStreamCreateWithFlags(&streams[k], cudaStreamNonBlocking));
      QSM_CUDA(cudaEventCreateWithFlags(&joins[k], cudaEventDisableTiming));
    }
    // one step of every volume on its branch stream; `pair` = two iterations
    auto enqueue = [&](bool pair, int q_single) {
      QSM_CUDA(cudaEventRecord(fork, s0));
      for (int k = 0; k < K; ++k) QSM_CUDA(cudaStreamWaitEvent(streams[k], fork, 0));
      for (size_t b : order) {
        ctx->stream = streams[lane[b]];
        if (pair) {
          tv_iter(ctx, V[b], 1);
          tv_iter(ctx, V[b], 0);
        } else {
          tv_iter(ctx, V[b], q_single);
        }
      }
      ctx->stream = s0;
      for (int k = 0; k < K; ++k) {
        QSM_CUDA(cudaEventRecord(joins[k], streams[k]));
        QSM_CUDA(cudaStreamWaitEvent(s0, joins[k], 0));
      }
    };
    const size_t max_iter = p.max_iter;
    std::vector<TvState> hs(n);
    size_t finished = 0;
    auto poll = [&]() {
      QSM_CUDA(cudaMemcpyAsync(hs.data(), states, sizeof(TvState) * n, cudaMemcpyDeviceToHost, s0));
      QSM_CUDA(cudaStreamSynchronize(s0));
      size_t f = 0;
      for (size_t b = 0; b < n; ++b) f += hs[b].done != 0;
      if (progress)
        for (; finished < f; ++finished) progress(user, finished + 1, n);
      return f == n;
    };
    bool all_done = false;
    const size_t pairs = max_iter / 2;
    if (pairs > 0 && ctx->profiling) {
      // eager launches for per-kernel timing
      for (size_t it = 0; it < pairs && !all_done; ++it) {
        enqueue(true, 0);
        if (p.tol > 0.0 && (it + 1) % 8 == 0) all_done = poll();
      }
    } else if (pairs > 0) {
      cudaGraph_t graph = nullptr;
      const uint64_t l0 = ctx->launches;
      QSM_CUDA(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
      try {
        enqueue(true, 0);
      } catch (...) {
        ctx->stream = s0;
        cudaStreamEndCapture(s0, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
      }
      QSM_CUDA(cudaStreamEndCapture(s0, &graph));
      const uint64_t per = ctx->launches - l0;
      ctx->launches = l0;
      exec = instantiate(ctx, graph);
      const bool watch = p.tol > 0.0;
      size_t launched = 0;
      while (launched < pairs && !all_done) {
        const size_t todo = watch ? std::min<size_t>(8, pairs - launched) : (pairs - launched);
        for (size_t c = 0; c < todo; ++c) {
          QSM_CUDA(cudaGraphLaunch(exec, s0));
          ctx->launches += per;
        }
        launched += todo;
        if (watch) all_done = poll();
      }
    }
    if (!all_done && (max_iter % 2 == 1)) enqueue(false, 1);
    all_done = poll();
    for (size_t b = 0; b < n; ++b) {
      size_t completed = hs[b].done ? (size_t)hs[b].conv_iter : max_iter;
      if (!hs[b].done && max_iter >= 1 && p.tol > 0.0) {
        tv_step_launch(ctx, V[b], (int)((max_iter + 1) % 2), 1);  // last-iterate test (tv.rs:85-91)
        completed = max_iter;
      }
      tv_out_launch(ctx, V[b], completed);
      if (out_iters) out_iters[b] = completed;
    }
    poll();
    if (progress)
      for (; finished < n; ++finished) progress(user, finished + 1, n);
  } catch (...) {
    cleanup();
    throw;
  }
  cleanup();
}

void tv_batch_device(qsm_ctx* ctx, const qsm_volume* vols, size_t n, const qsm_tv_params* p,
                     qsm_progress_fn progress, void* user, size_t* out_iters) {
  check_ptr(p, "params");
  check_finite(p->lambda, "lambda");
  check_finite(p->rho, "rho");
  if (std::isnan(p->tol)) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "tol is NaN");
  if (n == 0) return;
  check_ptr(vols, "volumes");
  for (size_t b = 0; b < n; ++b) {
    check_grid(&vols[b].grid);
    check_ptr(vols[b].local_field, "local_field");
    check_ptr(vols[b].mask, "mask");
    check_ptr(vols[b].out_chi, "out_chi");
    check_bdir(vols[b].bdir);
  }
  for (size_t b = 0; b < n; ++b) check_volume_finite(ctx, vols[b].local_field, check_grid(&vols[b].grid).n, "local_field");
  if (ctx->precision == QSM_PRECISION_MIXED) tv_admm_batch_impl<float>(ctx, vols, n, *p, progress, user, out_iters);
  else tv_admm_batch_impl<double>(ctx, vols, n, *p, progress, user, out_iters);
  sync(ctx);
}

void tv_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
               const qsm_tv_params* p, qsm_progress_fn progress, void* user, double* out) {
  GridDims d = check_grid(grid);
  check_ptr(f, "local_field");
  check_ptr(m, "mask");
  check_ptr(out, "out");
  check_ptr(p, "params");
  check_bdir(bdir);
  check_volume_finite(ctx, f, d.n, "local_field");
  check_finite(p->lambda, "lambda");
  check_finite(p->rho, "rho");
  if (std::isnan(p->tol)) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "tol is NaN");
  if (ctx->precision == QSM_PRECISION_MIXED) tv_admm_impl<float>(ctx, d, f, m, bdir, *p, progress, user, out);
  else tv_admm_impl<double>(ctx, d, f, m, bdir, *p, progress, user, out);
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
    with_host_io(ctx, d.n, local_field, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
      tv_device(ctx, f, m, grid, bdir, params, progress, user, o);
    });
  });
}

size_t qsm_tv_last_iterations(const qsm_ctx* ctx) { return ctx ? ctx->tv_last_iters : 0; }

qsm_status qsm_tv_admm_batch_device(qsm_ctx* ctx, const qsm_volume* vols, size_t n, const qsm_tv_params* params,
                                    qsm_progress_fn progress, void* user, size_t* out_iterations) {
  return guarded(ctx, [&] { tv_batch_device(ctx, vols, n, params, progress, user, out_iterations); });
}

qsm_status qsm_tv_admm_batch(qsm_ctx* ctx, const qsm_volume* vols, size_t n, const qsm_tv_params* params,
                             qsm_progress_fn progress, void* user, size_t* out_iterations) {
  return guarded(ctx, [&] {
    if (n == 0) return;
    check_ptr(vols, "volumes");
    // stage every volume on the device, solve the batch, copy every result back
    std::vector<qsm_volume> dv(vols, vols + n);
    for (size_t b = 0; b < n; ++b) {
      const GridDims d = check_grid(&vols[b].grid);
      check_ptr(vols[b].local_field, "local_field");
      check_ptr(vols[b].mask, "mask");
      check_ptr(vols[b].out_chi, "out_chi");
      const std::string k = "iob." + std::to_string(b) + ".";
      double* f = ws<double>(ctx, k + "in", (size_t)d.n);
      uint8_t* m = ws<uint8_t>(ctx, k + "mask", (size_t)d.n);
      double* o = ws<double>(ctx, k + "out", (size_t)d.n);
      h2d(ctx, f, vols[b].local_field, sizeof(double) * d.n);
      h2d(ctx, m, vols[b].mask, (size_t)d.n);
      dv[b].local_field = f;
      dv[b].mask = m;
      dv[b].out_chi = o;
    }
    tv_batch_device(ctx, dv.data(), n, params, progress, user, out_iterations);
    for (size_t b = 0; b < n; ++b) {
      const GridDims d = check_grid(&vols[b].grid);
      d2h(ctx, vols[b].out_chi, dv[b].out_chi, sizeof(double) * d.n);
    }
    sync(ctx);
  });
}

}  // extern "C"
