// Multi-echo field mapping on the GPU: the magnitude-weighted B0 average
// (src/utils/multi_echo.rs:450-506) and the magnitude-weighted linear fit with its
// reliability mask (src/utils/multi_echo.rs:631-804).
//
// Both are per-voxel reductions over the echoes, so one thread owns one voxel and
// reads the echo-major inputs (echo e of voxel v at e*n + v) with coalesced loads; the
// kernels are bound by HBM reads of the 2 * n_echoes float64 inputs.  The arithmetic
// is written with explicitly rounded double intrinsics (no fused multiply-add) in the
// reference's evaluation order, so every output is the reference's float64 result bit
// for bit.  The reliability threshold is an exact order statistic of the selected
// residuals (radix selection), which the reference takes from a full sort.
#include "common.cuh"
#include "select.h"
#include "solvers.h"

#include <cmath>

namespace qsm {

namespace {

constexpr int kMaxEchoes = 64;

struct EchoTimes {
  double te[kMaxEchoes];
};

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

// B0 (Hz) = (1/2pi) sum (phase/TE) w / sum w over the mask; 0 where sum w <= 1e-10
template <int WT>
__global__ void k_b0_weighted(long long n, int ne, const double* __restrict__ ph, const double* __restrict__ mg,
                              const __grid_constant__ EchoTimes tes, const uint8_t* __restrict__ mask,
                              double scale, double* __restrict__ out) {
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
    double r = 0.0;
    if (mask[v] != 0) {
      double ws = 0.0, wsum = 0.0;
      for (int e = 0; e < ne; ++e) {
        const double te = tes.te[e];
        const double p = dvd(ph[(long long)e * n + v], te);
        double w;
        if (WT == QSM_B0W_PHASE_SNR) w = mul(mg[(long long)e * n + v], te);
        else if (WT == QSM_B0W_PHASE_VAR) {
          const double m = mg[(long long)e * n + v];
          w = mul(mul(mul(m, m), te), te);
        } else if (WT == QSM_B0W_AVERAGE) w = 1.0;
        else if (WT == QSM_B0W_TES) w = te;
        else w = mg[(long long)e * n + v];
        ws = add(ws, mul(p, w));
        wsum = add(wsum, w);
      }
      if (wsum > 1e-10) r = dvd(mul(scale, ws), wsum);
    }
    out[v] = r;
  }
}

// Weighted fit per voxel; sel marks the residuals the reliability percentile ranks
// (mask > 0, r > 0, finite: multi_echo.rs:777-781).
__global__ void k_linear_fit(long long n, int ne, const double* __restrict__ ph, const double* __restrict__ mg,
                             const __grid_constant__ EchoTimes tes, const uint8_t* __restrict__ mask, int offset,
                             double* __restrict__ field, double* __restrict__ phase_offset,
                             double* __restrict__ resid, uint8_t* __restrict__ sel) {
  const double nef = (double)ne;
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
    double fv = 0.0, ov = 0.0, rv = 0.0;
    if (mask[v] != 0) {
      if (offset) {
        // centred weighted regression, multi_echo.rs:656-712
        double sw = 0.0, swt = 0.0, swp = 0.0;
        for (int e = 0; e < ne; ++e) {
          const double w = mg[(long long)e * n + v];
          sw = add(sw, w);
          swt = add(swt, mul(w, tes.te[e]));
          swp = add(swp, mul(w, ph[(long long)e * n + v]));
        }
        if (!(sw < 1e-10)) {
          const double te_mean = dvd(swt, sw), ph_mean = dvd(swp, sw);
          double sxx = 0.0, sxy = 0.0;
          for (int e = 0; e < ne; ++e) {
            const double w = mg[(long long)e * n + v];
            const double tc = sub(tes.te[e], te_mean);
            const double pc = sub(ph[(long long)e * n + v], ph_mean);
            sxx = add(sxx, mul(mul(w, tc), tc));
            sxy = add(sxy, mul(mul(w, tc), pc));
          }
          if (sxx > 1e-10) {
            const double slope = dvd(sxy, sxx);
            const double icpt = sub(ph_mean, mul(slope, te_mean));
            double srr = 0.0;
            for (int e = 0; e < ne; ++e) {
              const double w = mg[(long long)e * n + v];
              const double d = sub(ph[(long long)e * n + v], add(icpt, mul(slope, tes.te[e])));
              srr = add(srr, mul(mul(w, d), d));
            }
            fv = slope;
            ov = icpt;
            rv = mul(dvd(srr, sw), nef);
          }
        }
      } else {
        // through the origin, multi_echo.rs:713-752
        double stp = 0.0, stt = 0.0, sw = 0.0;
        for (int e = 0; e < ne; ++e) {
          const double w = mg[(long long)e * n + v];
          const double te = tes.te[e];
          stp = add(stp, mul(mul(w, te), ph[(long long)e * n + v]));
          stt = add(stt, mul(mul(w, te), te));
          sw = add(sw, w);
        }
        if (stt > 1e-10) {
          const double slope = dvd(stp, stt);
          fv = slope;
          double srr = 0.0;
          for (int e = 0; e < ne; ++e) {
            const double w = mg[(long long)e * n + v];
            const double d = sub(ph[(long long)e * n + v], mul(slope, tes.te[e]));
            srr = add(srr, mul(mul(w, d), d));
          }
          if (sw > 1e-10) rv = mul(dvd(srr, sw), nef);
        }
      }
    }
    field[v] = fv;
    phase_offset[v] = ov;
    resid[v] = rv;
    sel[v] = (mask[v] > 0 && rv > 0.0 && isfinite(rv)) ? 1 : 0;
  }
}

__global__ void k_reliability(long long n, const uint8_t* __restrict__ mask, const double* __restrict__ resid,
                              double thr, uint8_t* __restrict__ out) {
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
    out[v] = (mask[v] > 0 && resid[v] < thr) ? 1 : 0;
}

EchoTimes echo_times(const double* tes, size_t ne) {
  if (ne == 0) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "no echoes");
  if (ne > (size_t)kMaxEchoes) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "more than 64 echoes");
  check_ptr(tes, "tes");
  EchoTimes t{};
  for (size_t e = 0; e < ne; ++e) t.te[e] = tes[e];
  return t;
}

void check_n(size_t n) {
  if (n == 0) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "no voxels");
  if (n > (size_t)1 << 40) throw QsmError(QSM_ERR_UNSUPPORTED_SIZE, "too many voxels");
}

}  // namespace

void b0_weighted_device(qsm_ctx* ctx, const double* ph, const double* mg, const double* tes, size_t ne,
                        const uint8_t* mask, size_t n, int weight_type, double* out) {
  const EchoTimes t = echo_times(tes, ne);
  check_n(n);
  check_ptr(ph, "phases");
  check_ptr(mg, "mags");
  check_ptr(mask, "mask");
  check_ptr(out, "out");
  const long long N = (long long)n;
  const double scale = 1.0 / (2.0 * kPi);  // multi_echo.rs:465
  LaunchScope ls(ctx, "b0_weighted");
  const unsigned g = grid1d(N);
  switch (weight_type) {
    case QSM_B0W_PHASE_SNR:
      k_b0_weighted<QSM_B0W_PHASE_SNR><<<g, 256, 0, ctx->stream>>>(N, (int)ne, ph, mg, t, mask, scale, out);
      break;
    case QSM_B0W_PHASE_VAR:
      k_b0_weighted<QSM_B0W_PHASE_VAR><<<g, 256, 0, ctx->stream>>>(N, (int)ne, ph, mg, t, mask, scale, out);
      break;
    case QSM_B0W_AVERAGE:
      k_b0_weighted<QSM_B0W_AVERAGE><<<g, 256, 0, ctx->stream>>>(N, (int)ne, ph, mg, t, mask, scale, out);
      break;
    case QSM_B0W_TES:
      k_b0_weighted<QSM_B0W_TES><<<g, 256, 0, ctx->stream>>>(N, (int)ne, ph, mg, t, mask, scale, out);
      break;
    case QSM_B0W_MAG:
      k_b0_weighted<QSM_B0W_MAG><<<g, 256, 0, ctx->stream>>>(N, (int)ne, ph, mg, t, mask, scale, out);
      break;
    default:
      throw QsmError(QSM_ERR_INVALID_ARGUMENT, "unknown B0 weight type " + std::to_string(weight_type));
  }
  ls.done();
}

void linear_fit_device(qsm_ctx* ctx, const double* ph, const double* mg, const double* tes, size_t ne,
                       const uint8_t* mask, size_t n, const qsm_linear_fit_params* p, double* field,
                       double* phase_offset, double* resid, uint8_t* reliability) {
  const EchoTimes t = echo_times(tes, ne);
  check_n(n);
  check_ptr(ph, "phases");
  check_ptr(mg, "mags");
  check_ptr(mask, "mask");
  check_ptr(p, "params");
  check_ptr(field, "out_field");
  check_ptr(phase_offset, "out_phase_offset");
  check_ptr(resid, "out_fit_residual");
  check_ptr(reliability, "out_reliability");
  if (std::isnan(p->reliability_threshold_percentile))
    throw QsmError(QSM_ERR_INVALID_ARGUMENT, "reliability_threshold_percentile is NaN");
  const long long N = (long long)n;
  uint8_t* sel = ws<uint8_t>(ctx, "fit.sel", n);
  {
    LaunchScope ls(ctx, "linear_fit");
    k_linear_fit<<<grid1d(N), 256, 0, ctx->stream>>>(N, (int)ne, ph, mg, t, mask, p->estimate_offset ? 1 : 0, field,
                                                     phase_offset, resid, sel);
    ls.done();
  }
  const double pct = p->reliability_threshold_percentile;
  long long count = 0;
  if (pct > 0.0) count = count_selected(ctx, sel, N);
  if (!(pct > 0.0) || count == 0) {  // the mask itself (multi_echo.rs:760-763, 783-785)
    QSM_CUDA(cudaMemcpyAsync(reliability, mask, n, cudaMemcpyDeviceToDevice, ctx->stream));
    return;
  }
  // index (p/100 * count) truncated, clamped to count - 1 (multi_echo.rs:789-790)
  long long idx = (long long)((pct / 100.0) * (double)count);
  if (idx > count - 1) idx = count - 1;
  const double thr = select_ranks(ctx, resid, sel, N, {idx})[0];
  LaunchScope ls(ctx, "reliability");
  k_reliability<<<grid1d(N), 256, 0, ctx->stream>>>(N, mask, resid, thr, reliability);
  ls.done();
}

}  // namespace qsm

using namespace qsm;

extern "C" {

void qsm_linear_fit_params_default(qsm_linear_fit_params* p) {
  if (!p) return;
  // LinearFitParams::default, src/utils/multi_echo.rs:41-48
  p->estimate_offset = 1;
  p->reliability_threshold_percentile = 90.0;
}

qsm_status qsm_calculate_b0_weighted_device(qsm_ctx* ctx, const double* d_phases, const double* d_mags,
                                            const double* tes, size_t n_echoes, const uint8_t* d_mask, size_t n,
                                            int weight_type, double* d_out_b0_hz) {
  return guarded(ctx, [&] {
    b0_weighted_device(ctx, d_phases, d_mags, tes, n_echoes, d_mask, n, weight_type, d_out_b0_hz);
    sync(ctx);
  });
}

qsm_status qsm_calculate_b0_weighted(qsm_ctx* ctx, const double* phases, const double* mags, const double* tes,
                                     size_t n_echoes, const uint8_t* mask, size_t n, int weight_type,
                                     double* out_b0_hz) {
  return guarded(ctx, [&] {
    check_n(n);
    check_ptr(phases, "phases");
    check_ptr(mags, "mags");
    check_ptr(mask, "mask");
    check_ptr(out_b0_hz, "out_b0_hz");
    const size_t ne = n_echoes;
    (void)echo_times(tes, ne);
    double* dph = ws<double>(ctx, "fit.ph", ne * n);
    double* dmg = ws<double>(ctx, "fit.mg", ne * n);
    uint8_t* dm = ws<uint8_t>(ctx, "fit.mask", n);
    double* dout = ws<double>(ctx, "fit.out0", n);
    h2d(ctx, dph, phases, ne * n * sizeof(double));
    h2d(ctx, dmg, mags, ne * n * sizeof(double));
    h2d(ctx, dm, mask, n);
    b0_weighted_device(ctx, dph, dmg, tes, ne, dm, n, weight_type, dout);
    d2h(ctx, out_b0_hz, dout, n * sizeof(double));
    sync(ctx);
  });
}

qsm_status qsm_multi_echo_linear_fit_device(qsm_ctx* ctx, const double* d_phases, const double* d_mags,
                                            const double* tes, size_t n_echoes, const uint8_t* d_mask, size_t n,
                                            const qsm_linear_fit_params* params, double* d_out_field,
                                            double* d_out_phase_offset, double* d_out_fit_residual,
                                            uint8_t* d_out_reliability) {
  return guarded(ctx, [&] {
    linear_fit_device(ctx, d_phases, d_mags, tes, n_echoes, d_mask, n, params, d_out_field, d_out_phase_offset,
                      d_out_fit_residual, d_out_reliability);
    sync(ctx);
  });
}

qsm_status qsm_multi_echo_linear_fit(qsm_ctx* ctx, const double* phases, const double* mags, const double* tes,
                                     size_t n_echoes, const uint8_t* mask, size_t n,
                                     const qsm_linear_fit_params* params, double* out_field,
                                     double* out_phase_offset, double* out_fit_residual, uint8_t* out_reliability) {
  return guarded(ctx, [&] {
    check_n(n);
    check_ptr(phases, "phases");
    check_ptr(mags, "mags");
    check_ptr(mask, "mask");
    check_ptr(out_field, "out_field");
    check_ptr(out_phase_offset, "out_phase_offset");
    check_ptr(out_fit_residual, "out_fit_residual");
    check_ptr(out_reliability, "out_reliability");
    const size_t ne = n_echoes;
    (void)echo_times(tes, ne);
    double* dph = ws<double>(ctx, "fit.ph", ne * n);
    double* dmg = ws<double>(ctx, "fit.mg", ne * n);
    uint8_t* dm = ws<uint8_t>(ctx, "fit.mask", n);
    double* df = ws<double>(ctx, "fit.out0", n);
    double* dof = ws<double>(ctx, "fit.out1", n);
    double* dr = ws<double>(ctx, "fit.out2", n);
    uint8_t* drel = ws<uint8_t>(ctx, "fit.rel", n);
    h2d(ctx, dph, phases, ne * n * sizeof(double));
    h2d(ctx, dmg, mags, ne * n * sizeof(double));
    h2d(ctx, dm, mask, n);
    linear_fit_device(ctx, dph, dmg, tes, ne, dm, n, params, df, dof, dr, drel);
    d2h(ctx, out_field, df, n * sizeof(double));
    d2h(ctx, out_phase_offset, dof, n * sizeof(double));
    d2h(ctx, out_fit_residual, dr, n * sizeof(double));
    d2h(ctx, out_reliability, drel, n);
    sync(ctx);
  });
}

}  // extern "C"
