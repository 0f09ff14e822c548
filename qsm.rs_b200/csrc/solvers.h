// Device-pointer solver entry points shared between translation units (the C ABI
// wrappers and the pipeline dispatchers call these).
#pragma once

#include "internal.h"

namespace qsm {

void check_bdir(const double bdir[3]);

// All pointers are device pointers on ctx's GPU; work is enqueued on ctx->stream.
void tv_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
               const qsm_tv_params* p, qsm_progress_fn progress, void* user, double* out);
void tkd_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                const qsm_tkd_params* p, double* out, int tsvd);
void tikhonov_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                     const qsm_tikhonov_params* p, double* out);
// xsa, xfs, xlsqr may be null
void ilsqr_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                  const qsm_ilsqr_params* p, qsm_progress_fn progress, void* user, double* chi, double* xsa,
                  double* xfs, double* xlsqr);
void resharp_device(qsm_ctx* ctx, const double* field, const uint8_t* mask, const GridDims& d,
                    const qsm_resharp_params* p, qsm_progress_fn progress, void* user, double* out_local,
                    uint8_t* out_mask);
void apply_reference_device(qsm_ctx* ctx, long long N, const double* chi, const uint8_t* mask, int method,
                            double* out);
void rts_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                const qsm_rts_params* p, qsm_progress_fn progress, void* user, double* out);
void nltv_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                 const qsm_nltv_params* p, qsm_progress_fn progress, void* user, double* out);
void tgv_device(qsm_ctx* ctx, const double* phase, const uint8_t* mask, const qsm_grid* grid, const qsm_tgv_params* p,
                const double b0[3], qsm_progress_fn progress, void* user, double* out);

// Stage a host volume (and optional mask) on the device, run, copy the result back.
template <class Run>
void with_host_io(qsm_ctx* ctx, long long n, const double* h_in, const uint8_t* h_mask, double* h_out, Run run) {
  const size_t N = (size_t)n;
  double* din = reinterpret_cast<double*>(ws_get(ctx, "io.in", N * sizeof(double)));
  uint8_t* dm = h_mask ? reinterpret_cast<uint8_t*>(ws_get(ctx, "io.mask", N)) : nullptr;
  double* dout = reinterpret_cast<double*>(ws_get(ctx, "io.out", N * sizeof(double)));
  h2d(ctx, din, h_in, N * sizeof(double));
  if (h_mask) h2d(ctx, dm, h_mask, N);
  run(din, dm, dout);
  d2h(ctx, h_out, dout, N * sizeof(double));
  sync(ctx);
}

inline unsigned grid1d(long long n, int block = 256) {
  long long b = (n + block - 1) / block;
  const long long cap = 148LL * 16;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

}  // namespace qsm
