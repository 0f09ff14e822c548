// Closed-form dipole inversion on the GPU: TKD, TSVD, Tikhonov and the forward dipole
// model, plus the pipeline dispatcher run_dipole_inversion.
//
// Each method is one five-pass transform chain with its k-space multiplier
// evaluated in the fused z pass:
//   X r2c (f64 field -> working precision) -> Y fwd -> Z fwd*M*inv -> Y inv
//   -> X c2r (1/N, mask, write f64).
// Multipliers with thresholds are evaluated in double in both precisions, so the
// truncation decisions are the reference's.
#include "closed_form_ops.cuh"
#include "functors.cuh"
#include "solvers.h"

#include <algorithm>
#include <cstring>

namespace qsm {

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
  check_volume_finite(ctx, f, d.n, "local_field");
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
  check_volume_finite(ctx, f, d.n, "local_field");
  KSpace K = make_kspace(ctx, d, bdir);
  closed_form(ctx, d, f, m, OpTikhonov<float>{K, p->lambda, p->reg}, OpTikhonov<double>{K, p->lambda, p->reg}, out);
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

qsm_status qsm_tkd_device(qsm_ctx* ctx, const double* f, const uint8_t* m, const qsm_grid* grid, const double bdir[3],
                          const qsm_tkd_params* p, double* out) {
  return guarded(ctx, [&] {
    tkd_device(ctx, f, m, grid, bdir, p, out, 0);
    sync(ctx);
  });
}
qsm_status qsm_tkd_batch_device(qsm_ctx* ctx, const qsm_volume* vols, size_t n, const qsm_tkd_params* p) {
  return guarded(ctx, [&] {
    if (n == 0) return;
    check_ptr(vols, "volumes");
    for (size_t b = 0; b < n; ++b) {
      // volumes share the transform workspaces: the previous volume's pointers are dead
      // here, so the buffers may be regrown
      ctx->epoch++;
      tkd_device(ctx, vols[b].local_field, vols[b].mask, &vols[b].grid, vols[b].bdir, p, vols[b].out_chi, 0);
    }
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
    with_host_io(ctx, d.n, f, m, out, [&](const double* df, const uint8_t* dm, double* o) {
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
    with_host_io(ctx, d.n, f, m, out, [&](const double* df, const uint8_t* dm, double* o) {
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
    with_host_io(ctx, d.n, f, m, out, [&](const double* df, const uint8_t* dm, double* o) {
      tikhonov_device(ctx, df, dm, grid, bdir, p, o);
    });
  });
}

qsm_status qsm_dipole_forward_device(qsm_ctx* ctx, const double* d_chi, const qsm_grid* grid, const double bdir[3],
                                     double* d_out_field) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_ptr(d_chi, "chi");
    check_ptr(d_out_field, "out_field");
    check_bdir(bdir);
    KSpace K = make_kspace(ctx, d, bdir);
    closed_form(ctx, d, d_chi, nullptr, OpDipole<float>{K}, OpDipole<double>{K}, d_out_field);
    sync(ctx);
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
    with_host_io(ctx, d.n, chi, nullptr, out_field, [&](const double* df, const uint8_t*, double* o) {
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
  qsm_ilsqr_params_default(&c->ilsqr);
  qsm_rts_params_default(&c->rts);
  qsm_nltv_params_default(&c->nltv);
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
        with_host_io(ctx, d.n, local_field_ppm, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
          tkd_device(ctx, f, m, &g, b, &cfg->tkd, o, 0);
        });
        break;
      case QSM_INV_TSVD:
        with_host_io(ctx, d.n, local_field_ppm, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
          tkd_device(ctx, f, m, &g, b, &cfg->tsvd, o, 1);
        });
        break;
      case QSM_INV_TIKHONOV:
        with_host_io(ctx, d.n, local_field_ppm, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
          tikhonov_device(ctx, f, m, &g, b, &cfg->tikhonov, o);
        });
        break;
      case QSM_INV_TV:
        with_host_io(ctx, d.n, local_field_ppm, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
          tv_device(ctx, f, m, &g, b, &cfg->tv, progress, user, o);
        });
        break;
      case QSM_INV_RTS:
        with_host_io(ctx, d.n, local_field_ppm, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
          rts_device(ctx, f, m, &g, b, &cfg->rts, progress, user, o);
        });
        break;
      case QSM_INV_NLTV:
        with_host_io(ctx, d.n, local_field_ppm, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
          nltv_device(ctx, f, m, &g, b, &cfg->nltv, progress, user, o);
        });
        break;
      case QSM_INV_ILSQR:  // src/pipeline/inversion.rs:100-105: chi of the 4-tuple
        with_host_io(ctx, d.n, local_field_ppm, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
          ilsqr_device(ctx, f, m, &g, b, &cfg->ilsqr, progress, user, o, nullptr, nullptr, nullptr);
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
