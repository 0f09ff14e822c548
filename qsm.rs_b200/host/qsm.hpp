// qsm.hpp — C++ host mirror of QSM.rs's reconstruction API over the qsmgpu C ABI.
//
// The reference crate (astewartau/QSM.rs) exposes free functions taking borrowed
// slices and returning owned vectors; this header keeps those names, argument order,
// defaults and error behaviour:
//   * algorithm functions (inversion::tv_admm, tkd, tsvd, tikhonov, ilsqr, rts, nltv,
//     tgv_qsm, unwrap::laplacian_unwrap, bgremove::smv/sharp/vsharp/resharp/ismv,
//     multi_echo::*) throw qsm::Panic where the
//     Rust code would panic (length mismatch) or where the GPU call fails;
//   * pipeline functions (pipeline::run_dipole_inversion, run_bg_removal, run_tgv) return
//     a Result carrying PipelineError {DimensionMismatch, InvalidConfig, AlgorithmError};
//   * io functions (load_nifti, save_nifti, read_nifti_file, ...) return a Result with a
//     String error, as src/io.rs does.
//
// Header-only; link with libqsmgpu.so.  One Session (a qsm_ctx) per thread.
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <variant>
#include <vector>

#include "../../include/qsmgpu.h"

namespace qsm {

using Progress = std::function<void(size_t, size_t)>;

// src/grid.rs:9-44
struct Grid {
  std::tuple<size_t, size_t, size_t> dims;
  std::tuple<double, double, double> voxel_size{1.0, 1.0, 1.0};
  static Grid make(size_t nx, size_t ny, size_t nz, double vsx = 1, double vsy = 1, double vsz = 1) {
    return Grid{{nx, ny, nz}, {vsx, vsy, vsz}};
  }
  size_t nx() const { return std::get<0>(dims); }
  size_t ny() const { return std::get<1>(dims); }
  size_t nz() const { return std::get<2>(dims); }
  size_t n_total() const { return nx() * ny() * nz(); }
  qsm_grid c() const {
    return qsm_grid{nx(), ny(), nz(), std::get<0>(voxel_size), std::get<1>(voxel_size), std::get<2>(voxel_size)};
  }
};

using BDir = std::tuple<double, double, double>;

struct Panic : std::runtime_error {
  int status;
  Panic(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

// A GPU session: owns one qsm_ctx (device, stream, precision, workspaces).
class Session {
 public:
  explicit Session(int device = 0, qsm_precision precision = QSM_PRECISION_F64) {
    qsm_ctx* c = nullptr;
    int st = qsm_ctx_create(device, precision, &c);
    if (st != QSM_OK) throw Panic(st, "qsm_ctx_create failed");
    ctx_.reset(c);
  }
  qsm_ctx* get() const { return ctx_.get(); }
  void check(int st) const {
    if (st != QSM_OK) throw Panic(st, qsm_last_error(ctx_.get()));
  }
  static Session& default_session() {
    thread_local Session s;
    return s;
  }

 private:
  struct Del {
    void operator()(qsm_ctx* c) const { qsm_ctx_destroy(c); }
  };
  std::unique_ptr<qsm_ctx, Del> ctx_;
};

namespace detail {
inline void require_len(size_t got, const Grid& g, const char* what) {
  if (got != g.n_total())
    throw Panic(QSM_ERR_DIMENSION_MISMATCH, std::string(what) + ": index out of bounds (length " +
                                                std::to_string(got) + ", grid " + std::to_string(g.n_total()) + ")");
}
struct ProgressThunk {
  const Progress* p;
  static void call(void* user, size_t cur, size_t max) {
    auto* self = static_cast<ProgressThunk*>(user);
    if (self->p && *self->p) (*self->p)(cur, max);
  }
};
inline void bdir3(const BDir& b, double out[3]) {
  out[0] = std::get<0>(b);
  out[1] = std::get<1>(b);
  out[2] = std::get<2>(b);
}
}  // namespace detail

// ----------------------------------------------------------------- inversion --
namespace inversion {

// src/inversion/tv.rs:23-43
struct TvParams {
  double lambda = 2e-4;
  double rho = 2e-2;
  double tol = 1e-3;
  size_t max_iter = 250;
};
// src/inversion/tkd.rs:23-32
struct TkdParams {
  double threshold = 0.15;
};
// src/inversion/tikhonov.rs:26-49
enum class Regularization { Identity = 0, Gradient = 1, Laplacian = 2 };
struct TikhonovParams {
  double lambda = 0.01;
  Regularization reg = Regularization::Identity;
};

// src/inversion/tv.rs:63-97
inline std::vector<double> tv_admm(const std::vector<double>& local_field, const std::vector<uint8_t>& mask,
                                   const Grid& grid, BDir bdir, const TvParams& params,
                                   Progress progress = nullptr, Session& s = Session::default_session()) {
  detail::require_len(local_field.size(), grid, "local_field");
  detail::require_len(mask.size(), grid, "mask");
  std::vector<double> out(grid.n_total());
  qsm_grid g = grid.c();
  double b[3];
  detail::bdir3(bdir, b);
  qsm_tv_params p{params.lambda, params.rho, params.tol, params.max_iter};
  detail::ProgressThunk th{&progress};
  s.check(qsm_tv_admm(s.get(), local_field.data(), mask.data(), &g, b, &p,
                      progress ? &detail::ProgressThunk::call : nullptr, &th, out.data()));
  return out;
}

inline std::vector<double> tkd(const std::vector<double>& local_field, const std::vector<uint8_t>& mask,
                               const Grid& grid, BDir bdir, const TkdParams& params,
                               Session& s = Session::default_session()) {
  detail::require_len(local_field.size(), grid, "local_field");
  detail::require_len(mask.size(), grid, "mask");
  std::vector<double> out(grid.n_total());
  qsm_grid g = grid.c();
  double b[3];
  detail::bdir3(bdir, b);
  qsm_tkd_params p{params.threshold};
  s.check(qsm_tkd(s.get(), local_field.data(), mask.data(), &g, b, &p, out.data()));
  return out;
}

inline std::vector<double> tsvd(const std::vector<double>& local_field, const std::vector<uint8_t>& mask,
                                const Grid& grid, BDir bdir, const TkdParams& params,
                                Session& s = Session::default_session()) {
  detail::require_len(local_field.size(), grid, "local_field");
  detail::require_len(mask.size(), grid, "mask");
  std::vector<double> out(grid.n_total());
  qsm_grid g = grid.c();
  double b[3];
  detail::bdir3(bdir, b);
  qsm_tkd_params p{params.threshold};
  s.check(qsm_tsvd(s.get(), local_field.data(), mask.data(), &g, b, &p, out.data()));
  return out;
}

inline std::vector<double> tikhonov(const std::vector<double>& local_field, const std::vector<uint8_t>& mask,
                                    const Grid& grid, BDir bdir, const TikhonovParams& params,
                                    Session& s = Session::default_session()) {
  detail::require_len(local_field.size(), grid, "local_field");
  detail::require_len(mask.size(), grid, "mask");
  std::vector<double> out(grid.n_total());
  qsm_grid g = grid.c();
  double b[3];
  detail::bdir3(bdir, b);
  qsm_tikhonov_params p{params.lambda, (int)params.reg};
  s.check(qsm_tikhonov(s.get(), local_field.data(), mask.data(), &g, b, &p, out.data()));
  return out;
}

// src/inversion/ilsqr.rs:20-34
struct IlsqrParams {
  double tol = 0.01;
  size_t max_iter = 50;
};
// src/inversion/rts.rs:22-51
struct RtsParams {
  double delta = 0.15;
  double mu = 1e5;
  double rho = 10.0;
  double tol = 1e-2;
  size_t max_iter = 20;
  size_t lsmr_iter = 4;
};
// src/inversion/nltv.rs:24-48
struct NltvParams {
  double lambda = 1e-3;
  double mu = 1.0;
  double tol = 1e-3;
  size_t max_iter = 250;
  size_t newton_iter = 10;
};
// src/inversion/tgv.rs:39-76
struct TgvParams {
  float alpha1 = 0.0005f;
  float alpha0 = 0.0015f;
  size_t iterations = 1000;
  size_t erosions = 3;
  float step_size = 3.0f;
  float fieldstrength = 3.0f;
  float te = 0.020f;
  float tol = 1e-5f;
  qsm_tgv_params c() const {
    return qsm_tgv_params{alpha1, alpha0, iterations, erosions, step_size, fieldstrength, te, tol};
  }
};

// src/inversion/ilsqr.rs:1307-1351: (chi, xsa, xfs, xlsqr)
inline std::tuple<std::vector<double>, std::vector<double>, std::vector<double>, std::vector<double>> ilsqr(
    const std::vector<double>& local_field, const std::vector<uint8_t>& mask, const Grid& grid, BDir bdir,
    const IlsqrParams& params, Progress progress = nullptr, Session& s = Session::default_session()) {
  detail::require_len(local_field.size(), grid, "local_field");
  detail::require_len(mask.size(), grid, "mask");
  const size_t n = grid.n_total();
  std::vector<double> chi(n), xsa(n), xfs(n), xl(n);
  qsm_grid g = grid.c();
  double b[3];
  detail::bdir3(bdir, b);
  qsm_ilsqr_params p{params.tol, params.max_iter};
  detail::ProgressThunk th{&progress};
  s.check(qsm_ilsqr(s.get(), local_field.data(), mask.data(), &g, b, &p,
                    progress ? &detail::ProgressThunk::call : nullptr, &th, chi.data(), xsa.data(), xfs.data(),
                    xl.data()));
  return {std::move(chi), std::move(xsa), std::move(xfs), std::move(xl)};
}

// src/inversion/rts.rs:72-211
inline std::vector<double> rts(const std::vector<double>& local_field, const std::vector<uint8_t>& mask,
                               const Grid& grid, BDir bdir, const RtsParams& params, Progress progress = nullptr,
                               Session& s = Session::default_session()) {
  detail::require_len(local_field.size(), grid, "local_field");
  detail::require_len(mask.size(), grid, "mask");
  std::vector<double> out(grid.n_total());
  qsm_grid g = grid.c();
  double b[3];
  detail::bdir3(bdir, b);
  qsm_rts_params p{params.delta, params.mu, params.rho, params.tol, params.max_iter, params.lsmr_iter};
  detail::ProgressThunk th{&progress};
  s.check(qsm_rts(s.get(), local_field.data(), mask.data(), &g, b, &p,
                  progress ? &detail::ProgressThunk::call : nullptr, &th, out.data()));
  return out;
}

// src/inversion/nltv.rs:62-131
inline std::vector<double> nltv(const std::vector<double>& local_field, const std::vector<uint8_t>& mask,
                                const Grid& grid, BDir bdir, const NltvParams& params, Progress progress = nullptr,
                                Session& s = Session::default_session()) {
  detail::require_len(local_field.size(), grid, "local_field");
  detail::require_len(mask.size(), grid, "mask");
  std::vector<double> out(grid.n_total());
  qsm_grid g = grid.c();
  double b[3];
  detail::bdir3(bdir, b);
  qsm_nltv_params p{params.lambda, params.mu, params.tol, params.max_iter, params.newton_iter};
  detail::ProgressThunk th{&progress};
  s.check(qsm_nltv(s.get(), local_field.data(), mask.data(), &g, b, &p,
                   progress ? &detail::ProgressThunk::call : nullptr, &th, out.data()));
  return out;
}

// src/inversion/tgv.rs:1045-1052: parameters come before the field direction
inline std::vector<double> tgv_qsm(const std::vector<double>& phase, const std::vector<uint8_t>& mask,
                                   const Grid& grid, const TgvParams& params, BDir b0_dir,
                                   Progress progress = nullptr, Session& s = Session::default_session()) {
  detail::require_len(phase.size(), grid, "phase");
  detail::require_len(mask.size(), grid, "mask");
  std::vector<double> out(grid.n_total());
  qsm_grid g = grid.c();
  double b[3];
  detail::bdir3(b0_dir, b);
  qsm_tgv_params p = params.c();
  detail::ProgressThunk th{&progress};
  s.check(qsm_tgv_qsm(s.get(), phase.data(), mask.data(), &g, &p, b,
                      progress ? &detail::ProgressThunk::call : nullptr, &th, out.data()));
  return out;
}

}  // namespace inversion

// -------------------------------------------------------------------- unwrap --
namespace unwrap {
// src/unwrap/laplacian.rs:135-161
inline std::vector<double> laplacian_unwrap(const std::vector<double>& phase, const std::vector<uint8_t>& mask,
                                            const Grid& grid, Session& s = Session::default_session()) {
  detail::require_len(phase.size(), grid, "phase");
  detail::require_len(mask.size(), grid, "mask");
  std::vector<double> out(grid.n_total());
  qsm_grid g = grid.c();
  s.check(qsm_laplacian_unwrap(s.get(), phase.data(), mask.data(), &g, out.data()));
  return out;
}
}  // namespace unwrap

// ------------------------------------------------------------------ bgremove --
namespace bgremove {
// src/bgremove/sharp.rs:22-37
struct SharpParams {
  double threshold = 0.05;
  double radius = 6.0;
};
// src/bgremove/vsharp.rs:22-40
struct VsharpParams {
  double threshold = 0.05;
  double max_radius = 12.0;
  double min_radius = 1.0;
};
using FieldAndMask = std::pair<std::vector<double>, std::vector<uint8_t>>;

// src/bgremove/smv.rs:31-59
inline FieldAndMask smv(const std::vector<double>& field, const std::vector<uint8_t>& mask, const Grid& grid,
                        double radius, Session& s = Session::default_session()) {
  detail::require_len(field.size(), grid, "field");
  detail::require_len(mask.size(), grid, "mask");
  FieldAndMask r{std::vector<double>(grid.n_total()), std::vector<uint8_t>(grid.n_total())};
  qsm_grid g = grid.c();
  s.check(qsm_smv(s.get(), field.data(), mask.data(), &g, radius, r.first.data(), r.second.data()));
  return r;
}

// src/bgremove/sharp.rs:51-58
inline FieldAndMask sharp(const std::vector<double>& field, const std::vector<uint8_t>& mask, const Grid& grid,
                          const SharpParams& params, Session& s = Session::default_session()) {
  detail::require_len(field.size(), grid, "field");
  detail::require_len(mask.size(), grid, "mask");
  FieldAndMask r{std::vector<double>(grid.n_total()), std::vector<uint8_t>(grid.n_total())};
  qsm_grid g = grid.c();
  qsm_sharp_params p{params.threshold, params.radius};
  s.check(qsm_sharp(s.get(), field.data(), mask.data(), &g, &p, r.first.data(), r.second.data()));
  return r;
}

// src/bgremove/vsharp.rs:55-63
inline FieldAndMask vsharp(const std::vector<double>& field, const std::vector<uint8_t>& mask, const Grid& grid,
                           const VsharpParams& params, Progress progress = nullptr,
                           Session& s = Session::default_session()) {
  detail::require_len(field.size(), grid, "field");
  detail::require_len(mask.size(), grid, "mask");
  FieldAndMask r{std::vector<double>(grid.n_total()), std::vector<uint8_t>(grid.n_total())};
  qsm_grid g = grid.c();
  qsm_vsharp_params p{params.threshold, params.max_radius, params.min_radius};
  detail::ProgressThunk th{&progress};
  s.check(qsm_vsharp(s.get(), field.data(), mask.data(), &g, &p, progress ? &detail::ProgressThunk::call : nullptr,
                     &th, r.first.data(), r.second.data()));
  return r;
}
// src/bgremove/resharp.rs:22-45
struct ResharpParams {
  double radius = 6.0;
  double tik_reg = 1e-4;
  double tol = 1e-6;
  size_t max_iter = 30;
};
// src/bgremove/ismv.rs:19-35
struct IsmvParams {
  double tol = 1e-6;
  size_t max_iter = 50;
  double radius = 5.0;
};

// src/bgremove/resharp.rs:58-125
inline FieldAndMask resharp(const std::vector<double>& field, const std::vector<uint8_t>& mask, const Grid& grid,
                            const ResharpParams& params, Progress progress = nullptr,
                            Session& s = Session::default_session()) {
  detail::require_len(field.size(), grid, "field");
  detail::require_len(mask.size(), grid, "mask");
  FieldAndMask r{std::vector<double>(grid.n_total()), std::vector<uint8_t>(grid.n_total())};
  qsm_grid g = grid.c();
  qsm_resharp_params p{params.radius, params.tik_reg, params.tol, params.max_iter};
  detail::ProgressThunk th{&progress};
  s.check(qsm_resharp(s.get(), field.data(), mask.data(), &g, &p, progress ? &detail::ProgressThunk::call : nullptr,
                      &th, r.first.data(), r.second.data()));
  return r;
}

// src/bgremove/ismv.rs:48-56
inline FieldAndMask ismv(const std::vector<double>& field, const std::vector<uint8_t>& mask, const Grid& grid,
                         const IsmvParams& params, Progress progress = nullptr,
                         Session& s = Session::default_session()) {
  detail::require_len(field.size(), grid, "field");
  detail::require_len(mask.size(), grid, "mask");
  FieldAndMask r{std::vector<double>(grid.n_total()), std::vector<uint8_t>(grid.n_total())};
  qsm_grid g = grid.c();
  qsm_ismv_params p{params.tol, params.max_iter, params.radius};
  detail::ProgressThunk th{&progress};
  s.check(qsm_ismv(s.get(), field.data(), mask.data(), &g, &p, progress ? &detail::ProgressThunk::call : nullptr,
                   &th, r.first.data(), r.second.data()));
  return r;
}
}  // namespace bgremove

// --------------------------------------------------------- utils::multi_echo --
namespace multi_echo {
// src/utils/multi_echo.rs:78-91
enum class B0WeightType { PhaseSNR = 0, PhaseVar = 1, Average = 2, TEs = 3, Mag = 4 };

// src/utils/multi_echo.rs:603-613
struct LinearFitResult {
  std::vector<double> field;
  std::vector<double> phase_offset;
  std::vector<double> fit_residual;
  std::vector<uint8_t> reliability_mask;
};

namespace detail3 {
inline std::vector<double> stack(const std::vector<std::vector<double>>& v, size_t n, const char* what) {
  std::vector<double> out;
  out.reserve(v.size() * n);
  for (const auto& e : v) {
    if (e.size() != n) throw Panic(QSM_ERR_DIMENSION_MISMATCH, std::string(what) + ": index out of bounds");
    out.insert(out.end(), e.begin(), e.end());
  }
  return out;
}
}  // namespace detail3

// src/utils/multi_echo.rs:450-506 (B0 in Hz; the grid only gives the voxel count)
inline std::vector<double> calculate_b0_weighted(const std::vector<std::vector<double>>& unwrapped_phases,
                                                 const std::vector<std::vector<double>>& mags,
                                                 const std::vector<double>& tes, const std::vector<uint8_t>& mask,
                                                 B0WeightType weight_type, const Grid& grid,
                                                 Session& s = Session::default_session()) {
  const size_t n = grid.n_total();
  detail::require_len(mask.size(), grid, "mask");
  const std::vector<double> ph = detail3::stack(unwrapped_phases, n, "unwrapped_phases");
  const std::vector<double> mg = detail3::stack(mags, n, "mags");
  if (mags.size() != unwrapped_phases.size() || tes.size() != unwrapped_phases.size())
    throw Panic(QSM_ERR_DIMENSION_MISMATCH, "echo counts disagree: index out of bounds");
  std::vector<double> out(n);
  s.check(qsm_calculate_b0_weighted(s.get(), ph.data(), mg.data(), tes.data(), tes.size(), mask.data(), n,
                                    (int)weight_type, out.data()));
  return out;
}

// src/utils/multi_echo.rs:631-768
inline LinearFitResult multi_echo_linear_fit(const std::vector<std::vector<double>>& unwrapped_phases,
                                             const std::vector<std::vector<double>>& mags,
                                             const std::vector<double>& tes, const std::vector<uint8_t>& mask,
                                             bool estimate_offset, double reliability_threshold_percentile,
                                             Session& s = Session::default_session()) {
  if (unwrapped_phases.empty()) throw Panic(QSM_ERR_INVALID_ARGUMENT, "no echoes: index out of bounds");
  const size_t n = unwrapped_phases[0].size();
  if (mask.size() != n) throw Panic(QSM_ERR_DIMENSION_MISMATCH, "mask: index out of bounds");
  const std::vector<double> ph = detail3::stack(unwrapped_phases, n, "unwrapped_phases");
  const std::vector<double> mg = detail3::stack(mags, n, "mags");
  if (mags.size() != unwrapped_phases.size() || tes.size() != unwrapped_phases.size())
    throw Panic(QSM_ERR_DIMENSION_MISMATCH, "echo counts disagree: index out of bounds");
  LinearFitResult r{std::vector<double>(n), std::vector<double>(n), std::vector<double>(n), std::vector<uint8_t>(n)};
  qsm_linear_fit_params p{estimate_offset ? 1 : 0, reliability_threshold_percentile};
  s.check(qsm_multi_echo_linear_fit(s.get(), ph.data(), mg.data(), tes.data(), tes.size(), mask.data(), n, &p,
                                    r.field.data(), r.phase_offset.data(), r.fit_residual.data(),
                                    r.reliability_mask.data()));
  return r;
}
}  // namespace multi_echo

// ------------------------------------------------------------------------ io --
// src/io.rs: fallible functions return Result<T, String>, here std::variant<T, std::string>.
namespace io {
template <class T> using IoResult = std::variant<T, std::string>;

// src/io.rs:13-27
struct NiftiData {
  std::vector<double> data;
  std::tuple<size_t, size_t, size_t> dims;
  std::tuple<double, double, double> voxel_size;
  std::array<double, 16> affine;
  double scl_slope;
  double scl_inter;
};

namespace detail4 {
inline NiftiData from(std::vector<double>&& d, const qsm_nifti_header& h) {
  NiftiData r;
  r.data = std::move(d);
  r.dims = {h.nx, h.ny, h.nz};
  r.voxel_size = {h.voxel_size[0], h.voxel_size[1], h.voxel_size[2]};
  for (int i = 0; i < 16; ++i) r.affine[i] = h.affine[i];
  r.scl_slope = h.scl_slope;
  r.scl_inter = h.scl_inter;
  return r;
}
inline IoResult<NiftiData> load(const std::vector<uint8_t>& bytes, bool all, qsm_nifti_header* hout) {
  char err[1024];
  qsm_nifti_header h{};
  if (qsm_nifti_parse_header(bytes.data(), bytes.size(), &h, err, sizeof err) != QSM_OK) return std::string(err);
  std::vector<double> d(h.nx * h.ny * h.nz * (all ? h.nt : 1));
  if (qsm_nifti_load(bytes.data(), bytes.size(), all ? 1 : 0, d.data(), d.size(), &h, err, sizeof err) != QSM_OK)
    return std::string(err);
  if (hout) *hout = h;
  return from(std::move(d), h);
}
inline IoResult<std::vector<uint8_t>> save(const std::vector<double>& data, std::tuple<size_t, size_t, size_t> dims,
                                           std::tuple<double, double, double> vs,
                                           const std::array<double, 16>& affine, bool gz) {
  char err[1024];
  const double v[3] = {std::get<0>(vs), std::get<1>(vs), std::get<2>(vs)};
  const size_t nx = std::get<0>(dims), ny = std::get<1>(dims), nz = std::get<2>(dims);
  if (data.size() != nx * ny * nz) return std::string("data length does not match dims");
  size_t need = 0;
  if (qsm_nifti_save(data.data(), nx, ny, nz, v, affine.data(), gz ? 1 : 0, nullptr, 0, &need, err, sizeof err) !=
      QSM_OK)
    return std::string(err);
  std::vector<uint8_t> out(need);
  size_t got = 0;
  if (qsm_nifti_save(data.data(), nx, ny, nz, v, affine.data(), gz ? 1 : 0, out.data(), out.size(), &got, err,
                     sizeof err) != QSM_OK)
    return std::string(err);
  out.resize(got);
  return out;
}
}  // namespace detail4

// src/io.rs:62-158
inline IoResult<NiftiData> load_nifti(const std::vector<uint8_t>& bytes) { return detail4::load(bytes, false, nullptr); }

// src/io.rs:161-224: (data, (nx, ny, nz, nt), voxel size, affine)
inline IoResult<std::tuple<std::vector<double>, std::tuple<size_t, size_t, size_t, size_t>,
                           std::tuple<double, double, double>, std::array<double, 16>>>
load_nifti_4d(const std::vector<uint8_t>& bytes) {
  qsm_nifti_header h{};
  auto r = detail4::load(bytes, true, &h);
  if (std::holds_alternative<std::string>(r)) return std::get<std::string>(r);
  NiftiData& d = std::get<NiftiData>(r);
  return std::make_tuple(std::move(d.data), std::make_tuple(h.nx, h.ny, h.nz, h.nt), d.voxel_size, d.affine);
}

// src/io.rs:255-338
inline IoResult<std::vector<uint8_t>> save_nifti(const std::vector<double>& data,
                                                 std::tuple<size_t, size_t, size_t> dims,
                                                 std::tuple<double, double, double> voxel_size,
                                                 const std::array<double, 16>& affine) {
  return detail4::save(data, dims, voxel_size, affine, false);
}

// src/io.rs:340-364
inline IoResult<std::vector<uint8_t>> save_nifti_gz(const std::vector<double>& data,
                                                    std::tuple<size_t, size_t, size_t> dims,
                                                    std::tuple<double, double, double> voxel_size,
                                                    const std::array<double, 16>& affine) {
  return detail4::save(data, dims, voxel_size, affine, true);
}

// src/io.rs:366-421
inline IoResult<std::tuple<size_t, size_t, size_t>> read_nifti_dims(const std::string& path) {
  char err[1024];
  size_t d[3];
  if (qsm_nifti_read_dims(path.c_str(), d, err, sizeof err) != QSM_OK) return std::string(err);
  return std::make_tuple(d[0], d[1], d[2]);
}

// src/io.rs:424-431
inline IoResult<NiftiData> read_nifti_file(const std::string& path) {
  char err[1024];
  qsm_nifti_header h{};
  if (qsm_nifti_read_file_header(path.c_str(), &h, err, sizeof err) != QSM_OK) return std::string(err);
  std::vector<double> d(h.nx * h.ny * h.nz);
  if (qsm_nifti_read_file(path.c_str(), 0, d.data(), d.size(), &h, err, sizeof err) != QSM_OK) return std::string(err);
  return detail4::from(std::move(d), h);
}

// src/io.rs:434-452
inline IoResult<std::monostate> save_nifti_to_file(const std::string& path, const std::vector<double>& data,
                                                   std::tuple<size_t, size_t, size_t> dims,
                                                   std::tuple<double, double, double> voxel_size,
                                                   const std::array<double, 16>& affine) {
  char err[1024];
  const double v[3] = {std::get<0>(voxel_size), std::get<1>(voxel_size), std::get<2>(voxel_size)};
  const size_t nx = std::get<0>(dims), ny = std::get<1>(dims), nz = std::get<2>(dims);
  if (data.size() != nx * ny * nz) return std::string("data length does not match dims");
  if (qsm_nifti_save_file(path.c_str(), data.data(), nx, ny, nz, v, affine.data(), err, sizeof err) != QSM_OK)
    return std::string(err);
  return std::monostate{};
}
}  // namespace io

// ------------------------------------------------------------------ pipeline --
namespace pipeline {

enum class InversionAlgorithm { Tkd, Tsvd, Tikhonov, Tv, Rts, Nltv, Medi, Ilsqr, Tgv, Qsmart };
enum class BgRemovalAlgorithm { Vsharp, Pdf, Lbv, Ismv, Sharp, Resharp, Harperella, Iharperella };

// src/pipeline/config.rs:302-324
struct ScanMetadata {
  std::tuple<size_t, size_t, size_t> dims;
  std::tuple<double, double, double> voxel_size{1.0, 1.0, 1.0};
  std::vector<double> echo_times;
  double field_strength = 3.0;
  BDir b0_direction{0.0, 0.0, 1.0};
  Grid grid() const { return Grid{dims, voxel_size}; }
};

struct InversionConfig {
  InversionAlgorithm algorithm = InversionAlgorithm::Rts;  // src/pipeline/config.rs:251
  inversion::TkdParams tkd;
  inversion::TkdParams tsvd;
  inversion::TikhonovParams tikhonov;
  inversion::TvParams tv;
  inversion::IlsqrParams ilsqr;
  inversion::RtsParams rts;
  inversion::NltvParams nltv;
};

struct BgRemovalConfig {
  BgRemovalAlgorithm algorithm = BgRemovalAlgorithm::Vsharp;
  bgremove::VsharpParams vsharp;
  bgremove::SharpParams sharp;
  bgremove::ResharpParams resharp;
  bgremove::IsmvParams ismv;
};

// src/pipeline/config.rs:69-72
enum class QsmReference { Mean = 0, None = 1 };

// src/pipeline/config.rs:343-368
struct PipelineError {
  enum Kind { InvalidConfig, InvalidInput, AlgorithmError, DimensionMismatch } kind;
  std::string message;
  size_t expected = 0, got = 0;
};

template <class T> using Result = std::variant<T, PipelineError>;

struct BgRemovalResult {
  std::vector<double> local_field_ppm;
  std::vector<uint8_t> eroded_mask;
};

namespace detail2 {
inline qsm_scan_metadata md(const ScanMetadata& m) {
  qsm_scan_metadata c{};
  c.nx = std::get<0>(m.dims);
  c.ny = std::get<1>(m.dims);
  c.nz = std::get<2>(m.dims);
  c.vsx = std::get<0>(m.voxel_size);
  c.vsy = std::get<1>(m.voxel_size);
  c.vsz = std::get<2>(m.voxel_size);
  c.field_strength = m.field_strength;
  detail::bdir3(m.b0_direction, c.b0_direction);
  return c;
}
inline PipelineError to_error(int st, qsm_ctx* ctx, size_t expected, size_t got) {
  PipelineError e;
  e.message = qsm_last_error(ctx);
  e.expected = expected;
  e.got = got;
  e.kind = st == QSM_ERR_DIMENSION_MISMATCH ? PipelineError::DimensionMismatch
           : st == QSM_ERR_INVALID_CONFIG   ? PipelineError::InvalidConfig
           : st == QSM_ERR_INVALID_ARGUMENT ? PipelineError::InvalidInput
                                            : PipelineError::AlgorithmError;
  return e;
}
}  // namespace detail2

// src/pipeline/inversion.rs:28-114
inline Result<std::vector<double>> run_dipole_inversion(const std::vector<double>& local_field_ppm,
                                                        const std::vector<uint8_t>& mask,
                                                        const ScanMetadata& metadata, const InversionConfig& config,
                                                        const std::vector<double>* /*magnitude*/,
                                                        Progress progress = nullptr,
                                                        Session& s = Session::default_session()) {
  qsm_scan_metadata m = detail2::md(metadata);
  qsm_inversion_config c{};
  c.algorithm = (int)config.algorithm;
  c.tkd = {config.tkd.threshold};
  c.tsvd = {config.tsvd.threshold};
  c.tikhonov = {config.tikhonov.lambda, (int)config.tikhonov.reg};
  c.tv = {config.tv.lambda, config.tv.rho, config.tv.tol, config.tv.max_iter};
  c.ilsqr = {config.ilsqr.tol, config.ilsqr.max_iter};
  c.rts = {config.rts.delta, config.rts.mu, config.rts.rho, config.rts.tol, config.rts.max_iter, config.rts.lsmr_iter};
  c.nltv = {config.nltv.lambda, config.nltv.mu, config.nltv.tol, config.nltv.max_iter, config.nltv.newton_iter};
  const size_t n = metadata.grid().n_total();
  std::vector<double> out(local_field_ppm.size() == n ? n : 1);
  detail::ProgressThunk th{&progress};
  int st = qsm_run_dipole_inversion(s.get(), local_field_ppm.data(), local_field_ppm.size(), mask.data(), &m, &c,
                                    progress ? &detail::ProgressThunk::call : nullptr, &th, out.data());
  if (st != QSM_OK) return detail2::to_error(st, s.get(), n, local_field_ppm.size());
  return out;
}

// src/pipeline/bg_removal.rs:20-92
inline Result<BgRemovalResult> run_bg_removal(const std::vector<double>& field_ppm, const std::vector<uint8_t>& mask,
                                              const ScanMetadata& metadata, const BgRemovalConfig& config,
                                              Progress progress = nullptr,
                                              Session& s = Session::default_session()) {
  qsm_scan_metadata m = detail2::md(metadata);
  qsm_bg_removal_config c{};
  c.algorithm = (int)config.algorithm;
  c.vsharp = {config.vsharp.threshold, config.vsharp.max_radius, config.vsharp.min_radius};
  c.sharp = {config.sharp.threshold, config.sharp.radius};
  c.resharp = {config.resharp.radius, config.resharp.tik_reg, config.resharp.tol, config.resharp.max_iter};
  c.ismv = {config.ismv.tol, config.ismv.max_iter, config.ismv.radius};
  const size_t n = metadata.grid().n_total();
  BgRemovalResult r{std::vector<double>(field_ppm.size() == n ? n : 1),
                    std::vector<uint8_t>(field_ppm.size() == n ? n : 1)};
  detail::ProgressThunk th{&progress};
  int st = qsm_run_bg_removal(s.get(), field_ppm.data(), field_ppm.size(), mask.data(), &m, &c,
                              progress ? &detail::ProgressThunk::call : nullptr, &th, r.local_field_ppm.data(),
                              r.eroded_mask.data());
  if (st != QSM_OK) return detail2::to_error(st, s.get(), n, field_ppm.size());
  return r;
}

// src/pipeline/referencing.rs:12-43
inline std::vector<double> apply_reference(const std::vector<double>& chi, const std::vector<uint8_t>& mask,
                                           QsmReference method, Session& s = Session::default_session()) {
  if (mask.size() != chi.size()) throw Panic(QSM_ERR_DIMENSION_MISMATCH, "mask: index out of bounds");
  std::vector<double> out(chi.size());
  s.check(qsm_apply_reference(s.get(), chi.data(), mask.data(), chi.size(), (int)method, out.data()));
  return out;
}

// src/pipeline/inversion.rs:124-157 for single-echo wrapped phase (the multi-echo
// field-mapping step before TGV is not on this library's path)
inline Result<std::vector<double>> run_tgv(const std::vector<const std::vector<double>*>& phases,
                                           const std::vector<uint8_t>& mask, const ScanMetadata& metadata,
                                           const inversion::TgvParams& tgv_params, QsmReference reference,
                                           Progress progress = nullptr, Session& s = Session::default_session()) {
  qsm_scan_metadata m = detail2::md(metadata);
  std::vector<const double*> ptrs;
  size_t len = phases.empty() ? 0 : phases[0]->size();
  for (auto* p : phases) ptrs.push_back(p->data());
  const size_t n = metadata.grid().n_total();
  std::vector<double> out(len == n ? n : 1);
  qsm_tgv_params p = tgv_params.c();
  detail::ProgressThunk th{&progress};
  int st = qsm_run_tgv(s.get(), ptrs.data(), ptrs.size(), len, mask.data(), &m, &p, (int)reference,
                       progress ? &detail::ProgressThunk::call : nullptr, &th, out.data());
  if (st != QSM_OK) return detail2::to_error(st, s.get(), n, len);
  return out;
}

}  // namespace pipeline
}  // namespace qsm
