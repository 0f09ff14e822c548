// qsm.hpp — C++ host mirror of QSM.rs's reconstruction API over the qsmgpu C ABI.
//
// The reference crate (astewartau/QSM.rs) exposes free functions taking borrowed
// slices and returning owned vectors; this header keeps those names, argument order,
// defaults and error behaviour:
//   * algorithm functions (inversion::tv_admm, tkd, tsvd, tikhonov,
//     unwrap::laplacian_unwrap, bgremove::smv/sharp/vsharp) throw qsm::Panic where the
//     Rust code would panic (length mismatch) or where the GPU call fails;
//   * pipeline functions (pipeline::run_dipole_inversion, run_bg_removal) return a
//     Result carrying PipelineError {DimensionMismatch, InvalidConfig, AlgorithmError}.
//
// Header-only; link with libqsmgpu.so.  One Session (a qsm_ctx) per thread.
#pragma once

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
}  // namespace bgremove

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
};

struct BgRemovalConfig {
  BgRemovalAlgorithm algorithm = BgRemovalAlgorithm::Vsharp;
  bgremove::VsharpParams vsharp;
  bgremove::SharpParams sharp;
};

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

}  // namespace pipeline
}  // namespace qsm
