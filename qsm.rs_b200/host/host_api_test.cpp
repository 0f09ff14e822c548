// Exercise the C++ host mirror (qsm.hpp) on the GPU: run each algorithm on a small
// deterministic volume, write the results to a raw float64 file for comparison with
// the oracle, and check the pipeline error variants.
//
//   host_api_test OUT.bin      (exit 0 on success)
#include <cmath>
#include <cstdio>
#include <fstream>

#include "qsm.hpp"

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s OUT.bin\n", argv[0]);
    return 2;
  }
  const size_t n = 16;
  qsm::Grid grid = qsm::Grid::make(n, n, n, 1.0, 1.0, 1.0);
  std::vector<double> field(grid.n_total());
  std::vector<uint8_t> mask(grid.n_total(), 1);
  for (size_t i = 0; i < field.size(); ++i) field[i] = 0.01 * std::sin(0.7 * (double)i);
  qsm::BDir b{0.0, 0.0, 1.0};
  qsm::Session s(0, QSM_PRECISION_F64);

  std::vector<std::vector<double>> outs;
  outs.push_back(qsm::inversion::tkd(field, mask, grid, b, {0.15}, s));
  qsm::inversion::TvParams tv;
  tv.tol = 0.0;
  tv.max_iter = 10;
  size_t calls = 0;
  outs.push_back(qsm::inversion::tv_admm(field, mask, grid, b, tv, [&](size_t, size_t) { ++calls; }, s));
  if (calls != 10) {
    std::fprintf(stderr, "progress calls %zu != 10\n", calls);
    return 1;
  }
  std::vector<double> phase(field.size());
  for (size_t i = 0; i < phase.size(); ++i) phase[i] = 3.0 * std::sin(0.05 * (double)i);
  outs.push_back(qsm::unwrap::laplacian_unwrap(phase, mask, grid, s));
  auto sh = qsm::bgremove::sharp(field, mask, grid, {0.05, 3.0}, s);
  outs.push_back(sh.first);

  // the entry points added after the first set
  qsm::inversion::RtsParams rp;
  rp.tol = 0.0;
  rp.max_iter = 7;
  outs.push_back(qsm::inversion::rts(field, mask, grid, b, rp, nullptr, s));
  qsm::inversion::NltvParams np;
  np.tol = 0.0;
  np.max_iter = 5;
  np.newton_iter = 2;
  outs.push_back(qsm::inversion::nltv(field, mask, grid, b, np, nullptr, s));
  outs.push_back(qsm::bgremove::ismv(field, mask, grid, {1e-6, 20, 3.0}, nullptr, s).first);
  outs.push_back(qsm::bgremove::resharp(field, mask, grid, {3.0, 1e-4, 1e-6, 20}, nullptr, s).first);
  std::vector<double> tes{0.005, 0.010, 0.015};
  std::vector<std::vector<double>> ph3, mg3;
  for (double te : tes) {
    std::vector<double> p(field.size()), m(field.size());
    for (size_t i = 0; i < p.size(); ++i) {
      p[i] = 0.3 + 150.0 * std::sin(0.01 * (double)i) * te + 0.01 * std::cos(3.0 * (double)i + te);
      m[i] = 1.0 + 0.5 * std::sin(0.2 * (double)i);
    }
    ph3.push_back(p);
    mg3.push_back(m);
  }
  auto fit = qsm::multi_echo::multi_echo_linear_fit(ph3, mg3, tes, mask, true, 90.0, s);
  outs.push_back(fit.field);
  auto il = qsm::inversion::ilsqr(field, mask, grid, b, {0.01, 10}, nullptr, s);
  for (double v : std::get<0>(il))
    if (!std::isfinite(v)) {
      std::fprintf(stderr, "ilsqr not finite\n");
      return 1;
    }
  // NIfTI round trips: bytes and a .nii.gz file
  std::array<double, 16> aff{1.0, 0, 0, 10.0, 0, 2.0, 0, 20.0, 0, 0, 3.0, 30.0, 0, 0, 0, 1};
  auto bytes = qsm::io::save_nifti(field, {n, n, n}, {1.0, 2.0, 3.0}, aff);
  auto back = qsm::io::load_nifti(std::get<0>(bytes));
  const auto& nd = std::get<qsm::io::NiftiData>(back);
  for (size_t i = 0; i < field.size(); ++i)
    if (nd.data[i] != (double)(float)field[i]) {
      std::fprintf(stderr, "nifti round trip differs at %zu\n", i);
      return 1;
    }
  const std::string path = std::string(argv[1]) + ".nii.gz";
  if (!std::holds_alternative<std::monostate>(qsm::io::save_nifti_to_file(path, field, {n, n, n}, {1, 2, 3}, aff)) ||
      std::get<0>(qsm::io::read_nifti_file(path)).data != nd.data ||
      std::get<0>(qsm::io::read_nifti_dims(path)) != std::make_tuple(n, n, n) ||
      !std::holds_alternative<std::string>(qsm::io::read_nifti_file(path + ".missing"))) {
    std::fprintf(stderr, "nifti file round trip failed\n");
    return 1;
  }

  // pipeline: dispatch equals the direct call; error variants
  qsm::pipeline::ScanMetadata md;
  md.dims = {n, n, n};
  qsm::pipeline::InversionConfig cfg;
  cfg.algorithm = qsm::pipeline::InversionAlgorithm::Tkd;
  auto r = qsm::pipeline::run_dipole_inversion(field, mask, md, cfg, nullptr, nullptr, s);
  if (!std::holds_alternative<std::vector<double>>(r) || std::get<0>(r) != outs[0]) {
    std::fprintf(stderr, "pipeline TKD differs from direct TKD\n");
    return 1;
  }
  cfg.algorithm = qsm::pipeline::InversionAlgorithm::Rts;
  cfg.rts = rp;
  auto rr = qsm::pipeline::run_dipole_inversion(field, mask, md, cfg, nullptr, nullptr, s);
  if (!std::holds_alternative<std::vector<double>>(rr) || std::get<0>(rr) != outs[4]) {
    std::fprintf(stderr, "pipeline RTS differs from direct RTS\n");
    return 1;
  }
  auto ref = qsm::pipeline::apply_reference(outs[4], mask, qsm::pipeline::QsmReference::Mean, s);
  double mean = 0.0;
  for (double v : ref) mean += v;
  if (std::fabs(mean / (double)ref.size()) > 1e-12) {
    std::fprintf(stderr, "apply_reference mean %g\n", mean);
    return 1;
  }
  cfg.algorithm = qsm::pipeline::InversionAlgorithm::Tkd;
  std::vector<double> shortf(10, 0.0);
  auto e1 = qsm::pipeline::run_dipole_inversion(shortf, mask, md, cfg, nullptr, nullptr, s);
  if (!std::holds_alternative<qsm::pipeline::PipelineError>(e1) ||
      std::get<1>(e1).kind != qsm::pipeline::PipelineError::DimensionMismatch || std::get<1>(e1).expected != 4096 ||
      std::get<1>(e1).got != 10) {
    std::fprintf(stderr, "expected DimensionMismatch\n");
    return 1;
  }
  cfg.algorithm = qsm::pipeline::InversionAlgorithm::Tgv;
  auto e2 = qsm::pipeline::run_dipole_inversion(field, mask, md, cfg, nullptr, nullptr, s);
  if (!std::holds_alternative<qsm::pipeline::PipelineError>(e2) ||
      std::get<1>(e2).kind != qsm::pipeline::PipelineError::InvalidConfig) {
    std::fprintf(stderr, "expected InvalidConfig\n");
    return 1;
  }
  // algorithm functions panic on a length mismatch, as slice indexing does in Rust
  bool threw = false;
  try {
    qsm::inversion::tkd(shortf, mask, grid, b, {0.15}, s);
  } catch (const qsm::Panic&) {
    threw = true;
  }
  if (!threw) {
    std::fprintf(stderr, "expected a panic on a short input\n");
    return 1;
  }

  std::ofstream f(argv[1], std::ios::binary);
  for (auto& o : outs) f.write(reinterpret_cast<const char*>(o.data()), (std::streamsize)(o.size() * sizeof(double)));
  std::printf("host api ok\n");
  return 0;
}
