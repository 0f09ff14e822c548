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
