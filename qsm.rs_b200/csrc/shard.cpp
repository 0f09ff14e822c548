// Placement of a batch of independent volumes on several GPUs.
//
// A batch of volumes (the per-volume unit is inversion::tv_admm, src/inversion/tv.rs:63-97)
// shards across GPUs with no exchange: every volume is solved whole on one GPU, each GPU
// runs its own share as one batched call (one context, one graph), and the results are
// gathered on the host at the end.  The share of each GPU comes from the
// longest-processing-time-first rule: volumes in decreasing order of cost (ties in batch
// order), each placed on the part with the least total cost so far (ties to the lowest
// part index).  The cost of a volume is N*log2(N)*iterations, N its voxel count: every
// TV-ADMM iteration is five FFT passes plus one stencil over the volume.
//
// Host-only code: it needs no GPU, so launchers and tests can call it anywhere.
#include "internal.h"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace qsm {

double volume_cost(const qsm_grid& g, size_t iterations) {
  const double n = (double)g.nx * (double)g.ny * (double)g.nz;
  return n * std::log2(n + 2.0) * (double)iterations;
}

}  // namespace qsm

using namespace qsm;

extern "C" qsm_status qsm_batch_partition(const qsm_grid* grids, const size_t* iterations, size_t n, size_t n_parts,
                                          uint32_t* out_part, double* out_load) {
  if (n_parts == 0 || n_parts > 65536) return QSM_ERR_INVALID_ARGUMENT;
  if (n > 0 && (grids == nullptr || out_part == nullptr)) return QSM_ERR_INVALID_ARGUMENT;
  try {
    std::vector<double> cost(n);
    for (size_t b = 0; b < n; ++b) {
      const qsm_grid& g = grids[b];
      if (g.nx == 0 || g.ny == 0 || g.nz == 0) return QSM_ERR_INVALID_ARGUMENT;
      cost[b] = volume_cost(g, iterations ? iterations[b] : 1);
    }
    std::vector<size_t> order(n);
    std::iota(order.begin(), order.end(), (size_t)0);
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
    std::vector<double> load(n_parts, 0.0);
    for (size_t b : order) {
      const size_t k = (size_t)(std::min_element(load.begin(), load.end()) - load.begin());
      out_part[b] = (uint32_t)k;
      load[k] += cost[b];
    }
    if (out_load) std::copy(load.begin(), load.end(), out_load);
  } catch (const std::bad_alloc&) {
    return QSM_ERR_ALLOC;
  }
  return QSM_OK;
}
