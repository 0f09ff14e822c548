// Host-side context, workspace cache and error plumbing behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <functional>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/qsmgpu.h"
#include "fft_plan.h"

namespace qsm {

struct QsmError : std::runtime_error {
  qsm_status code;
  QsmError(qsm_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define QSM_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e__ = (call);                                                            \
    if (e__ != cudaSuccess)                                                              \
      throw ::qsm::QsmError(QSM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
  } while (0)

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  uint64_t epoch = 0;  // API call that last handed the pointer out
};

struct GraphCache {
  cudaGraphExec_t exec = nullptr;
  std::string key;
};

// One timed kernel launch (profiling mode): events recorded around the launch on
// the context's stream.
struct ProfRec {
  std::string name;
  cudaEvent_t start, stop;
};

// Largest launch-shape number of the autotuned passes (launch.cuh).
constexpr int kTuneMaxShape = 63;

// One autotuned launch shape: the chosen candidate and each candidate's best time.
struct TuneRec {
  int choice = 0;
  std::vector<std::pair<int, float>> us;  // (candidate, microseconds per launch)
};

struct ProfStat {
  uint64_t launches = 0;
  double total_ms = 0.0;
};

}  // namespace qsm

struct qsm_ctx {
  int device = 0;
  int precision = QSM_PRECISION_F64;
  int plan_mode = QSM_PLANS_COMPILED;  // qsm_ctx_set_plan_mode
  int krylov_precision = QSM_PRECISION_F64;  // qsm_ctx_set_krylov_precision (mixed contexts)
  bool check_inputs = false;  // qsm_ctx_set_input_check
  bool autotune = true;  // qsm_ctx_set_autotune
  int forced_shape = -1;  // qsm_ctx_force_launch_shape (-1: none)
  std::map<std::string, qsm::TuneRec> tuned;  // launch shapes chosen by the autotuner
  long long alloc_fail_after = -1;  // qsm_ctx_inject_alloc_failure: allocations left before one fails
  cudaStream_t stream = nullptr;
  std::string err;
  std::map<std::string, qsm::DevBuf> ws;
  uint64_t epoch = 0;  // incremented by every API call (guarded)
  std::map<long long, void*> twiddles;  // key n*2 + (double ? 1 : 0)
  std::map<std::string, void*> tables;  // small per-grid tables
  std::map<std::string, qsm::GraphCache> graphs;
  uint64_t launches = 0;
  size_t tv_last_iters = 0;
  // per-kernel CUDA-event profiling (qsm_ctx_set_profiling); iterative solvers run
  // without graph capture while it is on
  bool profiling = false;
  std::string prof_prefix;
  std::vector<qsm::ProfRec> prof_pending;
  std::vector<std::pair<std::string, qsm::ProfStat>> prof_stats;
  // pinned host staging ring for host<->device streaming (staged_h2d / staged_d2h)
  void* pinned[2] = {nullptr, nullptr};
  cudaEvent_t pinned_ev[2] = {nullptr, nullptr};
};

namespace qsm {

// Named device workspace, grown on demand and reused across calls.
void* ws_get(qsm_ctx* ctx, const std::string& name, size_t bytes);
template <typename P> P* ws(qsm_ctx* ctx, const std::string& name, size_t count) {
  return reinterpret_cast<P*>(ws_get(ctx, name, count * sizeof(P)));
}
void ws_release(qsm_ctx* ctx);

// Device table of a plan, float2 or double2: the forward twiddles W_m^k (k in [0, m))
// of its stages and, for Bluestein plans, the chirp (n values) and the convolution
// kernel spectrum (m values) after them.  Cached per length and precision.
const void* twiddle_table(qsm_ctx* ctx, const FftPlan1D& pl, bool dbl);
// The same table on the host (bytes).
std::vector<unsigned char> transform_table(const FftPlan1D& pl, bool dbl);
FftPlan1D plan_or_throw(int n);

// Upload a small host vector as a cached device table keyed by name.
const void* upload_table(qsm_ctx* ctx, const std::string& key, const void* host, size_t bytes);

// Validation helpers
struct GridDims {
  int nx, ny, nz;
  double vsx, vsy, vsz;
  long long n;
};
GridDims check_grid(const qsm_grid* g);
void check_ptr(const void* p, const char* name);
void check_finite(double v, const char* name);
// With the context's input check on (qsm_ctx_set_input_check), reject a device volume
// holding a NaN or an infinity (QSM_ERR_INVALID_ARGUMENT); otherwise do nothing.
void check_volume_finite(qsm_ctx* ctx, const double* d, long long n, const char* name);
// Device allocation for the context: cudaMalloc, or the failure requested by
// qsm_ctx_inject_alloc_failure.
cudaError_t ctx_malloc(qsm_ctx* ctx, void** p, size_t bytes);

// Host <-> device staging used by the host-pointer entry points.
// Copies through two pinned staging buffers (kStageBytes each): the host copy of one
// chunk overlaps the DMA of the previous one.  Both return with the copies complete.
constexpr size_t kStageBytes = (size_t)32 << 20;
void staged_h2d(qsm_ctx* ctx, void* dst, const void* src, size_t bytes);
void staged_d2h(qsm_ctx* ctx, void* dst, const void* src, size_t bytes);
void h2d(qsm_ctx* ctx, void* dst, const void* src, size_t bytes);
void d2h(qsm_ctx* ctx, void* dst, const void* src, size_t bytes);
void sync(qsm_ctx* ctx);

// Profiling scope around one launch: records a start event now and a stop event
// (plus the launch-error check and launch count) in done().
struct LaunchScope {
  qsm_ctx* ctx;
  const char* name;
  cudaEvent_t ev0 = nullptr;
  LaunchScope(qsm_ctx* c, const char* n) : ctx(c), name(n) {
    if (ctx->profiling) {
      QSM_CUDA(cudaEventCreate(&ev0));
      QSM_CUDA(cudaEventRecord(ev0, ctx->stream));
    }
  }
  void done();
};
void prof_collect(qsm_ctx* ctx);

// Run fn and convert exceptions into a status + last error string.
template <class F> qsm_status guarded(qsm_ctx* ctx, F&& fn) {
  if (ctx == nullptr) return QSM_ERR_INVALID_ARGUMENT;
  ctx->epoch++;
  try {
    QSM_CUDA(cudaSetDevice(ctx->device));
    fn();
    ctx->err.clear();
    return QSM_OK;
  } catch (const QsmError& e) {
    ctx->err = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    ctx->err = "host allocation failed";
    return QSM_ERR_ALLOC;
  } catch (const std::exception& e) {
    ctx->err = e.what();
    return QSM_ERR_CUDA;
  }
}

}  // namespace qsm
