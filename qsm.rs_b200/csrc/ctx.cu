// Context, workspace cache, twiddle tables, argument validation and the
// context-level C ABI entry points.
#include "internal.h"
#include "common.cuh"

#include <algorithm>
#include <cstring>

namespace qsm {

cudaError_t ctx_malloc(qsm_ctx* ctx, void** p, size_t bytes) {
  if (ctx->alloc_fail_after == 0) {
    ctx->alloc_fail_after = -1;  // one injected failure, then allocations succeed again
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  if (ctx->alloc_fail_after > 0) ctx->alloc_fail_after--;
  return cudaMalloc(p, bytes);
}

namespace {
__global__ void k_count_nonfinite(long long n, const double* __restrict__ a, unsigned long long* count) {
  unsigned long long c = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    c += isfinite(a[i]) ? 0ull : 1ull;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}
}  // namespace

void check_volume_finite(qsm_ctx* ctx, const double* d, long long n, const char* name) {
  if (!ctx->check_inputs || n <= 0) return;
  unsigned long long* cnt = ws<unsigned long long>(ctx, "check.count", 1);
  QSM_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), ctx->stream));
  long long blocks = (n + 255) / 256;
  if (blocks > 148LL * 8) blocks = 148LL * 8;
  LaunchScope ls(ctx, "check_finite");
  k_count_nonfinite<<<(unsigned)blocks, 256, 0, ctx->stream>>>(n, d, cnt);
  ls.done();
  unsigned long long h = 0;
  d2h(ctx, &h, cnt, sizeof(h));
  sync(ctx);
  if (h != 0)
    throw QsmError(QSM_ERR_INVALID_ARGUMENT, std::string(name) + " has " + std::to_string(h) +
                                                 " non-finite voxel(s) (NaN or infinity)");
}

void* ws_get(qsm_ctx* ctx, const std::string& name, size_t bytes) {
  if (bytes == 0) bytes = 16;
  DevBuf& b = ctx->ws[name];
  if (b.bytes < bytes) {
    // growing frees the old buffer: a pointer handed out earlier in this call would dangle
    if (b.p && b.epoch == ctx->epoch)
      throw QsmError(QSM_ERR_CUDA, "internal error: workspace '" + name + "' grown after use in the same call");
    if (b.p) {
      QSM_CUDA(cudaStreamSynchronize(ctx->stream));
      QSM_CUDA(cudaFree(b.p));
      b.p = nullptr;
      b.bytes = 0;
    }
    void* p = nullptr;
    cudaError_t e = ctx_malloc(ctx, &p, bytes);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      throw QsmError(QSM_ERR_ALLOC, "device allocation of " + std::to_string(bytes) + " bytes for '" + name +
                                        "' failed: " + cudaGetErrorString(e));
    }
    b.p = p;
    b.bytes = bytes;
  }
  b.epoch = ctx->epoch;
  return b.p;
}

bool stream_capturing(qsm_ctx* ctx) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  QSM_CUDA(cudaStreamIsCapturing(ctx->stream, &st));
  return st != cudaStreamCaptureStatusNone;
}

void autotune_pick(qsm_ctx* ctx, const std::string& key, const std::vector<int>& cands,
                   const std::function<void(int)>& launch, int rounds, int reps) {
  if (cands.empty()) return;
  TuneRec rec;
  if (cands.size() == 1) {
    rec.choice = cands[0];
    ctx->tuned[key] = rec;
    return;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  QSM_CUDA(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    throw QsmError(QSM_ERR_CUDA, "autotuner: event creation failed");
  }
  std::vector<float> best(cands.size(), 3.0e38f);
  try {
    for (int c : cands) launch(c);  // warm-up (raises shared-memory limits, loads the code)
    QSM_CUDA(cudaGetLastError());
    for (int r = 0; r < rounds; ++r) {
      for (size_t i = 0; i < cands.size(); ++i) {
        QSM_CUDA(cudaEventRecord(e0, ctx->stream));
        for (int k = 0; k < reps; ++k) launch(cands[i]);
        QSM_CUDA(cudaEventRecord(e1, ctx->stream));
        QSM_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        QSM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best[i] = std::min(best[i], 1000.f * ms / reps);
      }
    }
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  size_t k = 0;
  for (size_t i = 1; i < cands.size(); ++i)
    if (best[i] < best[k]) k = i;
  rec.choice = cands[k];
  for (size_t i = 0; i < cands.size(); ++i) rec.us.emplace_back(cands[i], best[i]);
  ctx->tuned[key] = rec;
}

void ws_release(qsm_ctx* ctx) {
  cudaStreamSynchronize(ctx->stream);
  for (auto& kv : ctx->ws)
    if (kv.second.p) cudaFree(kv.second.p);
  ctx->ws.clear();
  for (auto& kv : ctx->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  ctx->graphs.clear();
}

FftPlan1D plan_or_throw(int n) {
  FftPlan1D pl;
  if (!make_fft_plan(n, &pl))
    throw QsmError(QSM_ERR_UNSUPPORTED_SIZE,
                   "axis length " + std::to_string(n) + " has no transform plan (n <= " + std::to_string(kFftMaxLen) +
                       ", and n <= " + std::to_string(kBluesteinMaxLen) + " when n has a prime factor above 13)");
  return pl;
}

std::vector<unsigned char> transform_table(const FftPlan1D& pl, bool dbl) {
  const int n = pl.n, m = pl.m;
  const size_t elem = dbl ? sizeof(double2) : sizeof(float2);
  const size_t count = (size_t)m + (m != n ? (size_t)n + (size_t)m : 0);
  std::vector<unsigned char> host(elem * count);
  auto put = [&](size_t i, double re, double im) {
    if (dbl) {
      const double2 v = make_double2(re, im);
      std::memcpy(&host[elem * i], &v, elem);
    } else {
      const float2 v = make_float2((float)re, (float)im);
      std::memcpy(&host[elem * i], &v, elem);
    }
  };
  // forward twiddles exp(-2 pi i k / m) of the stages
  for (int k = 0; k < m; ++k) put((size_t)k, cos2pi(k, m), -sin2pi(k, m));
  if (m != n) {
    // chirp c_j = exp(-i pi j^2 / n) = exp(-2 pi i (j^2 mod 2n) / 2n)
    std::vector<double> cre((size_t)n), cim((size_t)n), cosm((size_t)m);
    for (int j = 0; j < n; ++j) {
      const long long jj = ((long long)j * j) % (2LL * n);
      cre[(size_t)j] = cos2pi(jj, 2LL * n);
      cim[(size_t)j] = sin2pi(jj, 2LL * n);
      put((size_t)m + j, cre[(size_t)j], -cim[(size_t)j]);
    }
    for (int x = 0; x < m; ++x) cosm[(size_t)x] = cos2pi(x, m);
    // K_k = (1/m) DFT_m(conj chirp wrapped cyclically)_k
    //     = (1/m) (1 + 2 sum_{l=1}^{n-1} cos(2 pi l k / m) exp(i pi l^2 / n)), an even sequence
    for (int k = 0; k < m; ++k) {
      long double re = 1.0L, im = 0.0L;
      long long lk = 0;
      for (int l = 1; l < n; ++l) {
        lk += k;
        if (lk >= m) lk %= m;
        const long double c = 2.0L * (long double)cosm[(size_t)lk];
        re += c * (long double)cre[(size_t)l];
        im += c * (long double)cim[(size_t)l];
      }
      put((size_t)m + n + k, (double)(re / m), (double)(im / m));
    }
  }
  return host;
}

const void* twiddle_table(qsm_ctx* ctx, const FftPlan1D& pl, bool dbl) {
  const long long key = (long long)pl.n * 2 + (dbl ? 1 : 0);
  auto it = ctx->twiddles.find(key);
  if (it != ctx->twiddles.end()) return it->second;
  const std::vector<unsigned char> host = transform_table(pl, dbl);
  void* d = nullptr;
  cudaError_t e = ctx_malloc(ctx, &d, host.size());
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    throw QsmError(QSM_ERR_ALLOC, "twiddle table allocation failed");
  }
  QSM_CUDA(cudaMemcpy(d, host.data(), host.size(), cudaMemcpyHostToDevice));
  ctx->twiddles[key] = d;
  return d;
}

const void* upload_table(qsm_ctx* ctx, const std::string& key, const void* host, size_t bytes) {
  auto it = ctx->tables.find(key);
  if (it != ctx->tables.end()) return it->second;
  void* d = nullptr;
  cudaError_t e = ctx_malloc(ctx, &d, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    throw QsmError(QSM_ERR_ALLOC, "table allocation failed");
  }
  if (bytes) QSM_CUDA(cudaMemcpy(d, host, bytes, cudaMemcpyHostToDevice));
  ctx->tables[key] = d;
  return d;
}

GridDims check_grid(const qsm_grid* g) {
  if (g == nullptr) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "grid is null");
  if (g->nx == 0 || g->ny == 0 || g->nz == 0) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "grid has a zero dimension");
  if (g->nx > (size_t)kFftMaxLen || g->ny > (size_t)kFftMaxLen || g->nz > (size_t)kFftMaxLen)
    throw QsmError(QSM_ERR_UNSUPPORTED_SIZE, "grid dimension above " + std::to_string(kFftMaxLen));
  for (double v : {g->vsx, g->vsy, g->vsz})
    if (!std::isfinite(v) || v <= 0.0) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "voxel size must be finite and > 0");
  GridDims d;
  d.nx = (int)g->nx;
  d.ny = (int)g->ny;
  d.nz = (int)g->nz;
  d.vsx = g->vsx;
  d.vsy = g->vsy;
  d.vsz = g->vsz;
  d.n = (long long)d.nx * d.ny * d.nz;
  if ((long long)d.ny * d.nz > (1LL << 30)) throw QsmError(QSM_ERR_UNSUPPORTED_SIZE, "too many rows");
  plan_or_throw(d.nx);
  plan_or_throw(d.ny);
  plan_or_throw(d.nz);
  return d;
}

void check_ptr(const void* p, const char* name) {
  if (p == nullptr) throw QsmError(QSM_ERR_INVALID_ARGUMENT, std::string(name) + " is null");
}

void check_finite(double v, const char* name) {
  if (!std::isfinite(v)) throw QsmError(QSM_ERR_INVALID_ARGUMENT, std::string(name) + " is not finite");
}

void h2d(qsm_ctx* ctx, void* dst, const void* src, size_t bytes) {
  QSM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
}
void d2h(qsm_ctx* ctx, void* dst, const void* src, size_t bytes) {
  QSM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
}
void sync(qsm_ctx* ctx) { QSM_CUDA(cudaStreamSynchronize(ctx->stream)); }

namespace {
void ensure_pinned(qsm_ctx* ctx) {
  for (int k = 0; k < 2; ++k) {
    if (!ctx->pinned[k]) {
      if (cudaHostAlloc(&ctx->pinned[k], kStageBytes, cudaHostAllocDefault) != cudaSuccess) {
        (void)cudaGetLastError();
        ctx->pinned[k] = nullptr;
        throw QsmError(QSM_ERR_ALLOC, "pinned staging allocation failed");
      }
    }
    if (!ctx->pinned_ev[k]) QSM_CUDA(cudaEventCreateWithFlags(&ctx->pinned_ev[k], cudaEventDisableTiming));
  }
}
}  // namespace

void staged_h2d(qsm_ctx* ctx, void* dst, const void* src, size_t bytes) {
  ensure_pinned(ctx);
  const uint8_t* s = static_cast<const uint8_t*>(src);
  uint8_t* d = static_cast<uint8_t*>(dst);
  bool used[2] = {false, false};
  for (size_t off = 0, c = 0; off < bytes; off += kStageBytes, ++c) {
    const int k = (int)(c % 2);
    const size_t n = std::min(kStageBytes, bytes - off);
    if (used[k]) QSM_CUDA(cudaEventSynchronize(ctx->pinned_ev[k]));  // this slot's previous DMA is done
    std::memcpy(ctx->pinned[k], s + off, n);
    QSM_CUDA(cudaMemcpyAsync(d + off, ctx->pinned[k], n, cudaMemcpyHostToDevice, ctx->stream));
    QSM_CUDA(cudaEventRecord(ctx->pinned_ev[k], ctx->stream));
    used[k] = true;
  }
  sync(ctx);
}

void staged_d2h(qsm_ctx* ctx, void* dst, const void* src, size_t bytes) {
  ensure_pinned(ctx);
  const uint8_t* s = static_cast<const uint8_t*>(src);
  uint8_t* d = static_cast<uint8_t*>(dst);
  const size_t nchunks = (bytes + kStageBytes - 1) / kStageBytes;
  auto issue = [&](size_t c) {
    const int k = (int)(c % 2);
    const size_t off = c * kStageBytes;
    QSM_CUDA(cudaMemcpyAsync(ctx->pinned[k], s + off, std::min(kStageBytes, bytes - off), cudaMemcpyDeviceToHost,
                             ctx->stream));
    QSM_CUDA(cudaEventRecord(ctx->pinned_ev[k], ctx->stream));
  };
  if (nchunks > 0) issue(0);
  for (size_t c = 0; c < nchunks; ++c) {
    if (c + 1 < nchunks) issue(c + 1);  // the other slot was drained in the previous step
    const int k = (int)(c % 2);
    QSM_CUDA(cudaEventSynchronize(ctx->pinned_ev[k]));
    const size_t off = c * kStageBytes;
    std::memcpy(d + off, ctx->pinned[k], std::min(kStageBytes, bytes - off));
  }
}

void LaunchScope::done() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw QsmError(QSM_ERR_CUDA, std::string("kernel launch (") + name + "): " + cudaGetErrorString(e));
  ctx->launches++;
  if (ctx->profiling && ev0) {
    cudaEvent_t ev1;
    QSM_CUDA(cudaEventCreate(&ev1));
    QSM_CUDA(cudaEventRecord(ev1, ctx->stream));
    ctx->prof_pending.push_back(ProfRec{ctx->prof_prefix + name, ev0, ev1});
    ev0 = nullptr;
  }
}

// Fold pending launch events into per-name totals (synchronises the stream).
void prof_collect(qsm_ctx* ctx) {
  if (ctx->prof_pending.empty()) return;
  QSM_CUDA(cudaStreamSynchronize(ctx->stream));
  for (ProfRec& r : ctx->prof_pending) {
    float ms = 0.f;
    QSM_CUDA(cudaEventElapsedTime(&ms, r.start, r.stop));
    cudaEventDestroy(r.start);
    cudaEventDestroy(r.stop);
    auto it = std::find_if(ctx->prof_stats.begin(), ctx->prof_stats.end(),
                           [&](const std::pair<std::string, ProfStat>& kv) { return kv.first == r.name; });
    if (it == ctx->prof_stats.end()) {
      ctx->prof_stats.push_back({r.name, ProfStat{}});
      it = ctx->prof_stats.end() - 1;
    }
    it->second.launches += 1;
    it->second.total_ms += ms;
  }
  ctx->prof_pending.clear();
}

}  // namespace qsm

using namespace qsm;

extern "C" {

qsm_status qsm_ctx_create(int device, int precision, qsm_ctx** out) {
  if (out == nullptr) return QSM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (precision != QSM_PRECISION_F64 && precision != QSM_PRECISION_MIXED) return QSM_ERR_INVALID_ARGUMENT;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    (void)cudaGetLastError();
    return QSM_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) return QSM_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) return QSM_ERR_CUDA;
  qsm_ctx* c = new (std::nothrow) qsm_ctx();
  if (!c) return QSM_ERR_ALLOC;
  c->device = device;
  c->precision = precision;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return QSM_ERR_CUDA;
  }
  *out = c;
  return QSM_OK;
}

qsm_status qsm_ctx_destroy(qsm_ctx* ctx) {
  if (ctx == nullptr) return QSM_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  ws_release(ctx);
  for (auto& kv : ctx->twiddles) cudaFree(kv.second);
  for (auto& kv : ctx->tables) cudaFree(kv.second);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  for (int k = 0; k < 2; ++k) {
    if (ctx->pinned[k]) cudaFreeHost(ctx->pinned[k]);
    if (ctx->pinned_ev[k]) cudaEventDestroy(ctx->pinned_ev[k]);
  }
  delete ctx;
  return QSM_OK;
}

qsm_status qsm_ctx_set_precision(qsm_ctx* ctx, int precision) {
  if (ctx == nullptr) return QSM_ERR_INVALID_ARGUMENT;
  if (precision != QSM_PRECISION_F64 && precision != QSM_PRECISION_MIXED) {
    ctx->err = "unknown precision";
    return QSM_ERR_INVALID_ARGUMENT;
  }
  ctx->precision = precision;
  return QSM_OK;
}

int qsm_ctx_get_precision(const qsm_ctx* ctx) { return ctx ? ctx->precision : -1; }

qsm_status qsm_ctx_set_plan_mode(qsm_ctx* ctx, int mode) {
  if (ctx == nullptr) return QSM_ERR_INVALID_ARGUMENT;
  if (mode != QSM_PLANS_COMPILED && mode != QSM_PLANS_RUNTIME) {
    ctx->err = "unknown plan mode";
    return QSM_ERR_INVALID_ARGUMENT;
  }
  ctx->plan_mode = mode;
  return QSM_OK;
}

int qsm_ctx_get_plan_mode(const qsm_ctx* ctx) { return ctx ? ctx->plan_mode : -1; }

qsm_status qsm_ctx_set_krylov_precision(qsm_ctx* ctx, int precision) {
  if (ctx == nullptr) return QSM_ERR_INVALID_ARGUMENT;
  if (precision != QSM_PRECISION_F64 && precision != QSM_PRECISION_MIXED) {
    ctx->err = "unknown precision";
    return QSM_ERR_INVALID_ARGUMENT;
  }
  ctx->krylov_precision = precision;
  return QSM_OK;
}

int qsm_ctx_get_krylov_precision(const qsm_ctx* ctx) { return ctx ? ctx->krylov_precision : -1; }

qsm_status qsm_ctx_set_input_check(qsm_ctx* ctx, int on) {
  if (ctx == nullptr) return QSM_ERR_INVALID_ARGUMENT;
  ctx->check_inputs = on != 0;
  return QSM_OK;
}

qsm_status qsm_ctx_set_autotune(qsm_ctx* ctx, int on) {
  if (ctx == nullptr) return QSM_ERR_INVALID_ARGUMENT;
  ctx->autotune = on != 0;
  return QSM_OK;
}

qsm_status qsm_ctx_force_launch_shape(qsm_ctx* ctx, int shape) {
  if (ctx == nullptr) return QSM_ERR_INVALID_ARGUMENT;
  if (shape < -1 || shape > kTuneMaxShape) {
    ctx->err = "launch shape must be -1 (none) or 0.." + std::to_string(kTuneMaxShape);
    return QSM_ERR_INVALID_ARGUMENT;
  }
  ctx->forced_shape = shape;
  return QSM_OK;
}

size_t qsm_ctx_autotune_count(const qsm_ctx* ctx) { return ctx ? ctx->tuned.size() : 0; }

qsm_status qsm_ctx_autotune_entry(const qsm_ctx* ctx, size_t i, char* key, size_t key_cap, int* choice,
                                  int* candidates, float* us, size_t cap, size_t* count) {
  if (ctx == nullptr || i >= ctx->tuned.size()) return QSM_ERR_INVALID_ARGUMENT;
  auto it = ctx->tuned.begin();
  std::advance(it, (long)i);
  if (key != nullptr && key_cap > 0) {
    const size_t n = std::min(key_cap - 1, it->first.size());
    std::memcpy(key, it->first.data(), n);
    key[n] = '\0';
  }
  if (choice) *choice = it->second.choice;
  const size_t n = it->second.us.size();
  if (count) *count = n;
  for (size_t k = 0; k < n && k < cap; ++k) {
    if (candidates) candidates[k] = it->second.us[k].first;
    if (us) us[k] = it->second.us[k].second;
  }
  return QSM_OK;
}

qsm_status qsm_ctx_inject_alloc_failure(qsm_ctx* ctx, long long after) {
  if (ctx == nullptr) return QSM_ERR_INVALID_ARGUMENT;
  ctx->alloc_fail_after = after < 0 ? -1 : after;
  return QSM_OK;
}

qsm_status qsm_ctx_release_workspace(qsm_ctx* ctx) {
  if (ctx == nullptr) return QSM_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  ws_release(ctx);
  return QSM_OK;
}

const char* qsm_last_error(const qsm_ctx* ctx) {
  if (ctx == nullptr) return "null context";
  return ctx->err.c_str();
}

uint64_t qsm_ctx_kernel_launches(const qsm_ctx* ctx) { return ctx ? ctx->launches : 0; }

void* qsm_ctx_stream(const qsm_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

const char* qsm_version(void) { return "qsmgpu 0.1.0 (sm_100a)"; }

qsm_status qsm_ctx_set_profiling(qsm_ctx* ctx, int on) {
  return guarded(ctx, [&] {
    prof_collect(ctx);
    ctx->profiling = on != 0;
  });
}

qsm_status qsm_ctx_profile_reset(qsm_ctx* ctx) {
  return guarded(ctx, [&] {
    prof_collect(ctx);
    ctx->prof_stats.clear();
  });
}

size_t qsm_ctx_profile_count(qsm_ctx* ctx) {
  if (!ctx) return 0;
  if (guarded(ctx, [&] { prof_collect(ctx); }) != QSM_OK) return 0;
  return ctx->prof_stats.size();
}

qsm_status qsm_ctx_profile_entry(qsm_ctx* ctx, size_t i, char* name, size_t name_cap, uint64_t* launches,
                                 double* total_ms) {
  return guarded(ctx, [&] {
    prof_collect(ctx);
    if (i >= ctx->prof_stats.size()) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "profile index out of range");
    const auto& kv = ctx->prof_stats[i];
    if (name && name_cap) {
      std::strncpy(name, kv.first.c_str(), name_cap - 1);
      name[name_cap - 1] = 0;
    }
    if (launches) *launches = kv.second.launches;
    if (total_ms) *total_ms = kv.second.total_ms;
  });
}

int qsm_grid_supported(const qsm_grid* grid) {
  if (grid == nullptr) return 0;
  return fft_length_supported((int)grid->nx) && fft_length_supported((int)grid->ny) &&
         fft_length_supported((int)grid->nz);
}

void qsm_tv_params_default(qsm_tv_params* p) {
  if (!p) return;
  p->lambda = 2e-4;
  p->rho = 2e-2;
  p->tol = 1e-3;
  p->max_iter = 250;
}
void qsm_tkd_params_default(qsm_tkd_params* p) {
  if (p) p->threshold = 0.15;
}
void qsm_tikhonov_params_default(qsm_tikhonov_params* p) {
  if (!p) return;
  p->lambda = 0.01;
  p->reg = QSM_REG_IDENTITY;
}
void qsm_sharp_params_default(qsm_sharp_params* p) {
  if (!p) return;
  p->threshold = 0.05;
  p->radius = 6.0;
}
void qsm_vsharp_params_default(qsm_vsharp_params* p) {
  if (!p) return;
  p->threshold = 0.05;
  p->max_radius = 12.0;
  p->min_radius = 1.0;
}

}  // extern "C"
