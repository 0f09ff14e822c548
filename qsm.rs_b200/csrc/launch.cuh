// Host launchers for the pass kernels, the per-grid transform bundle and the
// double-precision k-space geometry shared by every spectral multiplier.
#pragma once

#include "internal.h"
#include "passes.cuh"

namespace qsm {

template <typename T> struct Fft3 {
  Geom g;
  FftPlan1D px, py, pz;
  const cplx_t<T>* twx;
  const cplx_t<T>* twy;
  const cplx_t<T>* twz;
};

// Point each Bluestein plan at the chirp and kernel spectrum that follow the stage
// twiddles in its table.
template <typename T> void attach_tables(Fft3<T>& f) {
  f.px.ext = f.px.m != f.px.n ? (const void*)(f.twx + f.px.m) : nullptr;
  f.py.ext = f.py.m != f.py.n ? (const void*)(f.twy + f.py.m) : nullptr;
  f.pz.ext = f.pz.m != f.pz.n ? (const void*)(f.twz + f.pz.m) : nullptr;
}

template <typename T> Fft3<T> make_fft3(qsm_ctx* ctx, const GridDims& d) {
  Fft3<T> f;
  f.g.nx = d.nx;
  f.g.ny = d.ny;
  f.g.nz = d.nz;
  f.g.nxh = d.nx / 2 + 1;
  // rows start on 32-byte boundaries in both precisions, and float and double
  // spectra of one grid share a layout (mixed-precision ops index both)
  f.g.pitch = (f.g.nxh + 3) / 4 * 4;
  f.px = plan_or_throw(d.nx);
  f.py = plan_or_throw(d.ny);
  f.pz = plan_or_throw(d.nz);
  const bool dbl = sizeof(T) == 8;
  f.twx = (const cplx_t<T>*)twiddle_table(ctx, f.px, dbl);
  f.twy = (const cplx_t<T>*)twiddle_table(ctx, f.py, dbl);
  f.twz = (const cplx_t<T>*)twiddle_table(ctx, f.pz, dbl);
  attach_tables(f);
  return f;
}

// Raise a kernel's dynamic shared-memory limit when a launch needs more than the
// default 48 KB (tracked per kernel function and device, under a lock).
void raise_smem_limit(const void* func, int device, size_t bytes);
template <class K> void ensure_smem(K kernel, size_t bytes) {
  if (bytes > 227u * 1024u) throw QsmError(QSM_ERR_UNSUPPORTED_SIZE, "transform tile exceeds shared memory");
  int dev = 0;
  QSM_CUDA(cudaGetDevice(&dev));
  raise_smem_limit(reinterpret_cast<const void*>(kernel), dev, bytes);
}

// False when the context runs every pass on the runtime engine (QSM_PLANS_RUNTIME).
inline bool compiled_plans(const qsm_ctx* ctx) { return ctx->plan_mode == QSM_PLANS_COMPILED; }

inline void after_launch(qsm_ctx* ctx) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw QsmError(QSM_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  ctx->launches++;
}

// Threads per pencil in the X passes: the plan's T rounded up to a divisor of 32
// (T <= 32) or to a multiple of 32, so that a block is a whole number of warps.
inline int x_block_t(int T_) {
  if (T_ <= 32) {
    int b = 1;
    while (b < T_) b <<= 1;
    return b;
  }
  return (T_ + 31) / 32 * 32;
}

template <typename T> inline int x_pencils_per_block(int T_) {
  int P = 256 / x_block_t(T_);
  if (P < 1) P = 1;
  return P;
}

template <typename T> inline long long x_blocks(const Fft3<T>& f) {
  // the X kernels hold a row's elements (<= kFftEmax) and half-spectrum entries
  // (<= kXHalfMax) per thread in fixed register arrays
  if ((f.px.n + f.px.T - 1) / f.px.T > kFftEmax || (f.g.nxh + f.px.T - 1) / f.px.T > kXHalfMax)
    throw QsmError(QSM_ERR_UNSUPPORTED_SIZE, "x length outside the per-thread register budget");
  const int P = x_pencils_per_block<T>(f.px.T);
  const long long npairs = ((long long)f.g.nrows() + 1) / 2;
  return (npairs + P - 1) / P;
}

// Compile-time X kernels (float) for the lengths of QSM_FIXED_PLANS (and of
// QSM_FIXED_PLANS_WIDE when W); false when the plan is not one of them.
template <typename T, bool W, bool DEAD, class Load>
bool run_x_r2c_fixed(qsm_ctx* ctx, const Fft3<T>& f, cplx_t<T>* spec, const Load& ld, const int* done) {
  if (!compiled_plans(ctx)) return false;
  if constexpr (!std::is_same<T, float>::value && !W) {
    return false;
  } else {
    using C = cplx_t<T>;
#define QSM_TRY_XR(N_, T_, R0_, R1_, R2_)                                                          \
    if (FixedPlan<N_, T_, R0_, R1_, R2_>::matches(f.px)) {                                         \
      using FP = FixedPlan<N_, T_, R0_, R1_, R2_>;                                                 \
      const int Tt = x_block_t(T_);                                                                \
      const int P = x_pencils_per_block<T>(T_);                                                    \
      const size_t smem = (size_t)(x_tw_len<T>(N_) + P * x_rowlen<T>(N_)) * sizeof(C);            \
      auto kern = k_x_r2c_fx<T, FP, Load, DEAD>;                                                   \
      ensure_smem(kern, smem);                                                                     \
      LaunchScope ls(ctx, "fft_x_r2c");                                                            \
      kern<<<(unsigned)x_blocks(f), dim3(Tt, P), smem, ctx->stream>>>(f.g, f.twx, spec, ld, done); \
      ls.done();                                                                                   \
      return true;                                                                                 \
    }
    QSM_FIXED_PLANS(QSM_TRY_XR)
    if constexpr (W) {
      QSM_FIXED_PLANS_WIDE(QSM_TRY_XR)
    }
#undef QSM_TRY_XR
    return false;
  }
}

template <typename T, bool W, bool DEAD, class Store>
bool run_x_c2r_fixed(qsm_ctx* ctx, const Fft3<T>& f, const cplx_t<T>* spec, const Store& st, const int* done) {
  if (!compiled_plans(ctx)) return false;
  if constexpr (!std::is_same<T, float>::value && !W) {
    return false;
  } else {
    using C = cplx_t<T>;
#define QSM_TRY_XC(N_, T_, R0_, R1_, R2_)                                                          \
    if (FixedPlan<N_, T_, R0_, R1_, R2_>::matches(f.px)) {                                         \
      using FP = FixedPlan<N_, T_, R0_, R1_, R2_>;                                                 \
      const int Tt = x_block_t(T_);                                                                \
      const int P = x_pencils_per_block<T>(T_);                                                    \
      const size_t smem = (size_t)(x_tw_len<T>(N_) + P * x_rowlen<T>(N_)) * sizeof(C);            \
      auto kern = k_x_c2r_fx<T, FP, Store, DEAD>;                                                  \
      ensure_smem(kern, smem);                                                                     \
      LaunchScope ls(ctx, "fft_x_c2r");                                                            \
      kern<<<(unsigned)x_blocks(f), dim3(Tt, P), smem, ctx->stream>>>(f.g, f.twx, spec, st, done); \
      ls.done();                                                                                   \
      return true;                                                                                 \
    }
    QSM_FIXED_PLANS(QSM_TRY_XC)
    if constexpr (W) {
      QSM_FIXED_PLANS_WIDE(QSM_TRY_XC)
    }
#undef QSM_TRY_XC
    return false;
  }
}

// DEAD (compile-time kernels only): the pass reads ld's rows for the last time and drops
// their L2 lines (k_x_r2c_fx); ld then provides row_begin.
template <typename T, bool W = false, bool DEAD = false, class Load>
void run_x_r2c(qsm_ctx* ctx, const Fft3<T>& f, cplx_t<T>* spec, const Load& ld, const int* done) {
  if (run_x_r2c_fixed<T, W, DEAD>(ctx, f, spec, ld, done)) return;
  using C = cplx_t<T>;
  const int Tt = x_block_t(f.px.T);
  const int P = x_pencils_per_block<T>(f.px.T);
  const size_t smem = (size_t)(f.px.m + P * x_rowlen<T>(f.px.m)) * sizeof(C);
  auto kern = f.px.m != f.px.n ? k_x_r2c<T, Load, true> : k_x_r2c<T, Load, false>;
  ensure_smem(kern, smem);
  LaunchScope ls(ctx, "fft_x_r2c");
  kern<<<(unsigned)x_blocks(f), dim3(Tt, P), smem, ctx->stream>>>(f.g, f.px, f.twx, spec, ld, done);
  ls.done();
}

// DEAD (compile-time kernels only): the pass reads the half spectrum for the last time and
// drops its L2 lines (k_x_c2r_fx).
template <typename T, bool W = false, bool DEAD = false, class Store>
void run_x_c2r(qsm_ctx* ctx, const Fft3<T>& f, const cplx_t<T>* spec, const Store& st, const int* done) {
  if (run_x_c2r_fixed<T, W, DEAD>(ctx, f, spec, st, done)) return;
  using C = cplx_t<T>;
  const int Tt = x_block_t(f.px.T);
  const int P = x_pencils_per_block<T>(f.px.T);
  const size_t smem = (size_t)(f.px.m + P * x_rowlen<T>(f.px.m)) * sizeof(C);
  auto kern = f.px.m != f.px.n ? k_x_c2r<T, Store, true> : k_x_c2r<T, Store, false>;
  ensure_smem(kern, smem);
  LaunchScope ls(ctx, "fft_x_c2r");
  kern<<<(unsigned)x_blocks(f), dim3(Tt, P), smem, ctx->stream>>>(f.g, f.px, f.twx, spec, st, done);
  ls.done();
}

// Transform bundle for full complex spectra (complex-to-complex along x too): every
// x column is valid, rows padded to a multiple of 4 values.
template <typename T> Fft3<T> make_fft3_full(qsm_ctx* ctx, const GridDims& d) {
  Fft3<T> f = make_fft3<T>(ctx, d);
  f.g.nxh = d.nx;
  f.g.pitch = (d.nx + 3) / 4 * 4;
  return f;
}

// Identity pointwise hook of k_x_full.
template <typename T> struct MidId {
  __device__ __forceinline__ cplx_t<T> operator()(cplx_t<T> v, int, int) const { return v; }
};

// X pass over full complex rows: load -> FFT(D1) -> mid -> FFT(D2) -> store.
// W: a hot loop's pass; with both transforms it takes the compile-time kernel
// (k_x_full_fx) for the lengths of QSM_FIXED_PLANS (FP64 384: 96 registers against the
// runtime engine's 130, two blocks per SM instead of one).
template <typename T, int D1, int D2, bool W = false, class Load, class Mid, class Store>
void run_x_full(qsm_ctx* ctx, const Fft3<T>& f, const Load& ld, const Mid& mid, const Store& st, const int* done,
                const char* name) {
  using C = cplx_t<T>;
  if constexpr (W && D1 != 0 && D2 != 0) {
    if (compiled_plans(ctx)) {
#define QSM_TRY_XF(N_, T_, R0_, R1_, R2_)                                                          \
    if (FixedPlan<N_, T_, R0_, R1_, R2_>::matches(f.px)) {                                         \
      using FP = FixedPlan<N_, T_, R0_, R1_, R2_>;                                                 \
      const int Tt = x_block_t(T_);                                                                \
      const int P = x_pencils_per_block<T>(T_);                                                    \
      const size_t smem = (size_t)(x_tw_len<T>(N_) + P * x_rowlen<T>(N_)) * sizeof(C);            \
      auto kern = k_x_full_fx<T, FP, D1, D2, Load, Mid, Store>;                                    \
      ensure_smem(kern, smem);                                                                     \
      const long long blocks = ((long long)f.g.nrows() + P - 1) / P;                              \
      LaunchScope ls(ctx, name);                                                                   \
      kern<<<(unsigned)blocks, dim3(Tt, P), smem, ctx->stream>>>(f.g, f.twx, ld, mid, st, done);   \
      ls.done();                                                                                   \
      return;                                                                                      \
    }
    QSM_FIXED_PLANS(QSM_TRY_XF)
#undef QSM_TRY_XF
    }
  }
  if ((f.px.n + f.px.T - 1) / f.px.T > kFftEmax)
    throw QsmError(QSM_ERR_UNSUPPORTED_SIZE, "x length outside the per-thread register budget");
  const int Tt = x_block_t(f.px.T);
  const int P = x_pencils_per_block<T>(f.px.T);
  const size_t smem = (size_t)(f.px.m + P * x_rowlen<T>(f.px.m)) * sizeof(C);
  auto kern = f.px.m != f.px.n ? k_x_full<T, D1, D2, Load, Mid, Store, true>
                                : k_x_full<T, D1, D2, Load, Mid, Store, false>;
  ensure_smem(kern, smem);
  const long long blocks = ((long long)f.g.nrows() + P - 1) / P;
  LaunchScope ls(ctx, name);
  kern<<<(unsigned)blocks, dim3(Tt, P), smem, ctx->stream>>>(f.g, f.px, f.twx, ld, mid, st, done);
  ls.done();
}

template <typename T> inline int yz_cols() { return sizeof(T) == 4 ? 16 : 8; }

int sm_count_of(int device);  // multiprocessor count, cached per device under a lock
inline int sm_count(qsm_ctx* ctx) { return sm_count_of(ctx->device); }

// Persistent grid: as many CTAs as fit on the device at once, capped by the work.
template <class K> unsigned persistent_grid(qsm_ctx* ctx, K kernel, int threads, size_t smem, long long work) {
  int per_sm = 0;
  QSM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
  if (per_sm < 1) throw QsmError(QSM_ERR_UNSUPPORTED_SIZE, "transform tile does not fit on an SM");
  long long g = (long long)per_sm * sm_count(ctx);
  if (g > work) g = work;
  if (g < 1) g = 1;
  return (unsigned)g;
}

// Tile walk of a Y (axis 1) or Z (axis 2) pass with P-column tiles.  edge: walk a
// narrow column remainder (at most P/4 columns) as edge tiles (TileWalk); only the
// compile-time kernels read edge tiles.
template <typename T> TileWalk tile_walk(const Fft3<T>& f, int axis, int P, bool edge = false) {
  TileWalk w;
  w.ntx = (f.g.nxh + P - 1) / P;
  w.nouter = axis == 1 ? f.g.nz : f.g.ny;
  if (axis == 1) {  // Y: outer = z
    w.ostride = (long long)f.g.pitch * f.g.ny;
    w.estride = f.g.pitch;
  } else {  // Z: outer = y
    w.ostride = f.g.pitch;
    w.estride = (long long)f.g.pitch * f.g.ny;
  }
  const int rem = f.g.nxh % P;
  w.nedge = 0;
  w.col_edge = f.g.nxh;
  if (edge && rem > 0 && 4 * rem <= P) {
    w.ntx = f.g.nxh / P;
    w.nedge = rem;
    w.col_edge = w.ntx * P;
  }
  w.nmain = w.ntx * w.nouter;
  w.ntiles = w.nmain + w.nedge * ((w.nouter + P - 1) / P);
  return w;
}
// True when tile_walk(..., edge = true) has edge tiles.
template <typename T> bool has_edge_tiles(const Fft3<T>& f, int P) {
  const int rem = f.g.nxh % P;
  return rem > 0 && 4 * rem <= P;
}

// shared memory of the direct-fetch kernels: twiddles + one tile (the stage exchange)
template <typename T> inline size_t dx_smem(int n, int P) {
  return (size_t)(((n + 7) & ~7) + (size_t)n * P) * sizeof(cplx_t<T>);
}

template <typename T> inline size_t yz_smem(int n, int P) {
  return (size_t)(((n + 7) & ~7) + 2 * (size_t)n * P) * sizeof(cplx_t<T>);
}

// Tile width for a Y/Z pass: 128-byte rows, halved while the block (P x T threads)
// does not fit on an SM (long axes: many threads, registers, shared memory).
template <typename T, class K> int yz_tile_width(K kernel, int n, int Tn) {
  constexpr int kMinP = 16 / (int)sizeof(cplx_t<T>) > 0 ? 16 / (int)sizeof(cplx_t<T>) : 1;
  for (int P = yz_cols<T>(); P >= kMinP; P /= 2) {
    if (P * Tn > 1024) continue;
    const size_t smem = yz_smem<T>(n, P);
    if (smem > 227u * 1024u) continue;
    ensure_smem(kernel, smem);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, P * Tn, smem) != cudaSuccess) {
      (void)cudaGetLastError();
      continue;
    }
    if (per_sm >= 1) return P;
  }
  throw QsmError(QSM_ERR_UNSUPPORTED_SIZE, "axis of length " + std::to_string(n) + " does not fit one tile");
}

// Columns per tile of the compile-time Y/Z passes: 128-byte tile rows (16 float or 8
// double complex values).
template <typename T> constexpr int fx_cols() { return sizeof(T) == 4 ? 16 : 8; }
constexpr int kZmCols = 8;  // columns per tile of the fused Z pass

// ----------------------------------------------------------------- autotuner --
// Launch shapes of the compile-time Y/Z passes, as fields of a candidate number:
//   kTuneEdge         edge tiles for a narrow column remainder (TileWalk)
//   kTuneBlockPerTile one block per tile, scheduled by the hardware, instead of a
//                     persistent grid of resident blocks walking the tiles
//   bits 2..5         persistent grid: resident blocks per SM (0 = as many as fit)
// Every shape runs the same arithmetic on every column, so results do not depend on the
// choice.  The choice is made per context by timing each candidate once on scratch
// buffers (autotune_pick) and cached under a key naming the pass and its geometry;
// launches whose key is not cached use shape 0, the persistent grid without edge tiles.
constexpr int kTuneEdge = 1, kTuneBlockPerTile = 2, kTuneBpsmShift = 2;  // kTuneMaxShape: internal.h
inline int tune_bpsm(int shape) { return (shape >> kTuneBpsmShift) & 15; }
bool stream_capturing(qsm_ctx* ctx);
// Time launch(c) for every candidate c on ctx->stream (after one warm-up launch each,
// `rounds` rounds of `reps` launches; the best round counts) and cache the fastest under key.
void autotune_pick(qsm_ctx* ctx, const std::string& key, const std::vector<int>& cands,
                   const std::function<void(int)>& launch, int rounds = 3, int reps = 5);
inline int tuned_shape(const qsm_ctx* ctx, const std::string& key) {
  if (ctx->forced_shape >= 0) return ctx->forced_shape;
  if (!ctx->autotune) return 0;
  auto it = ctx->tuned.find(key);
  return it == ctx->tuned.end() ? 0 : it->second.choice;
}
// Whether a tuning run for key should happen now (autotuner on, key not cached, stream
// not capturing).
inline bool autotune_due(qsm_ctx* ctx, const std::string& key) {
  return ctx->autotune && ctx->forced_shape < 0 && ctx->tuned.find(key) == ctx->tuned.end() && !stream_capturing(ctx);
}
template <typename T> std::string yz_tune_key(const char* pass, const Fft3<T>& f, int axis, int dir) {
  return std::string(pass) + (axis == 1 ? ":y" : ":z") + (dir < 0 ? "-" : "+") + ":" + std::to_string(f.g.nx) +
         "x" + std::to_string(f.g.ny) + "x" + std::to_string(f.g.nz) + (sizeof(T) == 4 ? ":f32" : ":f64");
}
// Candidates: persistent grids of the occupancy limit and of one block per SM fewer,
// and one block per tile, each with and without edge tiles where the grid has them.
template <typename T, class K>
std::vector<int> yz_candidates(const Fft3<T>& f, int P, K kern, int threads, size_t smem) {
  int per_sm = 0;
  QSM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
  std::vector<int> base{0, kTuneBlockPerTile};
  if (per_sm >= 2 && per_sm - 1 <= 15) base.push_back((per_sm - 1) << kTuneBpsmShift);
  std::vector<int> c = base;
  if (has_edge_tiles(f, P))
    for (int b : base) c.push_back(b | kTuneEdge);
  return c;
}

// Grid of a compile-time Y/Z pass over `work` tiles: resident blocks (persistent) or one
// block per tile; false when the block does not fit on an SM.
template <class K>
bool fx_launch_ok(qsm_ctx* ctx, K kern, int threads, size_t smem, unsigned* grid, long long work,
                  bool per_tile = false, int bpsm = 0) {
  if (smem > 227u * 1024u) return false;
  ensure_smem(kern, smem);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  if (per_sm < 1) return false;
  if (bpsm > 0 && bpsm < per_sm) per_sm = bpsm;
  long long g = per_tile ? work : (long long)per_sm * sm_count(ctx);
  if (g > work) g = work;
  *grid = (unsigned)(g < 1 ? 1 : g);
  return true;
}

// One compile-time Y/Z pass (k_pass_yz_dx, FP a FixedPlan) in launch shape `shape`.
// scoped: count and (when profiling) time the launch under the pass's name.
template <typename T, int DIR, int AXIS, class FP>
bool launch_yz_fx(qsm_ctx* ctx, const Fft3<T>& f, int shape, const cplx_t<T>* src, cplx_t<T>* dst,
                  const int* done, bool scoped) {
  const cplx_t<T>* tw = (AXIS == 1) ? f.twy : f.twz;
  auto kern = k_pass_yz_dx<T, DIR, FP, fx_cols<T>()>;
  const size_t smem = dx_smem<T>(FP::n, fx_cols<T>());
  const TileWalk w = tile_walk(f, AXIS, fx_cols<T>(), (shape & kTuneEdge) != 0);
  unsigned grid = 0;
  if (!fx_launch_ok(ctx, kern, fx_cols<T>() * FP::T, smem, &grid, w.ntiles, (shape & kTuneBlockPerTile) != 0,
                    tune_bpsm(shape)))
    return false;
  if (!scoped) {
    kern<<<grid, dim3(fx_cols<T>(), FP::T), smem, ctx->stream>>>(f.g, w, tw, src, dst, done);
    return true;
  }
  LaunchScope ls(ctx, AXIS == 1 ? (DIR < 0 ? "fft_y_fwd" : "fft_y_inv") : (DIR < 0 ? "fft_z_fwd" : "fft_z_inv"));
  kern<<<grid, dim3(fx_cols<T>(), FP::T), smem, ctx->stream>>>(f.g, w, tw, src, dst, done);
  ls.done();
  return true;
}

// Compile-time Y/Z kernels (fx_cols<T>() columns per tile) for the axis lengths of
// QSM_FIXED_PLANS (and QSM_FIXED_PLANS_WIDE when W); returns false when the plan is not
// one of them.
template <typename T, int DIR, int AXIS, bool W>
bool run_yz_fixed(qsm_ctx* ctx, const Fft3<T>& f, const cplx_t<T>* src, cplx_t<T>* dst, const int* done) {
  if (!compiled_plans(ctx)) return false;
  {
    const FftPlan1D& pl = (AXIS == 1) ? f.py : f.pz;
#define QSM_TRY_YZ(N_, T_, R0_, R1_, R2_)                                                         \
    if (FixedPlan<N_, T_, R0_, R1_, R2_>::matches(pl) && fx_cols<T>() * T_ <= 1024) {                   \
      using FP = FixedPlan<N_, T_, R0_, R1_, R2_>;                                                \
      const int shape = tuned_shape(ctx, yz_tune_key<T>("yz_fx", f, AXIS, DIR));                  \
      return launch_yz_fx<T, DIR, AXIS, FP>(ctx, f, shape, src, dst, done, true);                 \
    }
    QSM_FIXED_PLANS(QSM_TRY_YZ)
    if constexpr (W) {
      QSM_FIXED_PLANS_WIDE(QSM_TRY_YZ)
    }
#undef QSM_TRY_YZ
    return false;
  }
}

constexpr int kMaxPersistentBlocks = 4096;

// One compile-time operator pass: k_pass_yz_dx_old when the op's epilogue reads a second
// array (ACC only), k_pass_yz_st_op when its pre hook wants a staged tile, else
// k_pass_yz_dx_op.  False when the block does not fit.
template <typename T, int DIR, int AXIS, bool ACC, class FP, class Op>
bool launch_yz_op_fx(qsm_ctx* ctx, const Fft3<T>& f, const cplx_t<T>* tw, const cplx_t<T>* src, cplx_t<T>* dst,
                     const Op& op, double* partials, unsigned* counter, const int* done, const char* name) {
  constexpr int P = fx_cols<T>();
  const TileWalk w = tile_walk(f, AXIS, P);
  unsigned grid = 0;
  if constexpr (ACC && ReadsOld<Op>::value) {
    auto kern = k_pass_yz_dx_old<T, DIR, AXIS, FP, P, Op>;
    const size_t smem = dx_smem<T>(FP::n, P) + (size_t)FP::n * P * sizeof(cplx_t<T>);
    if (!fx_launch_ok(ctx, kern, P * FP::T, smem, &grid, w.ntiles)) return false;
    if (grid > (unsigned)kMaxPersistentBlocks) return false;
    LaunchScope ls(ctx, name);
    kern<<<grid, dim3(P, FP::T), smem, ctx->stream>>>(f.g, w, tw, src, dst, op, partials, counter, done);
    ls.done();
  } else if constexpr (!ACC && StagedPre<Op>::value) {
    auto kern = k_pass_yz_st_op<T, DIR, AXIS, FP, P, Op>;
    const size_t smem = yz_smem<T>(FP::n, P);
    if (!fx_launch_ok(ctx, kern, P * FP::T, smem, &grid, w.ntiles)) return false;
    LaunchScope ls(ctx, name);
    kern<<<grid, dim3(P, FP::T), smem, ctx->stream>>>(f.g, w, tw, src, dst, op, done);
    ls.done();
  } else {
    auto kern = k_pass_yz_dx_op<T, DIR, AXIS, FP, P, Op, ACC>;
    const size_t smem = dx_smem<T>(FP::n, P);
    if (!fx_launch_ok(ctx, kern, P * FP::T, smem, &grid, w.ntiles)) return false;
    if (ACC && grid > (unsigned)kMaxPersistentBlocks) return false;
    LaunchScope ls(ctx, name);
    kern<<<grid, dim3(P, FP::T), smem, ctx->stream>>>(f.g, w, tw, src, dst, op, partials, counter, done);
    ls.done();
  }
  return true;
}

// Compile-time Y/Z pass that carries an operator (k_pass_yz_dx_op), lengths of
// QSM_FIXED_PLANS; ACC as in run_yz_acc.  Returns false when the plan is not one of them.
template <typename T, int DIR, int AXIS, bool ACC, class Op>
bool run_yz_op_fixed(qsm_ctx* ctx, const Fft3<T>& f, const cplx_t<T>* src, cplx_t<T>* dst, const Op& op,
                     double* partials, unsigned* counter, const int* done, const char* name) {
  if (!compiled_plans(ctx)) return false;
  {
    const FftPlan1D& pl = (AXIS == 1) ? f.py : f.pz;
    const cplx_t<T>* tw = (AXIS == 1) ? f.twy : f.twz;
#define QSM_TRY_YZO(N_, T_, R0_, R1_, R2_)                                                         \
    if (FixedPlan<N_, T_, R0_, R1_, R2_>::matches(pl) && fx_cols<T>() * T_ <= 1024)                \
      return launch_yz_op_fx<T, DIR, AXIS, ACC, FixedPlan<N_, T_, R0_, R1_, R2_>>(ctx, f, tw, src, dst, op, partials, \
                                                                                counter, done, name);
    QSM_FIXED_PLANS(QSM_TRY_YZO)
#undef QSM_TRY_YZO
    return false;
  }
}

// AXIS 1 = y, 2 = z; DIR -1 forward, +1 inverse; W adds QSM_FIXED_PLANS_WIDE for plain
// passes and the compile-time operator pass (QSM_FIXED_PLANS) for the others.
template <typename T, int DIR, int AXIS, bool W = false, class Op>
void run_yz(qsm_ctx* ctx, const Fft3<T>& f, const cplx_t<T>* src, cplx_t<T>* dst, const Op& op, const int* done) {
  if constexpr (IsPlainOp<Op>::value) {
    if (run_yz_fixed<T, DIR, AXIS, W>(ctx, f, src, dst, done)) return;
  } else if constexpr (W) {
    if (run_yz_op_fixed<T, DIR, AXIS, false>(ctx, f, src, dst, op, nullptr, nullptr, done,
                                             AXIS == 1 ? (DIR < 0 ? "fft_y_fwd" : "fft_y_inv")
                                                       : (DIR < 0 ? "fft_z_fwd" : "fft_z_inv")))
      return;
  }
  const FftPlan1D& pl = (AXIS == 1) ? f.py : f.pz;
  const cplx_t<T>* tw = (AXIS == 1) ? f.twy : f.twz;
  auto kern = pl.m != pl.n ? k_pass_yz<T, DIR, AXIS, Op, true> : k_pass_yz<T, DIR, AXIS, Op, false>;
  const int P = yz_tile_width<T>(kern, pl.m, pl.T);
  const size_t smem = yz_smem<T>(pl.m, P);
  const TileWalk w = tile_walk(f, AXIS, P);
  const unsigned grid = persistent_grid(ctx, kern, P * pl.T, smem, w.ntiles);
  LaunchScope ls(ctx, AXIS == 1 ? (DIR < 0 ? "fft_y_fwd" : "fft_y_inv") : (DIR < 0 ? "fft_z_fwd" : "fft_z_inv"));
  kern<<<grid, dim3(P, pl.T), smem, ctx->stream>>>(f.g, pl, w, tw, src, dst, op, done);
  ls.done();
}

// Y/Z pass with an FP64 accumulation in its post hook (k_pass_yz_acc).  `partials`
// holds at least kMaxPersistentBlocks doubles; `counter` is 0 between launches.
template <typename T, int DIR, int AXIS, bool W = false, class Op>
void run_yz_acc(qsm_ctx* ctx, const Fft3<T>& f, const cplx_t<T>* src, cplx_t<T>* dst, const Op& op,
                double* partials, unsigned* counter, const int* done, const char* name) {
  if constexpr (W) {
    if (run_yz_op_fixed<T, DIR, AXIS, true>(ctx, f, src, dst, op, partials, counter, done, name)) return;
  }
  const FftPlan1D& pl = (AXIS == 1) ? f.py : f.pz;
  const cplx_t<T>* tw = (AXIS == 1) ? f.twy : f.twz;
  auto kern = pl.m != pl.n ? k_pass_yz_acc<T, DIR, AXIS, Op, true> : k_pass_yz_acc<T, DIR, AXIS, Op, false>;
  const int P = yz_tile_width<T>(kern, pl.m, pl.T);
  const size_t smem = yz_smem<T>(pl.m, P);
  const TileWalk w = tile_walk(f, AXIS, P);
  unsigned grid = persistent_grid(ctx, kern, P * pl.T, smem, w.ntiles);
  if (grid > (unsigned)kMaxPersistentBlocks) grid = kMaxPersistentBlocks;
  LaunchScope ls(ctx, name);
  kern<<<grid, dim3(P, pl.T), smem, ctx->stream>>>(f.g, pl, w, tw, src, dst, op, partials, counter, done);
  ls.done();
}

// n multiplier rows, m tile-buffer rows (m = n except for Bluestein plans)
template <typename T> inline size_t zm_smem(int n, int m, int P) {
  return yz_smem<T>(m, P) + 2 * (((size_t)n * P + 3) & ~(size_t)3) * sizeof(T);
}

// Tile width of the multiplier-array Z pass, 0 when no width fits (very long axes).
template <typename T> int zm_tile_width(int n, int m, int Tn) {
  auto kern = m != n ? k_z_fused_m<T, true> : k_z_fused_m<T, false>;
  for (int p = yz_cols<T>(); p >= 16 / (int)sizeof(T); p /= 2) {
    if (p * Tn > 1024 || zm_smem<T>(n, m, p) > 227u * 1024u) continue;
    ensure_smem(kern, zm_smem<T>(n, m, p));
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, p * Tn, zm_smem<T>(n, m, p)) != cudaSuccess) {
      (void)cudaGetLastError();
      continue;
    }
    if (per_sm >= 1) return p;
  }
  return 0;
}

// One compile-time multiplier Z pass (k_z_fused_m_fx, FP a FixedPlan) in launch shape
// `shape`; scoped as in launch_yz_fx.
template <typename T, class FP>
bool launch_zm_fx(qsm_ctx* ctx, const Fft3<T>& f, int shape, const cplx_t<T>* src, cplx_t<T>* dst, const T* mult,
                  const int* done, bool scoped) {
  auto kfx = k_z_fused_m_fx<T, FP, kZmCols>;
  const size_t smem = zm_smem<T>(FP::n, FP::n, kZmCols);
  const TileWalk w = tile_walk(f, 2, kZmCols, (shape & kTuneEdge) != 0);
  unsigned grid = 0;
  if (!fx_launch_ok(ctx, kfx, kZmCols * FP::T, smem, &grid, w.ntiles, (shape & kTuneBlockPerTile) != 0,
                    tune_bpsm(shape)))
    return false;
  if (!scoped) {
    kfx<<<grid, dim3(kZmCols, FP::T), smem, ctx->stream>>>(f.g, w, f.twz, src, dst, mult, done);
    return true;
  }
  LaunchScope ls(ctx, "fft_z_fused");
  kfx<<<grid, dim3(kZmCols, FP::T), smem, ctx->stream>>>(f.g, w, f.twz, src, dst, mult, done);
  ls.done();
  return true;
}

// Tune the launch shape of the compile-time Y/Z pass (DIR, AXIS) and of the multiplier
// Z pass for grid f, running the candidates in place on `scratch` (a half spectrum of f
// whose contents may be overwritten) and `mscratch` (a real half-spectrum array).  With
// `chain`, each candidate is timed inside that sequence of launches instead (the solver's
// own chain of passes, which looks the shape up under the same key), so that it is judged
// where it runs: after the pass that fills the L2-resident spectrum, not back to back
// with itself.  No-op when the lengths have no compile-time pass, the shapes are cached,
// the autotuner is off or the stream is capturing.
template <typename T, int DIR, int AXIS, bool W>
void tune_yz_fixed(qsm_ctx* ctx, const Fft3<T>& f, cplx_t<T>* scratch, const std::function<void()>* chain = nullptr) {
  {
    if (!compiled_plans(ctx)) return;
    const std::string key = yz_tune_key<T>("yz_fx", f, AXIS, DIR);
    if (!autotune_due(ctx, key)) return;
    const FftPlan1D& pl = (AXIS == 1) ? f.py : f.pz;
#define QSM_TUNE_YZ(N_, T_, R0_, R1_, R2_)                                                        \
    if (FixedPlan<N_, T_, R0_, R1_, R2_>::matches(pl) && fx_cols<T>() * T_ <= 1024) {                   \
      using FP = FixedPlan<N_, T_, R0_, R1_, R2_>;                                                \
      auto kern = k_pass_yz_dx<T, DIR, FP, fx_cols<T>()>;                                              \
      const size_t smem = dx_smem<T>(FP::n, fx_cols<T>());                                             \
      ensure_smem(kern, smem);                                                                    \
      const auto cands = yz_candidates(f, fx_cols<T>(), kern, fx_cols<T>() * FP::T, smem);                  \
      if (chain != nullptr)                                                                       \
        autotune_pick(ctx, key, cands, [&](int c) { ctx->tuned[key] = TuneRec{c, {}}; (*chain)(); }, 3, 4); \
      else                                                                                        \
        autotune_pick(ctx, key, cands, [&](int c) {                                               \
          launch_yz_fx<T, DIR, AXIS, FP>(ctx, f, c, scratch, scratch, nullptr, false);             \
        });                                                                                       \
      return;                                                                                     \
    }
    QSM_FIXED_PLANS(QSM_TUNE_YZ)
    if constexpr (W) {
      QSM_FIXED_PLANS_WIDE(QSM_TUNE_YZ)
    }
#undef QSM_TUNE_YZ
  }
}

template <typename T, bool W>
void tune_z_fused_m(qsm_ctx* ctx, const Fft3<T>& f, cplx_t<T>* scratch, T* mscratch,
                    const std::function<void()>* chain = nullptr) {
  if constexpr (std::is_same<T, float>::value) {
    if (!compiled_plans(ctx)) return;
    const std::string key = yz_tune_key<T>("zm_fx", f, 2, -1);
    if (!autotune_due(ctx, key)) return;
    const FftPlan1D& pl = f.pz;
#define QSM_TUNE_ZM(N_, T_, R0_, R1_, R2_)                                                        \
    if (FixedPlan<N_, T_, R0_, R1_, R2_>::matches(pl) && kZmCols * T_ <= 1024) {                   \
      using FP = FixedPlan<N_, T_, R0_, R1_, R2_>;                                                \
      auto kfx = k_z_fused_m_fx<T, FP, kZmCols>;                                                  \
      const size_t smem = zm_smem<T>(FP::n, FP::n, kZmCols);                                      \
      ensure_smem(kfx, smem);                                                                     \
      const auto cands = yz_candidates(f, kZmCols, kfx, kZmCols * FP::T, smem);                   \
      if (chain != nullptr)                                                                       \
        autotune_pick(ctx, key, cands, [&](int c) { ctx->tuned[key] = TuneRec{c, {}}; (*chain)(); }, 3, 4); \
      else                                                                                        \
        autotune_pick(ctx, key, cands, [&](int c) {                                               \
          launch_zm_fx<T, FP>(ctx, f, c, scratch, scratch, mscratch, nullptr, false);              \
        });                                                                                       \
      return;                                                                                     \
    }
    QSM_FIXED_PLANS(QSM_TUNE_ZM)
    if constexpr (W) {
      QSM_FIXED_PLANS_WIDE(QSM_TUNE_ZM)
    }
#undef QSM_TUNE_ZM
  }
}

// Z fused pass with a precomputed real multiplier array (spectrum layout); W adds
// QSM_FIXED_PLANS_WIDE.
template <typename T, bool W = false>
void run_z_fused_m(qsm_ctx* ctx, const Fft3<T>& f, const cplx_t<T>* src, cplx_t<T>* dst, const T* mult,
                   const int* done) {
  const FftPlan1D& pl = f.pz;
  if constexpr (std::is_same<T, float>::value) {
    if (compiled_plans(ctx)) {
#define QSM_TRY_ZM(N_, T_, R0_, R1_, R2_)                                                         \
    if (FixedPlan<N_, T_, R0_, R1_, R2_>::matches(pl) && kZmCols * T_ <= 1024) {                   \
      using FP = FixedPlan<N_, T_, R0_, R1_, R2_>;                                                \
      const int shape = tuned_shape(ctx, yz_tune_key<T>("zm_fx", f, 2, -1));                      \
      if (launch_zm_fx<T, FP>(ctx, f, shape, src, dst, mult, done, true)) return;                 \
    }
    QSM_FIXED_PLANS(QSM_TRY_ZM)
    if constexpr (W) {
      QSM_FIXED_PLANS_WIDE(QSM_TRY_ZM)
    }
#undef QSM_TRY_ZM
    }
  }
  auto kern = pl.m != pl.n ? k_z_fused_m<T, true> : k_z_fused_m<T, false>;
  const int P = zm_tile_width<T>(pl.n, pl.m, pl.T);
  if (P == 0) throw QsmError(QSM_ERR_UNSUPPORTED_SIZE, "z axis does not fit one multiplier tile");
  const size_t smem = zm_smem<T>(pl.n, pl.m, P);
  const TileWalk w = tile_walk(f, 2, P);
  const unsigned grid = persistent_grid(ctx, kern, P * pl.T, smem, w.ntiles);
  LaunchScope ls(ctx, "fft_z_fused");
  kern<<<grid, dim3(P, pl.T), smem, ctx->stream>>>(f.g, pl, w, f.twz, src, dst, mult, done);
  ls.done();
}

template <typename T, class Op>
void run_z_fused(qsm_ctx* ctx, const Fft3<T>& f, const cplx_t<T>* src, cplx_t<T>* dst, const Op& op,
                 const int* done) {
  const FftPlan1D& pl = f.pz;
  auto kern = pl.m != pl.n ? k_z_fused<T, Op, true> : k_z_fused<T, Op, false>;
  const int P = yz_tile_width<T>(kern, pl.m, pl.T);
  const size_t smem = yz_smem<T>(pl.m, P);
  const TileWalk w = tile_walk(f, 2, P);
  const unsigned grid = persistent_grid(ctx, kern, P * pl.T, smem, w.ntiles);
  LaunchScope ls(ctx, "fft_z_fused");
  kern<<<grid, dim3(P, pl.T), smem, ctx->stream>>>(f.g, pl, w, f.twz, src, dst, op, done);
  ls.done();
}

// ---------------------------------------------------------------------------
// k-space geometry in double: fftfreq per axis (src/fft.rs:544-566), per-axis
// eigenvalues of the negative 7-point Laplacian (the FFT of
// laplacian_kernel(negative=true), src/kernels/laplacian.rs:20-61, which is a sum of
// per-axis terms), the Poisson eigenvalues of the unwrapping solver
// (src/unwrap/laplacian.rs:91-105), and the normalised B0 direction.
// ---------------------------------------------------------------------------
template <typename S> struct KSpaceT {
  const S* fx;
  const S* fy;
  const S* fz;
  const S* lx;
  const S* ly;
  const S* lz;
  const S* qx;
  const S* qy;
  const S* qz;
  int nyqx, nyqy, nyqz;  // index n/2 for even n, else -1
  S bx, by, bz;

  __device__ __forceinline__ S dipole(S kx, S ky, S kz) const {
    const S kdb = kx * bx + ky * by + kz * bz;
    const S k2 = kx * kx + ky * ky + kz * kz;
    return k2 > S(1e-20) ? S(1.0 / 3.0) - (kdb * kdb) / k2 : S(0);
  }
  __device__ __forceinline__ S lapneg(int ix, int iy, int iz) const {
    return (__ldg(lx + ix) + __ldg(ly + iy)) + __ldg(lz + iz);
  }
  __device__ __forceinline__ S poisson(int ix, int iy, int iz) const {
    return (__ldg(qx + ix) + __ldg(qy + iy)) + __ldg(qz + iz);
  }
  __device__ __forceinline__ bool on_nyquist(int ix, int iy, int iz) const {
    return ix == nyqx || iy == nyqy || iz == nyqz;
  }
  // Evaluate a multiplier M(kx,ky,kz,ix,iy,iz) symmetrised over k -> -k: the C2C
  // reference keeps Re(IFFT(F * M)), which equals IFFT(F * (M(k) + M(-k))/2) for real
  // input.  M(-k) differs from M(k) only on even-length Nyquist planes, where the
  // mirrored index keeps its frequency -n/2 while the other coordinates flip sign.
  template <class F>
  __device__ __forceinline__ S sym(int ix, int iy, int iz, const F& m) const {
    const S kx = __ldg(fx + ix), ky = __ldg(fy + iy), kz = __ldg(fz + iz);
    S v = m(kx, ky, kz, ix, iy, iz);
    if (on_nyquist(ix, iy, iz)) {
      const S v2 = m(ix == nyqx ? -kx : kx, iy == nyqy ? -ky : ky, iz == nyqz ? -kz : kz, ix, iy, iz);
      v = S(0.5) * (v + v2);
    }
    return v;
  }
};
using KSpace = KSpaceT<double>;

template <typename S> KSpaceT<S> make_kspace_t(qsm_ctx* ctx, const GridDims& d, const double bdir[3]);
KSpace make_kspace(qsm_ctx* ctx, const GridDims& d, const double bdir[3]);

}  // namespace qsm
