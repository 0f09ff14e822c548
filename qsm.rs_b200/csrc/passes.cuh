// The four 3D-FFT pass kernels the solvers are built from.
//
// Spectra use the half-spectrum layout of a real-to-complex transform along x:
// complex [nz][ny][pitch] with x' in [0, nx/2] valid (Fortran order like the
// reference, src/fft.rs:236-241, with x the contiguous axis).  The reference runs
// full complex-to-complex transforms of real data and keeps the real part
// (src/fft.rs:514-540); with real-symmetric (Nyquist-averaged) multipliers the
// half-spectrum chain computes the same values on half the bytes.
//
//   k_x_r2c   : two real rows per complex pencil (z = a + i b), forward FFT along x,
//               split into the two half spectra.  A loader functor produces the
//               real input on the fly (cast from f64, masked, stencil, kernel image).
//   k_pass_yz : C2C along y or z.  Persistent CTAs walk P-column tiles (128-byte rows);
//               each tile is staged into shared memory with cp.async, double
//               buffered so that the next tile's copy overlaps this tile's transform.
//               Optional pre/post pointwise hooks.
//   k_z_fused : same tiling; forward z FFT -> pointwise multiplier -> inverse z FFT.
//   k_x_c2r   : rebuild two Hermitian rows, inverse FFT along x, hand each real
//               value to a store functor (scale, mask, selection).
#pragma once

#include "fft_engine.cuh"

namespace qsm {

struct Geom {
  int nx, ny, nz;
  int nxh;    // nx/2 + 1
  int pitch;  // row pitch of the half spectrum, >= nxh, multiple of 4
  __host__ __device__ long long nvox() const { return (long long)nx * ny * nz; }
  __host__ __device__ long long hsize() const { return (long long)pitch * ny * nz; }
  __host__ __device__ int nrows() const { return ny * nz; }
};

template <typename T> struct PadG;
template <> struct PadG<float> { static constexpr int G = 16; };
template <> struct PadG<double> { static constexpr int G = 8; };

template <typename T> __host__ __device__ inline int x_rowlen(int n) { return n + n / PadG<T>::G + 1; }
// Twiddle table of the compile-time X passes: padded (tw_pad) in double, where it took
// iLSQR's FP64 X pass at length 384 from 523 to 504 us; dense in float, where the extra
// index arithmetic made the length-256 passes slower (r2c 25.5 -> 27.2 us).
template <typename T> constexpr bool x_tw_padded() { return sizeof(T) == 8; }
template <typename T> __host__ __device__ constexpr int x_tw_len(int n) {
  return x_tw_padded<T>() ? tw_table_len(n) : n;
}

// Identity pointwise op: Y/Z passes with it go smem -> registers -> global.
template <typename T> struct OpId {
  using C = cplx_t<T>;
  __device__ __forceinline__ C pre(C v, int, int, int, long long) const { return v; }
  __device__ __forceinline__ C post(C v, int, int, int, long long) const { return v; }
  __device__ __forceinline__ C mid(C v, int, int, int, long long) const { return v; }
};
template <class Op> struct IsPlainOp { static constexpr bool value = false; };
template <typename T> struct IsPlainOp<OpId<T>> { static constexpr bool value = true; };

// ------------------------------------------------------------------ cp.async --
// 16-byte global -> shared copy; when pred is false nothing is read and zeros are
// written.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int nbytes = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(nbytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Drops the L2 lines lying wholly inside [lo, hi) without writing them back
// (discard.global.L2: the lines then hold indeterminate values).  For data a block has
// read for the last time: dirty lines of a dead buffer would otherwise be written to HBM
// when evicted.  Lines shared with bytes outside the range are left alone.  Call after a
// barrier that follows the block's last reads of the range.
__device__ __forceinline__ void l2_discard_lines(const void* lo, const void* hi, int tid, int nthr) {
  const unsigned long long a = (__cvta_generic_to_global(lo) + 127ull) & ~127ull;
  const unsigned long long b = __cvta_generic_to_global(hi) & ~127ull;
  for (unsigned long long q = a + 128ull * (unsigned long long)tid; q < b; q += 128ull * (unsigned long long)nthr)
    asm volatile("discard.global.L2 [%0], 128;\n" ::"l"(q) : "memory");
}

// ---------------------------------------------------------------------------
// X forward: real rows -> half spectrum.  blockDim = (Tb, P) with Tb >= plan T
// (threads t >= T idle, so blocks stay whole warps); P pencils (row pairs).
// A thread holds at most kFftEmax elements of a row (T >= n/16), so the loader's
// global reads are issued as one unrolled batch before any is consumed.
// ---------------------------------------------------------------------------
template <typename T, class Load, bool BL>
__global__ void k_x_r2c(Geom g, const __grid_constant__ FftPlan1D pl, const cplx_t<T>* __restrict__ twg,
                        cplx_t<T>* __restrict__ spec, Load ld, const int* __restrict__ done) {
  using C = cplx_t<T>;
  if (done != nullptr && *done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  const int n = pl.n;
  const int m = pl.m;  // slot length: n, or the Bluestein convolution length
  const int rowlen = x_rowlen<T>(m);
  C* sm = tw + m;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int i = tid; i < m; i += blockDim.x * blockDim.y) tw[i] = twg[i];
  const int t = threadIdx.x;
  const int p = threadIdx.y;
  const long long q = (long long)blockIdx.x * blockDim.y + p;
  const long long nrows = g.nrows();
  const long long a = 2 * q, b = 2 * q + 1;
  const bool active = a < nrows && t < pl.T;
  const bool hasb = b < nrows;
  C* sp = sm + p * rowlen;
  SAPadded<PadG<T>::G> sa;
  {
    T va[kFftEmax], vb[kFftEmax];
#pragma unroll
    for (int c = 0; c < kFftEmax; ++c) {
      const int e = t + c * pl.T;
      va[c] = T(0);
      vb[c] = T(0);
      if (active && e < n) {
        va[c] = ld((int)a, e);
        if (hasb) vb[c] = ld((int)b, e);
      }
    }
#pragma unroll
    for (int c = 0; c < kFftEmax; ++c) {
      const int e = t + c * pl.T;
      if (active && e < n) sp[sa(e)] = mk<C>(va[c], vb[c]);
    }
  }
  __syncthreads();
  fft_pencil<-1, C, SAPadded<PadG<T>::G>, false, false, BL>(&pl, t, active, sp, sa, tw, nullptr, nullptr, 0, 0);
  if (active) {
    const T half = T(0.5);
    for (int k = t; k < g.nxh; k += pl.T) {
      C zk = sp[sa(k)];
      C zn = sp[sa(k == 0 ? 0 : n - k)];
      C A = mk<C>((zk.x + zn.x) * half, (zk.y - zn.y) * half);
      C B = mk<C>((zk.y + zn.y) * half, (zn.x - zk.x) * half);
      spec[a * g.pitch + k] = A;
      if (hasb) spec[b * g.pitch + k] = B;
    }
  }
}

// ---------------------------------------------------------------------------
// X pass over full complex rows (complex-to-complex spectra: [nz][ny][pitch] with all
// nx columns valid).  Per row: load -> FFT(D1) -> mid -> FFT(D2) -> store, where a
// direction of 0 skips that transform.  One row per pencil; blockDim = (Tb, P).
//   Load : C operator()(int row, int e)
//   Mid  : C operator()(C v, int row, int e)
//   Store: void operator()(int row, int e, C v); void finish()
// ---------------------------------------------------------------------------
template <typename T, int D1, int D2, class Load, class Mid, class Store, bool BL>
__global__ void k_x_full(Geom g, const __grid_constant__ FftPlan1D pl, const cplx_t<T>* __restrict__ twg, Load ld,
                         Mid mid, Store st0, const int* __restrict__ done) {
  using C = cplx_t<T>;
  if (done != nullptr && *done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  const int n = pl.n;
  const int m = pl.m;  // slot length: n, or the Bluestein convolution length
  const int rowlen = x_rowlen<T>(m);
  C* sm = tw + m;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int i = tid; i < m; i += blockDim.x * blockDim.y) tw[i] = twg[i];
  const int t = threadIdx.x;
  const long long row = (long long)blockIdx.x * blockDim.y + threadIdx.y;
  const bool active = row < g.nrows() && t < pl.T;
  C* sp = sm + threadIdx.y * rowlen;
  SAPadded<PadG<T>::G> sa;
  {
    C v[kFftEmax];
#pragma unroll
    for (int c = 0; c < kFftEmax; ++c) {
      const int e = t + c * pl.T;
      v[c] = mk<C>(T(0), T(0));
      if (active && e < n) v[c] = ld((int)row, e);
    }
#pragma unroll
    for (int c = 0; c < kFftEmax; ++c) {
      const int e = t + c * pl.T;
      if (active && e < n) sp[sa(e)] = v[c];
    }
  }
  __syncthreads();
  if constexpr (D1 != 0) fft_pencil<D1, C, SAPadded<PadG<T>::G>, false, false, BL>(&pl, t, active, sp, sa, tw, nullptr, nullptr, 0, 0);
  if (active)
    for (int e = t; e < n; e += pl.T) sp[sa(e)] = mid(sp[sa(e)], (int)row, e);
  __syncthreads();
  if constexpr (D2 != 0) fft_pencil<D2, C, SAPadded<PadG<T>::G>, false, false, BL>(&pl, t, active, sp, sa, tw, nullptr, nullptr, 0, 0);
  Store st = st0;
  {
    C v[kFftEmax];
#pragma unroll
    for (int c = 0; c < kFftEmax; ++c) {
      const int e = t + c * pl.T;
      if (active && e < n) v[c] = sp[sa(e)];
    }
#pragma unroll
    for (int c = 0; c < kFftEmax; ++c) {
      const int e = t + c * pl.T;
      if (active && e < n) st((int)row, e, v[c]);
    }
  }
  st.finish();
}

// Compile-time form of k_x_full with both transforms (FP a FixedPlan): the first
// transform's first stage fetches through the loader, its last stage applies the mid
// hook and passes the values in registers to the second transform (the reversed plan),
// whose last stage hands its values straight to the store functor, so a row makes three
// shared-memory round trips fewer than in k_x_full.  Every element of a row is fetched
// in the first stage, before any store of that row, so the loader and the store may
// address the same rows.
template <typename T, class FP, int D1, int D2, class Load, class Mid, class Store>
__global__ void k_x_full_fx(Geom g, const cplx_t<T>* __restrict__ twg, Load ld, Mid mid, Store st0,
                            const int* __restrict__ done) {
  using C = cplx_t<T>;
  constexpr int N = FP::n, TT = FP::T;
  static_assert(D1 != 0 && D2 != 0, "both transforms");
  if (done != nullptr && *done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  constexpr bool TWP = x_tw_padded<T>();
  C* tw = reinterpret_cast<C*>(smraw);
  C* sm = tw + x_tw_len<T>(N);
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int i = tid; i < N; i += blockDim.x * blockDim.y) tw[TWP ? tw_pad(i) : i] = twg[i];
  const int t = threadIdx.x;
  const int row = blockIdx.x * blockDim.y + threadIdx.y;
  const bool active = row < g.nrows() && t < TT;
  C* sp = sm + threadIdx.y * x_rowlen<T>(N);
  SAPadded<PadG<T>::G> sa;
  Store st = st0;
  auto fetch_g = [&](int e) -> C { return ld(row, e); };
  auto emit_g = [&](int e, C v) { st(row, e, v); };
  // The first transform's last stage applies the mid hook in registers and the second
  // transform, the reversed plan, starts from them (FetchInRegs): no shared-memory round
  // trip and no barrier between the two.
  C v[kFftEmax];
  auto hook = [&](int e, C x) -> C { return mid(x, row, e); };
  EmitInRegs<decltype(hook)> keep{hook};
  FetchInRegs in_regs;
  FP::template run_v<D1, TWP>(v, t, active, sp, sa, tw, fetch_g, keep);
  ReversePlan<FP>::type::template run_v<D2, TWP>(v, t, active, sp, sa, tw, in_regs, emit_g);
  st.finish();
}

// ---------------------------------------------------------------------------
// X inverse: half spectrum -> real rows.  blockDim = (Tb, P) as for k_x_r2c.
// A thread loads at most 9 half-spectrum entries per row (nx/2+1 <= 9T), issued as
// one batch; the results are handed to the store functor in one unrolled batch.
// ---------------------------------------------------------------------------
constexpr int kXHalfMax = 9;

template <typename T, class Store, bool BL>
__global__ void k_x_c2r(Geom g, const __grid_constant__ FftPlan1D pl, const cplx_t<T>* __restrict__ twg,
                        const cplx_t<T>* __restrict__ spec, Store st0, const int* __restrict__ done) {
  using C = cplx_t<T>;
  if (done != nullptr && *done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  const int n = pl.n;
  const int m = pl.m;  // slot length: n, or the Bluestein convolution length
  const int rowlen = x_rowlen<T>(m);
  C* sm = tw + m;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int i = tid; i < m; i += blockDim.x * blockDim.y) tw[i] = twg[i];
  const int t = threadIdx.x;
  const int p = threadIdx.y;
  const long long q = (long long)blockIdx.x * blockDim.y + p;
  const long long nrows = g.nrows();
  const long long a = 2 * q, b = 2 * q + 1;
  const bool active = a < nrows && t < pl.T;
  const bool hasb = b < nrows;
  C* sp = sm + p * rowlen;
  SAPadded<PadG<T>::G> sa;
  {
    C ga[kXHalfMax], gb[kXHalfMax];
#pragma unroll
    for (int c = 0; c < kXHalfMax; ++c) {
      const int k = t + c * pl.T;
      ga[c] = mk<C>(T(0), T(0));
      gb[c] = mk<C>(T(0), T(0));
      if (active && k < g.nxh) {
        ga[c] = spec[a * g.pitch + k];
        if (hasb) gb[c] = spec[b * g.pitch + k];
      }
    }
#pragma unroll
    for (int c = 0; c < kXHalfMax; ++c) {
      const int k = t + c * pl.T;
      if (active && k < g.nxh) {
        C xa = ga[c], xb = gb[c];
        const bool selfm = (k == 0) || (2 * k == n);
        if (selfm) {
          xa.y = T(0);
          xb.y = T(0);
        }
        sp[sa(k)] = mk<C>(xa.x - xb.y, xa.y + xb.x);
        if (!selfm) sp[sa(n - k)] = mk<C>(xa.x + xb.y, xb.x - xa.y);
      }
    }
  }
  __syncthreads();
  fft_pencil<+1, C, SAPadded<PadG<T>::G>, false, false, BL>(&pl, t, active, sp, sa, tw, nullptr, nullptr, 0, 0);
  Store st = st0;
  {
    C v[kFftEmax];
#pragma unroll
    for (int c = 0; c < kFftEmax; ++c) {
      const int e = t + c * pl.T;
      if (active && e < n) v[c] = sp[sa(e)];
    }
#pragma unroll
    for (int c = 0; c < kFftEmax; ++c) {
      const int e = t + c * pl.T;
      if (active && e < n) {
        st((int)a, e, v[c].x);
        if (hasb) st((int)b, e, v[c].y);
      }
    }
  }
  st.finish();
}

// ---------------------------------------------------------------------------
// Compile-time X passes (FP a FixedPlan): the first Stockham stage reads its inputs
// straight from global memory through the loader (r2c) or through the Hermitian
// rebuild of the two half-spectrum rows (c2r), and the c2r's last stage hands its
// values straight to the store functor, so each pass makes one shared-memory round
// trip fewer than k_x_r2c / k_x_c2r and runs with constant loop bounds.
// blockDim = (Tb >= FP::T, P) as for the runtime kernels.
// DEAD: the pass reads its input for the last time (r2c: the loader's rows, through
// ld.row_begin; c2r: the half spectrum), so each block drops the L2 lines of its rows
// (l2_discard_lines) once it has read them, instead of leaving them dirty.
// ---------------------------------------------------------------------------
template <typename T, class FP, class Load, bool DEAD = false>
__global__ void k_x_r2c_fx(Geom g, const cplx_t<T>* __restrict__ twg, cplx_t<T>* __restrict__ spec, Load ld,
                           const int* __restrict__ done) {
  using C = cplx_t<T>;
  constexpr int N = FP::n, TT = FP::T, NXH = N / 2 + 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  constexpr bool TWP = x_tw_padded<T>();
  C* tw = reinterpret_cast<C*>(smraw);
  C* sm = tw + x_tw_len<T>(N);
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int i = tid; i < N; i += blockDim.x * blockDim.y) tw[TWP ? tw_pad(i) : i] = twg[i];
  if (done != nullptr && *done) return;
  const int t = threadIdx.x;
  const int p = threadIdx.y;
  const int nrows = g.nrows();
  const int a = 2 * (blockIdx.x * blockDim.y + p), b = a + 1;
  const bool active = a < nrows && t < TT;
  const bool hasb = b < nrows;
  C* sp = sm + p * x_rowlen<T>(N);
  SAPadded<PadG<T>::G> sa;
  auto fetch = [&](int e) -> C { return mk<C>(ld(a, e), hasb ? ld(b, e) : T(0)); };
  auto emit = [&](int e, C v) { sp[sa(e)] = v; };
  FP::template run<-1, TWP>(t, active, sp, sa, tw, fetch, emit);
  // Here rather than between the stages, where the discards slowed the pass (27.0
  // against 25.3 us at 256x256x176); the c2r pass gains from the earlier point.
  if constexpr (DEAD) {
    const int r0 = 2 * blockIdx.x * blockDim.y, r1 = min(r0 + 2 * (int)blockDim.y, nrows);
    l2_discard_lines(ld.row_begin(r0), ld.row_begin(r1), tid, blockDim.x * blockDim.y);
  }
  if (active) {
    const T half = T(0.5);
    C* ra = spec + (long long)a * g.pitch;
    C* rb = spec + (long long)b * g.pitch;
#pragma unroll
    for (int c = 0; c < (NXH + TT - 1) / TT; ++c) {
      const int k = t + c * TT;
      if (k < NXH) {
        const C zk = sp[sa(k)];
        const C zn = sp[sa(k == 0 ? 0 : N - k)];
        ra[k] = mk<C>((zk.x + zn.x) * half, (zk.y - zn.y) * half);
        if (hasb) rb[k] = mk<C>((zk.y + zn.y) * half, (zn.x - zk.x) * half);
      }
    }
  }
}

template <typename T, class FP, class Store, bool DEAD = false>
__global__ void k_x_c2r_fx(Geom g, const cplx_t<T>* __restrict__ twg, const cplx_t<T>* __restrict__ spec, Store st0,
                           const int* __restrict__ done) {
  using C = cplx_t<T>;
  constexpr int N = FP::n, TT = FP::T;
  extern __shared__ __align__(16) unsigned char smraw[];
  constexpr bool TWP = x_tw_padded<T>();
  C* tw = reinterpret_cast<C*>(smraw);
  C* sm = tw + x_tw_len<T>(N);
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int i = tid; i < N; i += blockDim.x * blockDim.y) tw[TWP ? tw_pad(i) : i] = twg[i];
  if (done != nullptr && *done) return;
  const int t = threadIdx.x;
  const int p = threadIdx.y;
  const int nrows = g.nrows();
  const int a = 2 * (blockIdx.x * blockDim.y + p), b = a + 1;
  const bool active = a < nrows && t < TT;
  const bool hasb = b < nrows;
  C* sp = sm + p * x_rowlen<T>(N);
  SAPadded<PadG<T>::G> sa;
  const C* ra = spec + (long long)a * g.pitch;
  const C* rb = spec + (long long)b * g.pitch;
  // z[e] = A[e] + i B[e] from the two half spectra (A, B Hermitian)
  auto fetch = [&](int e) -> C {
    const bool lo = e <= N / 2;
    const int k = lo ? e : N - e;
    C xa = ra[k];
    C xb = hasb ? rb[k] : mk<C>(T(0), T(0));
    if (k == 0 || 2 * k == N) {
      xa.y = T(0);
      xb.y = T(0);
    }
    return lo ? mk<C>(xa.x - xb.y, xa.y + xb.x) : mk<C>(xa.x + xb.y, xb.x - xa.y);
  };
  Store st = st0;
  auto emit = [&](int e, C v) {
    st(a, e, v.x);
    if (hasb) st(b, e, v.y);
  };
  auto release = [&] {
    if constexpr (DEAD) {
      const int r0 = 2 * blockIdx.x * blockDim.y, r1 = min(r0 + 2 * (int)blockDim.y, nrows);
      l2_discard_lines(spec + (long long)r0 * g.pitch, spec + (long long)r1 * g.pitch, tid, blockDim.x * blockDim.y);
    }
  };
  C v[kFftEmax];
  FP::template run_v<+1, TWP>(v, t, active, sp, sa, tw, fetch, emit, release);
  st.finish();
}

// ---------------------------------------------------------------------------
// Tiled Y/Z passes.  A tile is P consecutive x' columns (P*sizeof(C) = 128 bytes, or
// narrower for long axes) at one outer index, all n elements along the transform
// axis.  blockDim = (P, T);
// the grid is persistent (a few CTAs per SM) and walks tiles with stride gridDim.x.
// ---------------------------------------------------------------------------
struct TileWalk {
  int ntx;        // column tiles along x'
  int ntiles;     // tiles in all: nmain, plus the edge tiles
  long long ostride;  // global stride of the outer index
  long long estride;  // global stride along the transform axis
  // Edge tiles (compile-time kernels only).  Main tiles are P consecutive columns at
  // one outer index.  When the last nedge columns (from col_edge) would fill only a
  // small part of a P-wide tile, as the one Nyquist column of an even length does
  // (129 = 8 * 16 + 1), they are left out of the main tiles and walked as edge tiles
  // instead: one of those columns at P consecutive outer indices, so no tile is mostly
  // idle lanes.  Their loads are scattered (one element per row and lane), so the walk
  // takes them first (tile indices below nfirst = ntiles - nmain) and the main tiles
  // after them, rather than leaving the slowest tiles for the end.  nedge = 0: none.
  int nmain;
  int nouter;
  int col_edge;
  int nedge;
};

// Column and outer index of lane px in a tile (main or edge), and whether it is a
// valid element column.
__device__ __forceinline__ bool tile_pos(const Geom& g, const TileWalk& w, int tile, int px, int P, int& col,
                                         int& outer) {
  const int nfirst = w.ntiles - w.nmain;
  if (tile >= nfirst) {
    const int mt = tile - nfirst;
    const int tx = mt % w.ntx;
    outer = mt / w.ntx;
    col = tx * P + px;
    return col < g.nxh;
  }
  const int et = tile;
  const int ob = (et / w.nedge) * P;
  col = w.col_edge + (et - (et / w.nedge) * w.nedge);
  outer = ob + px < w.nouter ? ob + px : w.nouter - 1;  // clamped: inactive lanes address a valid row
  return ob + px < w.nouter;
}

// 4- or 8-byte global -> shared copies (edge tiles: one element per lane)
template <int B> __device__ __forceinline__ void cp_async_small(void* smem, const void* gmem, bool pred) {
  static_assert(B == 4 || B == 8 || B == 16, "cp.async copies 4, 8 or 16 bytes");
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int nbytes = pred ? B : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(s), "l"(gmem), "n"(B), "r"(nbytes)
               : "memory");
}

// Stage an edge tile (element e of lane px at buf[e * P + px]) of complex (C) or real
// (C = T) values.
template <typename C>
__device__ __forceinline__ void issue_edge_tile(const C* __restrict__ src, C* buf, const TileWalk& w, int tile,
                                                int n, int P) {
  const int et = tile;
  const int ob = (et / w.nedge) * P;
  const int col = w.col_edge + (et - (et / w.nedge) * w.nedge);
  const int nth = blockDim.x * blockDim.y;
  for (int c = threadIdx.x + threadIdx.y * blockDim.x; c < n * P; c += nth) {
    const int e = c / P, px = c - e * P;
    const bool ok = ob + px < w.nouter;
    const C* gp = src + col + (long long)(ok ? ob + px : 0) * w.ostride + (long long)e * w.estride;
    cp_async_small<(int)sizeof(C)>(buf + e * P + px, gp, ok);
  }
}

template <typename C>
__device__ __forceinline__ void issue_tile(const C* __restrict__ src, C* buf, const Geom& g, const TileWalk& w,
                                           int tile, int n, int P) {
  const int tx = tile % w.ntx;
  const int outer = tile / w.ntx;
  const int col0 = tx * P;
  const long long base = col0 + (long long)outer * w.ostride;
  constexpr int kPer = 16 / (int)sizeof(C);  // complex values per 16-byte chunk
  const int cpr = P / kPer;                  // 16-byte chunks per tile row
  const int chunks = n * cpr;
  const int nth = blockDim.x * blockDim.y;
  for (int c = threadIdx.x + threadIdx.y * blockDim.x; c < chunks; c += nth) {
    const int e = c / cpr, ch = c - e * cpr;
    const int col = col0 + ch * kPer;
    const bool ok = col < g.nxh;
    const C* gp = src + base + (long long)e * w.estride + (ok ? ch * kPer : 0);
    cp_async16(buf + e * P + ch * kPer, gp, ok);
  }
}

// Register cap of the tiled Y/Z kernels: three 256-thread CTAs per SM in single
// precision, three 128-thread CTAs in double.
template <typename T> struct YzRegCap { static constexpr int value = sizeof(T) == 4 ? 80 : 128; };
// The fused Z kernels run two transforms around a pointwise op; under the Y/Z cap they
// spill (float: ~0.1 KB, double: ~1.5 KB per thread), so they get a larger one.
template <typename T> struct ZRegCap { static constexpr int value = sizeof(T) == 4 ? 128 : 168; };

template <typename T, int DIR, int AXIS, class Op, bool BL>
__global__ void __maxnreg__(YzRegCap<T>::value)
    k_pass_yz(Geom g, const __grid_constant__ FftPlan1D pl, TileWalk w, const cplx_t<T>* __restrict__ twg,
                          const cplx_t<T>* src, cplx_t<T>* dst, Op op, const int* __restrict__ done) {
  using C = cplx_t<T>;
  if (done != nullptr && *done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  const int n = pl.n;
  const int m = pl.m;  // rows of a tile buffer: n, or the Bluestein convolution length
  const int P = blockDim.x;
  C* buf0 = tw + ((m + 7) & ~7);
  C* buf1 = buf0 + (size_t)m * P;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int i = tid; i < m; i += blockDim.x * blockDim.y) tw[i] = twg[i];
  const int px = threadIdx.x;
  const int t = threadIdx.y;
  SAStrided sa{P};
  int tile = blockIdx.x;
  if (tile < w.ntiles) issue_tile(src, buf0, g, w, tile, n, P);
  cp_async_commit();
  for (int it = 0; tile < w.ntiles; tile += gridDim.x, ++it) {
    C* cur = (it & 1) ? buf1 : buf0;
    C* nxt = (it & 1) ? buf0 : buf1;
    const int next = tile + gridDim.x;
    if (next < w.ntiles) issue_tile(src, nxt, g, w, next, n, P);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const int tx = tile % w.ntx, outer = tile / w.ntx;
    const int col = tx * P + px;
    const bool active = col < g.nxh;
    const long long base = col + (long long)outer * w.ostride;
    C* sp = cur + px;
    if constexpr (IsPlainOp<Op>::value) {
      fft_pencil<DIR, C, SAStrided, false, true, BL>(&pl, t, active, sp, sa, tw, nullptr, dst, base, w.estride);
    } else {
      if (active) {
        for (int e = t; e < n; e += pl.T) {
          const long long idx = base + e * w.estride;
          sp[sa(e)] = (AXIS == 1) ? op.pre(sp[sa(e)], col, e, outer, idx) : op.pre(sp[sa(e)], col, outer, e, idx);
        }
      }
      __syncthreads();
      fft_pencil<DIR, C, SAStrided, false, false, BL>(&pl, t, active, sp, sa, tw, nullptr, nullptr, 0, 0);
      if (active) {
        for (int e = t; e < n; e += pl.T) {
          const long long idx = base + e * w.estride;
          const C v = sp[sa(e)];
          dst[idx] = (AXIS == 1) ? op.post(v, col, e, outer, idx) : op.post(v, col, outer, e, idx);
        }
      }
      __syncthreads();
    }
  }
  cp_async_wait<0>();
}

// ------------------------------------------------------------- reductions --
// Sum K doubles over a block of any shape (partial last warp included); the result
// is valid in thread 0.  Fixed order for a fixed block shape.
template <int K> __device__ __forceinline__ void block_sum_any(double (&a)[K]) {
  __shared__ double red[K][32];
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nth = blockDim.x * blockDim.y * blockDim.z;
  const int lane = tid & 31, wid = tid >> 5;
  const int wsz = imin(32, nth - (wid << 5));
  const unsigned m = wsz == 32 ? 0xffffffffu : ((1u << wsz) - 1u);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double b = __shfl_down_sync(m, a[k], o);
      if (lane + o < wsz) a[k] += b;
    }
  }
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) red[k][wid] = a[k];
  __syncthreads();
  const int nw = (nth + 31) >> 5;
  if (wid == 0) {  // warp 0 itself may be partial (blocks of fewer than 32 threads)
#pragma unroll
    for (int k = 0; k < K; ++k) a[k] = lane < nw ? red[k][lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const double b = __shfl_down_sync(m, a[k], o);
        if (lane + o < wsz) a[k] += b;
      }
    }
  }
}

// Deterministic grid-wide sum: every block passes its K values; the block that
// arrives last sums the per-block partials in block order and returns true with the
// totals valid in its thread 0.  `counter` must be 0 on entry and is reset.
template <int K>
__device__ __forceinline__ bool grid_sum_last(double (&a)[K], double* __restrict__ partials, unsigned* counter) {
  __shared__ int am_last;
  block_sum_any<K>(a);
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nth = blockDim.x * blockDim.y * blockDim.z;
  const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
  const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) partials[(size_t)bid * K + k] = a[k];
    __threadfence();
    const unsigned prev = atomicAdd(counter, 1u);
    am_last = (prev == nblocks - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < K; ++k) a[k] = 0.0;
  for (unsigned b = tid; b < nblocks; b += nth)
#pragma unroll
    for (int k = 0; k < K; ++k) a[k] += __ldcg(&partials[(size_t)b * K + k]);
  block_sum_any<K>(a);
  if (tid == 0) *counter = 0u;
  return true;
}

// Y/Z pass whose post hook also accumulates one FP64 value per element
// (post(v, ix, iy, iz, idx, acc) returns the value to store).  The block that
// finishes last reduces the sums and runs op.last(total) on its thread 0.
template <typename T, int DIR, int AXIS, class Op, bool BL>
__global__ void __maxnreg__(YzRegCap<T>::value)
    k_pass_yz_acc(Geom g, const __grid_constant__ FftPlan1D pl, TileWalk w, const cplx_t<T>* __restrict__ twg,
                  const cplx_t<T>* src, cplx_t<T>* dst, Op op, double* __restrict__ partials, unsigned* counter,
                  const int* __restrict__ done) {
  using C = cplx_t<T>;
  if (done != nullptr && *done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  const int n = pl.n;
  const int m = pl.m;  // rows of a tile buffer: n, or the Bluestein convolution length
  const int P = blockDim.x;
  C* buf0 = tw + ((m + 7) & ~7);
  C* buf1 = buf0 + (size_t)m * P;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int i = tid; i < m; i += blockDim.x * blockDim.y) tw[i] = twg[i];
  const int px = threadIdx.x;
  const int t = threadIdx.y;
  SAStrided sa{P};
  double acc[1] = {0.0};
  int tile = blockIdx.x;
  if (tile < w.ntiles) issue_tile(src, buf0, g, w, tile, n, P);
  cp_async_commit();
  for (int it = 0; tile < w.ntiles; tile += gridDim.x, ++it) {
    C* cur = (it & 1) ? buf1 : buf0;
    C* nxt = (it & 1) ? buf0 : buf1;
    const int next = tile + gridDim.x;
    if (next < w.ntiles) issue_tile(src, nxt, g, w, next, n, P);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const int tx = tile % w.ntx, outer = tile / w.ntx;
    const int col = tx * P + px;
    const bool active = col < g.nxh;
    const long long base = col + (long long)outer * w.ostride;
    C* sp = cur + px;
    if (active) {
      for (int e = t; e < n; e += pl.T) {
        const long long idx = base + e * w.estride;
        sp[sa(e)] = (AXIS == 1) ? op.pre(sp[sa(e)], col, e, outer, idx) : op.pre(sp[sa(e)], col, outer, e, idx);
      }
    }
    __syncthreads();
    fft_pencil<DIR, C, SAStrided, false, false, BL>(&pl, t, active, sp, sa, tw, nullptr, nullptr, 0, 0);
    if (active) {
      for (int e = t; e < n; e += pl.T) {
        const long long idx = base + e * w.estride;
        const C v = sp[sa(e)];
        dst[idx] = (AXIS == 1) ? op.post(v, col, e, outer, idx, acc[0]) : op.post(v, col, outer, e, idx, acc[0]);
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
  if (grid_sum_last<1>(acc, partials, counter) && tid == 0) op.last(acc[0]);
}

// ------------------------------------------------------------------------------
// Compile-time Y/Z passes: the same tile walk with the transform length, threads per
// column and radices fixed (FP, a FixedPlan) and P columns per tile, so that loop
// bounds, j mod Ns, twiddle strides and shared-memory addressing fold into constants.
// Plain copies (k_pass_yz_dx) and the multiplier Z pass (k_z_fused_m_fx).
// ------------------------------------------------------------------------------
// Resident blocks per SM the compile-time Y/Z passes are compiled for: four blocks of
// up to 256 threads in float (64 registers; no plan of the two lists spills more than 4
// bytes, and with the five-block multiplier Z pass the TV-ADMM iteration at 256x256x176
// went from 0.1956 to 0.1941 ms); in double (twice the registers
// per value) three blocks of up to 128 threads and two of up to 256, so the long plans
// (384: 208 threads) do not spill.
template <typename T, int THREADS> constexpr int yz_dx_min_blocks() {
  if constexpr (sizeof(T) == 4) return THREADS <= 256 ? 4 : 1;
  else return THREADS <= 128 ? 3 : (THREADS <= 256 ? 2 : 1);
}

template <int P> struct SAStridedC {
  __device__ __forceinline__ int operator()(int e) const { return e * P; }
};

template <typename T, class FP, int P>
__global__ void __launch_bounds__(P* FP::T, (P * FP::T <= 256 ? 3 : 1))
    k_z_fused_m_fx(Geom g, TileWalk w, const cplx_t<T>* __restrict__ twg, const cplx_t<T>* src, cplx_t<T>* dst,
                   const T* __restrict__ mult, const int* __restrict__ done);

// Real multiplier tile (same tile walk, element size sizeof(T)), 16-byte chunks.
template <typename T>
__device__ __forceinline__ void issue_mtile(const T* __restrict__ src, T* buf, const Geom& g, const TileWalk& w,
                                            int tile, int n, int P) {
  const int tx = tile % w.ntx;
  const int outer = tile / w.ntx;
  const int col0 = tx * P;
  const long long base = col0 + (long long)outer * w.ostride;
  constexpr int kPer = 16 / (int)sizeof(T);
  const int cpr = P / kPer;
  const int chunks = n * cpr;
  const int nth = blockDim.x * blockDim.y;
  for (int c = threadIdx.x + threadIdx.y * blockDim.x; c < chunks; c += nth) {
    const int e = c / cpr, ch = c - e * cpr;
    const int col = col0 + ch * kPer;
    const bool ok = col < g.nxh;
    const T* gp = src + base + (long long)e * w.estride + (ok ? ch * kPer : 0);
    cp_async16(buf + e * P + ch * kPer, gp, ok);
  }
}

// Z forward -> multiply by a precomputed real multiplier -> Z inverse.  The
// multiplier (spectrum layout, real) is staged with the spectrum tile, so the
// pointwise step is one shared-memory read per element.  Needs P*sizeof(T) >= 16.
template <typename T, bool BL>
__global__ void __maxnreg__(ZRegCap<T>::value) k_z_fused_m(Geom g, const __grid_constant__ FftPlan1D pl, TileWalk w,
                            const cplx_t<T>* __restrict__ twg, const cplx_t<T>* src, cplx_t<T>* dst,
                            const T* __restrict__ mult, const int* __restrict__ done) {
  using C = cplx_t<T>;
  if (done != nullptr && *done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  const int n = pl.n;
  const int m = pl.m;  // rows of a tile buffer: n, or the Bluestein convolution length
  const int P = blockDim.x;
  C* buf0 = tw + ((m + 7) & ~7);
  C* buf1 = buf0 + (size_t)m * P;
  T* mb0 = reinterpret_cast<T*>(buf1 + (size_t)m * P);
  T* mb1 = mb0 + (((size_t)n * P + 3) & ~(size_t)3);
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int i = tid; i < m; i += blockDim.x * blockDim.y) tw[i] = twg[i];
  const int px = threadIdx.x;
  const int t = threadIdx.y;
  SAStrided sa{P};
  int tile = blockIdx.x;
  if (tile < w.ntiles) {
    issue_tile(src, buf0, g, w, tile, n, P);
    issue_mtile(mult, mb0, g, w, tile, n, P);
  }
  cp_async_commit();
  for (int it = 0; tile < w.ntiles; tile += gridDim.x, ++it) {
    C* cur = (it & 1) ? buf1 : buf0;
    C* nxt = (it & 1) ? buf0 : buf1;
    T* mcur = (it & 1) ? mb1 : mb0;
    T* mnxt = (it & 1) ? mb0 : mb1;
    const int next = tile + gridDim.x;
    if (next < w.ntiles) {
      issue_tile(src, nxt, g, w, next, n, P);
      issue_mtile(mult, mnxt, g, w, next, n, P);
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const int tx = tile % w.ntx, iy = tile / w.ntx;
    const int col = tx * P + px;
    const bool active = col < g.nxh;
    const long long base = col + (long long)iy * w.ostride;
    C* sp = cur + px;
    fft_pencil<-1, C, SAStrided, false, false, BL>(&pl, t, active, sp, sa, tw, nullptr, nullptr, 0, 0);
    if (active) {
      for (int e = t; e < n; e += pl.T) sp[sa(e)] = cscale(sp[sa(e)], mcur[e * P + px]);
    }
    __syncthreads();
    fft_pencil<+1, C, SAStrided, false, true, BL>(&pl, t, active, sp, sa, tw, nullptr, dst, base, w.estride);
  }
  cp_async_wait<0>();
}

// Compile-time Y/Z pass (FP a FixedPlan, P columns per tile) in direct-fetch form: the
// first Stockham stage loads
// its column elements straight from global memory (for each radix-stage element r, the
// P columns of a tile are one contiguous row segment, so the loads coalesce) instead of
// staging the whole tile through shared memory first.  The spectrum between passes is
// L2-resident at the benchmark sizes, so this trades a shared-memory round trip per
// element for L2 loads that the block's warps issue together (21 us instead of 25 us for
// a 256-point Y pass at 256x256x176).  The fused Z pass keeps its double-buffered tile
// staging: at two blocks per SM the direct loads left its latency exposed.  One tile
// buffer (the stage exchange) per block; blocks walk tiles with stride gridDim.x.
template <typename T, int DIR, class FP, int P>
__global__ void __launch_bounds__(P* FP::T, yz_dx_min_blocks<T, P * FP::T>())
    k_pass_yz_dx(Geom g, TileWalk w, const cplx_t<T>* __restrict__ twg, const cplx_t<T>* src, cplx_t<T>* dst,
                 const int* __restrict__ done) {
  using C = cplx_t<T>;
  constexpr int n = FP::n;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  C* buf = tw + ((n + 7) & ~7);
  const int tid = threadIdx.x + threadIdx.y * P;
  for (int i = tid; i < n; i += P * FP::T) tw[i] = twg[i];
  if (done != nullptr && *done) return;
  const int px = threadIdx.x;
  const int t = threadIdx.y;
  SAStridedC<P> sa;
  C* sp = buf + px;
  for (int tile = blockIdx.x; tile < w.ntiles; tile += gridDim.x) {
    int col, outer;
    const bool active = tile_pos(g, w, tile, px, P, col, outer);
    const long long base = col + (long long)outer * w.ostride;
    auto fetch = [&](int e) -> C { return src[base + e * w.estride]; };
    auto emit = [&](int e, C v) { dst[base + e * w.estride] = v; };
    // the first stage's barrier also orders the twiddle table and the previous tile's
    // last reads of buf before this tile writes it
    FP::template run<DIR>(t, active, sp, sa, tw, fetch, emit);
  }
}

// k_pass_yz_dx with the pass's operator applied as elements are fetched (op.pre) and
// stored (op.post), for passes that carry one (k-space scalings, fused LSQR epilogues).
// ACC: op.post also adds to a per-thread FP64 sum that is reduced over the grid at the
// end (grid_sum_last) and handed to op.last, as in k_pass_yz_acc.  The element order of
// that sum follows the fixed plan's last stage, so the total is deterministic for a
// given launch shape.
template <typename T, int DIR, int AXIS, class FP, int P, class Op, bool ACC>
__global__ void __launch_bounds__(P* FP::T, yz_dx_min_blocks<T, P * FP::T>())
    k_pass_yz_dx_op(Geom g, TileWalk w, const cplx_t<T>* __restrict__ twg, const cplx_t<T>* src, cplx_t<T>* dst,
                    Op op, double* __restrict__ partials, unsigned* counter, const int* __restrict__ done) {
  using C = cplx_t<T>;
  constexpr int n = FP::n;
  if (done != nullptr && *done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  C* buf = tw + ((n + 7) & ~7);
  const int tid = threadIdx.x + threadIdx.y * P;
  for (int i = tid; i < n; i += P * FP::T) tw[i] = twg[i];
  const int px = threadIdx.x;
  const int t = threadIdx.y;
  SAStridedC<P> sa;
  C* sp = buf + px;
  double acc[1] = {0.0};
  for (int tile = blockIdx.x; tile < w.ntiles; tile += gridDim.x) {
    const int tx = tile % w.ntx, outer = tile / w.ntx;
    const int col = tx * P + px;
    const bool active = col < g.nxh;
    const long long base = col + (long long)outer * w.ostride;
    auto fetch = [&](int e) -> C {
      const long long idx = base + e * w.estride;
      const C v = src[idx];
      return (AXIS == 1) ? op.pre(v, col, e, outer, idx) : op.pre(v, col, outer, e, idx);
    };
    auto emit = [&](int e, C v) {
      const long long idx = base + e * w.estride;
      if constexpr (ACC)
        dst[idx] = (AXIS == 1) ? op.post(v, col, e, outer, idx, acc[0]) : op.post(v, col, outer, e, idx, acc[0]);
      else
        dst[idx] = (AXIS == 1) ? op.post(v, col, e, outer, idx) : op.post(v, col, outer, e, idx);
    };
    FP::template run<DIR>(t, active, sp, sa, tw, fetch, emit);
  }
  if constexpr (ACC) {
    if (grid_sum_last<1>(acc, partials, counter) && tid == 0) op.last(acc[0]);
  }
}

// Ops whose pre hook is costly enough (a k-space evaluation per element) that it should
// run on a staged tile rather than inside the first stage's loads (kStagedPre).
template <class Op, class = void> struct StagedPre : std::false_type {};
template <class Op> struct StagedPre<Op, std::void_t<decltype(Op::kStagedPre)>> : std::bool_constant<Op::kStagedPre> {};

// Compile-time Y/Z operator pass in staged form: the tile is copied into shared memory
// with cp.async, double-buffered so the next tile's copy overlaps this tile's work, the
// pre hook runs over the staged tile, and the transform (FP) reads its first stage from
// shared memory and hands each output to the post hook on its way to global memory.
template <typename T, int DIR, int AXIS, class FP, int P, class Op>
__global__ void __launch_bounds__(P* FP::T, yz_dx_min_blocks<T, P * FP::T>())
    k_pass_yz_st_op(Geom g, TileWalk w, const cplx_t<T>* __restrict__ twg, const cplx_t<T>* src, cplx_t<T>* dst,
                    Op op, const int* __restrict__ done) {
  using C = cplx_t<T>;
  constexpr int n = FP::n;
  if (done != nullptr && *done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  C* buf0 = tw + ((n + 7) & ~7);
  C* buf1 = buf0 + n * P;
  const int tid = threadIdx.x + threadIdx.y * P;
  for (int i = tid; i < n; i += P * FP::T) tw[i] = twg[i];
  const int px = threadIdx.x;
  const int t = threadIdx.y;
  SAStridedC<P> sa;
  int tile = blockIdx.x;
  if (tile < w.ntiles) issue_tile(src, buf0, g, w, tile, n, P);
  cp_async_commit();
  for (int it = 0; tile < w.ntiles; tile += gridDim.x, ++it) {
    C* cur = (it & 1) ? buf1 : buf0;
    C* nxt = (it & 1) ? buf0 : buf1;
    const int next = tile + gridDim.x;
    if (next < w.ntiles) issue_tile(src, nxt, g, w, next, n, P);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const int tx = tile % w.ntx, outer = tile / w.ntx;
    const int col = tx * P + px;
    const bool active = col < g.nxh;
    const long long base = col + (long long)outer * w.ostride;
    C* sp = cur + px;
    if (active) {
      for (int e = t; e < n; e += FP::T) {
        const long long idx = base + e * w.estride;
        sp[sa(e)] = (AXIS == 1) ? op.pre(sp[sa(e)], col, e, outer, idx) : op.pre(sp[sa(e)], col, outer, e, idx);
      }
    }
    __syncthreads();
    auto fetch = [&](int e) -> C { return sp[sa(e)]; };
    auto emit = [&](int e, C v) {
      const long long idx = base + e * w.estride;
      dst[idx] = (AXIS == 1) ? op.post(v, col, e, outer, idx) : op.post(v, col, outer, e, idx);
    };
    // the transform ends with a block barrier, so the buffer may be refilled next
    FP::template run<DIR>(t, active, sp, sa, tw, fetch, emit);
  }
  cp_async_wait<0>();
}

// Ops whose store epilogue reads a second array at the stored element (kReadsOld): the
// LSQR update u' = A v - alpha u reads u where it writes u' (the two may be the same
// buffer).  Inside the transform's last stage such a read sits between two stores that
// may alias it, so each of a thread's elements waited for its own load in turn.
template <class Op, class = void> struct ReadsOld : std::false_type {};
template <class Op> struct ReadsOld<Op, std::void_t<decltype(Op::kReadsOld)>> : std::bool_constant<Op::kReadsOld> {};

// k_pass_yz_dx_op (ACC) for ops that read a second array in the epilogue.  The tile of
// that array (op.old_src(), or none) is staged into shared memory with cp.async when the
// tile starts, so it arrives while the transform runs; the transform's last stage writes
// its values back into the tile buffer, and a coalesced epilogue then applies
// op.post_old(v, .., old, scalars, acc) and stores.  op.scalars() (read once per block)
// holds the op's scalars, which no block changes before the last one finishes.  The FP64
// sum runs in the epilogue's element order, fixed for a given launch shape.
template <typename T, int DIR, int AXIS, class FP, int P, class Op>
__global__ void __launch_bounds__(P* FP::T, yz_dx_min_blocks<T, P * FP::T>())
    k_pass_yz_dx_old(Geom g, TileWalk w, const cplx_t<T>* __restrict__ twg, const cplx_t<T>* src, cplx_t<T>* dst,
                     Op op, double* __restrict__ partials, unsigned* counter, const int* __restrict__ done) {
  using C = cplx_t<T>;
  constexpr int n = FP::n;
  if (done != nullptr && *done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  C* buf = tw + ((n + 7) & ~7);
  C* obuf = buf + n * P;
  const int tid = threadIdx.x + threadIdx.y * P;
  for (int i = tid; i < n; i += P * FP::T) tw[i] = twg[i];
  const int px = threadIdx.x;
  const int t = threadIdx.y;
  SAStridedC<P> sa;
  C* sp = buf + px;
  const C* osrc = op.old_src();
  const auto sc = op.scalars();
  double acc[1] = {0.0};
  for (int tile = blockIdx.x; tile < w.ntiles; tile += gridDim.x) {
    const int tx = tile % w.ntx, outer = tile / w.ntx;
    const int col = tx * P + px;
    const bool active = col < g.nxh;
    const long long base = col + (long long)outer * w.ostride;
    if (osrc != nullptr) issue_tile(osrc, obuf, g, w, tile, n, P);
    cp_async_commit();
    auto fetch = [&](int e) -> C {
      const long long idx = base + e * w.estride;
      const C v = src[idx];
      return (AXIS == 1) ? op.pre(v, col, e, outer, idx) : op.pre(v, col, outer, e, idx);
    };
    auto emit = [&](int e, C v) { sp[sa(e)] = v; };
    // the transform ends with a block barrier: the tile buffer holds its results
    FP::template run<DIR>(t, active, sp, sa, tw, fetch, emit);
    cp_async_wait<0>();
    __syncthreads();
    if (active) {
      for (int e = t; e < n; e += FP::T) {
        const long long idx = base + e * w.estride;
        const C o = osrc != nullptr ? obuf[e * P + px] : mk<C>(T(0), T(0));
        dst[idx] = (AXIS == 1) ? op.post_old(sp[sa(e)], col, e, outer, o, sc, acc[0])
                               : op.post_old(sp[sa(e)], col, outer, e, o, sc, acc[0]);
      }
    }
    __syncthreads();  // the next tile's copies and transform overwrite both buffers
  }
  if (grid_sum_last<1>(acc, partials, counter) && tid == 0) op.last(acc[0]);
}

// Compile-time form of k_z_fused_m (FP a FixedPlan, P columns per tile).  Both transforms are inlined,
// so it is compiled for 512 or 640 threads per SM (zm_budget): the 768-thread cap spills.  A
// block whose size is not a multiple of 32 still occupies whole warps, so the block
// count per SM is taken on the warp-rounded size.
template <int THREADS, int BUDGET = 512> constexpr int zm_min_blocks() {
  constexpr int rounded = (THREADS + 31) / 32 * 32;
  return rounded <= BUDGET ? BUDGET / rounded : 1;
}
// Threads per SM the multiplier Z pass of length N is compiled for: 640 (five 128-thread
// blocks, at most 102 registers) where that compiles without spills, as for the 176-point
// benchmark axis (TV-ADMM 256x256x176: 2 us per iteration less); 512 for the lengths whose
// plan spilled at 640 (ptxas: 4-92 bytes per thread).
template <int N> constexpr int zm_budget() {
  return (N == 75 || N == 125 || N == 128 || N == 135 || N == 150 || N == 180 || N == 216 || N == 224 ||
          N == 225 || N == 240 || N == 256)
             ? 512
             : 640;
}
template <typename T, class FP, int P>
__global__ void __launch_bounds__(P* FP::T, zm_min_blocks<P * FP::T, zm_budget<FP::n>()>())
    k_z_fused_m_fx(Geom g, TileWalk w, const cplx_t<T>* __restrict__ twg, const cplx_t<T>* src, cplx_t<T>* dst,
                   const T* __restrict__ mult, const int* __restrict__ done) {
  using C = cplx_t<T>;
  constexpr int n = FP::n;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  C* buf0 = tw + ((n + 7) & ~7);
  C* buf1 = buf0 + n * P;
  T* mb0 = reinterpret_cast<T*>(buf1 + n * P);
  T* mb1 = mb0 + ((n * P + 3) & ~3);
  const int tid = threadIdx.x + threadIdx.y * P;
  for (int i = tid; i < n; i += P * FP::T) tw[i] = twg[i];
  if (done != nullptr && *done) return;
  const int px = threadIdx.x;
  const int t = threadIdx.y;
  SAStridedC<P> sa;
  auto issue = [&](int tl, C* b, T* mb) {
    if (tl >= w.ntiles - w.nmain) {
      issue_tile(src, b, g, w, tl - (w.ntiles - w.nmain), n, P);
      issue_mtile(mult, mb, g, w, tl - (w.ntiles - w.nmain), n, P);
    } else {
      issue_edge_tile(src, b, w, tl, n, P);
      issue_edge_tile(mult, mb, w, tl, n, P);
    }
  };
  int tile = blockIdx.x;
  if (tile < w.ntiles) issue(tile, buf0, mb0);
  cp_async_commit();
  for (int it = 0; tile < w.ntiles; tile += gridDim.x, ++it) {
    C* cur = (it & 1) ? buf1 : buf0;
    C* nxt = (it & 1) ? buf0 : buf1;
    T* mcur = (it & 1) ? mb1 : mb0;
    T* mnxt = (it & 1) ? mb0 : mb1;
    const int next = tile + gridDim.x;
    if (next < w.ntiles) issue(next, nxt, mnxt);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    int col, iy;
    const bool active = tile_pos(g, w, tile, px, P, col, iy);
    const long long base = col + (long long)iy * w.ostride;
    C* sp = cur + px;
    auto fetch = [&](int e) -> C { return sp[sa(e)]; };
    // forward transform scaled by the multiplier in registers, handed to the inverse
    // transform (the reversed plan) without a shared-memory round trip (FetchInRegs)
    auto scale = [&](int e, C v) -> C { return cscale(v, mcur[e * P + px]); };
    EmitInRegs<decltype(scale)> keep{scale};
    FetchInRegs in_regs;
    auto emit = [&](int e, C v) { dst[base + e * w.estride] = v; };
    C v[kFftEmax];
    FP::template run_v<-1>(v, t, active, sp, sa, tw, fetch, keep);
    ReversePlan<FP>::type::template run_v<+1>(v, t, active, sp, sa, tw, in_regs, emit);
  }
  cp_async_wait<0>();
}

// Z forward -> Op::mid pointwise -> Z inverse, tiled like k_pass_yz (outer = y).
template <typename T, class Op, bool BL>
__global__ void __maxnreg__(ZRegCap<T>::value)
    k_z_fused(Geom g, const __grid_constant__ FftPlan1D pl, TileWalk w, const cplx_t<T>* __restrict__ twg,
                          const cplx_t<T>* src, cplx_t<T>* dst, Op op, const int* __restrict__ done) {
  using C = cplx_t<T>;
  if (done != nullptr && *done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  const int n = pl.n;
  const int m = pl.m;  // rows of a tile buffer: n, or the Bluestein convolution length
  const int P = blockDim.x;
  C* buf0 = tw + ((m + 7) & ~7);
  C* buf1 = buf0 + (size_t)m * P;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int i = tid; i < m; i += blockDim.x * blockDim.y) tw[i] = twg[i];
  const int px = threadIdx.x;
  const int t = threadIdx.y;
  SAStrided sa{P};
  int tile = blockIdx.x;
  if (tile < w.ntiles) issue_tile(src, buf0, g, w, tile, n, P);
  cp_async_commit();
  for (int it = 0; tile < w.ntiles; tile += gridDim.x, ++it) {
    C* cur = (it & 1) ? buf1 : buf0;
    C* nxt = (it & 1) ? buf0 : buf1;
    const int next = tile + gridDim.x;
    if (next < w.ntiles) issue_tile(src, nxt, g, w, next, n, P);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const int tx = tile % w.ntx, iy = tile / w.ntx;
    const int col = tx * P + px;
    const bool active = col < g.nxh;
    const long long base = col + (long long)iy * w.ostride;
    C* sp = cur + px;
    fft_pencil<-1, C, SAStrided, false, false, BL>(&pl, t, active, sp, sa, tw, nullptr, nullptr, 0, 0);
    if (active) {
#pragma unroll 1
      for (int e = t; e < n; e += pl.T) sp[sa(e)] = op.mid(sp[sa(e)], col, iy, e, base + e * w.estride);
    }
    __syncthreads();
    fft_pencil<+1, C, SAStrided, false, true, BL>(&pl, t, active, sp, sa, tw, nullptr, dst, base, w.estride);
  }
  cp_async_wait<0>();
}

}  // namespace qsm
