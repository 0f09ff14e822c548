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
//   k_pass_yz : C2C along y or z on a P-column tile (128-byte coalesced rows), with
//               pre/post pointwise hooks.
//   k_z_fused : forward z FFT -> pointwise multiplier -> inverse z FFT in one pass.
//   k_x_c2r   : rebuild two Hermitian rows, inverse FFT along x, hand each real
//               value to a store functor (scale, mask, FP64 reductions, selection).
#pragma once

#include "fft_engine.cuh"

namespace qsm {

struct Geom {
  int nx, ny, nz;
  int nxh;    // nx/2 + 1
  int pitch;  // row pitch of the half spectrum, >= nxh
  __host__ __device__ long long nvox() const { return (long long)nx * ny * nz; }
  __host__ __device__ long long hsize() const { return (long long)pitch * ny * nz; }
  __host__ __device__ int nrows() const { return ny * nz; }
};

template <typename T> struct PadG;
template <> struct PadG<float> { static constexpr int G = 16; };
template <> struct PadG<double> { static constexpr int G = 8; };

template <typename T> __host__ __device__ inline int x_rowlen(int n) { return n + n / PadG<T>::G + 1; }

// Identity pointwise op: Y/Z passes with it stream global -> registers -> global.
template <typename T> struct OpId {
  using C = cplx_t<T>;
  __device__ __forceinline__ C pre(C v, int, int, int, long long) const { return v; }
  __device__ __forceinline__ C post(C v, int, int, int, long long) const { return v; }
  __device__ __forceinline__ C mid(C v, int, int, int, long long) const { return v; }
};
template <class Op> struct IsPlainOp { static constexpr bool value = false; };
template <typename T> struct IsPlainOp<OpId<T>> { static constexpr bool value = true; };

// ---------------------------------------------------------------------------
// X forward: real rows -> half spectrum.  blockDim = (Tb, P) with Tb >= plan T
// (threads t >= T idle, so blocks stay whole warps); P pencils (row pairs).
// ---------------------------------------------------------------------------
template <typename T, class Load>
__global__ void k_x_r2c(Geom g, const __grid_constant__ FftPlan1D pl, const cplx_t<T>* __restrict__ twg,
                        cplx_t<T>* __restrict__ spec, Load ld, const int* __restrict__ done) {
  using C = cplx_t<T>;
  if (done != nullptr && *done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  const int n = pl.n;
  const int rowlen = x_rowlen<T>(n);
  C* sm = tw + n;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int i = tid; i < n; i += blockDim.x * blockDim.y) tw[i] = twg[i];
  const int t = threadIdx.x;
  const int p = threadIdx.y;
  const long long q = (long long)blockIdx.x * blockDim.y + p;
  const long long nrows = g.nrows();
  const long long a = 2 * q, b = 2 * q + 1;
  const bool active = a < nrows && t < pl.T;
  const bool hasb = b < nrows;
  C* sp = sm + p * rowlen;
  SAPadded<PadG<T>::G> sa;
  if (active) {
    for (int e = t; e < n; e += pl.T) {
      const T va = ld((int)a, e);
      const T vb = hasb ? ld((int)b, e) : T(0);
      sp[sa(e)] = mk<C>(va, vb);
    }
  }
  __syncthreads();
  fft_pencil<-1, C, SAPadded<PadG<T>::G>, false, false>(&pl, t, active, sp, sa, tw, nullptr, nullptr, 0, 0);
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
// X inverse: half spectrum -> real rows.  blockDim = (Tb, P) as for k_x_r2c.
// ---------------------------------------------------------------------------
template <typename T, class Store>
__global__ void k_x_c2r(Geom g, const __grid_constant__ FftPlan1D pl, const cplx_t<T>* __restrict__ twg,
                        const cplx_t<T>* __restrict__ spec, Store st0, const int* __restrict__ done) {
  using C = cplx_t<T>;
  if (done != nullptr && *done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  const int n = pl.n;
  const int rowlen = x_rowlen<T>(n);
  C* sm = tw + n;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int i = tid; i < n; i += blockDim.x * blockDim.y) tw[i] = twg[i];
  const int t = threadIdx.x;
  const int p = threadIdx.y;
  const long long q = (long long)blockIdx.x * blockDim.y + p;
  const long long nrows = g.nrows();
  const long long a = 2 * q, b = 2 * q + 1;
  const bool active = a < nrows && t < pl.T;
  const bool hasb = b < nrows;
  C* sp = sm + p * rowlen;
  SAPadded<PadG<T>::G> sa;
  if (active) {
    for (int k = t; k < g.nxh; k += pl.T) {
      C ga = spec[a * g.pitch + k];
      C gb = hasb ? spec[b * g.pitch + k] : mk<C>(T(0), T(0));
      const bool selfm = (k == 0) || (2 * k == n);
      if (selfm) {
        ga.y = T(0);
        gb.y = T(0);
      }
      sp[sa(k)] = mk<C>(ga.x - gb.y, ga.y + gb.x);
      if (!selfm) sp[sa(n - k)] = mk<C>(ga.x + gb.y, gb.x - ga.y);
    }
  }
  __syncthreads();
  fft_pencil<+1, C, SAPadded<PadG<T>::G>, false, false>(&pl, t, active, sp, sa, tw, nullptr, nullptr, 0, 0);
  Store st = st0;
  if (active) {
    for (int e = t; e < n; e += pl.T) {
      const C v = sp[sa(e)];
      st((int)a, e, v.x);
      if (hasb) st((int)b, e, v.y);
    }
  }
  st.finish();
}

// ---------------------------------------------------------------------------
// Y (AXIS=1) or Z (AXIS=2) C2C pass on the half spectrum.  blockDim = (P, T).
// grid = (ceil(nxh/P), nz) for Y, (ceil(nxh/P), ny) for Z.
// Op::pre(v, ix, iy, iz, idx) is applied on load and Op::post on store.
// ---------------------------------------------------------------------------
template <typename T, int DIR, int AXIS, class Op>
__global__ void k_pass_yz(Geom g, const __grid_constant__ FftPlan1D pl, const cplx_t<T>* __restrict__ twg,
                          const cplx_t<T>* src, cplx_t<T>* dst, Op op, const int* __restrict__ done) {
  using C = cplx_t<T>;
  if (done != nullptr && *done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  const int n = pl.n;
  C* sm = tw + n;
  const int P = blockDim.x;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int i = tid; i < n; i += blockDim.x * blockDim.y) tw[i] = twg[i];
  __syncthreads();
  const int px = threadIdx.x;
  const int t = threadIdx.y;
  const int col = blockIdx.x * P + px;
  const bool active = col < g.nxh;
  const int outer = blockIdx.y;
  long long base, estride;
  if (AXIS == 1) {
    base = col + (long long)outer * g.pitch * g.ny;
    estride = g.pitch;
  } else {
    base = col + (long long)outer * g.pitch;
    estride = (long long)g.pitch * g.ny;
  }
  C* sp = sm + px;
  SAStrided sa{P};
  if constexpr (IsPlainOp<Op>::value) {
    fft_pencil<DIR, C, SAStrided, true, true>(&pl, t, active, sp, sa, tw, src, dst, base, estride);
  } else {
    if (active) {
      for (int e = t; e < n; e += pl.T) {
        const long long idx = base + e * estride;
        const C v = src[idx];
        sp[sa(e)] = (AXIS == 1) ? op.pre(v, col, e, outer, idx) : op.pre(v, col, outer, e, idx);
      }
    }
    __syncthreads();
    fft_pencil<DIR, C, SAStrided, false, false>(&pl, t, active, sp, sa, tw, nullptr, nullptr, 0, 0);
    if (active) {
      for (int e = t; e < n; e += pl.T) {
        const long long idx = base + e * estride;
        const C v = sp[sa(e)];
        dst[idx] = (AXIS == 1) ? op.post(v, col, e, outer, idx) : op.post(v, col, outer, e, idx);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Z forward -> Op::mid pointwise -> Z inverse, one pass.  blockDim = (P, T),
// grid = (ceil(nxh/P), ny).
// ---------------------------------------------------------------------------
template <typename T, class Op>
__global__ void k_z_fused(Geom g, const __grid_constant__ FftPlan1D pl, const cplx_t<T>* __restrict__ twg,
                          const cplx_t<T>* src, cplx_t<T>* dst, Op op, const int* __restrict__ done) {
  using C = cplx_t<T>;
  if (done != nullptr && *done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* tw = reinterpret_cast<C*>(smraw);
  const int n = pl.n;
  C* sm = tw + n;
  const int P = blockDim.x;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  for (int i = tid; i < n; i += blockDim.x * blockDim.y) tw[i] = twg[i];
  __syncthreads();
  const int px = threadIdx.x;
  const int t = threadIdx.y;
  const int col = blockIdx.x * P + px;
  const bool active = col < g.nxh;
  const int iy = blockIdx.y;
  const long long base = col + (long long)iy * g.pitch;
  const long long estride = (long long)g.pitch * g.ny;
  C* sp = sm + px;
  SAStrided sa{P};
  fft_pencil<-1, C, SAStrided, true, false>(&pl, t, active, sp, sa, tw, src, nullptr, base, estride);
  if (active) {
    for (int e = t; e < n; e += pl.T) sp[sa(e)] = op.mid(sp[sa(e)], col, iy, e, base + e * estride);
  }
  __syncthreads();
  fft_pencil<+1, C, SAStrided, false, true>(&pl, t, active, sp, sa, tw, nullptr, dst, base, estride);
}

}  // namespace qsm
