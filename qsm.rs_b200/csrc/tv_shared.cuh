// TV-ADMM building blocks shared by the solver, the batched solver and the unrolled
// adjoint: the stencil kernels, the per-iteration multiplier, and the per-volume
// setup / iteration / output launchers.
#pragma once

#include "functors.cuh"
#include "solvers.h"

#include <algorithm>

namespace qsm {

template <typename S> __device__ __forceinline__ S sabs(S x) { return x < S(0) ? -x : x; }

// inv_a = 1/(D^2 + rho*Lneg), 0 where |a| <= 1e-20 (src/inversion/admm.rs:164-168)
template <typename S>
__device__ __forceinline__ S admm_inv_a(const KSpaceT<S>& K, S kx, S ky, S kz, int ix, int iy, int iz, S rho) {
  const S d = K.dipole(kx, ky, kz);
  const S a = d * d + rho * K.lapneg(ix, iy, iz);
  return sabs(a) > S(1e-20) ? S(1) / a : S(0);
}

// x0 = Re IFFT(F(f) * D * inv_a) (admm.rs:169-176), multiplier in double
template <typename T> struct OpAdmmRhs {
  using C = cplx_t<T>;
  KSpace K;
  double rho;
  __device__ __forceinline__ C mid(C v, int ix, int iy, int iz, long long) const {
    const KSpace& k = K;
    const double r = rho;
    const double m = K.sym(ix, iy, iz, [&](double kx, double ky, double kz, int a, int b, int c) {
      return k.dipole(kx, ky, kz) * admm_inv_a<double>(k, kx, ky, kz, a, b, c, r);
    });
    return cscale(v, (T)m);
  }
};

// per-iteration multiplier rho * sym(inv_a) (admm.rs:105-108), working precision
template <typename T> struct OpAdmmMul {
  using C = cplx_t<T>;
  KSpaceT<T> K;
  T rho;
  __device__ __forceinline__ C mid(C v, int ix, int iy, int iz, long long) const {
    const KSpaceT<T>& k = K;
    const T r = rho;
    const T ia = K.sym(ix, iy, iz, [&](T kx, T ky, T kz, int a, int b, int c) {
      return admm_inv_a<T>(k, kx, ky, kz, a, b, c, r);
    });
    return cscale(v, r * ia);
  }
};

// Per-iteration multiplier rho*sym(inv_a) as a real half-spectrum array (spectrum
// layout, padding columns 0), evaluated once per solve in double.
template <typename T>
__global__ void k_admm_mult(Geom g, KSpace K, double rho, T* __restrict__ out) {
  const long long H = g.hsize();
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < H; i += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(i % g.pitch);
    const long long r = i / g.pitch;
    const int iy = (int)(r % g.ny);
    const int iz = (int)(r / g.ny);
    double m = 0.0;
    if (ix < g.nxh) {
      const KSpace& k = K;
      m = rho * K.sym(ix, iy, iz, [&](double kx, double ky, double kz, int a, int b, int c) {
        return admm_inv_a<double>(k, kx, ky, kz, a, b, c, rho);
      });
    }
    out[i] = (T)m;
  }
}

template <typename T> struct StoreReal {
  T* __restrict__ out;
  int nx;
  T scale;
  __device__ __forceinline__ void operator()(int row, int e, T v) { out[(long long)row * nx + e] = v * scale; }
  __device__ __forceinline__ void finish() {}
};

struct TvState {
  int done;       // 1 once relative_change < tol
  int k;          // iteration whose k_tv_step runs next (1-based)
  unsigned counter;
  int conv_iter;  // iteration that converged
  double tol;
  double rc;      // last relative change
};

// Convergence test of x_{k-1} (k >= 2) + z/u update + divergence, periodic BC
// (src/utils/gradient.rs:21-108, src/utils/mod.rs:44-77, src/inversion/admm.rs:117-142).
// x_j = x0 - y_j.  u is read from ui and written to uo; the backward neighbours' g
// components are recomputed from x and ui there.
//
// blockDim = (32, 8): a warp spans 32 consecutive x, so x-neighbours come from
// shuffles; each thread marches through `zchunk` planes keeping x at k-1, k, k+1 and
// u_z at k-1 in registers.  grid = (ceil(nx/32), ceil(ny/8), ceil(nz/zchunk)).
constexpr int kStepBX = 32, kStepBY = 8;

template <typename T, bool WT>
__global__ void __launch_bounds__(kStepBX* kStepBY)
    k_tv_step(int nx, int ny, int nz, int zchunk, T hx, T hy, T hz, T thr, const T* __restrict__ w,
              const T* __restrict__ x0, const T* __restrict__ ycur, const T* __restrict__ yprev,
              const T* __restrict__ ui, T* __restrict__ uo, T* __restrict__ div, double2* __restrict__ partials,
              TvState* st, int check_only) {
  if (st->done) return;
  const int kiter = st->k;
  const bool check = kiter >= 2;
  const long long N = (long long)nx * ny * nz;
  const long long sz = (long long)nx * ny;
  const int lane = threadIdx.x;
  const int i0 = blockIdx.x * kStepBX + lane;
  const int j0 = blockIdx.y * kStepBY + threadIdx.y;
  const bool in = i0 < nx && j0 < ny;
  const int i = i0 < nx ? i0 : nx - 1;  // clamped for the shuffle partners
  const int j = j0 < ny ? j0 : ny - 1;
  const int ip = i + 1 < nx ? i + 1 : 0, im = i > 0 ? i - 1 : nx - 1;
  const int jp = j + 1 < ny ? j + 1 : 0, jm = j > 0 ? j - 1 : ny - 1;
  const int k0 = blockIdx.z * zchunk;
  const int k1 = k0 + zchunk < nz ? k0 + zchunk : nz;
  // x-neighbours through shuffles when the partner lane holds them
  const bool shf_p = (lane < 31) && (i + 1 < nx) && (i0 < nx);
  const bool shf_m = (lane > 0) && (i > 0) && (i0 < nx);
  auto X = [&](long long q) -> T { return x0[q] - ycur[q]; };
  const long long rowj = (long long)j * nx;
  const int kmm = k0 > 0 ? k0 - 1 : nz - 1;
  T x_km = X(kmm * sz + rowj + i);
  T uz_km = check_only ? T(0) : ui[2 * N + kmm * sz + rowj + i];
  T w_km = (WT && !check_only) ? w[kmm * sz + rowj + i] : T(1);
  T x_k = X(k0 * sz + rowj + i);
  double sd = 0.0, sx = 0.0;
  for (int k = k0; k < k1; ++k) {
    const int kp = k + 1 < nz ? k + 1 : 0;
    const long long base = k * sz;
    const long long c = base + rowj + i;
    const T x_kp = X(kp * sz + rowj + i);
    if (check && in) {
      const T xp = x0[c] - yprev[c];
      const double dd = (double)x_k - (double)xp;
      sd += dd * dd;
      sx += (double)x_k * (double)x_k;
    }
    if (!check_only) {
      const T ux = ui[c], uy = ui[N + c], uz = ui[2 * N + c];
      T xip = __shfl_down_sync(0xffffffffu, x_k, 1);
      T xim = __shfl_up_sync(0xffffffffu, x_k, 1);
      T uxm = __shfl_up_sync(0xffffffffu, ux, 1);
      if (!shf_p) xip = X(base + rowj + ip);
      if (!shf_m) {
        xim = X(base + rowj + im);
        uxm = ui[base + rowj + im];
      }
      const T xjp = X(base + (long long)jp * nx + i);
      const long long cjm = base + (long long)jm * nx + i;
      const T xjm = X(cjm);
      const T uym = ui[N + cjm];
      // shrink thresholds: thr, or thr * w at each voxel whose g is formed (weighted
      // shrink, src/utils/mod.rs:57-59)
      T tc = thr, txm = thr, tym = thr, tzm = thr, w_k = T(1);
      if (WT) {
        w_k = w[c];
        tc = thr * w_k;
        txm = thr * w[base + rowj + im];
        tym = thr * w[cjm];
        tzm = thr * w_km;
      }
      const T vx = (xip - x_k) * hx + ux;
      const T vy = (xjp - x_k) * hy + uy;
      const T vz = (x_kp - x_k) * hz + uz;
      const T zx = shrink(vx, tc), zy = shrink(vy, tc), zz = shrink(vz, tc);
      const T gx = T(2) * zx - vx, gy = T(2) * zy - vy, gz = T(2) * zz - vz;
      const T vxm = (x_k - xim) * hx + uxm;
      const T vym = (x_k - xjm) * hy + uym;
      const T vzm = (x_k - x_km) * hz + uz_km;
      const T gxm = T(2) * shrink(vxm, txm) - vxm;
      const T gym = T(2) * shrink(vym, tym) - vym;
      const T gzm = T(2) * shrink(vzm, tzm) - vzm;
      if (in) {
        // the first update sees x_0 = u = g = 0 (admm.rs:18-53): zeros, whatever x_0's
        // buffer holds (RTS keeps its starting iterate there for the first test)
        const bool z0 = kiter == 1;
        uo[c] = z0 ? T(0) : vx - zx;
        uo[N + c] = z0 ? T(0) : vy - zy;
        uo[2 * N + c] = z0 ? T(0) : vz - zz;
        div[c] = z0 ? T(0) : (gx - gxm) * hx + (gy - gym) * hy + (gz - gzm) * hz;
      }
      uz_km = uz;
      w_km = w_k;
    }
    x_km = x_k;
    x_k = x_kp;
  }
  // deterministic two-level reduction: per-block partials, summed in a fixed order
  // by the block that arrives last
  __shared__ int am_last;
  double a = sd, b = sx;
  block_sum2(a, b);
  const int tid = threadIdx.x + kStepBX * threadIdx.y;
  const int nblocks = gridDim.x * gridDim.y * gridDim.z;
  const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (tid == 0) {
    partials[bid] = make_double2(a, b);
    __threadfence();
    const unsigned prev = atomicAdd(&st->counter, 1u);
    am_last = (prev == (unsigned)nblocks - 1);
  }
  __syncthreads();
  if (am_last) {
    __threadfence();
    double pa = 0.0, pb = 0.0;
    for (int i = tid; i < nblocks; i += kStepBX * kStepBY) {
      const double2 p = __ldcg(&partials[i]);
      pa += p.x;
      pb += p.y;
    }
    block_sum2(pa, pb);
    if (tid == 0) {
      if (check) {
        const double rc = sqrt(pa) / (sqrt(pb) + 1e-20);  // src/utils/mod.rs:69-77
        st->rc = rc;
        if (rc < st->tol) {
          st->done = 1;
          st->conv_iter = kiter - 1;
        }
      }
      st->k = kiter + 1;
      st->counter = 0u;
    }
  }
}

// 16-byte vectors: 4 floats or 2 doubles per thread along x.
template <typename T> struct Vec16;
template <> struct Vec16<float> {
  static constexpr int n = 4;
  struct V { float v[4]; };
  static __device__ __forceinline__ V ld(const float* p) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p));
    return V{{a.x, a.y, a.z, a.w}};
  }
  static __device__ __forceinline__ void st(float* p, const V& a) {
    *reinterpret_cast<float4*>(p) = make_float4(a.v[0], a.v[1], a.v[2], a.v[3]);
  }
};
template <> struct Vec16<double> {
  static constexpr int n = 2;
  struct V { double v[2]; };
  static __device__ __forceinline__ V ld(const double* p) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    return V{{a.x, a.y}};
  }
  static __device__ __forceinline__ void st(double* p, const V& a) {
    *reinterpret_cast<double2*>(p) = make_double2(a.v[0], a.v[1]);
  }
};

// k_tv_step with 16-byte vector loads and stores: each thread owns Vec16<T>::n
// consecutive x (nx a multiple of that), x-neighbours across vectors come from the
// adjacent lanes.  Same arithmetic per voxel as k_tv_step.
template <typename T, bool WT>
__global__ void __launch_bounds__(kStepBX* kStepBY)
    k_tv_step_v(int nx, int ny, int nz, int zchunk, T hx, T hy, T hz, T thr, const T* __restrict__ w,
                const T* __restrict__ x0, const T* __restrict__ ycur, const T* __restrict__ yprev,
                const T* __restrict__ ui, T* __restrict__ uo, T* __restrict__ div, double2* __restrict__ partials,
                TvState* st, int check_only) {
  using W = Vec16<T>;
  using V = typename W::V;
  constexpr int NV = W::n;
  if (st->done) return;
  const int kiter = st->k;
  const bool check = kiter >= 2;
  const long long N = (long long)nx * ny * nz;
  const long long sz = (long long)nx * ny;
  const int lane = threadIdx.x;
  const int nxv = nx / NV;
  const int v0 = blockIdx.x * kStepBX + lane;
  const int j0 = blockIdx.y * kStepBY + threadIdx.y;
  const bool in = v0 < nxv && j0 < ny;
  const int i = (v0 < nxv ? v0 : nxv - 1) * NV;  // first x of this thread (clamped for the shuffles)
  const int j = j0 < ny ? j0 : ny - 1;
  const int ip = i + NV < nx ? i + NV : 0, im = i > 0 ? i - 1 : nx - 1;
  const int jp = j + 1 < ny ? j + 1 : 0, jm = j > 0 ? j - 1 : ny - 1;
  const int k0 = blockIdx.z * zchunk;
  const int k1 = k0 + zchunk < nz ? k0 + zchunk : nz;
  const bool shf_p = (lane < 31) && (v0 + 1 < nxv);
  const bool shf_m = (lane > 0) && (v0 > 0) && (v0 < nxv);
  auto X = [&](long long q) -> V {
    const V a = W::ld(x0 + q), b = W::ld(ycur + q);
    V r;
#pragma unroll
    for (int e = 0; e < NV; ++e) r.v[e] = a.v[e] - b.v[e];
    return r;
  };
  auto Xs = [&](long long q) -> T { return x0[q] - ycur[q]; };
  const long long rowj = (long long)j * nx;
  const int kmm = k0 > 0 ? k0 - 1 : nz - 1;
  V x_km = X(kmm * sz + rowj + i);
  V uz_km{}, w_km{};
  if (!check_only) uz_km = W::ld(ui + 2 * N + kmm * sz + rowj + i);
  if (WT && !check_only) w_km = W::ld(w + kmm * sz + rowj + i);
  V x_k = X(k0 * sz + rowj + i);
  double sd = 0.0, sx = 0.0;
  for (int k = k0; k < k1; ++k) {
    const int kp = k + 1 < nz ? k + 1 : 0;
    const long long base = k * sz;
    const long long c = base + rowj + i;
    const V x_kp = X(kp * sz + rowj + i);
    if (check && in) {
      const V a = W::ld(x0 + c), b = W::ld(yprev + c);
#pragma unroll
      for (int e = 0; e < NV; ++e) {
        const double dd = (double)x_k.v[e] - (double)(a.v[e] - b.v[e]);
        sd += dd * dd;
        sx += (double)x_k.v[e] * (double)x_k.v[e];
      }
    }
    if (!check_only) {
      const V ux = W::ld(ui + c), uy = W::ld(ui + N + c), uz = W::ld(ui + 2 * N + c);
      T xnext = __shfl_down_sync(0xffffffffu, x_k.v[0], 1);
      T xprev = __shfl_up_sync(0xffffffffu, x_k.v[NV - 1], 1);
      T uxprev = __shfl_up_sync(0xffffffffu, ux.v[NV - 1], 1);
      if (!shf_p) xnext = Xs(base + rowj + ip);
      if (!shf_m) {
        xprev = Xs(base + rowj + im);
        uxprev = ui[base + rowj + im];
      }
      const V xjp = X(base + (long long)jp * nx + i);
      const long long cjm = base + (long long)jm * nx + i;
      const V xjm = X(cjm);
      const V uym = W::ld(ui + N + cjm);
      // weighted shrink thresholds (src/utils/mod.rs:57-59), as in k_tv_step
      V w_k{}, wjm{};
      T wprev = T(1);
      if (WT) {
        w_k = W::ld(w + c);
        wjm = W::ld(w + cjm);
        wprev = __shfl_up_sync(0xffffffffu, w_k.v[NV - 1], 1);
        if (!shf_m) wprev = w[base + rowj + im];
      }
      V ox, oy, oz, dv;
#pragma unroll
      for (int e = 0; e < NV; ++e) {
        const T xe = x_k.v[e];
        const T xip = e + 1 < NV ? x_k.v[e + 1] : xnext;
        const T xim = e > 0 ? x_k.v[e - 1] : xprev;
        const T uxm = e > 0 ? ux.v[e - 1] : uxprev;
        const T tc = WT ? thr * w_k.v[e] : thr;
        const T txm = WT ? thr * (e > 0 ? w_k.v[e - 1] : wprev) : thr;
        const T tym = WT ? thr * wjm.v[e] : thr;
        const T tzm = WT ? thr * w_km.v[e] : thr;
        const T vx = (xip - xe) * hx + ux.v[e];
        const T vy = (xjp.v[e] - xe) * hy + uy.v[e];
        const T vz = (x_kp.v[e] - xe) * hz + uz.v[e];
        const T zx = shrink(vx, tc), zy = shrink(vy, tc), zz = shrink(vz, tc);
        const T gx = T(2) * zx - vx, gy = T(2) * zy - vy, gz = T(2) * zz - vz;
        const T vxm = (xe - xim) * hx + uxm;
        const T vym = (xe - xjm.v[e]) * hy + uym.v[e];
        const T vzm = (xe - x_km.v[e]) * hz + uz_km.v[e];
        const T gxm = T(2) * shrink(vxm, txm) - vxm;
        const T gym = T(2) * shrink(vym, tym) - vym;
        const T gzm = T(2) * shrink(vzm, tzm) - vzm;
        ox.v[e] = vx - zx;
        oy.v[e] = vy - zy;
        oz.v[e] = vz - zz;
        dv.v[e] = (gx - gxm) * hx + (gy - gym) * hy + (gz - gzm) * hz;
      }
      if (in) {
        if (kiter == 1) {  // first update: x_0 = u = g = 0 (see k_tv_step)
          ox = V{};
          oy = V{};
          oz = V{};
          dv = V{};
        }
        W::st(uo + c, ox);
        W::st(uo + N + c, oy);
        W::st(uo + 2 * N + c, oz);
        W::st(div + c, dv);
      }
      uz_km = uz;
      if (WT) w_km = w_k;
    }
    x_km = x_k;
    x_k = x_kp;
  }
  __shared__ int am_last;
  double a = sd, b = sx;
  block_sum2(a, b);
  const int tid = threadIdx.x + kStepBX * threadIdx.y;
  const int nblocks = gridDim.x * gridDim.y * gridDim.z;
  const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (tid == 0) {
    partials[bid] = make_double2(a, b);
    __threadfence();
    const unsigned prev = atomicAdd(&st->counter, 1u);
    am_last = (prev == (unsigned)nblocks - 1);
  }
  __syncthreads();
  if (am_last) {
    __threadfence();
    double pa = 0.0, pb = 0.0;
    for (int q = tid; q < nblocks; q += kStepBX * kStepBY) {
      const double2 p = __ldcg(&partials[q]);
      pa += p.x;
      pb += p.y;
    }
    block_sum2(pa, pb);
    if (tid == 0) {
      if (check) {
        const double rc = sqrt(pa) / (sqrt(pb) + 1e-20);  // src/utils/mod.rs:69-77
        st->rc = rc;
        if (rc < st->tol) {
          st->done = 1;
          st->conv_iter = kiter - 1;
        }
      }
      st->k = kiter + 1;
      st->counter = 0u;
    }
  }
}

// k_tv_step_v (unweighted, full update; float4 or double2 vectors) with every global read of the plane loop
// staged through shared memory by cp.async.  A four-slot ring per block holds, for
// plane k: x0 and y at plane k+1 for the block's 8 rows and its two halo rows (the
// rows j-1 of the first and j+1 of the last), y_{i-2} and u at plane k, uy of the
// lower halo row, and per row the x-halo scalars (x0, y at the neighbour across the
// warp's ends, ux at the lower one).  Two planes are in flight while one is computed,
// so loads hold no registers and no warp waits on L2 inside the loop.
// Slot s(kk) = (kk - k0 + 1) % 4; slot s(k0 - 1) holds only the plane-k0 part.
// Same arithmetic per voxel as k_tv_step.
constexpr int kStageSlots = 4;
// One ring slot; the vector entries are 16-byte chunks (4 floats or 2 doubles).
template <typename T> struct StepSlot {
  uint4 a[6][kStepBY][kStepBX];  // x0(k+1), y(k+1), y_{i-2}(k), ux(k), uy(k), uz(k)
  uint4 hx0[2][kStepBX];         // halo rows (0: lower, 1: upper) of x0(k+1)
  uint4 hy[2][kStepBX];          // ... and of y(k+1)
  uint4 huy[kStepBX];            // uy(k) of the lower halo row
  T xm[kStepBY][4];              // x0(k+1), y(k+1), ux(k) at the lower x neighbour
  T xp[kStepBY][4];              // x0(k+1), y(k+1) at the upper x neighbour
};
template <typename T> constexpr size_t step_staged_smem() { return (size_t)kStageSlots * sizeof(StepSlot<T>); }

// cp.async of one element (4 or 8 bytes)
template <typename T> __device__ __forceinline__ void cp_async_elem(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (sizeof(T) == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}

template <typename T>
__global__ void __launch_bounds__(kStepBX* kStepBY, 2)
    k_tv_step_s(int nx, int ny, int nz, int zchunk, T hx, T hy, T hz, T thr, const T* __restrict__ x0,
                const T* __restrict__ ycur, const T* __restrict__ yprev, const T* __restrict__ ui,
                T* __restrict__ uo, T* __restrict__ div, double2* __restrict__ partials, TvState* st) {
  using W = Vec16<T>;
  using V = typename W::V;
  using Slot = StepSlot<T>;
  constexpr int NV = W::n;
  if (st->done) return;
  extern __shared__ __align__(16) unsigned char stage_raw[];
  Slot* ring = reinterpret_cast<Slot*>(stage_raw);
  const int kiter = st->k;
  const bool check = kiter >= 2;
  const long long N = (long long)nx * ny * nz;
  const long long sz = (long long)nx * ny;
  const int lane = threadIdx.x, ty = threadIdx.y;
  const int nxv = nx / NV;
  const int v0 = blockIdx.x * kStepBX + lane;
  const int jb = blockIdx.y * kStepBY;
  const int j0 = jb + ty;
  const bool in = v0 < nxv && j0 < ny;
  const int i = (v0 < nxv ? v0 : nxv - 1) * NV;
  const int j = j0 < ny ? j0 : ny - 1;
  const int ip = i + NV < nx ? i + NV : 0, im = i > 0 ? i - 1 : nx - 1;
  const int k0 = blockIdx.z * zchunk;
  const int k1 = k0 + zchunk < nz ? k0 + zchunk : nz;
  const bool shf_p = (lane < 31) && (v0 + 1 < nxv);
  const bool shf_m = (lane > 0) && (v0 > 0) && (v0 < nxv);
  const bool need_p = v0 < nxv && !shf_p;  // the row's last vector: x-halo above
  const bool need_m = v0 < nxv && !shf_m;  // the row's first vector: x-halo below
  // y-neighbours staged by the sibling row (exactly rows j +- 1), else the halo rows
  const bool stj_p = ty + 1 < kStepBY && j0 + 1 < ny;
  const bool stj_m = ty > 0 && j0 < ny;
  const int jlast = jb + kStepBY - 1 < ny ? jb + kStepBY - 1 : ny - 1;
  const long long row_lo = (long long)(jb > 0 ? jb - 1 : ny - 1) * nx;  // row below the block
  const long long row_hi = (long long)(jlast + 1 < ny ? jlast + 1 : 0) * nx;  // row above its last row
  const int ilane = (v0 < nxv ? v0 : nxv - 1) * NV;
  const long long rowj = (long long)j * nx;
  auto slot = [&](int kk) -> Slot& { return ring[(kk - k0 + 1) & (kStageSlots - 1)]; };
  auto issue = [&](int kk) {  // stage for plane kk (kk = k0 - 1: the plane-k0 part only)
    Slot& S = slot(kk);
    const int kn = kk + 1 < nz ? kk + 1 : 0;
    const long long pn = (long long)kn * sz;
    cp_async16(&S.a[0][ty][lane], x0 + pn + rowj + i, true);
    cp_async16(&S.a[1][ty][lane], ycur + pn + rowj + i, true);
    if (ty == 0) {
      cp_async16(&S.hx0[0][lane], x0 + pn + row_lo + ilane, true);
      cp_async16(&S.hy[0][lane], ycur + pn + row_lo + ilane, true);
    } else if (ty == kStepBY - 1) {
      cp_async16(&S.hx0[1][lane], x0 + pn + row_hi + ilane, true);
      cp_async16(&S.hy[1][lane], ycur + pn + row_hi + ilane, true);
    }
    if (need_m) {
      cp_async_elem<T>(&S.xm[ty][0], x0 + pn + rowj + im);
      cp_async_elem<T>(&S.xm[ty][1], ycur + pn + rowj + im);
    }
    if (need_p) {
      cp_async_elem<T>(&S.xp[ty][0], x0 + pn + rowj + ip);
      cp_async_elem<T>(&S.xp[ty][1], ycur + pn + rowj + ip);
    }
    if (kk >= k0) {
      const long long pk = (long long)kk * sz;
      const long long c = pk + rowj + i;
      if (check) cp_async16(&S.a[2][ty][lane], yprev + c, true);
      cp_async16(&S.a[3][ty][lane], ui + c, true);
      cp_async16(&S.a[4][ty][lane], ui + N + c, true);
      cp_async16(&S.a[5][ty][lane], ui + 2 * N + c, true);
      if (ty == 0) cp_async16(&S.huy[lane], ui + N + pk + row_lo + ilane, true);
      if (need_m) cp_async_elem<T>(&S.xm[ty][2], ui + pk + rowj + im);
    }
  };
  auto ldv = [](const uint4& a) -> V {
    V r;
    memcpy(&r, &a, sizeof(V));
    return r;
  };
  auto diffv = [&](const uint4& a, const uint4& b) -> V {
    const V va = ldv(a), vb = ldv(b);
    V r;
#pragma unroll
    for (int e = 0; e < NV; ++e) r.v[e] = va.v[e] - vb.v[e];
    return r;
  };
  auto X = [&](long long q) -> V {
    const V a = W::ld(x0 + q), b = W::ld(ycur + q);
    V r;
#pragma unroll
    for (int e = 0; e < NV; ++e) r.v[e] = a.v[e] - b.v[e];
    return r;
  };
  const int kmm = k0 > 0 ? k0 - 1 : nz - 1;
  V x_km = X(kmm * sz + rowj + i);
  V uz_km = W::ld(ui + 2 * N + kmm * sz + rowj + i);
  issue(k0 - 1);
  cp_async_commit();
  issue(k0);
  cp_async_commit();
  if (k0 + 1 < k1) issue(k0 + 1);
  cp_async_commit();
  double sd = 0.0, sx = 0.0;
  for (int k = k0; k < k1; ++k) {
    if (k + 2 < k1) issue(k + 2);
    cp_async_commit();
    cp_async_wait<2>();  // the stages of planes k - 1 and k have landed
    __syncthreads();
    const Slot& Sp = slot(k - 1);  // x0, y at plane k
    const Slot& Sk = slot(k);      // x0, y at plane k + 1; y_{i-2}, u at plane k
    const long long c = (long long)k * sz + rowj + i;
    const V x_k = diffv(Sp.a[0][ty][lane], Sp.a[1][ty][lane]);
    const V x_kp = diffv(Sk.a[0][ty][lane], Sk.a[1][ty][lane]);
    if (check && in) {
      const V a = ldv(Sp.a[0][ty][lane]), b = ldv(Sk.a[2][ty][lane]);
#pragma unroll
      for (int e = 0; e < NV; ++e) {
        const double dd = (double)x_k.v[e] - (double)(a.v[e] - b.v[e]);
        sd += dd * dd;
        sx += (double)x_k.v[e] * (double)x_k.v[e];
      }
    }
    const V ux = ldv(Sk.a[3][ty][lane]), uy = ldv(Sk.a[4][ty][lane]), uz = ldv(Sk.a[5][ty][lane]);
    T xnext = __shfl_down_sync(0xffffffffu, x_k.v[0], 1);
    T xprev = __shfl_up_sync(0xffffffffu, x_k.v[NV - 1], 1);
    T uxprev = __shfl_up_sync(0xffffffffu, ux.v[NV - 1], 1);
    if (need_p) xnext = Sp.xp[ty][0] - Sp.xp[ty][1];
    if (need_m) {
      xprev = Sp.xm[ty][0] - Sp.xm[ty][1];
      uxprev = Sk.xm[ty][2];
    }
    const V xjp = stj_p ? diffv(Sp.a[0][ty + 1][lane], Sp.a[1][ty + 1][lane]) : diffv(Sp.hx0[1][lane], Sp.hy[1][lane]);
    const V xjm = stj_m ? diffv(Sp.a[0][ty - 1][lane], Sp.a[1][ty - 1][lane]) : diffv(Sp.hx0[0][lane], Sp.hy[0][lane]);
    const V uym = stj_m ? ldv(Sk.a[4][ty - 1][lane]) : ldv(Sk.huy[lane]);
    V ox, oy, oz, dv;
#pragma unroll
    for (int e = 0; e < NV; ++e) {
      const T xe = x_k.v[e];
      const T xip = e + 1 < NV ? x_k.v[e + 1] : xnext;
      const T xim = e > 0 ? x_k.v[e - 1] : xprev;
      const T uxm = e > 0 ? ux.v[e - 1] : uxprev;
      const T vx = (xip - xe) * hx + ux.v[e];
      const T vy = (xjp.v[e] - xe) * hy + uy.v[e];
      const T vz = (x_kp.v[e] - xe) * hz + uz.v[e];
      const T zx = shrink(vx, thr), zy = shrink(vy, thr), zz = shrink(vz, thr);
      const T gx = T(2) * zx - vx, gy = T(2) * zy - vy, gz = T(2) * zz - vz;
      const T vxm = (xe - xim) * hx + uxm;
      const T vym = (xe - xjm.v[e]) * hy + uym.v[e];
      const T vzm = (xe - x_km.v[e]) * hz + uz_km.v[e];
      const T gxm = T(2) * shrink(vxm, thr) - vxm;
      const T gym = T(2) * shrink(vym, thr) - vym;
      const T gzm = T(2) * shrink(vzm, thr) - vzm;
      ox.v[e] = vx - zx;
      oy.v[e] = vy - zy;
      oz.v[e] = vz - zz;
      dv.v[e] = (gx - gxm) * hx + (gy - gym) * hy + (gz - gzm) * hz;
    }
    if (in) {
      if (kiter == 1) {  // first update: x_0 = u = g = 0 (see k_tv_step)
        ox = V{};
        oy = V{};
        oz = V{};
        dv = V{};
      }
      W::st(uo + c, ox);
      W::st(uo + N + c, oy);
      W::st(uo + 2 * N + c, oz);
      W::st(div + c, dv);
    }
    uz_km = uz;
    x_km = x_k;
    __syncthreads();  // slot s(k - 1) is refilled by the next iteration
  }
  cp_async_wait<0>();
  __shared__ int am_last;
  double a = sd, b = sx;
  block_sum2(a, b);
  const int tid = threadIdx.x + kStepBX * threadIdx.y;
  const int nblocks = gridDim.x * gridDim.y * gridDim.z;
  const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (tid == 0) {
    partials[bid] = make_double2(a, b);
    __threadfence();
    const unsigned prev = atomicAdd(&st->counter, 1u);
    am_last = (prev == (unsigned)nblocks - 1);
  }
  __syncthreads();
  if (am_last) {
    __threadfence();
    double pa = 0.0, pb = 0.0;
    for (int q = tid; q < nblocks; q += kStepBX * kStepBY) {
      const double2 p = __ldcg(&partials[q]);
      pa += p.x;
      pb += p.y;
    }
    block_sum2(pa, pb);
    if (tid == 0) {
      if (check) {
        const double rc = sqrt(pa) / (sqrt(pb) + 1e-20);  // src/utils/mod.rs:69-77
        st->rc = rc;
        if (rc < st->tol) {
          st->done = 1;
          st->conv_iter = kiter - 1;
        }
      }
      st->k = kiter + 1;
      st->counter = 0u;
    }
  }
}

template <typename T>
__global__ void k_tv_out(long long N, const T* __restrict__ x0, const T* __restrict__ y,
                         const uint8_t* __restrict__ mask, double* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    out[i] = mask[i] != 0 ? (double)(x0[i] - y[i]) : 0.0;  // apply_mask_zero, src/utils/mask.rs:47-53
}

// Device buffers, launch shapes and constants of one TV-ADMM volume.
template <typename T> struct TvVol {
  GridDims d;
  Fft3<T> f;
  OpAdmmMul<T> mul;
  T* x0;
  T* yb[2];
  T* ub[2];
  T* div;
  T* mult;
  cplx_t<T>* spec;
  double2* partials;
  TvState* st;
  dim3 sgrid;
  int zchunk;
  bool vec, use_mult;
  bool staged = false;  // k_tv_step_s for the full update (unweighted, 16-byte vectors)
  dim3 sgrid_s;
  int zchunk_s = 0;
  T hx, hy, hz, thr, scale;
  const T* w = nullptr;  // per-voxel shrink weights (NLTV); nullptr: unweighted
  const uint8_t* mask;
  double* out;
};

// Autotune the launch shapes of the iteration's Y and fused Z passes for this volume's
// grid, on its spectrum and multiplier buffers before they hold data (instantiated once,
// in tv_fft.cu).
template <typename T> void tv_tune(qsm_ctx* ctx, const TvVol<T>& v);
extern template void tv_tune<float>(qsm_ctx*, const TvVol<float>&);
extern template void tv_tune<double>(qsm_ctx*, const TvVol<double>&);

// Allocate one volume's buffers (workspace names prefixed by `pre`), launch shapes and
// constants; `thr` is the shrink threshold.  The only work enqueued is the launch-shape
// tuning of a grid the context has not seen (tv_tune), which overwrites the new buffers.
template <typename T>
void tv_alloc(qsm_ctx* ctx, TvVol<T>& v, const std::string& pre, const GridDims& d, const double bdir[3],
              double rho_mul, double thr, TvState* st, const uint8_t* d_mask, double* d_out) {
  using C = cplx_t<T>;
  v.d = d;
  v.f = make_fft3<T>(ctx, d);
  v.mul = OpAdmmMul<T>{make_kspace_t<T>(ctx, d, bdir), (T)rho_mul};
  const long long N = d.n;
  const long long H = v.f.g.hsize();
  auto nm = [&](const char* s) { return pre + s; };
  v.x0 = ws<T>(ctx, nm("x0"), (size_t)N);
  v.yb[0] = ws<T>(ctx, nm("y0"), (size_t)N);
  v.yb[1] = ws<T>(ctx, nm("y1"), (size_t)N);
  v.ub[0] = ws<T>(ctx, nm("u0"), (size_t)(3 * N));
  v.ub[1] = ws<T>(ctx, nm("u1"), (size_t)(3 * N));
  v.div = ws<T>(ctx, nm("div"), (size_t)N);
  v.spec = ws<C>(ctx, nm("spec"), (size_t)H);
  // stencil grid: 32x8 threads per block (each thread one x, or one 16-byte vector of
  // x in single precision when nx allows), z split into chunks so that ~3000 blocks run
  v.vec = sizeof(T) == 4 && d.nx % Vec16<T>::n == 0;
  const int xper = v.vec ? Vec16<T>::n : 1;
  const int gbx = (d.nx / xper + kStepBX - 1) / kStepBX, gby = (d.ny + kStepBY - 1) / kStepBY;
  int zchunk = (int)std::max<long long>(2, (long long)d.nz * gbx * gby / 3000);
  if (zchunk > d.nz) zchunk = d.nz;
  v.zchunk = zchunk;
  v.sgrid = dim3(gbx, gby, (d.nz + zchunk - 1) / zchunk);
  size_t nblk = (size_t)v.sgrid.x * v.sgrid.y * v.sgrid.z;
  if (d.nx % Vec16<T>::n == 0) {
    // staged stencil (16-byte vectors): about two waves of 2 blocks per SM, each block
    // marching >= 4 planes
    const int gbxs = (d.nx / Vec16<T>::n + kStepBX - 1) / kStepBX;
    const long long resident = 2LL * sm_count(ctx);
    const long long zc = std::max<long long>(1, 2 * resident / ((long long)gbxs * gby));
    v.zchunk_s = (int)std::min<long long>(d.nz, std::max<long long>(4, (d.nz + zc - 1) / zc));
    v.sgrid_s = dim3(gbxs, gby, (d.nz + v.zchunk_s - 1) / v.zchunk_s);
    v.staged = true;
    nblk = std::max(nblk, (size_t)v.sgrid_s.x * v.sgrid_s.y * v.sgrid_s.z);
  }
  v.partials = ws<double2>(ctx, nm("partials"), nblk);
  v.st = st;
  v.scale = (T)(1.0 / (double)N);
  v.hx = (T)(1.0 / d.vsx);
  v.hy = (T)(1.0 / d.vsy);
  v.hz = (T)(1.0 / d.vsz);
  v.thr = (T)thr;
  v.mask = d_mask;
  v.out = d_out;
  v.mult = ws<T>(ctx, pre + "mult", (size_t)v.f.g.hsize());
  v.use_mult = zm_tile_width<T>(d.nz, v.f.pz.m, v.f.pz.T) > 0;
  tv_tune(ctx, v);
}

// Initial state on ctx->stream: y_0 = x0 (x_0 = 0), u = 0, iteration counter 1.
template <typename T> void tv_init_state(qsm_ctx* ctx, const TvVol<T>& v, double tol) {
  const long long N = v.d.n;
  QSM_CUDA(cudaMemcpyAsync(v.yb[0], v.x0, sizeof(T) * N, cudaMemcpyDeviceToDevice, ctx->stream));
  QSM_CUDA(cudaMemsetAsync(v.ub[0], 0, sizeof(T) * 3 * N, ctx->stream));
  TvState init{};
  init.k = 1;
  init.tol = tol;
  QSM_CUDA(cudaMemcpyAsync(v.st, &init, sizeof(TvState), cudaMemcpyHostToDevice, ctx->stream));
}

// TV-ADMM setup: buffers, x0 = Re IFFT(F(f) * sym(D * inv_a)), the per-iteration
// multiplier rho * sym(inv_a) and the initial state (st is this volume's device state).
template <typename T>
void tv_setup(qsm_ctx* ctx, TvVol<T>& v, const std::string& pre, const GridDims& d, const double* d_f,
              const uint8_t* d_mask, const double bdir[3], const qsm_tv_params& p, TvState* st, double* d_out) {
  tv_alloc<T>(ctx, v, pre, d, bdir, p.rho, p.lambda / p.rho, st, d_mask, d_out);
  const KSpace K64 = make_kspace(ctx, d, bdir);
  const long long H = v.f.g.hsize();
  run_x_r2c<T>(ctx, v.f, v.spec, LoadCast<double, T>{d_f, d.nx}, nullptr);
  run_yz<T, -1, 1>(ctx, v.f, v.spec, v.spec, OpId<T>{}, nullptr);
  run_z_fused<T>(ctx, v.f, v.spec, v.spec, OpAdmmRhs<T>{K64, p.rho}, nullptr);
  run_yz<T, +1, 1>(ctx, v.f, v.spec, v.spec, OpId<T>{}, nullptr);
  run_x_c2r<T>(ctx, v.f, v.spec, StoreReal<T>{v.x0, d.nx, v.scale}, nullptr);
  tv_init_state<T>(ctx, v, p.tol);
  // precomputed multiplier tiles need P*sizeof(T) >= 16 (always true for the
  // 128-byte tiles; narrow tiles of very long z axes use the in-kernel multiplier)
  LaunchScope ls(ctx, "admm_mult");
  k_admm_mult<T><<<grid1d(H), 256, 0, ctx->stream>>>(v.f.g, K64, p.rho, v.mult);
  ls.done();
}

// iteration i with parity q = i % 2: reads y_{i-1} = yb[1-q], y_{i-2} = yb[q],
// u = ub[1-q]; writes u' = ub[q], y_i = yb[q]
template <typename T> void tv_step_launch(qsm_ctx* ctx, const TvVol<T>& v, int q, int check_only) {
  {
    if (v.staged && !v.w && !check_only) {
      ensure_smem(k_tv_step_s<T>, step_staged_smem<T>());
      LaunchScope ls(ctx, "tv_step");
      k_tv_step_s<T><<<v.sgrid_s, dim3(kStepBX, kStepBY), step_staged_smem<T>(), ctx->stream>>>(
          v.d.nx, v.d.ny, v.d.nz, v.zchunk_s, v.hx, v.hy, v.hz, v.thr, v.x0, v.yb[1 - q], v.yb[q], v.ub[1 - q],
          v.ub[q], v.div, v.partials, v.st);
      ls.done();
      return;
    }
  }
  LaunchScope ls(ctx, "tv_step");
  auto kern = v.w ? (v.vec ? k_tv_step_v<T, true> : k_tv_step<T, true>)
                  : (v.vec ? k_tv_step_v<T, false> : k_tv_step<T, false>);
  kern<<<v.sgrid, dim3(kStepBX, kStepBY), 0, ctx->stream>>>(v.d.nx, v.d.ny, v.d.nz, v.zchunk, v.hx, v.hy, v.hz,
                                                              v.thr, v.w, v.x0, v.yb[1 - q], v.yb[q], v.ub[1 - q],
                                                              v.ub[q], v.div, v.partials, v.st, check_only);
  ls.done();
}

// y_i = Re IFFT(rho * sym(inv_a) * F(div)) into yb[q], skipped once the state is done
// (compile-time passes for the wide length list; instantiated once, in tv_fft.cu).
// div and the half spectrum are dead once the X passes have read them (the next step
// writes div and the next X r2c writes the spectrum before either is read again), so
// those passes drop their L2 lines rather than leave them to be written back to HBM
// while the stencil streams.
template <typename T> void tv_fft(qsm_ctx* ctx, const TvVol<T>& v, int q, const int* done) {
  run_x_r2c<T, true, true>(ctx, v.f, v.spec, LoadCast<T, T>{v.div, v.d.nx}, done);
  run_yz<T, -1, 1, true>(ctx, v.f, v.spec, v.spec, OpId<T>{}, done);
  if (v.use_mult) run_z_fused_m<T, true>(ctx, v.f, v.spec, v.spec, v.mult, done);
  else run_z_fused<T>(ctx, v.f, v.spec, v.spec, v.mul, done);
  run_yz<T, +1, 1, true>(ctx, v.f, v.spec, v.spec, OpId<T>{}, done);
  run_x_c2r<T, true, true>(ctx, v.f, v.spec, StoreReal<T>{v.yb[q], v.d.nx, v.scale}, done);
}
extern template void tv_fft<float>(qsm_ctx*, const TvVol<float>&, int, const int*);
extern template void tv_fft<double>(qsm_ctx*, const TvVol<double>&, int, const int*);
template <typename T> void tv_fft(qsm_ctx* ctx, const TvVol<T>& v, int q) { tv_fft(ctx, v, q, &v.st->done); }

// Each pass's candidates are timed inside a whole iteration (the stencil, then X r2c, Y,
// Z, Y, X c2r on the volume's buffers, which hold no data yet), one pass after the other
// with the passes already tuned at their choice.  Timed alone, back to back with itself,
// a pass favoured shapes that were slower in the iteration (one block per tile: 17.0
// against 18.6 us alone, 201.4 against 196.4 us per TV-ADMM iteration at 256x256x176);
// timed in the FFT passes without the stencil, with L2 holding the spectrum rather than
// the stencil's streams, the fused Z pass's pick changed from box to box (35.5 against
// 37.2 us in the iteration).  The stencil runs on a state made for the tuning (iteration
// 2, tol 0, so it never stops early); every caller initialises the state afterwards.
template <typename T> void tv_tune(qsm_ctx* ctx, const TvVol<T>& v) {
  TvState tune_state{};
  tune_state.k = 2;
  tune_state.tol = 0.0;
  QSM_CUDA(cudaMemcpyAsync(v.st, &tune_state, sizeof(TvState), cudaMemcpyHostToDevice, ctx->stream));
  const std::function<void()> chain = [&] {
    tv_step_launch(ctx, v, 0, 0);
    tv_fft(ctx, v, 0, nullptr);
  };
  tune_yz_fixed<T, -1, 1, true>(ctx, v.f, v.spec, &chain);
  tune_yz_fixed<T, +1, 1, true>(ctx, v.f, v.spec, &chain);
  if (v.use_mult) tune_z_fused_m<T, true>(ctx, v.f, v.spec, v.mult, &chain);
}

template <typename T> void tv_iter(qsm_ctx* ctx, const TvVol<T>& v, int q) {
  tv_step_launch(ctx, v, q, 0);
  tv_fft(ctx, v, q);
}

template <typename T> void tv_out_launch(qsm_ctx* ctx, const TvVol<T>& v, size_t completed) {
  LaunchScope ls(ctx, "tv_out");
  k_tv_out<T><<<grid1d(v.d.n), 256, 0, ctx->stream>>>(v.d.n, v.x0, v.yb[completed % 2], v.mask, v.out);
  ls.done();
}

// Instantiate a captured graph; the launch count it holds is returned in *per.
inline cudaGraphExec_t instantiate(qsm_ctx* ctx, cudaGraph_t graph) {
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) throw QsmError(QSM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
  return exec;
}


// Enqueue iterations first..last (1-based, inclusive) of an initialised volume whose
// TvState has k == first.  Pairs of iterations run as one CUDA graph; when `watch`,
// poll() (which reads the device state and returns true once done) runs every
// `poll_launches` graph launches (2 * poll_launches iterations), so that a converged
// solve stops launching and progress reaches the caller.  Returns poll()'s last answer
// (false when it never ran).
template <typename T, class Poll>
bool tv_iterate(qsm_ctx* ctx, const TvVol<T>& v, size_t first, size_t last, bool watch, const Poll& poll,
                size_t poll_launches = 8) {
  if (poll_launches < 1) poll_launches = 1;
  if (last < first) return false;
  const size_t count = last - first + 1;
  bool converged = false;
  if (ctx->profiling || count < 2) {
    // eager launches (per-kernel timing, or too short to be worth a graph)
    for (size_t it = first; it <= last && !converged; ++it) {
      tv_iter(ctx, v, (int)(it % 2));
      if (watch && ((it - first + 1) % (2 * poll_launches) == 0)) converged = poll();
    }
    return converged;
  }
  const int q0 = (int)(first % 2);
  cudaGraph_t graph = nullptr;
  const uint64_t l0 = ctx->launches;
  QSM_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  try {
    tv_iter(ctx, v, q0);
    tv_iter(ctx, v, 1 - q0);
  } catch (...) {
    cudaStreamEndCapture(ctx->stream, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  QSM_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
  const uint64_t per_pair = ctx->launches - l0;
  ctx->launches = l0;
  cudaGraphExec_t exec = instantiate(ctx, graph);
  const size_t pairs = count / 2;
  const size_t chunk = poll_launches;  // graph launches between host polls when watching
  try {
    size_t launched = 0;
    while (launched < pairs && !converged) {
      const size_t todo = watch ? std::min(chunk, pairs - launched) : (pairs - launched);
      for (size_t c = 0; c < todo; ++c) {
        QSM_CUDA(cudaGraphLaunch(exec, ctx->stream));
        ctx->launches += per_pair;
      }
      launched += todo;
      if (watch) converged = poll();
    }
    if (!converged && (count % 2 == 1)) tv_iter(ctx, v, (int)(last % 2));
  } catch (...) {
    cudaGraphExecDestroy(exec);
    throw;
  }
  cudaGraphExecDestroy(exec);
  return converged;
}

// Graph launches between host polls: with a progress callback after every launch (the
// caller hears of each iteration at most two iterations late), otherwise every 8
// launches (only the convergence flag is read; launches after convergence return at
// once on the device).
inline size_t tv_poll_launches(qsm_progress_fn progress) { return progress != nullptr ? 1 : 8; }

// Iterate an initialised volume (tv_setup or an equivalent) until relative_change < tol
// or max_iter iterations, write chi, and deliver progress as (iter, max_iter) per
// iteration plus (iters, iters) on convergence (src/inversion/tv.rs:78-93).  Returns the
// iterations run.
template <typename T>
size_t tv_run(qsm_ctx* ctx, const TvVol<T>& v, size_t max_iter, double tol, qsm_progress_fn progress, void* user) {
  TvState* st = v.st;
  const bool watch = (progress != nullptr) || (tol > 0.0);
  TvState hs{};
  size_t reported = 0;
  auto poll = [&]() {
    QSM_CUDA(cudaMemcpyAsync(&hs, st, sizeof(TvState), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    // the test-only step after the last iteration also advances k: clamp to max_iter
    const size_t completed = std::min(max_iter, hs.done ? (size_t)hs.conv_iter : (size_t)(hs.k - 1));
    if (progress)
      for (; reported < completed; ++reported) progress(user, reported + 1, max_iter);
    return hs.done != 0;
  };
  tv_iterate(ctx, v, 1, max_iter, watch, poll, tv_poll_launches(progress));
  bool converged = poll();
  size_t completed = converged ? (size_t)hs.conv_iter : max_iter;
  if (!converged && max_iter >= 1 && tol > 0.0) {
    // the reference also tests the last iterate (tv.rs:85-91)
    tv_step_launch(ctx, v, (int)((max_iter + 1) % 2), 1);
    converged = poll();
    completed = max_iter;
  }
  tv_out_launch(ctx, v, completed);
  sync(ctx);
  if (progress) {
    for (; reported < completed; ++reported) progress(user, reported + 1, max_iter);
    if (converged) progress(user, completed, completed);
  }
  return completed;
}

}  // namespace qsm
