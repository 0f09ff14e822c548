// Loaders (real input of an X forward pass), stores (real output of an X inverse
// pass) and small reductions shared by the solvers.
#pragma once

#include "launch.cuh"

namespace qsm {

// ---------------------------------------------------------------- loaders --
template <typename Tin, typename T> struct LoadCast {
  const Tin* p;
  int nx;
  __device__ __forceinline__ T operator()(int row, int e) const { return (T)p[(long long)row * nx + e]; }
  __device__ __forceinline__ const Tin* row_begin(int row) const { return p + (long long)row * nx; }
};

// value where mask != 0, else 0
template <typename Tin, typename T> struct LoadMasked {
  const Tin* p;
  const uint8_t* mask;
  int nx;
  __device__ __forceinline__ T operator()(int row, int e) const {
    const long long i = (long long)row * nx + e;
    return mask[i] != 0 ? (T)p[i] : T(0);
  }
};

// ----------------------------------------------------------------- stores --
// out[i] = mask[i] != 0 ? v*scale : 0, written as double
template <typename T> struct StoreMaskedF64 {
  double* __restrict__ out;
  const uint8_t* __restrict__ mask;
  int nx;
  T scale;
  __device__ __forceinline__ void operator()(int row, int e, T v) {
    const long long i = (long long)row * nx + e;
    out[i] = mask == nullptr || __ldg(mask + i) != 0 ? (double)(v * scale) : 0.0;
  }
  __device__ __forceinline__ void finish() {}
};

// out[i] = (mask == null || mask[i] == 1) ? v*scale : 0 in working precision
template <typename T> struct StoreMaskEqOne {
  T* __restrict__ out;
  const uint8_t* __restrict__ mask;
  int nx;
  T scale;
  __device__ __forceinline__ void operator()(int row, int e, T v) {
    const long long i = (long long)row * nx + e;
    out[i] = (mask == nullptr || __ldg(mask + i) == 1) ? v * scale : T(0);
  }
  __device__ __forceinline__ void finish() {}
};

// ------------------------------------------------------------- reductions --
// Sum two doubles over the block; the result is valid in thread 0.
__device__ __forceinline__ void block_sum2(double& a, double& b) {
  __shared__ double red[2][32];
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nth = blockDim.x * blockDim.y * blockDim.z;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const int lane = tid & 31, wid = tid >> 5;
  __syncthreads();
  if (lane == 0) {
    red[0][wid] = a;
    red[1][wid] = b;
  }
  __syncthreads();
  const int nw = (nth + 31) >> 5;
  if (wid == 0) {
    a = lane < nw ? red[0][lane] : 0.0;
    b = lane < nw ? red[1][lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
  }
}

}  // namespace qsm
