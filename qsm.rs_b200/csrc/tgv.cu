// TGV-QSM (src/inversion/tgv.rs:1045-1299): single-step susceptibility from wrapped
// phase with a TGV prior, primal-dual iterations in single precision like the reference.
//
// Setup: mask erosions (src/utils/mask.rs:59-92) and the bounding box of the innermost
// mask (padding 2) on the device; the 27-point dipole stencil fitted by least squares to
// the dipole field through DST-I Poisson solves on a 64^3 grid (tgv.rs:272-479) on the
// host in double (13 solves in parallel threads, cached per voxel size and field
// direction); the wrapped-phase Laplacian (tgv.rs:716-777) minus its mean over the mask.
//
// Iteration (all arrays over the bounding box, float):
//   k_tgv_dual   : eta += sigma(-L(phi_) + S(chi_) - L0)      (L: masked Neumann Laplacian,
//                  p   = proj_a1(p + s*grad chi_ - s*w_)        S: 27-point stencil)
//                  q   = proj_a0(q + s*symgrad w_)
//   k_tgv_primal : phi = (phi + tau L(m0 eta)) / (1 + tau m)
//                  chi = chi + ts(div_m0 p - S(m0 eta));  w = w + m ts(p + symdiv(m0 q))
//                  and the extrapolations x_ = 2x_new - x_old in the same pass.
// The current iterate and its extrapolation share two buffers per variable: the primal
// kernel reads x_old from one, writes x_new to the other and 2x_new - x_old back to the
// first, so the roles alternate with the iteration parity.  Every 100 iterations a check
// kernel computes the relative change of chi over the mask (tgv.rs:923-941) and sets a
// device flag that stops the remaining launches; 100 iterations are replayed as one
// CUDA graph.
#include "functors.cuh"
#include "solvers.h"

#include <array>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>

namespace qsm {

namespace {

// ================================================================== stencil ==
// Jacobi eigen-decomposition pseudo-inverse solve of the 13x13 normal equations
// (src/inversion/tgv.rs:558-654).
std::vector<double> jacobi_pinv_solve(std::vector<std::vector<double>> a, const std::vector<double>& h) {
  const int n = (int)h.size();
  std::vector<std::vector<double>> v(n, std::vector<double>(n, 0.0));
  for (int i = 0; i < n; ++i) v[i][i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double max_off = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) max_off = std::max(max_off, std::fabs(a[i][j]));
    if (max_off < 1e-15) break;
    for (int p = 0; p < n; ++p) {
      for (int q = p + 1; q < n; ++q) {
        if (std::fabs(a[p][q]) < 1e-15) continue;
        const double app = a[p][p], aqq = a[q][q], apq = a[p][q];
        const double tau = (aqq - app) / (2.0 * apq);
        const double t = tau >= 0.0 ? 1.0 / (tau + std::sqrt(1.0 + tau * tau))
                                    : -1.0 / (-tau + std::sqrt(1.0 + tau * tau));
        const double c = 1.0 / std::sqrt(1.0 + t * t);
        const double s = t * c;
        for (int i = 0; i < n; ++i) {
          if (i == p || i == q) continue;
          const double aip = a[i][p], aiq = a[i][q];
          a[i][p] = c * aip - s * aiq;
          a[p][i] = a[i][p];
          a[i][q] = s * aip + c * aiq;
          a[q][i] = a[i][q];
        }
        a[p][p] = c * c * app - 2.0 * c * s * apq + s * s * aqq;
        a[q][q] = s * s * app + 2.0 * c * s * apq + c * c * aqq;
        a[p][q] = 0.0;
        a[q][p] = 0.0;
        for (int i = 0; i < n; ++i) {
          const double vip = v[i][p], viq = v[i][q];
          v[i][p] = c * vip - s * viq;
          v[i][q] = s * vip + c * viq;
        }
      }
    }
  }
  double max_eigen = 0.0;
  for (int i = 0; i < n; ++i) max_eigen = std::max(max_eigen, std::fabs(a[i][i]));
  const double thr = 1e-10 * max_eigen;
  std::vector<double> vth(n, 0.0), x(n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) vth[i] += v[j][i] * h[j];
  for (int i = 0; i < n; ++i) vth[i] = std::fabs(a[i][i]) > thr ? vth[i] / a[i][i] : 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) x[i] += v[i][j] * vth[j];
  return x;
}

// st[di][dj][dk] (each in 0..2) of the fitted oblique stencil, float, tgv.rs:272-479.
using Stencil = std::array<float, 27>;
inline int sidx(int di, int dj, int dk) { return (di * 3 + dj) * 3 + dk; }

Stencil oblique_stencil(float rx, float ry, float rz, float b0x, float b0y, float b0z) {
  constexpr int n = 64, mid = 32, n2 = n * n, n3 = n * n * n;
  const double dx = rx, dy = ry, dz = rz;
  const double bn = std::sqrt((double)(b0x * b0x + b0y * b0y + b0z * b0z));
  const double bd[3] = {(double)b0x / bn, (double)b0y / bn, (double)b0z / bn};
  // sin table S[j][k] = sin(pi (j+1)(k+1)/(n+1)) and DST-I eigenvalues
  std::vector<double> S(n * n), c2(n), lam(n3);
  const double scale = kPi / (n + 1.0);
  for (int j = 0; j < n; ++j)
    for (int k = 0; k < n; ++k) S[j * n + k] = std::sin((j + 1.0) * (k + 1.0) * scale);
  for (int k = 0; k < n; ++k) {
    const double v = 2.0 * std::sin(kPi * (k + 1.0) / (2.0 * (n + 1.0)));
    c2[k] = v * v;
  }
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) lam[i + j * n + k * n2] = c2[i] + c2[j] + c2[k];
  // dipole field at points with r >= 4 (flat order, x fastest)
  std::vector<int> valid;
  std::vector<double> dval;
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        const double x = i - (double)mid, y = j - (double)mid, z = k - (double)mid;
        const double r = std::sqrt(x * x + y * y + z * z);
        if (r < 4.0) continue;
        const double xz = (bd[0] * x + bd[1] * y + bd[2] * z) / r;
        valid.push_back(i + j * n + k * n2);
        dval.push_back((3.0 * xz * xz - 1.0) / (4.0 * kPi * r * r * r));
      }
  std::vector<std::array<int, 3>> pos;
  for (int dk = -1; dk <= 1; ++dk)
    for (int dj = -1; dj <= 1; ++dj)
      for (int di = -1; di <= 1; ++di)
        if (di || dj || dk) pos.push_back({di, dj, dk});
  const double iscale = std::pow(2.0 / (n + 1.0), 3);
  std::vector<std::vector<double>> rows(13);
  auto solve_pair = [&](int p) {
    // forward DST-I of the delta (+1 at mid+I and mid-I, -2 at mid), divided by -lambda
    const int pts[3][3] = {{mid + pos[p][0], mid + pos[p][1], mid + pos[p][2]},
                           {mid - pos[p][0], mid - pos[p][1], mid - pos[p][2]},
                           {mid, mid, mid}};
    const double val[3] = {1.0, 1.0, -2.0};
    std::vector<double> a(n3), b(n3);
    for (int k3 = 0; k3 < n; ++k3)
      for (int k2 = 0; k2 < n; ++k2)
        for (int k1 = 0; k1 < n; ++k1) {
          double s = 0.0;
          for (int t = 0; t < 3; ++t)
            s += val[t] * S[pts[t][0] * n + k1] * S[pts[t][1] * n + k2] * S[pts[t][2] * n + k3];
          const int idx = k1 + k2 * n + k3 * n2;
          a[idx] = s / -lam[idx];
        }
    // inverse DST-I (= forward up to the scale), separable along x, y, z
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j) {
        const double* in = &a[j * n + k * n2];
        double* out = &b[j * n + k * n2];
        for (int q = 0; q < n; ++q) {
          double s = 0.0;
          for (int t = 0; t < n; ++t) s += in[t] * S[t * n + q];
          out[q] = s;
        }
      }
    for (int k = 0; k < n; ++k)
      for (int i = 0; i < n; ++i)
        for (int q = 0; q < n; ++q) {
          double s = 0.0;
          for (int t = 0; t < n; ++t) s += b[i + t * n + k * n2] * S[t * n + q];
          a[i + q * n + k * n2] = s;
        }
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i)
        for (int q = 0; q < n; ++q) {
          double s = 0.0;
          for (int t = 0; t < n; ++t) s += a[i + j * n + t * n2] * S[t * n + q];
          b[i + j * n + q * n2] = s;
        }
    std::vector<double>& row = rows[p];
    row.resize(valid.size());
    for (size_t v = 0; v < valid.size(); ++v) row[v] = b[valid[v]] * iscale;
  };
  std::vector<std::thread> th;
  for (int p = 0; p < 13; ++p) th.emplace_back(solve_pair, p);
  for (auto& t : th) t.join();
  std::vector<std::vector<double>> g(13, std::vector<double>(13, 0.0));
  std::vector<double> h(13, 0.0);
  for (int i = 0; i < 13; ++i) {
    for (int j = 0; j <= i; ++j) {
      double dot = 0.0;
      for (size_t v = 0; v < valid.size(); ++v) dot += rows[i][v] * rows[j][v];
      g[i][j] = g[j][i] = dot;
    }
    double dot = 0.0;
    for (size_t v = 0; v < valid.size(); ++v) dot += rows[i][v] * dval[v];
    h[i] = dot;
  }
  const std::vector<double> y = jacobi_pinv_solve(g, h);
  Stencil st{};
  for (int p = 0; p < 13; ++p) {
    const float c = (float)y[p];
    st[sidx(pos[p][0] + 1, pos[p][1] + 1, pos[p][2] + 1)] = c;
    st[sidx(pos[25 - p][0] + 1, pos[25 - p][1] + 1, pos[25 - p][2] + 1)] = c;
  }
  for (int dk = -1; dk <= 1; ++dk)
    for (int dj = -1; dj <= 1; ++dj)
      for (int di = -1; di <= 1; ++di) {
        if (!di && !dj && !dk) continue;
        const double i2 = di * di, j2 = dj * dj, k2 = dk * dk;
        const double w = (i2 / (dx * dx) + j2 / (dy * dy) + k2 / (dz * dz)) / (i2 + j2 + k2);
        st[sidx(di + 1, dj + 1, dk + 1)] *= (float)w;
      }
  float total = 0.0f;
  for (int dk = 0; dk < 3; ++dk)
    for (int dj = 0; dj < 3; ++dj)
      for (int di = 0; di < 3; ++di)
        if (!(di == 1 && dj == 1 && dk == 1)) total += st[sidx(di, dj, dk)];
  st[sidx(1, 1, 1)] = -total;
  return st;
}

const Stencil& cached_stencil(float rx, float ry, float rz, float bx, float by, float bz) {
  static std::mutex mu;
  static std::map<std::array<float, 6>, Stencil> cache;
  const std::array<float, 6> key{rx, ry, rz, bx, by, bz};
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(key);
  if (it == cache.end()) it = cache.emplace(key, oblique_stencil(rx, ry, rz, bx, by, bz)).first;
  return it->second;
}

// compute_operator_norm_sqr, src/inversion/tgv.rs:839-876 (float power iteration)
float operator_norm_sqr(float g, float g2, float w) {
  const float g4 = g2 * g2, g2w = g2 * w, g2w2 = g2 + w * w, g21 = g2 + 1.0f;
  float v[3] = {1.0f, 1.0f, 1.0f};
  for (int it = 0; it < 20; ++it) {
    const float y0 = g4 * v[0] + g2w * v[1];
    const float y1 = g2w * v[0] + g2w2 * v[1] + g * v[2];
    const float y2 = g * v[1] + g21 * v[2];
    const float nrm = std::sqrt(y0 * y0 + y1 * y1 + y2 * y2);
    if (nrm < 1e-10f) break;
    v[0] = y0 / nrm;
    v[1] = y1 / nrm;
    v[2] = y2 / nrm;
  }
  const float y0 = g4 * v[0] + g2w * v[1];
  const float y1 = g2w * v[0] + g2w2 * v[1] + g * v[2];
  const float y2 = g * v[1] + g21 * v[2];
  return v[0] * y0 + v[1] * y1 + v[2] * y2;
}

struct TgvConst {
  float st[27];  // st[(di*3+dj)*3+dk]
};

// ============================================================ setup kernels ==
// erode_mask one step (src/utils/mask.rs:59-92): faces of the volume and voxels with a
// zero 6-neighbour are removed
__global__ void k_erode(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int nx, int ny, int nz) {
  const long long N = (long long)nx * ny * nz, sxy = (long long)nx * ny;
  for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(l % nx), y = (int)((l / nx) % ny), z = (int)(l / sxy);
    uint8_t v = in[l];
    if (v != 0 && (x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || z == 0 || z == nz - 1 || in[l - 1] == 0 ||
                   in[l + 1] == 0 || in[l - nx] == 0 || in[l + nx] == 0 || in[l - sxy] == 0 || in[l + sxy] == 0))
      v = 0;
    out[l] = v;
  }
}

// min/max coordinates of the nonzero voxels: box[0..2] = min x,y,z; box[3..5] = max
__global__ void k_mask_bbox(const uint8_t* __restrict__ m, int nx, int ny, int nz, int* box) {
  const long long N = (long long)nx * ny * nz, sxy = (long long)nx * ny;
  int lo[3] = {nx, ny, nz}, hi[3] = {-1, -1, -1};
  for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += (long long)gridDim.x * blockDim.x) {
    if (m[l] == 0) continue;
    const int c[3] = {(int)(l % nx), (int)((l / nx) % ny), (int)(l / sxy)};
    for (int a = 0; a < 3; ++a) {
      lo[a] = min(lo[a], c[a]);
      hi[a] = max(hi[a], c[a]);
    }
  }
  for (int a = 0; a < 3; ++a) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[a] = min(lo[a], __shfl_down_sync(0xffffffffu, lo[a], o));
      hi[a] = max(hi[a], __shfl_down_sync(0xffffffffu, hi[a], o));
    }
  }
  if ((threadIdx.x & 31) == 0)
    for (int a = 0; a < 3; ++a) {
      atomicMin(&box[a], lo[a]);
      atomicMax(&box[3 + a], hi[a]);
    }
}

struct Box {
  int x0, y0, z0, bx, by, bz;
  __host__ __device__ long long n() const { return (long long)bx * by * bz; }
};

// sub-volume extraction: phase as float, both masks
__global__ void k_tgv_extract(Box b, int nx, int ny, const double* __restrict__ phase, const uint8_t* __restrict__ m0,
                              const uint8_t* __restrict__ me, float* __restrict__ ph, uint8_t* __restrict__ m0s,
                              uint8_t* __restrict__ mes) {
  const long long N = b.n();
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < N; s += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(s % b.bx), j = (int)((s / b.bx) % b.by), k = (int)(s / ((long long)b.bx * b.by));
    const long long f = (b.x0 + i) + (long long)(b.y0 + j) * nx + (long long)(b.z0 + k) * nx * ny;
    ph[s] = (float)phase[f];
    m0s[s] = m0[f];
    mes[s] = me[f];
  }
}

// sin and cos of the phase (float, like f32::sin / f32::cos)
__global__ void k_tgv_sincos(long long N, const float* __restrict__ ph, float* __restrict__ sn, float* __restrict__ cs) {
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < N; s += (long long)gridDim.x * blockDim.x) {
    sn[s] = sinf(ph[s]);
    cs[s] = cosf(ph[s]);
  }
}

// compute_phase_laplacian (tgv.rs:716-738) with the clamped 7-point Laplacian of
// tgv.rs:741-777; also accumulates the masked sum for the mean (FP64)
__global__ void k_tgv_phase_lap(Box b, float hx2, float hy2, float hz2, const float* __restrict__ sn,
                                const float* __restrict__ cs, const uint8_t* __restrict__ m0, float* __restrict__ lap,
                                double* partials, unsigned* counter, double* sum_out) {
  const long long N = b.n(), sxy = (long long)b.bx * b.by;
  const float centre = -2.0f * (hx2 + hy2 + hz2);
  double acc[2] = {0.0, 0.0};
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < N; s += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(s % b.bx), j = (int)((s / b.bx) % b.by), k = (int)(s / sxy);
    float v = 0.0f;
    if (m0[s] != 0) {
      const long long xm = s - (i > 0), xp = s + (i + 1 < b.bx), ym = s - (j > 0 ? b.bx : 0),
                      yp = s + (j + 1 < b.by ? b.bx : 0), zm = s - (k > 0 ? sxy : 0), zp = s + (k + 1 < b.bz ? sxy : 0);
      auto L = [&](const float* a) {
        return centre * a[s] + hx2 * (a[xm] + a[xp]) + hy2 * (a[ym] + a[yp]) + hz2 * (a[zm] + a[zp]);
      };
      v = L(sn) * cs[s] - L(cs) * sn[s];
      acc[0] += (double)v;
      acc[1] += 1.0;
    }
    lap[s] = v;
  }
  if (grid_sum_last<2>(acc, partials, counter) && threadIdx.x == 0) {
    sum_out[0] = acc[0];
    sum_out[1] = acc[1];
  }
}

__global__ void k_tgv_sub_mean(long long N, const uint8_t* __restrict__ m0, const double* __restrict__ sums,
                               float* __restrict__ lap) {
  const float mean = sums[1] > 0.0 ? (float)(sums[0] / sums[1]) : 0.0f;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < N; s += (long long)gridDim.x * blockDim.x)
    if (m0[s] != 0) lap[s] -= mean;
}

// ============================================================ iteration ==
struct TgvArrays {
  const float* lphi;
  const uint8_t* m0;
  const uint8_t* me;
  float* eta;
  float* p[3];
  float* q[6];  // xx, xy, xz, yy, yz, zz
  float* phi[2];
  float* chi[2];
  float* w[2][3];
  float* chi_prev;
};

struct TgvScalars {
  float hx, hy, hz, hx2, hy2, hz2;
  float sigma, sstep, tau, tstep, alpha0, alpha1;
};

struct TgvFlag {
  int done;
  int final_iter;
  unsigned counter;
  int pad;
};

// masked Neumann Laplacian at s (apply_laplacian_inplace, tgv.rs:780-824); the caller
// handles mask0 == 0
template <class F>
__device__ __forceinline__ float lap_neumann(const F& a, long long s, int i, int j, int k, const Box& b, long long sxy,
                                             const TgvScalars& c) {
  const float a0 = a(s);
  const float xm = i > 0 ? a(s - 1) : a0, xp = i + 1 < b.bx ? a(s + 1) : a0;
  const float ym = j > 0 ? a(s - b.bx) : a0, yp = j + 1 < b.by ? a(s + b.bx) : a0;
  const float zm = k > 0 ? a(s - sxy) : a0, zp = k + 1 < b.bz ? a(s + sxy) : a0;
  return c.hx2 * (xm - 2.0f * a0 + xp) + c.hy2 * (ym - 2.0f * a0 + yp) + c.hz2 * (zm - 2.0f * a0 + zp);
}

// 27-point stencil at an interior voxel (apply_stencil, tgv.rs:667-713; dk, dj, di order)
template <class F>
__device__ __forceinline__ float stencil27(const F& a, long long s, long long bx, long long sxy, const TgvConst& K) {
  float sum = 0.0f;
#pragma unroll
  for (int dk = 0; dk < 3; ++dk)
#pragma unroll
    for (int dj = 0; dj < 3; ++dj)
#pragma unroll
      for (int di = 0; di < 3; ++di)
        sum += K.st[(di * 3 + dj) * 3 + dk] * a(s + (di - 1) + (dj - 1) * bx + (dk - 1) * sxy);
  return sum;
}

__device__ __forceinline__ bool interior(int i, int j, int k, const Box& b) {
  return !(i == 0 || j == 0 || k == 0 || i + 1 >= b.bx || j + 1 >= b.by || k + 1 >= b.bz);
}

// The primal and dual kernels run 32x8 (x, y) tiles, each thread marching through
// `zchunk` planes of one (i, j) column: no index division, and the y/z neighbours of a
// voxel are the tile's own recent loads (L1) rather than another block's (L2).
constexpr int kTgvBX = 32, kTgvBY = 8;
// Resident blocks per SM the primal and dual kernels are compiled for (their register
// budgets: 85 registers a thread, no spills; the plane's values are held in registers).
constexpr int kTgvPrimalBlocks = 3;
constexpr int kTgvDualBlocks = 3;

// Dual update (tgv.rs:1157-1213).  q selects the buffers holding phi_, chi_, w_.
// Every array is accessed through a restrict-qualified pointer (no two alias, and no
// voxel reads what another voxel writes in the same launch); the two masks of the next
// plane are fetched while the current plane computes, and every value a plane needs is
// loaded into registers before its update, so a plane waits on one round of loads.  The
// arithmetic is that of the reference, in its order.
__global__ void __launch_bounds__(kTgvBX* kTgvBY, kTgvDualBlocks) k_tgv_dual(Box b, TgvArrays A, TgvScalars c, TgvConst K, int q,
                                                             int zchunk, const TgvFlag* flag) {
  if (flag->done) return;
  const long long sxy = (long long)b.bx * b.by;
  const float* __restrict__ phb = A.phi[q];
  const float* __restrict__ chb = A.chi[q];
  const float* __restrict__ wbx = A.w[q][0];
  const float* __restrict__ wby = A.w[q][1];
  const float* __restrict__ wbz = A.w[q][2];
  const uint8_t* __restrict__ m0 = A.m0;
  const uint8_t* __restrict__ me = A.me;
  const float* __restrict__ lphi = A.lphi;
  float* __restrict__ eta = A.eta;
  float* __restrict__ p0 = A.p[0];
  float* __restrict__ p1 = A.p[1];
  float* __restrict__ p2 = A.p[2];
  float* __restrict__ q0 = A.q[0];
  float* __restrict__ q1 = A.q[1];
  float* __restrict__ q2 = A.q[2];
  float* __restrict__ q3 = A.q[3];
  float* __restrict__ q4 = A.q[4];
  float* __restrict__ q5 = A.q[5];
  const int i = blockIdx.x * kTgvBX + threadIdx.x, j = blockIdx.y * kTgvBY + threadIdx.y;
  if (i >= b.bx || j >= b.by) return;
  const int kbeg = blockIdx.z * zchunk;
  const int kend = min(b.bz, (int)(blockIdx.z + 1) * zchunk);
  if (kbeg >= kend) return;
  long long s = (long long)kbeg * sxy + (long long)j * b.bx + i;
  uint8_t nm0 = m0[s], nme = me[s];
  for (int k = kbeg; k < kend; ++k, s += sxy) {
    const bool in0 = nm0 != 0, inm = nme != 0;
    if (k + 1 < kend) {
      nm0 = m0[s + sxy];
      nme = me[s + sxy];
    }
    if (!(in0 || inm)) continue;
    // Every load of the plane first, into registers, then the update in the reference's
    // order.  Neighbour offsets are clamped to the box, which gives exactly the values the
    // Neumann Laplacian substitutes at its faces (the centre), and loads that the
    // zero-on-the-far-face differences and the interior-only stencil never use.
    const long long dxm = i > 0 ? -1 : 0, dxp = i + 1 < b.bx ? 1 : 0;
    const long long dym = j > 0 ? -(long long)b.bx : 0, dyp = j + 1 < b.by ? (long long)b.bx : 0;
    const long long dzm = k > 0 ? -sxy : 0, dzp = k + 1 < b.bz ? sxy : 0;
    const long long ox[3] = {dxm, 0, dxp}, oy[3] = {dym, 0, dyp}, oz[3] = {dzm, 0, dzp};
    float ch[27];  // chi_ at (i + di - 1, j + dj - 1, k + dk - 1): ch[(dk * 3 + dj) * 3 + di]
    float ph[7];   // phi_: centre, x-, x+, y-, y+, z-, z+
    float wc[3], wx[3], wy[3], wz[3];  // w_ at the voxel and its x+1, y+1, z+1 neighbours
    float lph = 0.0f, et = 0.0f, pc[3], qc[6];
#pragma unroll
    for (int dk = 0; dk < 3; ++dk)
#pragma unroll
      for (int dj = 0; dj < 3; ++dj)
#pragma unroll
        for (int di = 0; di < 3; ++di) ch[(dk * 3 + dj) * 3 + di] = 0.0f;
    if (in0) {
#pragma unroll
      for (int dk = 0; dk < 3; ++dk)
#pragma unroll
        for (int dj = 0; dj < 3; ++dj)
#pragma unroll
          for (int di = 0; di < 3; ++di) ch[(dk * 3 + dj) * 3 + di] = chb[s + ox[di] + oy[dj] + oz[dk]];
      ph[0] = phb[s];
      ph[1] = phb[s + dxm];
      ph[2] = phb[s + dxp];
      ph[3] = phb[s + dym];
      ph[4] = phb[s + dyp];
      ph[5] = phb[s + dzm];
      ph[6] = phb[s + dzp];
      lph = lphi[s];
      et = eta[s];
#pragma unroll
      for (int t = 0; t < 6; ++t) qc[t] = A.q[t][s];
      wx[0] = wbx[s + dxp];
      wx[1] = wby[s + dxp];
      wx[2] = wbz[s + dxp];
      wy[0] = wbx[s + dyp];
      wy[1] = wby[s + dyp];
      wy[2] = wbz[s + dyp];
      wz[0] = wbx[s + dzp];
      wz[1] = wby[s + dzp];
      wz[2] = wbz[s + dzp];
    } else {
      ch[13] = chb[s];
      ch[14] = chb[s + dxp];
      ch[16] = chb[s + dyp];
      ch[22] = chb[s + dzp];
    }
    wc[0] = wbx[s];
    wc[1] = wby[s];
    wc[2] = wbz[s];
    pc[0] = p0[s];
    pc[1] = p1[s];
    pc[2] = p2[s];
    const float cb = ch[13];
    if (in0) {
      const float a0 = ph[0];
      const float t1 = c.hx2 * (ph[1] - 2.0f * a0 + ph[2]) + c.hy2 * (ph[3] - 2.0f * a0 + ph[4]) +
                       c.hz2 * (ph[5] - 2.0f * a0 + ph[6]);
      float t2 = 0.0f;
      if (interior(i, j, k, b)) {
        float sum = 0.0f;
#pragma unroll
        for (int dk = 0; dk < 3; ++dk)
#pragma unroll
          for (int dj = 0; dj < 3; ++dj)
#pragma unroll
            for (int di = 0; di < 3; ++di) sum += K.st[(di * 3 + dj) * 3 + dk] * ch[(dk * 3 + dj) * 3 + di];
        t2 = sum;
      }
      et += c.sigma * (-t1 + t2 - lph);
      eta[s] = et;
    }
    {
      const float gx = i + 1 < b.bx ? (ch[14] - cb) * c.hx : 0.0f;
      const float gy = j + 1 < b.by ? (ch[16] - cb) * c.hy : 0.0f;
      const float gz = k + 1 < b.bz ? (ch[22] - cb) * c.hz : 0.0f;
      const float s0 = in0 ? c.sstep : 0.0f, s1 = inm ? c.sstep : 0.0f;
      float px = pc[0] + (s0 * gx - s1 * wc[0]);
      float py = pc[1] + (s0 * gy - s1 * wc[1]);
      float pz = pc[2] + (s0 * gz - s1 * wc[2]);
      const float nrm = sqrtf(px * px + py * py + pz * pz);
      if (nrm > c.alpha1) {
        const float sc = c.alpha1 / nrm;
        px *= sc;
        py *= sc;
        pz *= sc;
      }
      p0[s] = px;
      p1[s] = py;
      p2[s] = pz;
    }
    if (in0) {
      // symgrad (src/utils/gradient.rs:300-372), zero on the far faces
      const float wx0 = wc[0], wy0 = wc[1], wz0 = wc[2];
      float sxx = 0.0f, sxy_ = 0.0f, sxz = 0.0f, syy = 0.0f, syz = 0.0f, szz = 0.0f;
      if (i + 1 < b.bx) {
        sxx = (wx[0] - wx0) * c.hx;
        sxy_ = ((wx[1] - wy0) * c.hx) * 0.5f;
        sxz = ((wx[2] - wz0) * c.hx) * 0.5f;
      }
      if (j + 1 < b.by) {
        syy = (wy[1] - wy0) * c.hy;
        sxy_ += ((wy[0] - wx0) * c.hy) * 0.5f;
        syz = ((wy[2] - wz0) * c.hy) * 0.5f;
      }
      if (k + 1 < b.bz) {
        szz = (wz[2] - wz0) * c.hz;
        sxz += ((wz[0] - wx0) * c.hz) * 0.5f;
        syz += ((wz[1] - wy0) * c.hz) * 0.5f;
      }
      float qq[6] = {qc[0] + c.sstep * sxx, qc[1] + c.sstep * sxy_, qc[2] + c.sstep * sxz,
                     qc[3] + c.sstep * syy, qc[4] + c.sstep * syz, qc[5] + c.sstep * szz};
      const float fro = sqrtf(qq[0] * qq[0] + qq[3] * qq[3] + qq[5] * qq[5] +
                              2.0f * (qq[1] * qq[1] + qq[2] * qq[2] + qq[4] * qq[4]));
      if (fro > c.alpha0) {
        const float sc = c.alpha0 / fro;
#pragma unroll
        for (int t = 0; t < 6; ++t) qq[t] *= sc;
      }
      q0[s] = qq[0];
      q1[s] = qq[1];
      q2[s] = qq[2];
      q3[s] = qq[3];
      q4[s] = qq[4];
      q5[s] = qq[5];
    }
  }
}

// Primal update and extrapolation (tgv.rs:1215-1271).  Buffers [1-q] hold the current
// iterate x (read), [q] the extrapolation consumed by the dual step (overwritten with
// x_new); [1-q] then receives 2 x_new - x.  Restrict-qualified pointers, the next
// plane's masks fetched ahead and the plane's values loaded before the update, as in
// k_tgv_dual.
__global__ void __launch_bounds__(kTgvBX* kTgvBY, kTgvPrimalBlocks) k_tgv_primal(Box b, TgvArrays A, TgvScalars c,
                                                                              TgvConst K, int q, int zchunk,
                                                                              const TgvFlag* flag) {
  if (flag->done) return;
  const long long sxy = (long long)b.bx * b.by;
  const uint8_t* __restrict__ m0 = A.m0;
  const uint8_t* __restrict__ me = A.me;
  const float* __restrict__ etab = A.eta;
  const float* __restrict__ p0 = A.p[0];
  const float* __restrict__ p1 = A.p[1];
  const float* __restrict__ p2 = A.p[2];
  const float* __restrict__ qb[6] = {A.q[0], A.q[1], A.q[2], A.q[3], A.q[4], A.q[5]};
  const float* __restrict__ phr = A.phi[1 - q];
  float* __restrict__ phw = A.phi[q];
  float* __restrict__ phx = A.phi[1 - q];
  const float* __restrict__ chr = A.chi[1 - q];
  float* __restrict__ chw = A.chi[q];
  float* __restrict__ chx = A.chi[1 - q];
  // eta and q are only ever updated inside mask0 (k_tgv_dual) and start at zero, so
  // m0*eta = eta and m0*q = q
  auto mq = [&](int comp, long long t) { return qb[comp][t]; };
  const int i = blockIdx.x * kTgvBX + threadIdx.x, j = blockIdx.y * kTgvBY + threadIdx.y;
  if (i >= b.bx || j >= b.by) return;
  const int kbeg = blockIdx.z * zchunk;
  const int kend = min(b.bz, (int)(blockIdx.z + 1) * zchunk);
  if (kbeg >= kend) return;
  long long s = (long long)kbeg * sxy + (long long)j * b.bx + i;
  uint8_t nm0 = m0[s], nme = me[s];
  for (int k = kbeg; k < kend; ++k, s += sxy) {
    const bool in0 = nm0 != 0, inm = nme != 0;
    if (k + 1 < kend) {
      nm0 = m0[s + sxy];
      nme = me[s + sxy];
    }
    // every load of the plane first (clamped neighbour offsets give the values the
    // Neumann faces substitute), then the update in the reference's order
    const long long dxm = i > 0 ? -1 : 0, dxp = i + 1 < b.bx ? 1 : 0;
    const long long dym = j > 0 ? -(long long)b.bx : 0, dyp = j + 1 < b.by ? (long long)b.bx : 0;
    const long long dzm = k > 0 ? -sxy : 0, dzp = k + 1 < b.bz ? sxy : 0;
    const long long ox[3] = {dxm, 0, dxp}, oy[3] = {dym, 0, dyp}, oz[3] = {dzm, 0, dzp};
    float e27[27];  // eta at (i + di - 1, j + dj - 1, k + dk - 1): e27[(dk * 3 + dj) * 3 + di]
    float pc[3] = {0.0f, 0.0f, 0.0f}, pm[3] = {0.0f, 0.0f, 0.0f};  // p at the voxel; p_a at the voxel - e_a
    float mm[3] = {0.0f, 0.0f, 0.0f};  // mask0 at the voxel - e_a (1 or 0)
    float qc[6], qx[3], qy[3], qz[3];  // q at the voxel; (q0,q1,q2)(x-1), (q1,q3,q4)(y-1), (q2,q4,q5)(z-1)
#pragma unroll
    for (int t = 0; t < 27; ++t) e27[t] = 0.0f;
    if (in0) {
#pragma unroll
      for (int dk = 0; dk < 3; ++dk)
#pragma unroll
        for (int dj = 0; dj < 3; ++dj)
#pragma unroll
          for (int di = 0; di < 3; ++di) e27[(dk * 3 + dj) * 3 + di] = etab[s + ox[di] + oy[dj] + oz[dk]];
      pm[0] = p0[s + dxm];
      pm[1] = p1[s + dym];
      pm[2] = p2[s + dzm];
      mm[0] = m0[s + dxm] ? 1.0f : 0.0f;
      mm[1] = m0[s + dym] ? 1.0f : 0.0f;
      mm[2] = m0[s + dzm] ? 1.0f : 0.0f;
    }
    if (in0 || inm) {
      pc[0] = p0[s];
      pc[1] = p1[s];
      pc[2] = p2[s];
    }
    if (inm) {
#pragma unroll
      for (int t = 0; t < 6; ++t) qc[t] = mq(t, s);
      qx[0] = mq(0, s + dxm);
      qx[1] = mq(1, s + dxm);
      qx[2] = mq(2, s + dxm);
      qy[0] = mq(1, s + dym);
      qy[1] = mq(3, s + dym);
      qy[2] = mq(4, s + dym);
      qz[0] = mq(2, s + dzm);
      qz[1] = mq(4, s + dzm);
      qz[2] = mq(5, s + dzm);
    }
    const float phi_old = phr[s];
    const float chi_old = chr[s];
    float wn[3], wo[3];
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) wo[comp] = wn[comp] = A.w[1 - q][comp][s];
    // phi
    float lap = 0.0f;
    if (in0) {
      const float a0 = e27[13];
      lap = c.hx2 * (e27[12] - 2.0f * a0 + e27[14]) + c.hy2 * (e27[10] - 2.0f * a0 + e27[16]) +
            c.hz2 * (e27[4] - 2.0f * a0 + e27[22]);
    }
    const float phi_new = (phi_old + c.tau * lap) / (1.0f + (inm ? c.tau : 0.0f));
    // chi: bdiv_masked (src/utils/gradient.rs:497-565) minus the stencil of m0*eta
    float t1 = 0.0f;
    if (in0) {
      const float gxt = 1.0f * pc[0] * c.hx - (i > 0 ? mm[0] * pm[0] * c.hx : 0.0f);
      const float gyt = 1.0f * pc[1] * c.hy - (j > 0 ? mm[1] * pm[1] * c.hy : 0.0f);
      const float gzt = 1.0f * pc[2] * c.hz - (k > 0 ? mm[2] * pm[2] * c.hz : 0.0f);
      t1 = gxt + gyt + gzt;
    }
    float t2 = 0.0f;
    if (in0 && interior(i, j, k, b)) {
      float sum = 0.0f;
#pragma unroll
      for (int dk = 0; dk < 3; ++dk)
#pragma unroll
        for (int dj = 0; dj < 3; ++dj)
#pragma unroll
          for (int di = 0; di < 3; ++di) sum += K.st[(di * 3 + dj) * 3 + dk] * e27[(dk * 3 + dj) * 3 + di];
      t2 = sum;
    }
    const float chi_new = chi_old + c.tstep * (t1 - t2);
    // w: symdiv of m0*q (src/utils/gradient.rs:380-432), zero on the near faces
    if (inm) {
      const float bx0 = i > 0 ? qx[0] : 0.0f, bx1 = i > 0 ? qx[1] : 0.0f, bx2 = i > 0 ? qx[2] : 0.0f;
      const float by1 = j > 0 ? qy[0] : 0.0f, by3 = j > 0 ? qy[1] : 0.0f, by4 = j > 0 ? qy[2] : 0.0f;
      const float bz2 = k > 0 ? qz[0] : 0.0f, bz4 = k > 0 ? qz[1] : 0.0f, bz5 = k > 0 ? qz[2] : 0.0f;
      const float dqx = (qc[0] - bx0) * c.hx + (qc[1] - by1) * c.hy + (qc[2] - bz2) * c.hz;
      const float dqy = (qc[1] - bx1) * c.hx + (qc[3] - by3) * c.hy + (qc[4] - bz4) * c.hz;
      const float dqz = (qc[2] - bx2) * c.hx + (qc[4] - by4) * c.hy + (qc[5] - bz5) * c.hz;
      wn[0] += c.tstep * (pc[0] + dqx);
      wn[1] += c.tstep * (pc[1] + dqy);
      wn[2] += c.tstep * (pc[2] + dqz);
    }
    phw[s] = phi_new;
    phx[s] = 2.0f * phi_new - phi_old;
    chw[s] = chi_new;
    chx[s] = 2.0f * chi_new - chi_old;
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
      A.w[q][comp][s] = wn[comp];
      A.w[1 - q][comp][s] = 2.0f * wn[comp] - wo[comp];
    }
  }
}

// Relative change of chi over mask0 at iteration `it` (tgv.rs:923-941, 1146-1154); sets
// the flag below tol, else saves chi for the next check.
__global__ void k_tgv_check(long long N, const float* __restrict__ chi, float* __restrict__ chi_prev,
                            const uint8_t* __restrict__ m0, float tol, int it, TgvFlag* flag, double* partials) {
  if (flag->done) return;
  double acc[2] = {0.0, 0.0};
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < N; s += (long long)gridDim.x * blockDim.x) {
    const float x = chi[s];
    if (m0[s] != 0) {
      const float d = x - chi_prev[s];
      acc[0] += (double)d * (double)d;
      acc[1] += (double)x * (double)x;
    }
    chi_prev[s] = x;
  }
  if (grid_sum_last<2>(acc, partials, &flag->counter) && threadIdx.x == 0) {
    const float d = (float)acc[0], nrm = (float)acc[1];
    const float rc = nrm > 1e-10f ? sqrtf(d / nrm) : 1.0f;
    if (rc < tol) {
      flag->done = 1;
      flag->final_iter = it;
    }
  }
}

__global__ void k_tgv_output(Box b, int nx, int ny, const float* __restrict__ chi, const uint8_t* __restrict__ me,
                             float scale, double* __restrict__ out) {
  const long long N = b.n();
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < N; s += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(s % b.bx), j = (int)((s / b.bx) % b.by), k = (int)(s / ((long long)b.bx * b.by));
    const long long f = (b.x0 + i) + (long long)(b.y0 + j) * nx + (long long)(b.z0 + k) * nx * ny;
    out[f] = me[s] != 0 ? (double)(chi[s] * scale) : 0.0;
  }
}

}  // namespace

// Host copy of the fitted stencil for parity tests: st[(di*3+dj)*3+dk].
void tgv_stencil_host(const double res[3], const double b0[3], float out[27]) {
  const Stencil& st = cached_stencil((float)res[0], (float)res[1], (float)res[2], (float)b0[0], (float)b0[1],
                                     (float)b0[2]);
  std::memcpy(out, st.data(), sizeof(float) * 27);
}

void tgv_device(qsm_ctx* ctx, const double* phase, const uint8_t* mask, const qsm_grid* grid, const qsm_tgv_params* p,
                const double b0[3], qsm_progress_fn progress, void* user, double* out) {
  GridDims d = check_grid(grid);
  check_ptr(phase, "phase");
  check_ptr(mask, "mask");
  check_ptr(out, "out");
  check_ptr(p, "params");
  check_bdir(b0);
  for (double v : {(double)p->alpha0, (double)p->alpha1, (double)p->step_size, (double)p->fieldstrength, (double)p->te})
    check_finite(v, "TGV parameter");
  if (std::isnan(p->tol)) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "tol is NaN");
  check_volume_finite(ctx, phase, d.n, "phase");
  const long long N = d.n;
  // erosions: mask_eroded = erode^erosions(mask), mask0 = erode(mask_eroded)
  uint8_t* ea = ws<uint8_t>(ctx, "tgv.er_a", (size_t)N);
  uint8_t* eb = ws<uint8_t>(ctx, "tgv.er_b", (size_t)N);
  uint8_t* m0f = ws<uint8_t>(ctx, "tgv.m0", (size_t)N);
  QSM_CUDA(cudaMemcpyAsync(ea, mask, (size_t)N, cudaMemcpyDeviceToDevice, ctx->stream));
  uint8_t* cur = ea;
  uint8_t* nxt = eb;
  for (size_t e = 0; e < p->erosions; ++e) {
    LaunchScope ls(ctx, "tgv_erode");
    k_erode<<<grid1d(N), 256, 0, ctx->stream>>>(cur, nxt, d.nx, d.ny, d.nz);
    ls.done();
    std::swap(cur, nxt);
  }
  const uint8_t* mef = cur;
  {
    LaunchScope ls(ctx, "tgv_erode");
    k_erode<<<grid1d(N), 256, 0, ctx->stream>>>(mef, m0f, d.nx, d.ny, d.nz);
    ls.done();
  }
  int* dbox = ws<int>(ctx, "tgv.box", 6);
  int hbox[6] = {d.nx, d.ny, d.nz, -1, -1, -1};
  h2d(ctx, dbox, hbox, sizeof(hbox));
  {
    LaunchScope ls(ctx, "tgv_bbox");
    k_mask_bbox<<<grid1d(N), 256, 0, ctx->stream>>>(m0f, d.nx, d.ny, d.nz, dbox);
    ls.done();
  }
  d2h(ctx, hbox, dbox, sizeof(hbox));
  sync(ctx);
  if (hbox[3] < 0)
    throw QsmError(QSM_ERR_INVALID_ARGUMENT, "the mask is empty after the TGV erosions (the reference panics here)");
  const int pad = 2;
  Box b;
  b.x0 = std::max(hbox[0] - pad, 0);
  b.y0 = std::max(hbox[1] - pad, 0);
  b.z0 = std::max(hbox[2] - pad, 0);
  b.bx = std::min(hbox[3] + pad + 1, d.nx) - b.x0;
  b.by = std::min(hbox[4] + pad + 1, d.ny) - b.y0;
  b.bz = std::min(hbox[5] + pad + 1, d.nz) - b.z0;
  const long long B = b.n();
  if (B >= (1LL << 32)) throw QsmError(QSM_ERR_UNSUPPORTED_SIZE, "TGV bounding box holds 2^32 voxels or more");
  // sub-volume arrays
  auto F = [&](const char* name) { return ws<float>(ctx, std::string("tgv.") + name, (size_t)B); };
  float* ph = F("phase");
  uint8_t* m0s = ws<uint8_t>(ctx, "tgv.m0s", (size_t)B);
  uint8_t* mes = ws<uint8_t>(ctx, "tgv.mes", (size_t)B);
  {
    LaunchScope ls(ctx, "tgv_extract");
    k_tgv_extract<<<grid1d(B), 256, 0, ctx->stream>>>(b, d.nx, d.ny, phase, m0f, mef, ph, m0s, mes);
    ls.done();
  }
  const float vsx = (float)d.vsx, vsy = (float)d.vsy, vsz = (float)d.vsz;
  TgvScalars c;
  c.hx = 1.0f / vsx;
  c.hy = 1.0f / vsy;
  c.hz = 1.0f / vsz;
  c.hx2 = 1.0f / (vsx * vsx);
  c.hy2 = 1.0f / (vsy * vsy);
  c.hz2 = 1.0f / (vsz * vsz);
  float* sn = F("sin");
  float* cs = F("cos");
  float* lphi = F("lphi");
  double* partials = ws<double>(ctx, "tgv.partials", (size_t)kMaxPersistentBlocks * 2);
  TgvFlag* flag = ws<TgvFlag>(ctx, "tgv.flag", 1);
  double* sums = ws<double>(ctx, "tgv.sums", 2);
  {
    TgvFlag f0{};
    h2d(ctx, flag, &f0, sizeof(f0));
    LaunchScope ls(ctx, "tgv_phase_lap");
    k_tgv_sincos<<<grid1d(B), 256, 0, ctx->stream>>>(B, ph, sn, cs);
    k_tgv_phase_lap<<<grid1d(B), 256, 0, ctx->stream>>>(b, c.hx2, c.hy2, c.hz2, sn, cs, m0s, lphi, partials,
                                                         &flag->counter, sums);
    k_tgv_sub_mean<<<grid1d(B), 256, 0, ctx->stream>>>(B, m0s, sums, lphi);
    ls.done();
  }
  // stencil and step sizes (tgv.rs:1107-1124)
  TgvConst K;
  {
    const Stencil& st = cached_stencil(vsx, vsy, vsz, (float)b0[0], (float)b0[1], (float)b0[2]);
    std::memcpy(K.st, st.data(), sizeof(K.st));
  }
  const float gns = 4.0f * (1.0f / (vsx * vsx) + 1.0f / (vsy * vsy) + 1.0f / (vsz * vsz));
  const float gn = std::sqrt(gns);
  float wave = 0.0f;
  for (int t = 0; t < 27; ++t) wave += std::fabs(K.st[t]);  // [di][dj][dk] order, dk fastest
  const float ns = operator_norm_sqr(gn, gns, wave);
  c.tau = 1.0f / std::sqrt(ns);
  c.sigma = c.tau;
  c.sstep = c.sigma * p->step_size;
  c.tstep = c.tau * p->step_size;
  c.alpha0 = p->alpha0;
  c.alpha1 = p->alpha1;
  // state, zero initialised
  TgvArrays A;
  A.lphi = lphi;
  A.m0 = m0s;
  A.me = mes;
  const char* names[] = {"eta", "px", "py", "pz", "qxx", "qxy", "qxz", "qyy", "qyz", "qzz", "phi0", "phi1",
                         "chi0", "chi1", "wx0", "wy0", "wz0", "wx1", "wy1", "wz1", "chi_prev"};
  float* buf[21];
  for (int t = 0; t < 21; ++t) {
    buf[t] = F(names[t]);
    QSM_CUDA(cudaMemsetAsync(buf[t], 0, sizeof(float) * B, ctx->stream));
  }
  A.eta = buf[0];
  for (int t = 0; t < 3; ++t) A.p[t] = buf[1 + t];
  for (int t = 0; t < 6; ++t) A.q[t] = buf[4 + t];
  A.phi[0] = buf[10];
  A.phi[1] = buf[11];
  A.chi[0] = buf[12];
  A.chi[1] = buf[13];
  for (int t = 0; t < 3; ++t) {
    A.w[0][t] = buf[14 + t];
    A.w[1][t] = buf[17 + t];
  }
  A.chi_prev = buf[20];
  // before iteration t the current iterate sits in [t % 2] and its extrapolation in
  // [(t + 1) % 2]; the dual step reads the extrapolation
  const unsigned gblocks = grid1d(B);
  // primal/dual tiles: ~16 blocks per SM in all, each marching zchunk planes
  const unsigned tgx = (unsigned)((b.bx + kTgvBX - 1) / kTgvBX), tgy = (unsigned)((b.by + kTgvBY - 1) / kTgvBY);
  const long long nzc = std::max<long long>(1, 16LL * sm_count(ctx) / ((long long)tgx * tgy));
  const int zchunk = (int)((b.bz + nzc - 1) / nzc);
  const dim3 tgrid(tgx, tgy, (unsigned)((b.bz + zchunk - 1) / zchunk)), tblock(kTgvBX, kTgvBY);
  auto one_iter = [&](size_t t) {
    const int q = (int)((t + 1) % 2);
    {
      LaunchScope ls(ctx, "tgv_dual");
      k_tgv_dual<<<tgrid, tblock, 0, ctx->stream>>>(b, A, c, K, q, zchunk, flag);
      ls.done();
    }
    LaunchScope ls(ctx, "tgv_primal");
    k_tgv_primal<<<tgrid, tblock, 0, ctx->stream>>>(b, A, c, K, q, zchunk, flag);
    ls.done();
  };
  auto check = [&](size_t t) {
    LaunchScope ls(ctx, "tgv_check");
    k_tgv_check<<<gblocks, 256, 0, ctx->stream>>>(B, A.chi[t % 2], A.chi_prev, m0s, p->tol, (int)t, flag, partials);
    ls.done();
  };
  const size_t iters = p->iterations;
  size_t reported = 0;  // progress calls issued for iterations [0, reported)
  auto report_to = [&](size_t upto) {
    if (progress)
      for (; reported < upto; ++reported) progress(user, reported, iters);
  };
  TgvFlag hf{};
  auto poll = [&]() {
    d2h(ctx, &hf, flag, sizeof(hf));
    sync(ctx);
    return hf.done != 0;
  };
  constexpr size_t kChunk = 100;  // convergence checks at multiples of 100 (tgv.rs:1146)
  bool converged = false;
  size_t t0 = 0;
  cudaGraphExec_t exec = nullptr;
  uint64_t per_graph = 0;
  try {
    while (t0 < iters && !converged) {
      const size_t len = std::min(kChunk, iters - t0);
      if (len == kChunk && t0 > 0 && !ctx->profiling) {
        if (exec == nullptr) {
          cudaGraph_t graph = nullptr;
          const uint64_t l0 = ctx->launches;
          QSM_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
          try {
            for (size_t t = 0; t < kChunk; ++t) one_iter(t);  // even start: same parities
          } catch (...) {
            cudaStreamEndCapture(ctx->stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
          }
          QSM_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
          per_graph = ctx->launches - l0;
          ctx->launches = l0;
          const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
          cudaGraphDestroy(graph);
          if (ie != cudaSuccess)
            throw QsmError(QSM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
        }
        check(t0);
        QSM_CUDA(cudaGraphLaunch(exec, ctx->stream));
        ctx->launches += per_graph;
      } else {
        if (t0 > 0) check(t0);
        for (size_t t = t0; t < t0 + len; ++t) one_iter(t);
      }
      converged = poll();
      report_to(converged ? (size_t)hf.final_iter + 1 : t0 + len);
      t0 += len;
    }
  } catch (...) {
    if (exec) cudaGraphExecDestroy(exec);
    throw;
  }
  if (exec) cudaGraphExecDestroy(exec);
  const size_t final_iter = converged ? (size_t)hf.final_iter : iters;
  if (progress) progress(user, final_iter, iters);
  // chi in ppm inside the eroded mask, zero elsewhere (tgv.rs:1275-1298)
  const float gamma = 42.5781f;
  const float scale = 1.0f / (2.0f * (float)kPi * p->te * p->fieldstrength * gamma);
  QSM_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * N, ctx->stream));
  {
    LaunchScope ls(ctx, "tgv_output");
    k_tgv_output<<<grid1d(B), 256, 0, ctx->stream>>>(b, d.nx, d.ny, A.chi[final_iter % 2], mes, scale, out);
    ls.done();
  }
  sync(ctx);
}

}  // namespace qsm

using namespace qsm;

extern "C" {

void qsm_tgv_params_default(qsm_tgv_params* p) {
  if (!p) return;
  // TgvParams::default, src/inversion/tgv.rs:59-75
  p->alpha1 = 0.0005f;
  p->alpha0 = 0.0015f;
  p->iterations = 1000;
  p->erosions = 3;
  p->step_size = 3.0f;
  p->fieldstrength = 3.0f;
  p->te = 0.020f;
  p->tol = 1e-5f;
}

qsm_status qsm_tgv_qsm_device(qsm_ctx* ctx, const double* d_phase, const uint8_t* d_mask, const qsm_grid* grid,
                              const qsm_tgv_params* params, const double b0_dir[3], qsm_progress_fn progress,
                              void* user, double* d_out_chi) {
  return guarded(ctx, [&] { tgv_device(ctx, d_phase, d_mask, grid, params, b0_dir, progress, user, d_out_chi); });
}

qsm_status qsm_tgv_qsm(qsm_ctx* ctx, const double* phase, const uint8_t* mask, const qsm_grid* grid,
                       const qsm_tgv_params* params, const double b0_dir[3], qsm_progress_fn progress, void* user,
                       double* out_chi) {
  return guarded(ctx, [&] {
    GridDims d = check_grid(grid);
    check_ptr(phase, "phase");
    check_ptr(mask, "mask");
    check_ptr(out_chi, "out_chi");
    with_host_io(ctx, d.n, phase, mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
      tgv_device(ctx, f, m, grid, params, b0_dir, progress, user, o);
    });
  });
}

qsm_status qsm_tgv_oblique_stencil(const double res[3], const double b0_dir[3], float out_stencil[27]) {
  if (!res || !b0_dir || !out_stencil) return QSM_ERR_INVALID_ARGUMENT;
  try {
    tgv_stencil_host(res, b0_dir, out_stencil);
  } catch (...) {
    return QSM_ERR_ALLOC;
  }
  return QSM_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ pipeline --
namespace qsm {
namespace {

// apply_reference (src/pipeline/referencing.rs:12-43): Mean subtracts the mean over
// mask > 0, None keeps the values; zero outside the mask in both
__global__ void k_ref_sum(long long N, const double* __restrict__ chi, const uint8_t* __restrict__ m,
                          double* partials, unsigned* counter, double* out) {
  double acc[2] = {0.0, 0.0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    if (m[i] > 0) {
      acc[0] += chi[i];
      acc[1] += 1.0;
    }
  if (grid_sum_last<2>(acc, partials, counter) && threadIdx.x == 0) {
    out[0] = acc[0];
    out[1] = acc[1];
  }
}

__global__ void k_ref_apply(long long N, const double* __restrict__ chi, const uint8_t* __restrict__ m,
                            const double* __restrict__ sums, int mean, double* __restrict__ out) {
  const double mu = (mean && sums[1] > 0.0) ? sums[0] / sums[1] : 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    out[i] = m[i] > 0 ? chi[i] - mu : 0.0;
}

}  // namespace

void apply_reference_device(qsm_ctx* ctx, long long N, const double* chi, const uint8_t* mask, int method,
                            double* out) {
  if (method != QSM_REFERENCE_MEAN && method != QSM_REFERENCE_NONE)
    throw QsmError(QSM_ERR_INVALID_ARGUMENT, "unknown QSM reference method " + std::to_string(method));
  double* partials = ws<double>(ctx, "ref.partials", (size_t)kMaxPersistentBlocks * 2);
  unsigned* counter = ws<unsigned>(ctx, "ref.counter", 1);
  double* sums = ws<double>(ctx, "ref.sums", 2);
  QSM_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), ctx->stream));
  QSM_CUDA(cudaMemsetAsync(sums, 0, 2 * sizeof(double), ctx->stream));
  LaunchScope ls(ctx, "apply_reference");
  if (method == QSM_REFERENCE_MEAN)
    k_ref_sum<<<grid1d(N), 256, 0, ctx->stream>>>(N, chi, mask, partials, counter, sums);
  k_ref_apply<<<grid1d(N), 256, 0, ctx->stream>>>(N, chi, mask, sums, method == QSM_REFERENCE_MEAN, out);
  ls.done();
}

}  // namespace qsm

extern "C" {

qsm_status qsm_apply_reference(qsm_ctx* ctx, const double* chi, const uint8_t* mask, size_t n, int method,
                               double* out) {
  return guarded(ctx, [&] {
    if (n == 0) return;
    check_ptr(chi, "chi");
    check_ptr(mask, "mask");
    check_ptr(out, "out");
    double* din = ws<double>(ctx, "io.in", n);
    uint8_t* dm = ws<uint8_t>(ctx, "io.mask", n);
    double* dout = ws<double>(ctx, "io.out", n);
    h2d(ctx, din, chi, n * sizeof(double));
    h2d(ctx, dm, mask, n);
    apply_reference_device(ctx, (long long)n, din, dm, method, dout);
    d2h(ctx, out, dout, n * sizeof(double));
    sync(ctx);
  });
}

qsm_status qsm_run_tgv(qsm_ctx* ctx, const double* const* phases, size_t n_echoes, size_t len, const uint8_t* mask,
                       const qsm_scan_metadata* md, const qsm_tgv_params* params, int reference,
                       qsm_progress_fn progress, void* user, double* out_chi) {
  return guarded(ctx, [&] {
    check_ptr(md, "metadata");
    check_ptr(params, "params");
    check_ptr(phases, "phases");
    if (n_echoes == 0) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "no echoes");
    if (n_echoes > 1)
      throw QsmError(QSM_ERR_INVALID_CONFIG,
                     "invalid config: multi-echo run_tgv needs field mapping, which this library does not provide");
    qsm_grid g{md->nx, md->ny, md->nz, md->vsx, md->vsy, md->vsz};
    GridDims d = check_grid(&g);
    if (len != (size_t)d.n)
      throw QsmError(QSM_ERR_DIMENSION_MISMATCH,
                     "dimension mismatch: expected " + std::to_string(d.n) + ", got " + std::to_string(len));
    if (reference != QSM_REFERENCE_MEAN && reference != QSM_REFERENCE_NONE)
      throw QsmError(QSM_ERR_INVALID_ARGUMENT, "unknown QSM reference method");
    check_ptr(phases[0], "phases[0]");
    check_ptr(mask, "mask");
    check_ptr(out_chi, "out_chi");
    // single echo: the wrapped phase goes to tgv_qsm directly (src/pipeline/inversion.rs:124-157)
    with_host_io(ctx, d.n, phases[0], mask, out_chi, [&](const double* f, const uint8_t* m, double* o) {
      double* chi = ws<double>(ctx, "tgv.chi_full", (size_t)d.n);
      tgv_device(ctx, f, m, &g, params, md->b0_direction, progress, user, chi);
      apply_reference_device(ctx, d.n, chi, m, reference, o);
    });
  });
}

}  // extern "C"
