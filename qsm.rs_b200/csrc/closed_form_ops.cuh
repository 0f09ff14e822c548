// k-space multipliers of the closed-form dipole inversions, evaluated in double and
// symmetrised over k -> -k (see KSpaceT::sym).
#pragma once

#include "launch.cuh"

namespace qsm {

// TKD: |D| <= t -> sign(D)/t with sign(0) = +, else 1/D  (src/inversion/tkd.rs:62-72)
// TSVD: |D| <= t -> 0, else 1/D                             (src/inversion/tkd.rs:117-124)
template <typename T> struct OpTkd {
  using C = cplx_t<T>;
  KSpace K;
  double t;
  int tsvd;
  __device__ __forceinline__ C mid(C v, int ix, int iy, int iz, long long) const {
    const double th = t;
    const int zero_mode = tsvd;
    const KSpace& k = K;
    const double m = K.sym(ix, iy, iz, [&](double kx, double ky, double kz, int, int, int) {
      const double d = k.dipole(kx, ky, kz);
      if (fabs(d) <= th) return zero_mode ? 0.0 : (d >= 0.0 ? 1.0 / th : -1.0 / th);
      return 1.0 / d;
    });
    return cscale(v, (T)m);
  }
};

// Tikhonov: D / (D^2 + lambda*Gamma), Gamma in {1, Lneg, Lpos^2}; |denom| <= 1e-20 -> 0
// (src/inversion/tikhonov.rs:71-115)
template <typename T> struct OpTikhonov {
  using C = cplx_t<T>;
  KSpace K;
  double lambda;
  int reg;
  __device__ __forceinline__ C mid(C v, int ix, int iy, int iz, long long) const {
    const double lam = lambda;
    const int r = reg;
    const KSpace& k = K;
    const double m = K.sym(ix, iy, iz, [&](double kx, double ky, double kz, int a, int b, int c) {
      const double d = k.dipole(kx, ky, kz);
      double gam = 1.0;
      if (r == 1) gam = k.lapneg(a, b, c);
      else if (r == 2) {
        const double lp = -k.lapneg(a, b, c);
        gam = lp * lp;
      }
      const double den = d * d + lam * gam;
      return fabs(den) > 1e-20 ? d / den : 0.0;
    });
    return cscale(v, (T)m);
  }
};

// Forward dipole model multiplier D (src/fft.rs:214-233)
template <typename T> struct OpDipole {
  using C = cplx_t<T>;
  KSpace K;
  __device__ __forceinline__ C mid(C v, int ix, int iy, int iz, long long) const {
    const KSpace& k = K;
    const double m =
        K.sym(ix, iy, iz, [&](double kx, double ky, double kz, int, int, int) { return k.dipole(kx, ky, kz); });
    return cscale(v, (T)m);
  }
};

}  // namespace qsm
