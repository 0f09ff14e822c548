// Register/shared-memory Stockham FFT engine for one pencil per thread group.
//
// A 1D transform of length n is split into stages of radix R (2..16).  Each stage
// is the autosort (Stockham) step: butterfly j reads its R inputs at j + r*(n/R),
// twiddles input r by W_{Ns*R}^{(j mod Ns)*r} (Ns = product of the radices already
// done), runs a register DFT of size R, and writes output r to
// (j - j mod Ns)*R + (j mod Ns) + r*Ns.  The first stage reads straight from the
// caller's fetch functor (global memory, coalesced across j) and the last stage
// writes natural-order outputs straight through the emit functor, so a two-stage
// transform crosses shared memory once.  Radices and the per-pencil thread count T
// come from a host-side plan, so one kernel binary serves every supported length.
//
// Replaces the per-axis rustfft plans of the reference (src/fft.rs:42-234,
// 423-479); the 3D passes built on this engine live in passes.cuh.
#pragma once

#include <type_traits>
#include <utility>
#include "common.cuh"
#include "fft_plan.h"

namespace qsm {

template <long long P, long long Q> inline constexpr double kCos2pi = cos2pi(P, Q);
template <long long P, long long Q> inline constexpr double kSin2pi = sin2pi(P, Q);

// a * exp(DIR * 2*pi*i * M / R), M and R compile-time
template <int DIR, int M, int R, typename C>
__device__ __forceinline__ C tw_const(C a) {
  constexpr int m = ((M % R) + R) % R;
  using S = decltype(a.x);
  if constexpr (m == 0) {
    return a;
  } else if constexpr (2 * m == R) {
    return mk<C>(-a.x, -a.y);
  } else if constexpr (4 * m == R) {
    if constexpr (DIR < 0) return cmul_mi(a); else return cmul_i(a);
  } else if constexpr (4 * m == 3 * R) {
    if constexpr (DIR < 0) return cmul_i(a); else return cmul_mi(a);
  } else {
    constexpr S c = (S)kCos2pi<m, R>;
    constexpr S s = (S)((double)DIR * kSin2pi<m, R>);
    return mk<C>(c * a.x - s * a.y, c * a.y + s * a.x);
  }
}

template <int R, int DIR, typename C> struct Dft;

template <int DIR, typename C> struct Dft<1, DIR, C> {
  static __device__ __forceinline__ void run(C*) {}
};

template <int DIR, typename C> struct Dft<2, DIR, C> {
  static __device__ __forceinline__ void run(C* v) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <int DIR, typename C> struct Dft<4, DIR, C> {
  static __device__ __forceinline__ void run(C* v) {
    C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    C t2 = cadd(v[1], v[3]), d = csub(v[1], v[3]);
    C t3 = (DIR < 0) ? cmul_mi(d) : cmul_i(d);  // (v1 - v3) * (DIR * i)
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};

// Odd prime R via symmetric pairs: y_k = v0 + sum_m (v_m + v_{R-m}) cos(2 pi m k/R)
//                                      + i*DIR*sum_m (v_m - v_{R-m}) sin(2 pi m k/R)
template <int R, int DIR, typename C> struct DftOdd {
  static constexpr int H = (R - 1) / 2;
  template <int K, int... M>
  static __device__ __forceinline__ void out_k(const C* s, const C* d, C v0, C* y, std::integer_sequence<int, M...>) {
    using S = decltype(v0.x);
    C A = v0;
    C B = mk<C>(S(0), S(0));
    ((A = mk<C>(A.x + (S)kCos2pi<(M + 1) * K, R> * s[M].x, A.y + (S)kCos2pi<(M + 1) * K, R> * s[M].y)), ...);
    ((B = mk<C>(B.x + (S)kSin2pi<(M + 1) * K, R> * d[M].x, B.y + (S)kSin2pi<(M + 1) * K, R> * d[M].y)), ...);
    C iB = (DIR < 0) ? cmul_mi(B) : cmul_i(B);
    y[K] = cadd(A, iB);
    y[R - K] = csub(A, iB);
  }
  template <int... K>
  static __device__ __forceinline__ void all_k(const C* s, const C* d, C v0, C* y, std::integer_sequence<int, K...>) {
    (out_k<K + 1>(s, d, v0, y, std::make_integer_sequence<int, H>{}), ...);
  }
  static __device__ __forceinline__ void run(C* v) {
    C s[H], d[H];
    C y0 = v[0];
#pragma unroll
    for (int m = 1; m <= H; ++m) {
      s[m - 1] = cadd(v[m], v[R - m]);
      d[m - 1] = csub(v[m], v[R - m]);
      y0 = cadd(y0, s[m - 1]);
    }
    C y[R];
    all_k(s, d, v[0], y, std::make_integer_sequence<int, H>{});
    v[0] = y0;
#pragma unroll
    for (int k = 1; k < R; ++k) v[k] = y[k];
  }
};
template <int DIR, typename C> struct Dft<3, DIR, C> : DftOdd<3, DIR, C> {};
template <int DIR, typename C> struct Dft<5, DIR, C> : DftOdd<5, DIR, C> {};
template <int DIR, typename C> struct Dft<7, DIR, C> : DftOdd<7, DIR, C> {};
template <int DIR, typename C> struct Dft<11, DIR, C> : DftOdd<11, DIR, C> {};
template <int DIR, typename C> struct Dft<13, DIR, C> : DftOdd<13, DIR, C> {};

// Composite R = R1*R2 in registers (Cooley-Tukey with constant twiddles):
// n = R2*n1 + n2, k = k1 + R1*k2.
template <int R1, int R2, int DIR, typename C> struct DftSplit {
  static constexpr int R = R1 * R2;
  template <int N2, int... K1>
  static __device__ __forceinline__ void twid(const C* t, C* a, std::integer_sequence<int, K1...>) {
    ((a[N2 * R1 + K1] = tw_const<DIR, N2 * K1, R>(t[K1])), ...);
  }
  template <int N2>
  static __device__ __forceinline__ void col(const C* v, C* a) {
    C t[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) t[n1] = v[R2 * n1 + N2];
    Dft<R1, DIR, C>::run(t);
    twid<N2>(t, a, std::make_integer_sequence<int, R1>{});
  }
  template <int... N2>
  static __device__ __forceinline__ void step1(const C* v, C* a, std::integer_sequence<int, N2...>) {
    (col<N2>(v, a), ...);
  }
  static __device__ __forceinline__ void run(C* v) {
    C a[R];
    step1(v, a, std::make_integer_sequence<int, R2>{});
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      C t[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) t[n2] = a[n2 * R1 + k1];
      Dft<R2, DIR, C>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = t[k2];
    }
  }
};
template <int DIR, typename C> struct Dft<6, DIR, C> : DftSplit<2, 3, DIR, C> {};
template <int DIR, typename C> struct Dft<8, DIR, C> : DftSplit<2, 4, DIR, C> {};
template <int DIR, typename C> struct Dft<9, DIR, C> : DftSplit<3, 3, DIR, C> {};
template <int DIR, typename C> struct Dft<10, DIR, C> : DftSplit<2, 5, DIR, C> {};
template <int DIR, typename C> struct Dft<12, DIR, C> : DftSplit<4, 3, DIR, C> {};
template <int DIR, typename C> struct Dft<15, DIR, C> : DftSplit<3, 5, DIR, C> {};
template <int DIR, typename C> struct Dft<16, DIR, C> : DftSplit<4, 4, DIR, C> {};

// ---------------------------------------------------------------------------
// Shared-memory addressing of one pencil.  Strided: element e of column px of a
// P-wide tile at sm[e*P + px] (Y/Z passes, 128-byte rows, conflict-free).
// Padded: element e of a contiguous row at row[e + e/G] (X pass; the skew keeps
// the stride-R writes of the first stage off a single bank).
// ---------------------------------------------------------------------------
struct SAStrided {
  int P;
  __device__ __forceinline__ int operator()(int e) const { return e * P; }
};
template <int G> struct SAPadded {
  __device__ __forceinline__ int operator()(int e) const { return e + e / G; }
};

// One Stockham stage of compile-time radix R.  Every thread of the block must call
// this (it contains __syncthreads); inactive threads skip the memory traffic.
template <int R, int DIR, int EMAX, typename C, class SA, class Fetch, class Emit>
__device__ __forceinline__ void fft_stage(C (&v)[EMAX], const FftPlan1D& pl, int s, int t, bool active,
                                          C* sp, const SA& sa, const C* tw, Fetch& fetch, Emit& emit) {
  constexpr int CM = EMAX / R;
  const int n = pl.m;
  const int nb = n / R;
  const int T = pl.T;
  const int Ns = pl.ns[s];
  const int tws = pl.tws[s];
  const bool first = (s == 0);
  const bool last = (s == pl.nstages - 1);
  if (active) {
#pragma unroll
    for (int c = 0; c < CM; ++c) {
      const int j = t + c * T;
      if (j < nb) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int e = j + r * nb;
          v[c * R + r] = first ? fetch(e) : sp[sa(e)];
        }
      }
    }
  }
  __syncthreads();
  if (active) {
#pragma unroll
    for (int c = 0; c < CM; ++c) {
      const int j = t + c * T;
      if (j < nb) {
        const int k = j % Ns;
        if (!first) {
#pragma unroll
          for (int r = 1; r < R; ++r) {
            const C w = tw[k * r * tws];
            v[c * R + r] = (DIR < 0) ? cmul(v[c * R + r], w) : cmulc(v[c * R + r], w);
          }
        }
        Dft<R, DIR, C>::run(&v[c * R]);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int e = base + r * Ns;
          if (last) emit(e, v[c * R + r]);
          else sp[sa(e)] = v[c * R + r];
        }
      }
    }
  }
  __syncthreads();
}

// The same Stockham stage with every size known at compile time (radix R, span NS,
// length N, threads per pencil TT): loop bounds, guards, j mod NS and the twiddle
// strides fold into constants.  Used for the axis lengths of the benchmark volumes.
// Fetch tag for a first stage whose inputs are already in the thread's registers, and
// emit tag for a last stage that leaves its outputs there after applying a hook
// (hook(e, value) -> value): a plan's last stage leaves thread j holding elements
// j + r * (N / R_last) in v[c * R + r], the layout the first stage of the plan with the
// reversed radices reads, so two transforms in a row can pass their values in registers.
struct FetchInRegs {};
template <class Hook> struct EmitInRegs {
  Hook& hook;
};
template <class E> struct IsEmitInRegs : std::false_type {};
template <class H> struct IsEmitInRegs<EmitInRegs<H>> : std::true_type {};

// Twiddle tables with one gap entry after every 16 (TWP in the compile-time stages).  In
// the X passes the 16 threads of a row read W^(j*r*s) for 16 consecutive j, a stride that
// puts power-of-two r on a few shared-memory banks in the dense table (r = 8 at length
// 256: eight-way conflicts) and on distinct banks in the padded one.
__host__ __device__ constexpr int tw_pad(int i) { return i + (i >> 4); }
// Complex entries a padded table of n twiddles occupies (even, so what follows it stays
// 16-byte aligned).
__host__ __device__ constexpr int tw_table_len(int n) { return (tw_pad(n - 1) + 2) & ~1; }

template <int R, int NS, int N, int TT, int DIR, bool FIRST, bool LAST, bool TWP, typename C, class SA,
          class Fetch, class Emit>
__device__ __forceinline__ void fft_stage_fixed(C (&v)[kFftEmax], int t, bool active, C* sp, const SA& sa,
                                                const C* tw, Fetch& fetch, Emit& emit) {
  constexpr int NB = N / R;
  constexpr int CM = (NB + TT - 1) / TT;
  constexpr int TWS = N / (NS * R);
  constexpr bool kRegsIn = FIRST && std::is_same<Fetch, FetchInRegs>::value;
  constexpr bool kRegsOut = LAST && IsEmitInRegs<Emit>::value;
  static_assert(CM * R <= kFftEmax, "stage does not fit the register budget");
  if constexpr (!kRegsIn) {
    if (active) {
#pragma unroll
      for (int c = 0; c < CM; ++c) {
        const int j = t + c * TT;
        if ((NB % TT == 0) || j < NB) {
#pragma unroll
          for (int r = 0; r < R; ++r) {
            if constexpr (FIRST) v[c * R + r] = fetch(j + r * NB);
            else v[c * R + r] = sp[sa(j + r * NB)];
          }
        }
      }
    }
    // With the inputs in registers there is nothing to order here: the stage before
    // (the other transform's last) read shared memory only ahead of its own barrier.
    __syncthreads();
  }
  if (active) {
#pragma unroll
    for (int c = 0; c < CM; ++c) {
      const int j = t + c * TT;
      if ((NB % TT == 0) || j < NB) {
        const int k = j % NS;
        if constexpr (NS > 1) {
#pragma unroll
          for (int r = 1; r < R; ++r) {
            const C w = tw[TWP ? tw_pad(k * r * TWS) : k * r * TWS];
            v[c * R + r] = (DIR < 0) ? cmul(v[c * R + r], w) : cmulc(v[c * R + r], w);
          }
        }
        Dft<R, DIR, C>::run(&v[c * R]);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int e = base + r * NS;
          if constexpr (kRegsOut) v[c * R + r] = emit.hook(e, v[c * R + r]);
          else if constexpr (LAST) emit(e, v[c * R + r]);
          else sp[sa(e)] = v[c * R + r];
        }
      }
    }
  }
  // A last stage that keeps its outputs in registers wrote no shared memory.
  if constexpr (!kRegsOut) __syncthreads();
}

// A compile-time plan: length N, TT threads per pencil, radices R0, R1[, R2].
template <int N, int TT, int R0, int R1, int R2 = 1> struct FixedPlan;
// The plan with its radices in reverse order (see FetchInRegs).
template <class FP> struct ReversePlan;
template <int N, int TT, int R0, int R1> struct ReversePlan<FixedPlan<N, TT, R0, R1, 1>> {
  using type = FixedPlan<N, TT, R1, R0, 1>;
};
template <int N, int TT, int R0, int R1, int R2> struct ReversePlan<FixedPlan<N, TT, R0, R1, R2>> {
  using type = FixedPlan<N, TT, R2, R1, R0>;
};

template <int N, int TT, int R0, int R1, int R2> struct FixedPlan {
  static constexpr int n = N, T = TT;
  static __host__ __device__ constexpr bool matches(const FftPlan1D& pl) {
    return pl.n == N && pl.m == N && pl.T == TT && pl.radix[0] == R0 && pl.radix[1] == R1 &&
           (R2 == 1 ? pl.nstages == 2 : (pl.nstages == 3 && pl.radix[2] == R2));
  }
  // TWP: tw is a padded table (tw_pad).
  template <int DIR, bool TWP = false, typename C, class SA, class Fetch, class Emit>
  static __device__ __forceinline__ void run(int t, bool active, C* sp, const SA& sa, const C* tw, Fetch& fetch,
                                             Emit& emit) {
    C v[kFftEmax];
    run_v<DIR, TWP>(v, t, active, sp, sa, tw, fetch, emit);
  }
  // The stages over a caller-held register array (FetchInRegs / EmitInRegs).
  template <int DIR, bool TWP = false, typename C, class SA, class Fetch, class Emit>
  static __device__ __forceinline__ void run_v(C (&v)[kFftEmax], int t, bool active, C* sp, const SA& sa,
                                               const C* tw, Fetch& fetch, Emit& emit) {
    auto none = [] {};
    run_v<DIR, TWP>(v, t, active, sp, sa, tw, fetch, emit, none);
  }
  // ... calling after_first() once the first stage has fetched every input and passed its
  // barrier, so a pass can release its input while the later stages run.
  template <int DIR, bool TWP = false, typename C, class SA, class Fetch, class Emit, class Hook>
  static __device__ __forceinline__ void run_v(C (&v)[kFftEmax], int t, bool active, C* sp, const SA& sa,
                                               const C* tw, Fetch& fetch, Emit& emit, Hook& after_first) {
    fft_stage_fixed<R0, 1, N, TT, DIR, true, false, TWP>(v, t, active, sp, sa, tw, fetch, emit);
    after_first();
    if constexpr (R2 == 1) {
      fft_stage_fixed<R1, R0, N, TT, DIR, false, true, TWP>(v, t, active, sp, sa, tw, fetch, emit);
    } else {
      fft_stage_fixed<R1, R0, N, TT, DIR, false, false, TWP>(v, t, active, sp, sa, tw, fetch, emit);
      fft_stage_fixed<R2, R0 * R1, N, TT, DIR, false, true, TWP>(v, t, active, sp, sa, tw, fetch, emit);
    }
  }
};

// Axis lengths with a compile-time transform (the host planner produces exactly
// these plans for them; any other plan takes the runtime path).
#define QSM_FIXED_PLANS(X)                                                                        \
  X(64, 4, 16, 4, 1) X(96, 8, 16, 6, 1) X(128, 8, 16, 8, 1) X(160, 16, 16, 10, 1)                 \
  X(176, 16, 16, 11, 1) X(192, 16, 16, 12, 1) X(256, 16, 16, 16, 1) X(384, 26, 16, 8, 3)

// Further 5- and 7-smooth lengths from 72 to 240 (the planner's own radices and threads
// per pencil): compiled only for the passes of the TV-ADMM iteration, whose launchers
// take the wide list (W = true), so that uneven clinical grids avoid the runtime engine
// in the loop that runs hundreds of times per solve.
#define QSM_FIXED_PLANS_WIDE(X)                                                                   \
  X(72, 6, 12, 6, 1) X(75, 5, 15, 5, 1) X(80, 6, 16, 5, 1) X(81, 9, 9, 9, 1) X(90, 8, 15, 6, 1)   \
  X(100, 10, 10, 10, 1) X(108, 12, 12, 9, 1) X(112, 8, 16, 7, 1) X(120, 8, 15, 8, 1)              \
  X(125, 9, 5, 5, 5) X(135, 15, 15, 9, 1) X(144, 12, 12, 12, 1) X(150, 15, 15, 10, 1)             \
  X(162, 18, 9, 9, 2) X(168, 12, 8, 7, 3) X(180, 15, 15, 12, 1) X(200, 14, 8, 5, 5)               \
  X(216, 18, 12, 6, 3) X(224, 16, 16, 7, 2) X(225, 15, 15, 15, 1) X(240, 16, 16, 15, 1)

// The runtime stages of a plan's length-m transform, reading through fetch (first
// stage) and writing through emit (last stage).
template <int DIR, typename C, class SA, class Fetch, class Emit>
__device__ __forceinline__ void run_stages(const FftPlan1D& pl, int t, bool active, C* sp, const SA& sa, const C* tw,
                                           Fetch& fetch, Emit& emit) {
  constexpr int EMAX = kFftEmax;
  C v[EMAX];
  for (int s = 0; s < pl.nstages; ++s) {
    switch (pl.radix[s]) {
      case 1: fft_stage<1, DIR>(v, pl, s, t, active, sp, sa, tw, fetch, emit); break;
      case 2: fft_stage<2, DIR>(v, pl, s, t, active, sp, sa, tw, fetch, emit); break;
      case 3: fft_stage<3, DIR>(v, pl, s, t, active, sp, sa, tw, fetch, emit); break;
      case 4: fft_stage<4, DIR>(v, pl, s, t, active, sp, sa, tw, fetch, emit); break;
      case 5: fft_stage<5, DIR>(v, pl, s, t, active, sp, sa, tw, fetch, emit); break;
      case 6: fft_stage<6, DIR>(v, pl, s, t, active, sp, sa, tw, fetch, emit); break;
      case 7: fft_stage<7, DIR>(v, pl, s, t, active, sp, sa, tw, fetch, emit); break;
      case 8: fft_stage<8, DIR>(v, pl, s, t, active, sp, sa, tw, fetch, emit); break;
      case 9: fft_stage<9, DIR>(v, pl, s, t, active, sp, sa, tw, fetch, emit); break;
      case 10: fft_stage<10, DIR>(v, pl, s, t, active, sp, sa, tw, fetch, emit); break;
      case 11: fft_stage<11, DIR>(v, pl, s, t, active, sp, sa, tw, fetch, emit); break;
      case 12: fft_stage<12, DIR>(v, pl, s, t, active, sp, sa, tw, fetch, emit); break;
      case 13: fft_stage<13, DIR>(v, pl, s, t, active, sp, sa, tw, fetch, emit); break;
      case 15: fft_stage<15, DIR>(v, pl, s, t, active, sp, sa, tw, fetch, emit); break;
      default: fft_stage<16, DIR>(v, pl, s, t, active, sp, sa, tw, fetch, emit); break;
    }
  }
}

// Full 1D transform of one pencil. DIR = -1 forward (exp(-2 pi i nk/n)), +1 inverse
// (unnormalised).  tw points at the forward table W_m^k, k in [0, m) (m = n except for
// Bluestein plans).
//
// The pencil is read from global memory (SRC_G: gsrc[base + e*stride]) or from its
// shared-memory slot (sp[sa(e)]), and written likewise (DST_G).  Solver-specific
// work (loaders, multipliers, stores) runs in coalesced loops around this call, so
// the engine is compiled once per I/O shape instead of once per solver operator.
// Direct transform (m = n), or the length-m stages of a Bluestein plan in place.  BL
// only separates the instances the Bluestein kernels call from the direct kernels' own:
// a function shared by both gets the smaller register budget and spills.
template <int DIR, typename C, class SA, bool SRC_G, bool DST_G, bool BL = false>
__device__ __noinline__ void fft_pencil_direct(const FftPlan1D* plp, int t, bool active, C* sp, SA sa, const C* tw,
                                               const C* gsrc, C* gdst, long long base, long long stride) {
  const FftPlan1D& pl = *plp;
  auto fetch = [&](int e) -> C {
    if constexpr (SRC_G) return gsrc[base + e * stride];
    else return sp[sa(e)];
  };
  auto emit = [&](int e, C v) {
    if constexpr (DST_G) gdst[base + e * stride] = v;
    else sp[sa(e)] = v;
  };
  // Compile-time plans only for the contiguous (X) passes in single precision:
  // inlining every plan into the strided Y/Z engine, or into the double-precision
  // engine, raises the register count past the occupancy budget.
  if constexpr (!std::is_same<SA, SAStrided>::value && sizeof(C) == 8) {
#define QSM_TRY_FIXED(N_, T_, R0_, R1_, R2_)                                                \
    if (FixedPlan<N_, T_, R0_, R1_, R2_>::matches(pl)) {                                    \
      FixedPlan<N_, T_, R0_, R1_, R2_>::template run<DIR>(t, active, sp, sa, tw, fetch, emit); \
      return;                                                                               \
    }
    QSM_FIXED_PLANS(QSM_TRY_FIXED)
#undef QSM_TRY_FIXED
  }
  run_stages<DIR>(pl, t, active, sp, sa, tw, fetch, emit);
}

// Bluestein (chirp-z) transform of one pencil of length n through a cyclic convolution
// of length m >= 2n - 1 (Bluestein 1970; Rabiner, Schafer and Rader 1969).  With
// q_j = exp(DIR i pi j^2 / n), jk = (j^2 + k^2 - (k - j)^2) / 2 gives
//   X_k = q_k * sum_j (x_j q_j) conj(q_{k-j}),
// a convolution of a_j = x_j q_j (zero-padded to m) with the conjugate chirp.  The table
// holds c_j = exp(-i pi j^2 / n) (so q = c forward, conj(c) inverse) and K = DFT_m of the
// conjugate chirp wrapped cyclically, divided by m.  That sequence is even, so K is even
// and the inverse direction's kernel spectrum is conj(K).  The pencil's slot holds m
// elements; the two length-m transforms are the plan's own stages, run in place by the
// direct engine, with the pointwise steps inline in the kernel.  BL selects this path at
// compile time: every runtime pass kernel is instantiated separately for Bluestein plans,
// because any second call path next to the direct engine in the same kernel (inline or
// out of line) shrinks the engine's register budget and makes it spill.
template <int DIR, typename C, class SA, bool SRC_G, bool DST_G, bool BL>
__device__ __forceinline__ void fft_pencil(const FftPlan1D* plp, int t, bool active, C* sp, SA sa, const C* tw,
                                           const C* gsrc, C* gdst, long long base, long long stride) {
  if constexpr (!BL) {
    fft_pencil_direct<DIR, C, SA, SRC_G, DST_G>(plp, t, active, sp, sa, tw, gsrc, gdst, base, stride);
    return;
  }
  const int n = plp->n, m = plp->m, T = plp->T;
  const C* chirp = static_cast<const C*>(plp->ext);
  const C* kspec = chirp + n;
  if (active) {
    for (int j = t; j < m; j += T) {
      C a = mk<C>(decltype(a.x)(0), decltype(a.x)(0));
      if (j < n) {
        C x;
        if constexpr (SRC_G) x = gsrc[base + j * stride];
        else x = sp[sa(j)];
        const C c = chirp[j];
        a = (DIR < 0) ? cmul(x, c) : cmulc(x, c);
      }
      sp[sa(j)] = a;
    }
  }
  __syncthreads();
  fft_pencil_direct<-1, C, SA, false, false, true>(plp, t, active, sp, sa, tw, nullptr, nullptr, 0, 0);
  if (active) {
    for (int j = t; j < m; j += T) {
      const C k = kspec[j];
      sp[sa(j)] = (DIR < 0) ? cmul(sp[sa(j)], k) : cmulc(sp[sa(j)], k);
    }
  }
  __syncthreads();
  fft_pencil_direct<+1, C, SA, false, false, true>(plp, t, active, sp, sa, tw, nullptr, nullptr, 0, 0);
  if (active) {
    for (int j = t; j < n; j += T) {
      const C c = chirp[j];
      const C y = (DIR < 0) ? cmul(sp[sa(j)], c) : cmulc(sp[sa(j)], c);
      if constexpr (DST_G) gdst[base + j * stride] = y;
      else sp[sa(j)] = y;
    }
  }
  __syncthreads();
}

}  // namespace qsm
