// 1D FFT plan shared by host planner and device engine.
#pragma once

namespace qsm {

constexpr int kFftEmax = 16;        // complex values held in registers per thread
constexpr int kFftMaxStages = 12;
constexpr int kFftMaxLen = 4096;
// Longest axis with a prime factor above 13: its Bluestein convolution length (a
// 7-smooth m >= 2n - 1) must stay within kFftMaxLen.
constexpr int kBluesteinMaxLen = 2048;

struct FftPlan1D {
  int n;        // transform length
  int m;        // length of the transform the stages run: n, or the Bluestein length
  int nstages;  // number of Stockham stages (of the length-m transform)
  int T;        // threads cooperating on one pencil
  int radix[kFftMaxStages];
  int ns[kFftMaxStages];   // product of radices before this stage
  int tws[kFftMaxStages];  // twiddle-table stride m / (ns * radix)
  // Bluestein plans (m != n): device table of the chirp c_j = exp(-i pi j^2 / n), j < n,
  // followed by the m-point DFT of the conjugate chirp divided by m.  Set by the
  // transform bundle; null for direct plans.
  const void* ext;
};

// Factor n into supported radices (2,3,4,5,6,7,8,9,10,11,12,13,15,16) and choose the
// per-pencil thread count so every stage fits kFftEmax registers per thread.  A length
// with a prime factor above 13 (up to kBluesteinMaxLen) gets a Bluestein plan: the
// stages of the smallest 7-smooth m >= 2n - 1.  Returns false when n exceeds
// kFftMaxLen, or has a prime factor above 13 and exceeds kBluesteinMaxLen.
bool make_fft_plan(int n, FftPlan1D* out);

// Number of supported lengths helper: true when make_fft_plan would succeed.
bool fft_length_supported(int n);

}  // namespace qsm
