// 1D FFT plan shared by host planner and device engine.
#pragma once

namespace qsm {

constexpr int kFftEmax = 16;        // complex values held in registers per thread
constexpr int kFftMaxStages = 12;
constexpr int kFftMaxLen = 4096;

struct FftPlan1D {
  int n;        // transform length
  int nstages;  // number of Stockham stages
  int T;        // threads cooperating on one pencil
  int radix[kFftMaxStages];
  int ns[kFftMaxStages];   // product of radices before this stage
  int tws[kFftMaxStages];  // twiddle-table stride n / (ns * radix)
};

// Factor n into supported radices (2,3,4,5,6,7,8,9,10,11,12,13,15,16) and choose the
// per-pencil thread count so every stage fits kFftEmax registers per thread.
// Returns false when n has a prime factor above 13 or exceeds kFftMaxLen.
bool make_fft_plan(int n, FftPlan1D* out);

// Number of supported lengths helper: true when make_fft_plan would succeed.
bool fft_length_supported(int n);

}  // namespace qsm
