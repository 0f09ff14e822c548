// Host-side radix planner for the Stockham engine (fft_engine.cuh).
#include "fft_plan.h"

#include <initializer_list>
#include <vector>

namespace qsm {

namespace {

const int kRadices[] = {16, 15, 13, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2};

struct Best {
  bool found = false;
  int stages = 1 << 30;
  int T = 1 << 30;
  int waste = 1 << 30;
  std::vector<int> seq;
};

int ceil_div(int a, int b) { return (a + b - 1) / b; }

void evaluate(int n, const std::vector<int>& seq, Best& best) {
  int T = 1;
  for (int R : seq) {
    int nb = n / R;
    int per = kFftEmax / R;  // butterflies a thread can hold
    int need = ceil_div(nb, per);
    if (need > T) T = need;
  }
  // idle butterfly slots summed over stages (smaller is better)
  int waste = 0;
  for (int R : seq) {
    int nb = n / R;
    int c = ceil_div(nb, T);
    waste += c * T - nb;
  }
  int st = (int)seq.size();
  bool better = !best.found || st < best.stages || (st == best.stages && T < best.T) ||
                (st == best.stages && T == best.T && waste < best.waste);
  if (better) {
    best.found = true;
    best.stages = st;
    best.T = T;
    best.waste = waste;
    best.seq = seq;
  }
}

void search(int n, int rem, int max_r, std::vector<int>& seq, Best& best) {
  if (rem == 1) {
    evaluate(n, seq, best);
    return;
  }
  if ((int)seq.size() >= kFftMaxStages) return;
  for (int R : kRadices) {
    if (R > max_r || rem % R != 0) continue;
    seq.push_back(R);
    search(n, rem / R, R, seq, best);
    seq.pop_back();
  }
}

bool smooth(int n, std::initializer_list<int> primes) {
  for (int p : primes)
    while (n % p == 0) n /= p;
  return n == 1;
}

}  // namespace

bool make_fft_plan(int n, FftPlan1D* out) {
  if (n < 1 || n > kFftMaxLen) return false;
  if (!smooth(n, {2, 3, 5, 7, 11, 13})) {
    // Bluestein: an n-point DFT as a cyclic convolution of length m >= 2n - 1
    if (n > kBluesteinMaxLen) return false;
    int m = 2 * n - 1;
    while (!smooth(m, {2, 3, 5, 7})) ++m;
    FftPlan1D inner{};
    if (!make_fft_plan(m, &inner)) return false;
    inner.n = n;
    if (out) *out = inner;
    return true;
  }
  FftPlan1D pl{};
  pl.n = n;
  pl.m = n;
  if (n == 1) {
    pl.nstages = 1;
    pl.T = 1;
    pl.radix[0] = 1;
    pl.ns[0] = 1;
    pl.tws[0] = 1;
    if (out) *out = pl;
    return true;
  }
  Best best;
  std::vector<int> seq;
  search(n, n, 16, seq, best);
  if (!best.found) return false;
  pl.nstages = (int)best.seq.size();
  pl.T = best.T;
  int ns = 1;
  for (int s = 0; s < pl.nstages; ++s) {
    int R = best.seq[s];
    pl.radix[s] = R;
    pl.ns[s] = ns;
    pl.tws[s] = n / (ns * R);
    ns *= R;
  }
  if (out) *out = pl;
  return true;
}

bool fft_length_supported(int n) { return make_fft_plan(n, nullptr); }

}  // namespace qsm
