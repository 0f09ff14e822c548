// Radix selection of order statistics (see select.h).
//
// Each double maps to a 64-bit key whose unsigned order is the numeric order
// (negative values: all bits flipped; others: sign bit set).  Six passes fix the key
// 11 bits at a time (the last pass 9 bits): a histogram kernel counts, per requested
// rank, the selected values whose higher bits equal the rank's prefix so far, binned by
// the current digit (shared-memory histograms, merged with global atomics); a scan
// kernel then picks the digit whose cumulative count covers the remaining rank.  Every
// pass reads the values once, so one selection of up to four ranks costs six reads of
// the array.
#include "select.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "solvers.h"

namespace qsm {

namespace {

constexpr int kSelMaxRanks = 4;
constexpr int kSelBins = 2048;  // 11-bit digits
constexpr int kSelThreads = 256;

struct SelState {
  unsigned long long prefix[kSelMaxRanks];
  unsigned long long rem[kSelMaxRanks];
};

__device__ __forceinline__ unsigned long long order_key(double v) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(v);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

double key_to_double(unsigned long long k) {
  const unsigned long long u = (k >> 63) ? (k ^ 0x8000000000000000ull) : ~k;
  double d;
  std::memcpy(&d, &u, sizeof(d));
  return d;
}

__global__ void __launch_bounds__(kSelThreads)
    k_sel_hist(const double* __restrict__ vals, const uint8_t* __restrict__ mask, long long n, int nr, int shift,
               int width, const SelState* __restrict__ st, unsigned* __restrict__ hist) {
  __shared__ unsigned sh[kSelMaxRanks * kSelBins];
  for (int i = threadIdx.x; i < nr * kSelBins; i += blockDim.x) sh[i] = 0u;
  unsigned long long pre[kSelMaxRanks];
#pragma unroll
  for (int r = 0; r < kSelMaxRanks; ++r) pre[r] = r < nr ? st->prefix[r] : 0ull;
  __syncthreads();
  const int hs = shift + width;  // bits above the current digit
  const unsigned dmask = (1u << width) - 1u;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (mask != nullptr && mask[i] == 0) continue;
    const unsigned long long k = order_key(vals[i]);
    const unsigned bin = (unsigned)(k >> shift) & dmask;
#pragma unroll
    for (int r = 0; r < kSelMaxRanks; ++r) {
      if (r >= nr) break;
      const bool match = hs >= 64 || (k >> hs) == (pre[r] >> hs);
      if (match) atomicAdd(&sh[r * kSelBins + bin], 1u);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nr * kSelBins; i += blockDim.x)
    if (sh[i] != 0u) atomicAdd(&hist[i], sh[i]);
}

// One warp per rank: find the digit whose cumulative count covers the remaining rank.
__global__ void k_sel_scan(int nr, int shift, int width, SelState* st, const unsigned* __restrict__ hist) {
  const int r = threadIdx.y, lane = threadIdx.x;
  if (r >= nr) return;
  const int per = (1 << width) / 32;
  const unsigned* h = hist + r * kSelBins;
  const unsigned long long rem = st->rem[r];
  unsigned long long s = 0;
  for (int b = lane * per; b < (lane + 1) * per; ++b) s += h[b];
  unsigned long long incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  const unsigned long long excl = incl - s;
  if (rem >= excl && rem < incl) {
    unsigned long long c = excl;
    for (int b = lane * per; b < (lane + 1) * per; ++b) {
      if (rem < c + h[b]) {
        st->prefix[r] |= (unsigned long long)b << shift;
        st->rem[r] = rem - c;
        break;
      }
      c += h[b];
    }
  }
}

__global__ void k_count_selected(const uint8_t* __restrict__ mask, long long n, unsigned long long* out) {
  unsigned long long c = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    c += mask[i] != 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

}  // namespace

long long count_selected(qsm_ctx* ctx, const uint8_t* mask, long long n) {
  if (mask == nullptr) return n;
  unsigned long long* d = ws<unsigned long long>(ctx, "sel.count", 1);
  QSM_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), ctx->stream));
  {
    LaunchScope ls(ctx, "count_selected");
    k_count_selected<<<grid1d(n), 256, 0, ctx->stream>>>(mask, n, d);
    ls.done();
  }
  unsigned long long h = 0;
  d2h(ctx, &h, d, sizeof(h));
  sync(ctx);
  return (long long)h;
}

std::vector<double> select_ranks(qsm_ctx* ctx, const double* vals, const uint8_t* mask, long long n,
                                 const std::vector<long long>& ranks) {
  const int nr = (int)ranks.size();
  if (nr < 1 || nr > kSelMaxRanks) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "select_ranks: 1 to 4 ranks");
  SelState h{};
  for (int r = 0; r < nr; ++r) {
    if (ranks[r] < 0) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "select_ranks: negative rank");
    h.rem[r] = (unsigned long long)ranks[r];
  }
  SelState* st = ws<SelState>(ctx, "sel.state", 1);
  unsigned* hist = ws<unsigned>(ctx, "sel.hist", (size_t)kSelMaxRanks * kSelBins);
  h2d(ctx, st, &h, sizeof(h));
  int sm = 0;
  QSM_CUDA(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, ctx->device));
  long long blocks = (n + kSelThreads - 1) / kSelThreads;
  if (blocks > 2LL * sm) blocks = 2LL * sm;
  if (blocks < 1) blocks = 1;
  static const int kShift[6] = {53, 42, 31, 20, 9, 0};
  static const int kWidth[6] = {11, 11, 11, 11, 11, 9};
  for (int p = 0; p < 6; ++p) {
    QSM_CUDA(cudaMemsetAsync(hist, 0, sizeof(unsigned) * nr * kSelBins, ctx->stream));
    {
      LaunchScope ls(ctx, "select_hist");
      k_sel_hist<<<(unsigned)blocks, kSelThreads, 0, ctx->stream>>>(vals, mask, n, nr, kShift[p], kWidth[p], st,
                                                                    hist);
      ls.done();
    }
    {
      LaunchScope ls(ctx, "select_scan");
      k_sel_scan<<<1, dim3(32, nr), 0, ctx->stream>>>(nr, kShift[p], kWidth[p], st, hist);
      ls.done();
    }
  }
  d2h(ctx, &h, st, sizeof(h));
  sync(ctx);
  std::vector<double> out(nr);
  for (int r = 0; r < nr; ++r) out[r] = key_to_double(h.prefix[r]);
  return out;
}

std::vector<double> percentiles(qsm_ctx* ctx, const double* vals, const uint8_t* mask, long long n,
                                long long count, const std::vector<double>& p) {
  if (count <= 0) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "percentiles of an empty selection");
  if (p.size() > 2) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "percentiles: at most two per call");
  std::vector<double> out(p.size());
  if (count == 1) {
    const std::vector<double> v = select_ranks(ctx, vals, mask, n, {0});
    for (size_t i = 0; i < p.size(); ++i) out[i] = v[0];
    return out;
  }
  std::vector<long long> ranks;
  std::vector<double> frac;
  for (double pi : p) {
    const double hpos = (pi / 100.0) * (double)(count - 1);
    const long long lo = (long long)std::floor(hpos);
    const long long hi = std::min(lo + 1, count - 1);
    ranks.push_back(lo);
    ranks.push_back(hi);
    frac.push_back(hpos - (double)lo);
  }
  const std::vector<double> v = select_ranks(ctx, vals, mask, n, ranks);
  for (size_t i = 0; i < p.size(); ++i) {
    const double lo = v[2 * i], hi = v[2 * i + 1];
    out[i] = lo + frac[i] * (hi - lo);
  }
  return out;
}

}  // namespace qsm

using namespace qsm;

extern "C" qsm_status qsm_prctile_device(qsm_ctx* ctx, const double* d_vals, const uint8_t* d_mask, size_t n,
                                         const double* p, size_t np, double* out) {
  return guarded(ctx, [&] {
    if (np == 0) return;
    check_ptr(p, "p");
    check_ptr(out, "out");
    if (n > 0) check_ptr(d_vals, "vals");
    const long long count = n == 0 ? 0 : count_selected(ctx, d_mask, (long long)n);
    for (size_t i = 0; i < np; i += 2) {
      std::vector<double> pi(p + i, p + std::min(np, i + 2));
      for (double v : pi)
        if (!(v >= 0.0 && v <= 100.0)) throw QsmError(QSM_ERR_INVALID_ARGUMENT, "percent outside [0, 100]");
      if (count == 0) {
        for (size_t k = 0; k < pi.size(); ++k) out[i + k] = 0.0;
        continue;
      }
      const std::vector<double> r = percentiles(ctx, d_vals, d_mask, (long long)n, count, pi);
      for (size_t k = 0; k < r.size(); ++k) out[i + k] = r[k];
    }
  });
}
