// Host construction of the per-grid k-space tables (cached per context).
#include "launch.cuh"

#include <cmath>
#include <map>
#include <mutex>

namespace qsm {

namespace {

// numpy-style fftfreq, src/fft.rs:544-566
std::vector<double> fftfreq(int n, double d) {
  std::vector<double> f(n);
  const double val = 1.0 / ((double)n * d);
  if (n % 2 == 0) {
    for (int i = 0; i < n / 2; ++i) f[i] = (double)i * val;
    for (int i = n / 2; i < n; ++i) f[i] = (double)(i - n) * val;
  } else {
    for (int i = 0; i <= (n - 1) / 2; ++i) f[i] = (double)i * val;
    for (int i = (n + 1) / 2; i < n; ++i) f[i] = (double)(i - n) * val;
  }
  return f;
}

// One axis of Re(FFT(laplacian_kernel(negative=true))): the kernel holds 2h at 0 and
// -h at indices 1 and n-1 (one entry when they coincide, none when n == 1),
// src/kernels/laplacian.rs:20-61.
std::vector<double> lapneg_axis(int n, double vs) {
  const double h = 1.0 / (vs * vs);
  std::vector<double> l(n);
  for (int i = 0; i < n; ++i) {
    double v = 2.0 * h;
    if (n > 1) {
      v -= h * cos2pi((long long)i * 1, n);
      if (n - 1 != 1) v -= h * cos2pi((long long)i * (n - 1), n);
    }
    l[i] = v;
  }
  return l;
}

// Poisson eigenvalue of one axis, src/unwrap/laplacian.rs:91-105:
// 2*(cos(2*pi*f) - 1)/h^2 with f = i/n (i <= n/2) or (i - n)/n.
std::vector<double> poisson_axis(int n, double vs) {
  const double idx2 = 1.0 / (vs * vs);
  std::vector<double> q(n);
  for (int i = 0; i < n; ++i) {
    const double f = (i <= n / 2) ? (double)i / (double)n : ((double)i - (double)n) / (double)n;
    q[i] = 2.0 * (std::cos(2.0 * kPi * f) - 1.0) * idx2;
  }
  return q;
}

template <typename S> const S* table(qsm_ctx* ctx, const std::string& key, const std::vector<double>& v) {
  std::vector<S> h(v.begin(), v.end());
  return (const S*)upload_table(ctx, key + (sizeof(S) == 4 ? ":f" : ":d"), h.data(), h.size() * sizeof(S));
}

std::string k(const char* what, int n, double vs) {
  char buf[96];
  std::snprintf(buf, sizeof buf, "%s:%d:%.17g", what, n, vs);
  return buf;
}

}  // namespace

template <typename S> KSpaceT<S> make_kspace_t(qsm_ctx* ctx, const GridDims& d, const double bdir[3]) {
  KSpaceT<S> K;
  K.fx = table<S>(ctx, k("freq", d.nx, d.vsx), fftfreq(d.nx, d.vsx));
  K.fy = table<S>(ctx, k("freq", d.ny, d.vsy), fftfreq(d.ny, d.vsy));
  K.fz = table<S>(ctx, k("freq", d.nz, d.vsz), fftfreq(d.nz, d.vsz));
  K.lx = table<S>(ctx, k("lap", d.nx, d.vsx), lapneg_axis(d.nx, d.vsx));
  K.ly = table<S>(ctx, k("lap", d.ny, d.vsy), lapneg_axis(d.ny, d.vsy));
  K.lz = table<S>(ctx, k("lap", d.nz, d.vsz), lapneg_axis(d.nz, d.vsz));
  K.qx = table<S>(ctx, k("poi", d.nx, d.vsx), poisson_axis(d.nx, d.vsx));
  K.qy = table<S>(ctx, k("poi", d.ny, d.vsy), poisson_axis(d.ny, d.vsy));
  K.qz = table<S>(ctx, k("poi", d.nz, d.vsz), poisson_axis(d.nz, d.vsz));
  K.nyqx = (d.nx % 2 == 0) ? d.nx / 2 : -1;
  K.nyqy = (d.ny % 2 == 0) ? d.ny / 2 : -1;
  K.nyqz = (d.nz % 2 == 0) ? d.nz / 2 : -1;
  double bx = 0, by = 0, bz = 1;
  if (bdir) {
    bx = bdir[0];
    by = bdir[1];
    bz = bdir[2];
  }
  // src/kernels/dipole.rs:38-43 normalises b (a zero vector yields NaN there too)
  const double bn = std::sqrt(bx * bx + by * by + bz * bz);
  K.bx = (S)(bx / bn);
  K.by = (S)(by / bn);
  K.bz = (S)(bz / bn);
  return K;
}

template KSpaceT<float> make_kspace_t<float>(qsm_ctx*, const GridDims&, const double*);
template KSpaceT<double> make_kspace_t<double>(qsm_ctx*, const GridDims&, const double*);

// Host copy of one per-axis k-space table: "freq", "lap" or "poi" (as uploaded by
// make_kspace_t), for callers that place the tables in memory they manage.
std::vector<double> kspace_axis_table(const char* what, int n, double vs) {
  const std::string w(what);
  if (w == "freq") return fftfreq(n, vs);
  if (w == "lap") return lapneg_axis(n, vs);
  return poisson_axis(n, vs);
}

void raise_smem_limit(const void* func, int device, size_t bytes) {
  // the compare, the attribute call and the update run under one lock, so contexts on
  // other host threads never skip a raise that another thread has not finished
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> limits;
  std::lock_guard<std::mutex> lock(mu);
  auto it = limits.find({func, device});
  if (it == limits.end()) it = limits.emplace(std::make_pair(func, device), (size_t)48 * 1024).first;
  if (bytes > it->second) {
    QSM_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    it->second = bytes;
  }
}

int sm_count_of(int device) {
  static std::mutex mu;
  static std::map<int, int> counts;
  std::lock_guard<std::mutex> lock(mu);
  auto it = counts.find(device);
  if (it != counts.end()) return it->second;
  int c = 0;
  QSM_CUDA(cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, device));
  counts[device] = c;
  return c;
}

KSpace make_kspace(qsm_ctx* ctx, const GridDims& d, const double bdir[3]) {
  return make_kspace_t<double>(ctx, d, bdir);
}

}  // namespace qsm
