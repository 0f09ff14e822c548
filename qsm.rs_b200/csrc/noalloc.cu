// TKD dipole inversion that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code that runs while another framework's
// caching allocator has reserved the whole GPU, real-time reconstruction loops that
// must not hit the implicit device synchronisation of cudaMalloc/cudaFree, and hosts
// that run under a fixed device-memory budget.  qsm_tkd_device_noalloc serves them:
// it runs the same five-pass TKD chain as qsm_tkd_device (f64), but its scratch (the
// half spectrum, the twiddle tables and the k-space tables) lives in the file-scope
// array g_tkd_scratch below instead of in a context's workspace.
//
//   * Limit: kNoAllocScratchBytes (48 MiB) per device; volumes whose scratch does not
//     fit (above about 160^3) are rejected with QSM_ERR_UNSUPPORTED_SIZE.
//   * Every GPU that loads this library holds the array until the process exits.
//   * All calls on a device share the array and it keeps the last call's contents;
//     calls that overlap on the GPU (different streams, or host threads racing) race
//     on it and must be serialised by the caller.
//   * Every call resolves the array's device address on the current device with
//     cudaGetSymbolAddress (nothing is cached, so a context torn down and recreated
//     by cudaDeviceReset cannot leave a stale address behind).
//   * The call uploads its tables with cudaMemcpyAsync from pageable host memory and
//     synchronises its stream, so it must not be called while that stream is being
//     captured into a CUDA graph; such a call is refused with QSM_ERR_INVALID_ARGUMENT.
#include "closed_form_ops.cuh"
#include "functors.cuh"
#include "solvers.h"

namespace qsm {

std::vector<double> kspace_axis_table(const char* what, int n, double vs);

namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)48 << 20;
__device__ __align__(256) unsigned char g_tkd_scratch[kNoAllocScratchBytes];

// Device address of g_tkd_scratch on the current device, resolved on every call.
unsigned char* scratch_address() {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_tkd_scratch);
  if (e != cudaSuccess || p == nullptr)
    throw QsmError(QSM_ERR_CUDA, std::string("cudaGetSymbolAddress(g_tkd_scratch): ") + cudaGetErrorString(e));
  return static_cast<unsigned char*>(p);
}

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace
}  // namespace qsm

using namespace qsm;

extern "C" qsm_status qsm_tkd_device_noalloc(const double* d_local_field, const uint8_t* d_mask, const qsm_grid* grid,
                                             const double bdir[3], const qsm_tkd_params* params, double* d_out_chi,
                                             void* stream) {
  qsm_ctx local;  // host-side bookkeeping only: no device memory behind it
  if (cudaGetDevice(&local.device) != cudaSuccess) {
    (void)cudaGetLastError();
    return QSM_ERR_NO_DEVICE;
  }
  local.precision = QSM_PRECISION_F64;
  local.stream = static_cast<cudaStream_t>(stream);
  return guarded(&local, [&] {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    QSM_CUDA(cudaStreamIsCapturing(local.stream, &cap));
    if (cap != cudaStreamCaptureStatusNone)
      throw QsmError(QSM_ERR_INVALID_ARGUMENT, "the allocation-free TKD cannot run while its stream is capturing");
    GridDims d = check_grid(grid);
    check_ptr(d_local_field, "local_field");
    check_ptr(d_mask, "mask");
    check_ptr(d_out_chi, "out_chi");
    check_ptr(params, "params");
    check_bdir(bdir);
    check_finite(params->threshold, "threshold");

    Fft3<double> f;
    f.g.nx = d.nx;
    f.g.ny = d.ny;
    f.g.nz = d.nz;
    f.g.nxh = d.nx / 2 + 1;
    f.g.pitch = (f.g.nxh + 3) / 4 * 4;
    f.px = plan_or_throw(d.nx);
    f.py = plan_or_throw(d.ny);
    f.pz = plan_or_throw(d.nz);

    // scratch layout: spectrum | transform tables x, y, z | 9 per-axis k-space tables
    const size_t spec_b = round256((size_t)f.g.hsize() * sizeof(double2));
    const std::vector<unsigned char> tw_h[3] = {transform_table(f.px, true), transform_table(f.py, true),
                                                transform_table(f.pz, true)};
    const size_t tw_b[3] = {round256(tw_h[0].size()), round256(tw_h[1].size()), round256(tw_h[2].size())};
    const int ns[3] = {d.nx, d.ny, d.nz};
    const double vs[3] = {d.vsx, d.vsy, d.vsz};
    size_t tab_b = 0;
    for (int a = 0; a < 3; ++a) tab_b += 3 * round256((size_t)ns[a] * sizeof(double));
    const size_t need = spec_b + tw_b[0] + tw_b[1] + tw_b[2] + tab_b;
    if (need > kNoAllocScratchBytes)
      throw QsmError(QSM_ERR_UNSUPPORTED_SIZE, "volume needs " + std::to_string(need) +
                                                   " bytes of scratch; the allocation-free TKD holds " +
                                                   std::to_string(kNoAllocScratchBytes));
    unsigned char* base = scratch_address();
    unsigned char* cur = base;
    double2* spec = reinterpret_cast<double2*>(cur);
    cur += spec_b;
    const double2* tw[3];
    for (int a = 0; a < 3; ++a) {
      QSM_CUDA(cudaMemcpyAsync(cur, tw_h[a].data(), tw_h[a].size(), cudaMemcpyHostToDevice, local.stream));
      tw[a] = reinterpret_cast<const double2*>(cur);
      cur += tw_b[a];
    }
    f.twx = tw[0];
    f.twy = tw[1];
    f.twz = tw[2];
    attach_tables(f);
    const double* tabs[3][3];  // [kind freq/lap/poi][axis]
    const char* kinds[3] = {"freq", "lap", "poi"};
    for (int kd = 0; kd < 3; ++kd)
      for (int a = 0; a < 3; ++a) {
        const std::vector<double> h = kspace_axis_table(kinds[kd], ns[a], vs[a]);
        QSM_CUDA(cudaMemcpyAsync(cur, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, local.stream));
        tabs[kd][a] = reinterpret_cast<const double*>(cur);
        cur += round256((size_t)ns[a] * sizeof(double));
      }
    KSpace K;
    K.fx = tabs[0][0];
    K.fy = tabs[0][1];
    K.fz = tabs[0][2];
    K.lx = tabs[1][0];
    K.ly = tabs[1][1];
    K.lz = tabs[1][2];
    K.qx = tabs[2][0];
    K.qy = tabs[2][1];
    K.qz = tabs[2][2];
    K.nyqx = (d.nx % 2 == 0) ? d.nx / 2 : -1;
    K.nyqy = (d.ny % 2 == 0) ? d.ny / 2 : -1;
    K.nyqz = (d.nz % 2 == 0) ? d.nz / 2 : -1;
    const double bn = std::sqrt(bdir[0] * bdir[0] + bdir[1] * bdir[1] + bdir[2] * bdir[2]);
    K.bx = bdir[0] / bn;
    K.by = bdir[1] / bn;
    K.bz = bdir[2] / bn;

    // the same chain as qsm_tkd_device in double (src/inversion/tkd.rs:48-99); the
    // spectrum is fully written by the first pass, so nothing needs clearing
    run_x_r2c<double>(&local, f, spec, LoadCast<double, double>{d_local_field, d.nx}, nullptr);
    run_yz<double, -1, 1>(&local, f, spec, spec, OpId<double>{}, nullptr);
    run_z_fused<double>(&local, f, spec, spec, OpTkd<double>{K, params->threshold, 0}, nullptr);
    run_yz<double, +1, 1>(&local, f, spec, spec, OpId<double>{}, nullptr);
    run_x_c2r<double>(&local, f, spec, StoreMaskedF64<double>{d_out_chi, d_mask, d.nx, 1.0 / (double)d.n}, nullptr);
    QSM_CUDA(cudaStreamSynchronize(local.stream));
  });
}
