// NIfTI voxels to and from device memory.
//
// Loading: the header is parsed on the host (nifti.cpp); the stored voxels (1-8 bytes
// each, often int16 or float32) cross PCIe in their own type through the context's
// pinned staging buffers, and one kernel swaps bytes when the file is big-endian,
// converts to double and applies raw * scl_slope + scl_inter (slope != 0) with
// explicitly rounded operations, as the host decoder does.  Saving: one kernel rounds
// the doubles to float32 and the 4-byte voxels come back through the same staging.
#include "nifti.h"
#include "solvers.h"

#include <cstring>

namespace qsm {

namespace {

template <typename S> __device__ __forceinline__ S load_swapped(const uint8_t* p, bool big) {
  S v;
  if (sizeof(S) == 1 || !big) {
    v = *reinterpret_cast<const S*>(p);
  } else {
    uint8_t t[sizeof(S)];
#pragma unroll
    for (int k = 0; k < (int)sizeof(S); ++k) t[k] = p[sizeof(S) - 1 - k];
    memcpy(&v, t, sizeof(S));
  }
  return v;
}

template <typename S>
__global__ void k_nifti_decode(const uint8_t* __restrict__ raw, long long n, int big, int scale, double slope,
                               double inter, double* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double d = (double)load_swapped<S>(raw + i * (long long)sizeof(S), big != 0);
    out[i] = scale ? __dadd_rn(__dmul_rn(d, slope), inter) : d;
  }
}

__global__ void k_to_f32(long long n, const double* __restrict__ in, float* __restrict__ out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = __double2float_rn(in[i]);
}

template <typename S>
void launch_decode(qsm_ctx* ctx, const uint8_t* raw, long long n, const qsm_nifti_header& h, double* out) {
  LaunchScope ls(ctx, "nifti_decode");
  k_nifti_decode<S><<<grid1d(n), 256, 0, ctx->stream>>>(raw, n, h.big_endian, h.raw_slope != 0.0 ? 1 : 0,
                                                        h.raw_slope, h.scl_inter, out);
  ls.done();
}

template <class F> void as_qsm_error(F&& f) {
  try {
    f();
  } catch (const nifti::Error& e) {
    throw QsmError(e.code, e.msg);
  }
}

}  // namespace

}  // namespace qsm

using namespace qsm;

extern "C" {

qsm_status qsm_nifti_load_device(qsm_ctx* ctx, const uint8_t* bytes, size_t len, int all_volumes, double* d_out,
                                 size_t out_len, qsm_nifti_header* hdr) {
  return guarded(ctx, [&] {
    check_ptr(d_out, "d_out");
    as_qsm_error([&] {
      const nifti::Image im = nifti::image_of(bytes, len);
      const qsm_nifti_header h = nifti::parse(im.p, im.n, im.gz);
      const size_t count = nifti::voxel_count(h, all_volumes != 0);
      if (out_len != count)
        throw QsmError(QSM_ERR_DIMENSION_MISMATCH,
                       "out_len " + std::to_string(out_len) + " != " + std::to_string(count) + " voxels");
      const uint8_t* src = nifti::voxels_of(im, h, count);
      const size_t eb = (size_t)nifti::element_bytes(h.datatype);
      uint8_t* raw = ws<uint8_t>(ctx, "nifti.raw", count * eb);
      staged_h2d(ctx, raw, src, count * eb);
      const long long n = (long long)count;
      switch (h.datatype) {
        case QSM_NIFTI_UINT8: launch_decode<uint8_t>(ctx, raw, n, h, d_out); break;
        case QSM_NIFTI_INT8: launch_decode<int8_t>(ctx, raw, n, h, d_out); break;
        case QSM_NIFTI_INT16: launch_decode<int16_t>(ctx, raw, n, h, d_out); break;
        case QSM_NIFTI_UINT16: launch_decode<uint16_t>(ctx, raw, n, h, d_out); break;
        case QSM_NIFTI_INT32: launch_decode<int32_t>(ctx, raw, n, h, d_out); break;
        case QSM_NIFTI_UINT32: launch_decode<uint32_t>(ctx, raw, n, h, d_out); break;
        case QSM_NIFTI_FLOAT32: launch_decode<float>(ctx, raw, n, h, d_out); break;
        case QSM_NIFTI_FLOAT64: launch_decode<double>(ctx, raw, n, h, d_out); break;
        case QSM_NIFTI_INT64: launch_decode<long long>(ctx, raw, n, h, d_out); break;
        case QSM_NIFTI_UINT64: launch_decode<unsigned long long>(ctx, raw, n, h, d_out); break;
        default: throw QsmError(QSM_ERR_IO, "unsupported datatype " + std::to_string(h.datatype));
      }
      sync(ctx);
      if (hdr) *hdr = h;
    });
  });
}

qsm_status qsm_nifti_save_device(qsm_ctx* ctx, const double* d_data, size_t nx, size_t ny, size_t nz,
                                 const double voxel_size[3], const double affine[16], int gzip_out, uint8_t* out,
                                 size_t out_cap, size_t* out_len) {
  return guarded(ctx, [&] {
    check_ptr(out_len, "out_len");
    as_qsm_error([&] {
      nifti::check_save_args(d_data, nx, ny, nz, voxel_size, affine);
      const size_t n = nx * ny * nz;
      const size_t raw = 352 + 4 * n;
      if (!out) {  // size query, as qsm_nifti_save
        *out_len = gzip_out ? nifti::gzip_bound(raw) : raw;
        return;
      }
      float* f32 = ws<float>(ctx, "nifti.f32", n);
      {
        LaunchScope ls(ctx, "nifti_to_f32");
        k_to_f32<<<grid1d((long long)n), 256, 0, ctx->stream>>>((long long)n, d_data, f32);
        ls.done();
      }
      std::vector<uint8_t> img = nifti::header_bytes(nx, ny, nz, voxel_size, affine);
      img.resize(raw);
      staged_d2h(ctx, img.data() + 352, f32, 4 * n);  // float32, little-endian on x86-64 hosts
      if (gzip_out) img = nifti::gzip(img.data(), img.size());
      if (out_cap < img.size())
        throw QsmError(QSM_ERR_INVALID_ARGUMENT,
                       "out_cap " + std::to_string(out_cap) + " < " + std::to_string(img.size()) + " bytes");
      std::memcpy(out, img.data(), img.size());
      *out_len = img.size();
    });
  });
}

}  // extern "C"
