// NIfTI-1 single-file I/O (src/io.rs:62-460), host side.
//
// Reading restates what the reference gets from the `nifti` crate (0.17.0, pinned in
// its Cargo.lock; not part of the reference tree) through load_nifti / load_nifti_4d
// (io.rs:62-224): the 348-byte NIfTI-1 header in either byte order, voxels from
// vox_offset in the stored datatype, cast to double and, when scl_slope != 0, mapped
// to raw * scl_slope + scl_inter; dims from dim[1..], the first volume for 4D data
// (all volumes for load_nifti_4d), the affine from the sform rows when sform_code > 0,
// else diag(pixdim) (io.rs:226-253).  gzip input is detected by its magic bytes
// (io.rs:29-31) and inflated with zlib.
//
// Writing follows save_nifti (io.rs:255-338) byte for byte: header fields, 4 zero
// extension bytes, float32 little-endian voxels; save_nifti_gz (io.rs:340-364) gzips
// that image at zlib's default level.
#include "nifti.h"

#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <new>
#include <stdexcept>

namespace qsm {
namespace nifti {

namespace {

[[noreturn]] void fail(const std::string& m, qsm_status c = QSM_ERR_IO) { throw Error{c, m}; }

bool host_le() {
  const uint16_t one = 1;
  uint8_t b;
  std::memcpy(&b, &one, 1);
  return b == 1;
}

template <typename T> T rd(const uint8_t* p, bool big) {
  uint8_t tmp[sizeof(T)];
  std::memcpy(tmp, p, sizeof(T));
  if (big == host_le())
    for (size_t i = 0; i < sizeof(T) / 2; ++i) std::swap(tmp[i], tmp[sizeof(T) - 1 - i]);
  T v;
  std::memcpy(&v, tmp, sizeof(T));
  return v;
}

template <typename T> void wr_le(uint8_t* p, T v) {
  uint8_t tmp[sizeof(T)];
  std::memcpy(tmp, &v, sizeof(T));
  if (!host_le())
    for (size_t i = 0; i < sizeof(T) / 2; ++i) std::swap(tmp[i], tmp[sizeof(T) - 1 - i]);
  std::memcpy(p, tmp, sizeof(T));
}

constexpr size_t kZChunk = (size_t)1 << 30;  // zlib counts in 32-bit units

}  // namespace

bool is_gzip(const uint8_t* b, size_t n) { return n >= 2 && b[0] == 0x1f && b[1] == 0x8b; }

std::vector<uint8_t> gunzip(const uint8_t* b, size_t n) {
  z_stream zs{};
  if (inflateInit2(&zs, 15 + 32) != Z_OK) fail("Failed to read gzipped NIfTI: inflateInit failed");
  std::vector<uint8_t> out(std::max<size_t>(n * 4, 1024));
  size_t fed = 0, produced = 0;
  while (true) {
    if (zs.avail_in == 0 && fed < n) {
      const size_t chunk = std::min(n - fed, kZChunk);
      zs.next_in = const_cast<Bytef*>(b + fed);
      zs.avail_in = (uInt)chunk;
      fed += chunk;
    }
    if (produced == out.size()) out.resize(out.size() * 2);
    const size_t room = std::min(out.size() - produced, kZChunk);
    zs.next_out = out.data() + produced;
    zs.avail_out = (uInt)room;
    const int rc = inflate(&zs, Z_NO_FLUSH);
    produced += room - zs.avail_out;
    if (rc == Z_STREAM_END) break;
    if (rc != Z_OK && rc != Z_BUF_ERROR) {
      const std::string m = zs.msg ? zs.msg : "zlib error";
      inflateEnd(&zs);
      fail("Failed to read gzipped NIfTI: corrupt gzip stream (" + m + ")");
    }
    if (rc == Z_BUF_ERROR && zs.avail_in == 0 && fed >= n && zs.avail_out > 0) {
      inflateEnd(&zs);
      fail("Failed to read gzipped NIfTI: truncated gzip stream");
    }
  }
  inflateEnd(&zs);
  out.resize(produced);
  return out;
}

size_t gzip_bound(size_t n) {
  // deflate's stored-block worst case (5 bytes per 16 KB block) plus the gzip wrapper
  return n + (n >> 12) + (n >> 14) + 5 * (n / 16384 + 1) + 64;
}

std::vector<uint8_t> gzip(const uint8_t* b, size_t n) {
  z_stream zs{};
  // zlib's default level (6), gzip wrapper (window bits 15 + 16)
  if (deflateInit2(&zs, Z_DEFAULT_COMPRESSION, Z_DEFLATED, 15 + 16, 8, Z_DEFAULT_STRATEGY) != Z_OK)
    fail("Gzip compression failed: deflateInit");
  std::vector<uint8_t> out(gzip_bound(n));
  size_t fed = 0, produced = 0;
  int rc = Z_OK;
  while (rc != Z_STREAM_END) {
    if (zs.avail_in == 0 && fed < n) {
      const size_t chunk = std::min(n - fed, kZChunk);
      zs.next_in = const_cast<Bytef*>(b + fed);
      zs.avail_in = (uInt)chunk;
      fed += chunk;
    }
    if (produced == out.size()) out.resize(out.size() * 2);
    const size_t room = std::min(out.size() - produced, kZChunk);
    zs.next_out = out.data() + produced;
    zs.avail_out = (uInt)room;
    rc = deflate(&zs, (fed >= n && zs.avail_in == 0) ? Z_FINISH : Z_NO_FLUSH);
    produced += room - zs.avail_out;
    if (rc == Z_STREAM_ERROR) {
      deflateEnd(&zs);
      fail("Gzip compression failed");
    }
  }
  deflateEnd(&zs);
  out.resize(produced);
  return out;
}

// get_header_info (io.rs:34-59): diagnostics appended to parse errors
std::string header_info(const uint8_t* b, size_t n) {
  char buf[160];
  if (n < 348) {
    std::snprintf(buf, sizeof buf, "File too small (%zu bytes, need at least 348)", n);
    return buf;
  }
  char magic[5] = {0, 0, 0, 0, 0};
  for (int i = 0; i < 4; ++i) magic[i] = (b[344 + i] >= 32 && b[344 + i] < 127) ? (char)b[344 + i] : '?';
  std::snprintf(buf, sizeof buf, "sizeof_hdr=%d, magic='%s', datatype=%d", (int)rd<int32_t>(b, false), magic,
                (int)rd<int16_t>(b + 70, false));
  return buf;
}

int element_bytes(int dt) {
  switch (dt) {
    case QSM_NIFTI_UINT8:
    case QSM_NIFTI_INT8:
      return 1;
    case QSM_NIFTI_INT16:
    case QSM_NIFTI_UINT16:
      return 2;
    case QSM_NIFTI_INT32:
    case QSM_NIFTI_UINT32:
    case QSM_NIFTI_FLOAT32:
      return 4;
    case QSM_NIFTI_FLOAT64:
    case QSM_NIFTI_INT64:
    case QSM_NIFTI_UINT64:
      return 8;
    default:
      return 0;
  }
}

qsm_nifti_header parse(const uint8_t* b, size_t n, bool gz) {
  const std::string what = gz ? "Failed to read gzipped NIfTI" : "Failed to read NIfTI";
  if (n < 348) fail(what + ": header too short (" + header_info(b, n) + ")");
  bool big;
  if (rd<int32_t>(b, false) == 348) big = false;
  else if (rd<int32_t>(b, true) == 348) big = true;
  else fail(what + ": invalid sizeof_hdr (" + header_info(b, n) + ")");
  if (!(b[344] == 'n' && b[345] == '+' && b[346] == '1' && b[347] == 0))
    fail(what + ": not a single-file NIfTI-1 image (" + header_info(b, n) + ")");
  qsm_nifti_header h{};
  int16_t dim[8];
  for (int i = 0; i < 8; ++i) dim[i] = rd<int16_t>(b + 40 + 2 * i, big);
  h.ndim = dim[0];
  if (dim[0] < 3) fail("Expected at least 3D volume, got " + std::to_string(dim[0]) + "D");  // io.rs:88-90
  if (dim[0] > 7) fail(what + ": dim[0] = " + std::to_string(dim[0]) + " is out of range");
  for (int i = 1; i <= dim[0]; ++i)
    if (dim[i] < 1) fail(what + ": dim[" + std::to_string(i) + "] < 1");
  for (int i = 5; i <= dim[0]; ++i)
    if (dim[i] != 1) fail(what + ": more than 4 non-singleton dimensions are not supported");
  h.nx = (size_t)dim[1];
  h.ny = (size_t)dim[2];
  h.nz = (size_t)dim[3];
  h.nt = dim[0] >= 4 ? (size_t)dim[4] : 1;
  h.datatype = rd<int16_t>(b + 70, big);
  if (element_bytes(h.datatype) == 0) fail(what + ": unsupported datatype " + std::to_string(h.datatype));
  float pix[8];
  for (int i = 0; i < 8; ++i) pix[i] = rd<float>(b + 76 + 4 * i, big);
  h.voxel_size[0] = (double)pix[1];  // io.rs:93-96
  h.voxel_size[1] = (double)pix[2];
  h.voxel_size[2] = (double)pix[3];
  const float vo = rd<float>(b + 108, big);
  if (!(vo >= 0.0f) || vo > 1e18f) fail(what + ": invalid vox_offset");
  h.vox_offset = (size_t)vo;
  if (h.vox_offset < 348) h.vox_offset = 352;  // single-file images keep voxels after the extension word
  const float slope = rd<float>(b + 112, big), inter = rd<float>(b + 116, big);
  h.scl_slope = slope == 0.0f ? 1.0 : (double)slope;  // io.rs:99
  h.scl_inter = (double)inter;
  h.raw_slope = (double)slope;
  if (rd<int16_t>(b + 254, big) > 0) {  // sform rows, io.rs:228-240
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 4; ++c) h.affine[4 * r + c] = (double)rd<float>(b + 280 + 16 * r + 4 * c, big);
  } else {  // diag(pixdim), io.rs:241-252
    h.affine[0] = (double)pix[1];
    h.affine[5] = (double)pix[2];
    h.affine[10] = (double)pix[3];
  }
  h.affine[15] = 1.0;
  h.big_endian = big ? 1 : 0;
  h.gzip = gz ? 1 : 0;
  return h;
}

size_t voxel_count(const qsm_nifti_header& h, bool all) { return h.nx * h.ny * h.nz * (all ? h.nt : 1); }

std::vector<uint8_t> header_bytes(size_t nx, size_t ny, size_t nz, const double vs[3], const double affine[16]) {
  std::vector<uint8_t> h(352, 0);
  wr_le<int32_t>(&h[0], 348);
  const int16_t dim[8] = {3, (int16_t)nx, (int16_t)ny, (int16_t)nz, 1, 1, 1, 1};
  for (int i = 0; i < 8; ++i) wr_le<int16_t>(&h[40 + 2 * i], dim[i]);
  wr_le<int16_t>(&h[70], 16);  // FLOAT32
  wr_le<int16_t>(&h[72], 32);  // bitpix
  const float pix[8] = {1.0f, (float)vs[0], (float)vs[1], (float)vs[2], 1.0f, 1.0f, 1.0f, 1.0f};
  for (int i = 0; i < 8; ++i) wr_le<float>(&h[76 + 4 * i], pix[i]);
  wr_le<float>(&h[108], 352.0f);  // vox_offset
  wr_le<float>(&h[112], 1.0f);    // scl_slope
  wr_le<float>(&h[116], 0.0f);    // scl_inter
  wr_le<int16_t>(&h[254], 1);     // sform_code
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 4; ++c) wr_le<float>(&h[280 + 16 * r + 4 * c], (float)affine[4 * r + c]);
  h[344] = 'n';
  h[345] = '+';
  h[346] = '1';
  h[347] = 0;
  return h;
}

Image image_of(const uint8_t* bytes, size_t len) {
  if (!bytes) fail("bytes is null", QSM_ERR_INVALID_ARGUMENT);
  Image im;
  im.gz = is_gzip(bytes, len);
  if (im.gz) {
    im.owned = gunzip(bytes, len);
    im.p = im.owned.data();
    im.n = im.owned.size();
  } else {
    im.p = bytes;
    im.n = len;
  }
  return im;
}

const uint8_t* voxels_of(const Image& im, const qsm_nifti_header& h, size_t count) {
  const size_t need = h.vox_offset + count * (size_t)element_bytes(h.datatype);
  if (im.n < need)
    fail(std::string(im.gz ? "Failed to read gzipped NIfTI" : "Failed to read NIfTI") + ": expected " +
         std::to_string(need) + " bytes of header and voxels, got " + std::to_string(im.n));
  return im.p + h.vox_offset;
}

void check_save_args(const double* data, size_t nx, size_t ny, size_t nz, const double* vs, const double* affine) {
  if (!data || !vs || !affine) fail("null argument", QSM_ERR_INVALID_ARGUMENT);
  if (nx == 0 || ny == 0 || nz == 0 || nx > 32767 || ny > 32767 || nz > 32767)
    fail("dims must be in 1..32767 (NIfTI-1 stores them as int16)", QSM_ERR_INVALID_ARGUMENT);
}

}  // namespace nifti
}  // namespace qsm

using namespace qsm::nifti;

namespace {

bool host_le_check() {
  const uint16_t one = 1;
  uint8_t b;
  std::memcpy(&b, &one, 1);
  return b == 1;
}

void set_err(char* err, size_t cap, const std::string& m) {
  if (!err || cap == 0) return;
  const size_t k = std::min(cap - 1, m.size());
  std::memcpy(err, m.data(), k);
  err[k] = 0;
}

template <class F> qsm_status io_guard(char* err, size_t cap, F&& f) {
  try {
    f();
    set_err(err, cap, "");
    return QSM_OK;
  } catch (const Error& e) {
    set_err(err, cap, e.msg);
    return e.code;
  } catch (const std::bad_alloc&) {
    set_err(err, cap, "host allocation failed");
    return QSM_ERR_ALLOC;
  } catch (const std::exception& e) {
    set_err(err, cap, e.what());
    return QSM_ERR_IO;
  }
}

[[noreturn]] void raise(const std::string& m, qsm_status c = QSM_ERR_IO) { throw Error{c, m}; }

template <typename S>
void decode_as(const uint8_t* src, bool big, size_t n, bool scale, double slope, double inter, double* out) {
  const bool swap = sizeof(S) > 1 && big == host_le_check();
  for (size_t i = 0; i < n; ++i) {
    uint8_t tmp[sizeof(S)];
    std::memcpy(tmp, src + i * sizeof(S), sizeof(S));
    if (swap)
      for (size_t k = 0; k < sizeof(S) / 2; ++k) std::swap(tmp[k], tmp[sizeof(S) - 1 - k]);
    S v;
    std::memcpy(&v, tmp, sizeof(S));
    const double d = (double)v;
    if (scale) {
      volatile double p = d * slope;  // raw * slope, rounded, then + inter (no contraction)
      out[i] = p + inter;
    } else {
      out[i] = d;
    }
  }
}

void decode(const qsm_nifti_header& h, const uint8_t* src, size_t n, double* out) {
  const bool big = h.big_endian != 0;
  const bool scale = h.raw_slope != 0.0;
  const double s = h.raw_slope, c = h.scl_inter;
  switch (h.datatype) {
    case QSM_NIFTI_UINT8: decode_as<uint8_t>(src, big, n, scale, s, c, out); break;
    case QSM_NIFTI_INT8: decode_as<int8_t>(src, big, n, scale, s, c, out); break;
    case QSM_NIFTI_INT16: decode_as<int16_t>(src, big, n, scale, s, c, out); break;
    case QSM_NIFTI_UINT16: decode_as<uint16_t>(src, big, n, scale, s, c, out); break;
    case QSM_NIFTI_INT32: decode_as<int32_t>(src, big, n, scale, s, c, out); break;
    case QSM_NIFTI_UINT32: decode_as<uint32_t>(src, big, n, scale, s, c, out); break;
    case QSM_NIFTI_FLOAT32: decode_as<float>(src, big, n, scale, s, c, out); break;
    case QSM_NIFTI_FLOAT64: decode_as<double>(src, big, n, scale, s, c, out); break;
    case QSM_NIFTI_INT64: decode_as<int64_t>(src, big, n, scale, s, c, out); break;
    case QSM_NIFTI_UINT64: decode_as<uint64_t>(src, big, n, scale, s, c, out); break;
    default: raise("unsupported datatype " + std::to_string(h.datatype));
  }
}

std::vector<uint8_t> read_all(const char* path) {
  if (!path) raise("path is null", QSM_ERR_INVALID_ARGUMENT);
  std::ifstream f(path, std::ios::binary);
  if (!f) raise(std::string("Failed to read file '") + path + "': cannot open");  // io.rs:425-426
  f.seekg(0, std::ios::end);
  const std::streamoff sz = f.tellg();
  if (sz < 0) raise(std::string("Failed to read file '") + path + "': cannot size");
  f.seekg(0, std::ios::beg);
  std::vector<uint8_t> b((size_t)sz);
  if (sz > 0 && !f.read(reinterpret_cast<char*>(b.data()), sz))
    raise(std::string("Failed to read file '") + path + "': short read");
  return b;
}

bool ends_with(const std::string& s, const char* suf) {
  const size_t k = std::strlen(suf);
  return s.size() >= k && s.compare(s.size() - k, k, suf) == 0;
}

// save_nifti's uncompressed image
std::vector<uint8_t> encode(const double* data, size_t nx, size_t ny, size_t nz, const double* vs,
                            const double* affine) {
  std::vector<uint8_t> img = header_bytes(nx, ny, nz, vs, affine);
  const size_t n = nx * ny * nz;
  img.resize(352 + 4 * n);
  uint8_t* p = img.data() + 352;
  const bool le = host_le_check();
  for (size_t i = 0; i < n; ++i) {
    const float f = (float)data[i];
    std::memcpy(p + 4 * i, &f, 4);
    if (!le) {
      std::swap(p[4 * i], p[4 * i + 3]);
      std::swap(p[4 * i + 1], p[4 * i + 2]);
    }
  }
  return img;
}

}  // namespace

extern "C" {

qsm_status qsm_nifti_parse_header(const uint8_t* bytes, size_t len, qsm_nifti_header* out, char* err,
                                  size_t err_cap) {
  return io_guard(err, err_cap, [&] {
    if (!out) raise("out is null", QSM_ERR_INVALID_ARGUMENT);
    const Image im = image_of(bytes, len);
    *out = parse(im.p, im.n, im.gz);
  });
}

qsm_status qsm_nifti_load(const uint8_t* bytes, size_t len, int all_volumes, double* out, size_t out_len,
                          qsm_nifti_header* hdr, char* err, size_t err_cap) {
  return io_guard(err, err_cap, [&] {
    if (!out) raise("out is null", QSM_ERR_INVALID_ARGUMENT);
    const Image im = image_of(bytes, len);
    const qsm_nifti_header h = parse(im.p, im.n, im.gz);
    const size_t count = voxel_count(h, all_volumes != 0);
    if (out_len != count)
      raise("out_len " + std::to_string(out_len) + " != " + std::to_string(count) + " voxels",
            QSM_ERR_DIMENSION_MISMATCH);
    decode(h, voxels_of(im, h, count), count, out);
    if (hdr) *hdr = h;
  });
}

qsm_status qsm_nifti_save(const double* data, size_t nx, size_t ny, size_t nz, const double voxel_size[3],
                          const double affine[16], int gzip_out, uint8_t* out, size_t out_cap, size_t* out_len,
                          char* err, size_t err_cap) {
  return io_guard(err, err_cap, [&] {
    if (!out_len) raise("out_len is null", QSM_ERR_INVALID_ARGUMENT);
    check_save_args(data, nx, ny, nz, voxel_size, affine);
    const size_t raw = 352 + 4 * nx * ny * nz;
    if (!out) {  // size query: exact when uncompressed, an upper bound for gzip
      *out_len = gzip_out ? gzip_bound(raw) : raw;
      return;
    }
    std::vector<uint8_t> img = encode(data, nx, ny, nz, voxel_size, affine);
    if (gzip_out) img = gzip(img.data(), img.size());
    if (out_cap < img.size())
      raise("out_cap " + std::to_string(out_cap) + " < " + std::to_string(img.size()) + " bytes",
            QSM_ERR_INVALID_ARGUMENT);
    std::memcpy(out, img.data(), img.size());
    *out_len = img.size();
  });
}

qsm_status qsm_nifti_read_dims(const char* path, size_t dims[3], char* err, size_t err_cap) {
  return io_guard(err, err_cap, [&] {
    if (!dims) raise("dims is null", QSM_ERR_INVALID_ARGUMENT);
    const std::vector<uint8_t> b = read_all(path);
    const Image im = image_of(b.data(), b.size());
    const qsm_nifti_header h = parse(im.p, im.n, im.gz);
    dims[0] = h.nx;
    dims[1] = h.ny;
    dims[2] = h.nz;
  });
}

qsm_status qsm_nifti_read_file_header(const char* path, qsm_nifti_header* out, char* err, size_t err_cap) {
  return io_guard(err, err_cap, [&] {
    if (!out) raise("out is null", QSM_ERR_INVALID_ARGUMENT);
    const std::vector<uint8_t> b = read_all(path);
    const Image im = image_of(b.data(), b.size());
    *out = parse(im.p, im.n, im.gz);
  });
}

qsm_status qsm_nifti_read_file(const char* path, int all_volumes, double* out, size_t out_len, qsm_nifti_header* hdr,
                               char* err, size_t err_cap) {
  return io_guard(err, err_cap, [&] {
    const std::vector<uint8_t> b = read_all(path);
    char e2[512] = {0};
    const qsm_status s = qsm_nifti_load(b.data(), b.size(), all_volumes, out, out_len, hdr, e2, sizeof e2);
    if (s != QSM_OK) raise(e2, s);
  });
}

qsm_status qsm_nifti_save_file(const char* path, const double* data, size_t nx, size_t ny, size_t nz,
                               const double voxel_size[3], const double affine[16], char* err, size_t err_cap) {
  return io_guard(err, err_cap, [&] {
    if (!path) raise("path is null", QSM_ERR_INVALID_ARGUMENT);
    check_save_args(data, nx, ny, nz, voxel_size, affine);
    std::vector<uint8_t> img = encode(data, nx, ny, nz, voxel_size, affine);
    if (ends_with(path, ".nii.gz")) img = gzip(img.data(), img.size());  // io.rs:441-446
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f) raise(std::string("Failed to write file '") + path + "': cannot open");
    f.write(reinterpret_cast<const char*>(img.data()), (std::streamsize)img.size());
    if (!f) raise(std::string("Failed to write file '") + path + "': short write");
  });
}

}  // extern "C"
