// NIfTI-1 single-file (.nii / .nii.gz) parsing and writing, host side.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/qsmgpu.h"

namespace qsm {
namespace nifti {

struct Error {
  qsm_status code;
  std::string msg;
};

bool is_gzip(const uint8_t* b, size_t n);
// Whole gzip stream -> bytes (throws Error).
std::vector<uint8_t> gunzip(const uint8_t* b, size_t n);
// Parse a 348-byte NIfTI-1 header at the start of uncompressed bytes (throws Error).
qsm_nifti_header parse(const uint8_t* b, size_t n, bool gzip);
// Bytes of one stored element of a datatype (0: unsupported).
int element_bytes(int datatype);
// Voxels the output holds: nx*ny*nz, times nt when all_volumes.
size_t voxel_count(const qsm_nifti_header& h, bool all_volumes);
// The 352 leading bytes (header and the zero extension word) of save_nifti's image.
std::vector<uint8_t> header_bytes(size_t nx, size_t ny, size_t nz, const double vs[3], const double affine[16]);
std::vector<uint8_t> gzip(const uint8_t* b, size_t n);
// Upper bound of gzip()'s output size for n input bytes.
size_t gzip_bound(size_t n);
std::string header_info(const uint8_t* b, size_t n);

// The uncompressed image of an in-memory file: the input itself, or its inflation.
struct Image {
  std::vector<uint8_t> owned;
  const uint8_t* p = nullptr;
  size_t n = 0;
  bool gz = false;
};
Image image_of(const uint8_t* bytes, size_t len);
// Start of `count` stored voxels (throws Error when the image is too short).
const uint8_t* voxels_of(const Image& im, const qsm_nifti_header& h, size_t count);
void check_save_args(const double* data, size_t nx, size_t ny, size_t nz, const double* vs, const double* affine);

}  // namespace nifti
}  // namespace qsm
