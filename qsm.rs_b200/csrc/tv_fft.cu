// The FFT half of a TV-ADMM iteration (tv_fft) and the tuning of its launch shapes
// (tv_tune), instantiated here only: its
// compile-time passes cover the wide axis-length list, and one translation unit keeps
// those kernels out of the solver files that share the iteration.
#include "tv_shared.cuh"

namespace qsm {

template void tv_fft<float>(qsm_ctx*, const TvVol<float>&, int, const int*);
template void tv_fft<double>(qsm_ctx*, const TvVol<double>&, int, const int*);
template void tv_tune<float>(qsm_ctx*, const TvVol<float>&);
template void tv_tune<double>(qsm_ctx*, const TvVol<double>&);

}  // namespace qsm
