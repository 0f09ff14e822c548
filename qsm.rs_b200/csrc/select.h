// Exact order statistics of device arrays: the percentile thresholds of iLSQR's
// weights (src/inversion/ilsqr.rs:672-760, 854-900), which the reference takes from a
// full sort of the values.  A radix selection on the order-preserving 64-bit keys of
// the doubles finds the same elements without sorting.
#pragma once

#include <vector>

#include "internal.h"

namespace qsm {

// Number of i < n with mask[i] != 0 (n when mask is null).
long long count_selected(qsm_ctx* ctx, const uint8_t* mask, long long n);

// Values of the given 0-based ranks in ascending order (at most 4 ranks per call)
// among vals[i] with mask[i] != 0 (all n values when mask is null).  Every rank must
// be below the number of selected values.
std::vector<double> select_ranks(qsm_ctx* ctx, const double* vals, const uint8_t* mask, long long n,
                                 const std::vector<long long>& ranks);

// prctile of the selected values for each percent in p (linear interpolation between
// the order statistics around (p/100)*(count-1), src/inversion/ilsqr.rs:937-946).
// `count` is the number of selected values (> 0); at most two percents per call.
std::vector<double> percentiles(qsm_ctx* ctx, const double* vals, const uint8_t* mask, long long n,
                                long long count, const std::vector<double>& p);

}  // namespace qsm
