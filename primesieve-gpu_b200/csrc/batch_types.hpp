// batch_types.hpp -- work descriptors of the persistent batch kernel
// (plain structs shared by host code and batch_kernel.cuh).
#pragma once
#include <stdint.h>

namespace psg {

// One range of a batch with its prime tiers.
struct BatchRange {
  uint64_t seg_low0;            // multiple of 30
  uint64_t lo, hi;              // inclusive, 7 <= lo <= hi
  uint32_t n_small;             // primes[0, n_small): warp per prime
  uint32_t n_med_end;           // primes[n_small, n_med_end): carried state
  uint32_t n_end;               // primes[n_med_end, n_end): direct
  uint32_t kinds;
};

// A stripe of consecutive segments of one range.
struct BatchItem {
  uint32_t range;
  uint32_t seg0;                // first segment of the stripe
  uint32_t nseg;                // >= 1
  uint32_t pad;
};

} // namespace psg
