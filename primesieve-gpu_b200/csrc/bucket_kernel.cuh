// bucket_kernel.cuh -- device-side EratBig: fill the per-segment bucket lists.
//
// The range is processed in windows of W consecutive segments. For every
// big sieving prime (p >= big limit) this kernel enumerates all of its
// multiples inside the window and appends one 4-byte entry
//     (byte index inside the segment) << 3 | bit
// to the list of the segment the multiple falls into. The sieve kernel then
// streams each segment's lists from HBM and applies them with shared-memory
// atomics. A bucket entry needs no sieving prime: the prime's position is
// recomputed once per window (one reciprocal multiply), so nothing but the
// entries themselves crosses HBM.
//
// One CTA owns a contiguous chunk of big primes and one list per segment;
// it counts the entries of each of the window's segments in shared memory
// (shared atomicAdd gives each entry its slot), so no global atomics are
// needed. A list has a fixed capacity (its expected length plus a generous
// margin); entries beyond it are dropped and the overflow flag is raised, and
// the host then recounts the range with larger lists.
//
// Reference counterpart: the CPU bucket sieve EratBig (src/EratBig.cpp:127-243,
// src/Bucket.hpp:32-148), which stores (sievingPrime, multipleIndex,
// wheelIndex) per entry in 8 KiB buckets; the reference GPU kernel has no
// bucket phase at all (doc/GPU.md:120-125).
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>
#include "wheel.hpp"
#include "sieve_kernel.cuh"

namespace psg {

struct BucketArgs {
  uint64_t win_low;           // segLow of the window's first segment
  uint32_t win_segments;      // segments in this window (<= counters in smem)
  uint32_t seg_bytes;
  uint64_t seg_rcp;           // floor((2^64-1)/seg_bytes)
  const uint32_t* primes;
  const uint64_t* recip;
  uint32_t first, last;       // big primes: primes[first, last)
  uint32_t primes_per_list;   // chunk of primes per CTA (= per list)
  uint32_t num_lists;
  const uint32_t* list_off;   // [num_lists] entry offset inside a segment region
  const uint32_t* list_cap;   // [num_lists] capacity
  uint64_t seg_stride;        // entries per segment region
  uint32_t* entries;
  uint32_t* counts;           // [win_segments][num_lists]
  uint32_t* overflow;         // set to 1 if any list overflowed
};

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
bucket_fill_kernel(const __grid_constant__ BucketArgs a)
{
  extern __shared__ uint32_t seg_count[];
  const uint32_t tid = threadIdx.x;
  const uint32_t W = a.win_segments;
  for (uint32_t i = tid; i < W; i += BLOCK) seg_count[i] = 0;
  __syncthreads();

  const uint32_t list = blockIdx.x;
  const uint32_t cap = a.list_cap[list];
  uint32_t* const out = a.entries + a.list_off[list];
  const uint64_t win_bytes = (uint64_t) W * a.seg_bytes;
  const uint32_t seg_bytes = a.seg_bytes;

  const uint64_t lo = (uint64_t) a.first + (uint64_t) list * a.primes_per_list;
  uint64_t hi = lo + a.primes_per_list;
  if (hi > a.last) hi = a.last;

  for (uint64_t i = lo + tid; i < hi; i += BLOCK) {
    const uint32_t p = a.primes[i];
    const uint64_t rcp = a.recip[i];
    uint64_t d; uint32_t c0;
    first_multiple(a.win_low, p, rcp, d, c0);
    if (d / 30u >= win_bytes) continue;
    const uint32_t pm = p % 30u;
#pragma unroll 1
    for (uint32_t j = 0; j < 8; j++) {
      const uint32_t Q = cofactor_class(j);
      const uint32_t k = (Q + 30u - c0) % 30u;
      uint64_t b = (d + (uint64_t) k * p) / 30u;      // byte index in window
      if (b >= win_bytes) continue;
      const uint32_t bit = residue_to_bit((Q * pm) % 30u);
      do {
        // segment = b / seg_bytes via the reciprocal, then correct
        uint64_t sg = __umul64hi(b, a.seg_rcp);
        uint64_t bo = b - sg * seg_bytes;
        if (bo >= seg_bytes) { bo -= seg_bytes; sg++; }
        if (bo >= seg_bytes) { bo -= seg_bytes; sg++; }
        const uint32_t pos = atomicAdd(&seg_count[sg], 1u);
        if (pos < cap)
          out[sg * a.seg_stride + pos] = ((uint32_t) bo << 3) | bit;
        b += p;
      } while (b < win_bytes);
    }
  }
  __syncthreads();

  for (uint32_t sgi = tid; sgi < W; sgi += BLOCK) {
    uint32_t c = seg_count[sgi];
    if (c > cap) { atomicOr(a.overflow, 1u); c = cap; }
    a.counts[(uint64_t) sgi * a.num_lists + list] = c;
  }
}

} // namespace psg
