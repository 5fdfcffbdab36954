// batch_kernel.cuh -- persistent kernel for many ranges at once.
//
// The reference counts one range per call (src/api.cpp:48-118), each call a
// full GPU pass with its own launches and host round trips. Here a batch of
// ranges becomes a device work queue of (range, segment stripe) items; a
// persistent grid (one CTA per SM) takes items from a global counter, so
// ranges of very different sizes share the GPU without a launch per range
// and without load imbalance between them. Each item runs the same segment
// phases as the range kernel (pre-sieve, small, medium with carried state,
// direct), with the prime tiers of its own range, and adds its counts to the
// range's row. Ranges that need the bucket tier are not items; the host runs
// them through the windowed range path.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>
#include "sieve_kernel.cuh"
#include "batch_types.hpp"

namespace psg {

struct BatchArgs {
  SieveArgs common;             // tables, primes, segment size (range fields unused)
  const BatchRange* ranges;
  const BatchItem* items;       // most expensive first
  uint32_t num_items;
  uint32_t* queue;              // next item; zero before the launch
  unsigned long long* counts;   // [range][6], added to
};

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
batch_sieve_kernel(const __grid_constant__ BatchArgs b)
{
  const SieveArgs& a = b.common;
  extern __shared__ uint4 smem4[];
  uint32_t* const sieve32 = reinterpret_cast<uint32_t*>(smem4);
  uint32_t* const mstate = sieve32 + (a.seg_bytes >> 2);
  const uint32_t tid = threadIdx.x;
  const uint32_t lane = tid & 31u;
  const uint32_t warp = tid >> 5;
  const uint64_t span = (uint64_t) a.seg_bytes * 30u;

  __shared__ uint32_t wheel_tab[16];
  __shared__ uint32_t s_item;
  if (tid < 16) wheel_tab[tid] = a.wheel_tab[tid];

  uint64_t acc[6] = { 0, 0, 0, 0, 0, 0 };
  uint32_t sp[kSmallRegs], sr[kSmallRegs], sdl[kSmallRegs];

  for (;;) {
    if (tid == 0) s_item = atomicAdd(b.queue, 1u);
    __syncthreads();
    const uint32_t it = s_item;
    __syncthreads();                    // s_item is rewritten only after this
    if (it >= b.num_items) break;
    const BatchItem item = b.items[it];
    const BatchRange r = b.ranges[item.range];
    const uint64_t low0 = r.seg_low0 + (uint64_t) item.seg0 * span;
    const uint32_t n_med = r.n_med_end - r.n_small;

    small_setup<BLOCK>(a, r.n_small, low0 + 7, true, warp, lane, sp, sr, sdl);
    medium_setup<BLOCK>(a, r.n_small, n_med, mstate, low0, tid);
    for (uint32_t s = 0; s < item.nseg; s++) {
      const uint64_t segLow = low0 + (uint64_t) s * span;
      phase_presieve<BLOCK>(a, smem4, segLow, tid);
      __syncthreads();
      phase_small<BLOCK>(a, r.n_small, sieve32, segLow, warp, lane, sp, sr);
      phase_medium<BLOCK>(a, r.n_small, n_med, mstate, sieve32, wheel_tab, segLow, tid);
      phase_direct<BLOCK>(a, r.n_med_end, r.n_end, sieve32, wheel_tab, segLow, tid);
      __syncthreads();
      phase_count<BLOCK, true>(smem4, a.seg_bytes, segLow, r.lo, r.hi, tid, acc);
      small_advance(sp, sr, sdl);
      __syncthreads();
    }
    flush_counts<true>(acc, r.kinds, b.counts + 6ull * item.range, lane);
  }
}

} // namespace psg
