// sweep_kernel.cuh -- device EratBig, segment-major: fill the bucket lists
// of a window with coalesced writes.
//
// Scattered 4-byte appends to thousands of lists run at ~1e11 stores/s on
// B200 (each one a partial DRAM sector), so the prime-major bucket fill
// (bucket_kernel.cuh) is store-bound for primes with many hits per window.
// This kernel walks the window segment by segment instead: every lane owns
// K sieving primes whose wheel state (next multiple's byte offset in the
// window, wheel index) it keeps in registers. For segment s the warp emits
// all hits below the segment end with a ballot: each round the active lanes
// write one entry each to consecutive slots of the CTA's list for segment s
// (one shared atomicAdd per warp and round reserves the slots), so the
// stores of a round are one contiguous 128-byte run.
//
// The state lives in HBM between windows (8 bytes per prime, read at kernel
// start and written back at the end); the first window of a count computes
// it from scratch (first multiple >= window start, cofactor >= p).
//
// Entries have the same format as the prime-major kernel's:
//   (byte index inside the segment) << 3 | bit
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>
#include "wheel.hpp"
#include "sieve_kernel.cuh"

namespace psg {

struct SweepArgs {
  uint64_t win_low;             // segLow of the window's first segment
  uint32_t win_segments;        // W (<= shared counters)
  uint32_t seg_bytes;
  const uint32_t* primes;       // sweep primes: primes[first, first + n)
  const uint64_t* recip;
  uint32_t first, n;
  uint32_t init;                // 1: compute the state from win_low
  uint32_t* state_b;            // [n] byte offset of the next multiple in the window
  uint32_t* state_i;            // [n] pdiv30 | cls << 22 | j << 25
  uint32_t list_base;           // index of this kernel's first list
  uint32_t num_lists_total;     // lists per segment (all kernels)
  const uint32_t* list_off;     // [num_lists_total]
  const uint32_t* list_cap;
  uint64_t seg_stride;
  uint32_t* entries;
  uint32_t* counts;             // [W][num_lists_total]
  uint32_t* overflow;
  unsigned long long* entry_total;
  uint32_t wheel_tab[16];       // per class: bits, corr
};

constexpr uint32_t kFarState = 0xfffffffeu;

template <int BLOCK, int K>
__global__ void __launch_bounds__(BLOCK)
bucket_sweep_kernel(const __grid_constant__ SweepArgs a)
{
  extern __shared__ uint32_t seg_count[];      // [W]
  __shared__ uint32_t wheel_tab[16];
  constexpr int NWARPS = BLOCK / 32;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t W = a.win_segments;
  for (uint32_t i = tid; i < W; i += BLOCK) seg_count[i] = 0;
  if (tid < 16) wheel_tab[tid] = a.wheel_tab[tid];
  __syncthreads();

  const uint32_t list = a.list_base + blockIdx.x;
  const uint32_t cap = a.list_cap[list];
  uint32_t* const out = a.entries + a.list_off[list];
  const uint32_t seg_bytes = a.seg_bytes;
  const uint32_t win_bytes = W * seg_bytes;          // < 2^31 (host-checked)
  const uint32_t gw = blockIdx.x * NWARPS + warp;    // global warp
  const uint32_t nw = gridDim.x * NWARPS;
  const uint32_t lanemask_lt = (1u << lane) - 1u;

  // slot k of this lane <-> sweep prime (k * nw + gw) * 32 + lane
  uint32_t sb[K], si[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    const uint32_t idx = ((uint32_t) k * nw + gw) * 32u + lane;
    sb[k] = 0xffffffffu; si[k] = 0;
    if (idx < a.n) {
      // kFarState: the first multiple was >= 2^32 bytes past a window start;
      // recompute it for this window
      const bool fresh = a.init || a.state_b[idx] == kFarState;
      if (fresh) {
        const uint32_t p = a.primes[a.first + idx];
        uint64_t d; uint32_t c0;
        first_multiple(a.win_low, p, a.recip[a.first + idx], d, c0);
        const uint32_t j = first_class_ge(c0);
        const uint64_t b = (d + (uint64_t) (cofactor_class(j) - c0) * p) / 30u;
        const uint32_t pdiv30 = p / 30u;
        sb[k] = (b < (uint64_t) kFarState) ? (uint32_t) b : kFarState;
        si[k] = pdiv30 | (residue_to_bit(p - 30u * pdiv30) << 22) | (j << 25);
      } else {
        sb[k] = a.state_b[idx];
        si[k] = a.state_i[idx];
      }
    }
  }

  uint32_t written = 0;
  for (uint32_t s = 0; s < W; s++) {
    const uint32_t seg_lo = s * seg_bytes;
    const uint32_t seg_end = seg_lo + seg_bytes;
    uint32_t* const seg_out = out + (uint64_t) s * a.seg_stride;
#pragma unroll
    for (int k = 0; k < K; k++) {
      uint32_t b = sb[k];
      uint32_t info = si[k];
      for (;;) {
        const bool act = b < seg_end;
        const uint32_t m = __ballot_sync(0xffffffffu, act);
        if (!m) break;
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&seg_count[s], (uint32_t) __popc(m));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (act) {
          const uint32_t j = (info >> 25) & 7u;
          const uint32_t cls = (info >> 22) & 7u;
          const uint32_t sh = 3u * j;
          const uint32_t bit = (wheel_tab[2 * cls] >> sh) & 7u;
          const uint32_t pos = base + __popc(m & lanemask_lt);
          if (pos < cap) seg_out[pos] = ((b - seg_lo) << 3) | bit;
          const uint32_t inc = (info & 0x3fffffu) * ((kGapPacked >> sh) & 7u) +
                               ((wheel_tab[2 * cls + 1] >> sh) & 7u);
          b += inc;                                   // < 2^31 + 2^25: no wrap
          info = (info & ~(7u << 25)) | (((j + 1u) & 7u) << 25);
        }
      }
      sb[k] = b;
      si[k] = info;
    }
  }

  // carry the state into the next window
#pragma unroll
  for (int k = 0; k < K; k++) {
    const uint32_t idx = ((uint32_t) k * nw + gw) * 32u + lane;
    if (idx < a.n) {
      a.state_b[idx] = (sb[k] == kFarState) ? kFarState : sb[k] - win_bytes;
      a.state_i[idx] = si[k];
    }
  }
  __syncthreads();
  for (uint32_t sgi = tid; sgi < W; sgi += BLOCK) {
    uint32_t c = seg_count[sgi];
    if (c > cap) { atomicOr(a.overflow, 1u); c = cap; }
    a.counts[(uint64_t) sgi * a.num_lists_total + list] = c;
    written += c;
  }
  for (int o = 16; o > 0; o >>= 1) written += __shfl_xor_sync(0xffffffffu, written, o);
  if (lane == 0 && written) atomicAdd(a.entry_total, (unsigned long long) written);
}

} // namespace psg
