// primegen_kernel.cuh -- device generation of the sieving-prime table.
//
// The reference generates its sieving primes on the CPU
// (primesieve::generate_primes(7, sqrt(hi)), src/gpu/cuda/CudaBackend.cpp:353)
// and uploads them; near 2^64 that is all primes below 2^32 (203 million).
// Here the same wheel-30 segment sieve produces them on the device, in two
// passes over the segments of (lo, hi]: pass 0 counts the primes of every
// segment, the host turns the counts into output offsets, and pass 1 sieves
// again and writes each segment's primes in ascending order at its offset.
// Base primes (<= 2^16) are crossed off warp-cooperatively when small and
// by one thread per prime (wheel walk) otherwise, exactly like the count
// kernel's small and medium tiers.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>
#include "wheel.hpp"
#include "sieve_kernel.cuh"

namespace psg {

struct PrimeGenArgs {
  uint64_t seg_low0;            // multiple of 30
  uint64_t lo, hi;              // emit primes p with lo <= p <= hi (lo >= 7, hi < 2^32)
  uint32_t num_segments;
  uint32_t seg_bytes;           // multiple of 16 * BLOCK
  const uint32_t* base;         // base primes 7 <= q <= sqrt(hi), ascending
  const uint64_t* base_recip;
  uint32_t n_base_small;        // base[0, n_base_small): one warp per prime
  uint32_t n_base;
  uint32_t pass;                // 0: count, 1: emit
  uint32_t* seg_counts;         // [num_segments] (pass 0)
  const uint64_t* seg_offsets;  // [num_segments] (pass 1)
  uint32_t* out;                // pass 1 output
  uint32_t wheel_tab[16];
};

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
primegen_kernel(const __grid_constant__ PrimeGenArgs a)
{
  extern __shared__ uint4 smem4[];
  uint32_t* const sieve32 = reinterpret_cast<uint32_t*>(smem4);
  __shared__ uint32_t wheel_tab[16];
  __shared__ uint32_t wtot[BLOCK / 32];
  constexpr uint32_t NWARPS = BLOCK / 32;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t seg_bytes = a.seg_bytes;
  const uint32_t nchunks = seg_bytes >> 4;
  const uint32_t nwords = seg_bytes >> 2;
  const uint64_t span = (uint64_t) seg_bytes * 30u;
  if (tid < 16) wheel_tab[tid] = a.wheel_tab[tid];

  for (uint32_t s = blockIdx.x; s < a.num_segments; s += gridDim.x) {
    const uint64_t segLow = a.seg_low0 + (uint64_t) s * span;
    for (uint32_t c = tid; c < nchunks; c += BLOCK) smem4[c] = make_uint4(~0u, ~0u, ~0u, ~0u);
    __syncthreads();

    // small base primes: one warp per prime, lane = (wheel class, phase)
    {
      const uint32_t j = lane & 7u, r = lane >> 3;
      const uint32_t Q = cofactor_class(j);
      for (uint32_t i = warp; i < a.n_base_small; i += NWARPS) {
        const uint32_t p = a.base[i];
        uint64_t d; uint32_t c0;
        first_multiple(segLow, p, a.base_recip[i], d, c0);
        if (d >= span) continue;
        const uint32_t k = (Q >= c0) ? Q - c0 : Q + 30u - c0;
        const uint64_t b64 = (d + (uint64_t) k * p) / 30u + (uint64_t) r * p;
        if (b64 < seg_bytes) {
          const uint32_t b = (uint32_t) b64;
          const uint32_t bit = residue_to_bit((Q * (p % 30u)) % 30u);
          const uint32_t mask = ~(1u << (bit + 8u * (b & 3u)));
          for (uint32_t w = b >> 2; w < nwords; w += p) atomicAnd(&sieve32[w], mask);
        }
      }
    }
    // other base primes: one thread per prime, sequential wheel walk
    for (uint32_t i = a.n_base_small + tid; i < a.n_base; i += BLOCK) {
      const uint32_t p = a.base[i];
      uint64_t d; uint32_t c0;
      first_multiple(segLow, p, a.base_recip[i], d, c0);
      if (d >= span) continue;
      uint32_t j = first_class_ge(c0);
      const uint64_t off = d + (uint64_t) (cofactor_class(j) - c0) * p;
      if (off >= span) continue;
      uint32_t b = (uint32_t) off / 30u;
      const uint32_t pdiv30 = p / 30u;
      const uint32_t cls = residue_to_bit(p - 30u * pdiv30);
      const uint32_t bits = wheel_tab[2 * cls], corr = wheel_tab[2 * cls + 1];
      while (b < seg_bytes) {
        const uint32_t sh = 3u * j;
        atomicAnd(&sieve32[b >> 2], ~(1u << (((bits >> sh) & 7u) + 8u * (b & 3u))));
        b += pdiv30 * ((kGapPacked >> sh) & 7u) + ((corr >> sh) & 7u);
        j = (j + 1u) & 7u;
      }
    }
    __syncthreads();

    // mask to [lo, hi]; warp w owns the contiguous words [w*per, (w+1)*per)
    const uint64_t rhi = (a.hi >= segLow) ? a.hi - segLow : 0;
    const uint64_t rlo = (a.lo > segLow) ? a.lo - segLow : 0;
    const uint32_t per = nwords / NWARPS;
    uint32_t cnt = 0;
    for (uint32_t x = lane; x < per; x += 32) {
      const uint32_t wi = warp * per + x;
      uint32_t m = 0;
#pragma unroll
      for (int by = 0; by < 4; by++) m |= byte_keep(30ull * (4ull * wi + by), rlo, rhi) << (8 * by);
      const uint32_t v = sieve32[wi] & m;
      sieve32[wi] = v;
      cnt += __popc(v);
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0) wtot[warp] = cnt;
    __syncthreads();

    if (a.pass == 0) {
      if (tid == 0) {
        uint32_t t = 0;
        for (uint32_t w = 0; w < NWARPS; w++) t += wtot[w];
        a.seg_counts[s] = t;
      }
    } else {
      uint64_t pos = a.seg_offsets[s];
      for (uint32_t w = 0; w < warp; w++) pos += wtot[w];
      for (uint32_t x0 = 0; x0 < per; x0 += 32) {
        const uint32_t x = x0 + lane;
        const uint32_t wi = warp * per + x;
        const uint32_t v = (x < per) ? sieve32[wi] : 0u;
        const uint32_t c = __popc(v);
        uint32_t incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= (uint32_t) o) incl += t;
        }
        uint64_t q = pos + incl - c;
        uint32_t bitsleft = v;
        while (bitsleft) {
          const uint32_t bpos = __ffs(bitsleft) - 1u;
          bitsleft &= bitsleft - 1u;
          const uint32_t byte = 4u * wi + (bpos >> 3);
          const uint32_t bv = bpos & 7u;
          const uint32_t offv = (bv == 0) ? 7u : (bv == 1) ? 11u : (bv == 2) ? 13u : (bv == 3) ? 17u
                              : (bv == 4) ? 19u : (bv == 5) ? 23u : (bv == 6) ? 29u : 31u;
          a.out[q++] = (uint32_t) (segLow + 30ull * byte + offv);
        }
        pos += __shfl_sync(0xffffffffu, incl, 31);
      }
    }
    __syncthreads();
  }
}

} // namespace psg
