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
// it counts the entries of each of the window's segments in shared memory,
// so no global atomics are needed. A list has a fixed capacity (its expected length plus a generous
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
  uint32_t seg_magic;         // floor(2^32 / seg_bytes) + 1 (segment index)
  uint32_t entry_bits;        // bits of an entry (byte << 3 | bit); segment above
  const uint32_t* primes;
  const uint64_t* recip;
  const uint32_t* chunk_begin;  // [CTAs + 1] prime index range per CTA
  uint32_t list_base;         // list of CTA 0 (the sweep kernel's lists come first)
  uint32_t num_lists;         // lists per segment, all kernels
  const uint32_t* list_off;   // [num_lists] entry offset inside a segment region
  const uint32_t* list_cap;   // [num_lists] capacity
  uint64_t seg_stride;        // entries per segment region
  uint32_t* entries;
  uint32_t* counts;           // [win_segments][num_lists]
  uint32_t* overflow;         // set to 1 if any list overflowed
  unsigned long long* entry_total;  // running total of entries written
};

// Byte index b (< 2^31) -> (segment, byte in segment) without a divide:
// with magic = floor(2^32/d) + 1 > 2^32/d, mulhi(b, magic) is floor(b/d) or
// one more (the excess b*(magic - 2^32/d)/2^32 < b/2^32 < 1/2), so one
// correction step suffices.
__device__ __forceinline__ uint32_t seg_of(uint32_t b, uint32_t seg_bytes, uint32_t magic, uint32_t& bo) {
  uint32_t sg = __umulhi(b, magic);
  int32_t r = (int32_t) (b - sg * seg_bytes);
  if (r < 0) { r += (int32_t) seg_bytes; sg--; }
  bo = (uint32_t) r;
  return sg;
}

// Tile-sorted prime-major fill. A warp takes 4 big primes at a time; lane
// (g = lane>>3, c = lane&7) walks the multiples of prime g whose cofactor is
// in wheel class c -- one arithmetic progression of stride p bytes with a
// fixed bit -- emitting one entry per step. Each step the active lanes
// append their entries to a shared-memory tile at consecutive slots (one
// shared atomicAdd per warp), and each entry's rank within its segment comes
// from a shared atomicAdd on that segment's histogram. When the tile is
// full, the CTA scans the histogram into segment offsets, scatters the tile
// into segment order and writes every segment's run to the CTA's list for
// that segment as one contiguous, coalesced run. HBM therefore sees whole
// sectors instead of scattered 4-byte writes.
constexpr uint32_t kFillSteps = 16;             // emit steps per warp and tile
template <int BLOCK> struct FillTile {
  static constexpr uint32_t kTile = BLOCK * kFillSteps;   // one entry per lane and step
};

// smem: hist[W] off[W] gcnt[W] | warp sums [32] | tile_n [32] |
//       tile_e[kTile] (packed) tile_r[kTile] (u16 rank) sorted[kTile]
template <int BLOCK>
constexpr size_t fill_smem_bytes(uint32_t W) {
  return (3ull * W + 64) * 4 + (size_t) FillTile<BLOCK>::kTile * (4 + 2 + 4);
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1)
bucket_fill_kernel(const __grid_constant__ BucketArgs a)
{
  constexpr uint32_t kTile = FillTile<BLOCK>::kTile;
  constexpr uint32_t NWARPS = BLOCK / 32;
  extern __shared__ uint32_t smem_u32[];
  const uint32_t W = a.win_segments;
  uint32_t* const hist = smem_u32;               // [W] entries of the tile per segment
  uint32_t* const off = hist + W;                // [W] exclusive scan of hist
  uint32_t* const gcnt = off + W;                // [W] entries already in HBM
  uint32_t* const wsum = gcnt + W;               // [32] scan scratch
  uint32_t* const tile_n = wsum + 32;            // [1]
  uint32_t* const tile_e = tile_n + 32;          // [kTile] sg << entry_bits | entry
  uint16_t* const tile_r = reinterpret_cast<uint16_t*>(tile_e + kTile);  // [kTile]
  uint32_t* const sorted = reinterpret_cast<uint32_t*>(tile_r + kTile);  // [kTile]
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  for (uint32_t i = tid; i < 3 * W + 64; i += BLOCK) smem_u32[i] = 0;
  __syncthreads();

  const uint32_t list = a.list_base + blockIdx.x;
  const uint32_t cap = a.list_cap[list];
  uint32_t* const out = a.entries + a.list_off[list];
  const uint32_t win_bytes = W * a.seg_bytes;       // < 2^31 (host-checked)
  const uint32_t seg_bytes = a.seg_bytes;
  const uint32_t magic = a.seg_magic;
  const uint64_t stride = a.seg_stride;
  const uint32_t lo = a.chunk_begin[blockIdx.x];
  const uint32_t hi = a.chunk_begin[blockIdx.x + 1];
  const uint32_t ebits = a.entry_bits;             // entry = byte << 3 | bit
  const uint32_t emask = (1u << ebits) - 1u;
  const uint32_t lanemask_lt = (1u << lane) - 1u;
  const uint32_t g = lane >> 3;
  const uint32_t Q = cofactor_class(lane & 7u);
  constexpr uint32_t kDone = 0xffffffffu;

  uint32_t b = kDone, p = 0, ebit = 0;    // this lane's progression
  uint32_t group = warp;                  // next group of 4 primes of this warp
  bool warp_done = false;
  // prefetched prime of the next group (its loads overlap the current walk)
  uint32_t p_nx = 0;
  uint64_t r_nx = 0;
  {
    const uint32_t idx = lo + group * 4u + g;
    if (idx < hi) { p_nx = a.primes[idx]; r_nx = a.recip[idx]; }
  }

  for (;;) {
    // ---- 1. generate: kFillSteps steps per warp into the tile
    for (uint32_t step = 0; step < kFillSteps && !warp_done; step++) {
      uint32_t act = __ballot_sync(0xffffffffu, b != kDone);
      if (act == 0) {
        const uint32_t base = lo + group * 4u;
        if (base >= hi) { warp_done = true; break; }
        group += NWARPS;
        const uint32_t idx = base + g;
        const uint32_t p_cur = p_nx;
        const uint64_t r_cur = r_nx;
        {
          const uint32_t nidx = lo + group * 4u + g;
          if (nidx < hi) { p_nx = a.primes[nidx]; r_nx = a.recip[nidx]; }
        }
        if (idx < hi) {
          p = p_cur;
          uint64_t d; uint32_t c0;
          first_multiple(a.win_low, p, r_cur, d, c0);
          const uint32_t k = (Q >= c0) ? Q - c0 : Q + 30u - c0;
          const uint64_t b64 = (d + (uint64_t) k * p) / 30u;   // byte index in window
          if (b64 < win_bytes) b = (uint32_t) b64;
          ebit = residue_to_bit((Q * (p % 30u)) % 30u);
        }
        act = __ballot_sync(0xffffffffu, b != kDone);
        if (act == 0) continue;
      }
      uint32_t slot = 0;
      if (lane == 0) slot = atomicAdd(tile_n, (uint32_t) __popc(act));
      slot = __shfl_sync(0xffffffffu, slot, 0) + __popc(act & lanemask_lt);
      if (b != kDone) {
        uint32_t bo;
        const uint32_t sg = seg_of(b, seg_bytes, magic, bo);
        const uint32_t rank = atomicAdd(&hist[sg], 1u);
        tile_e[slot] = (sg << ebits) | (bo << 3) | ebit;
        tile_r[slot] = (uint16_t) rank;
        // p >= win_bytes - b: no further hit (also keeps b + p from wrapping)
        b = (p >= win_bytes - b) ? kDone : b + p;
      }
    }
    const int more = __syncthreads_or(warp_done ? 0 : 1);
    const uint32_t n = *tile_n;

    // ---- 2. exclusive scan of the histogram -> segment offsets in the tile
    {
      constexpr uint32_t PER = 8;                   // W <= BLOCK * PER (host-checked)
      uint32_t v[PER], sum = 0;
#pragma unroll
      for (uint32_t q = 0; q < PER; q++) {
        const uint32_t i = tid * PER + q;
        v[q] = (i < W) ? hist[i] : 0u;
        sum += v[q];
      }
      uint32_t incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t) o) incl += t;
      }
      if (lane == 31) wsum[warp] = incl;
      __syncthreads();
      if (warp == 0) {
        uint32_t w = (lane < NWARPS) ? wsum[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
          if (lane >= (uint32_t) o) wi += t;
        }
        if (lane < NWARPS) wsum[lane] = wi - w;      // exclusive warp offsets
      }
      __syncthreads();
      uint32_t run = wsum[warp] + incl - sum;
#pragma unroll
      for (uint32_t q = 0; q < PER; q++) {
        const uint32_t i = tid * PER + q;
        if (i < W) off[i] = run;
        run += v[q];
      }
    }
    __syncthreads();

    // ---- 3. scatter into segment order
    for (uint32_t i = tid; i < n; i += BLOCK) {
      const uint32_t e = tile_e[i];
      sorted[off[e >> ebits] + tile_r[i]] = e;
    }
    __syncthreads();

    // ---- 4. write each segment's run contiguously to its HBM list
    for (uint32_t i = tid; i < n; i += BLOCK) {
      const uint32_t e = sorted[i];
      const uint32_t sg = e >> ebits;
      const uint32_t pos = gcnt[sg] + (i - off[sg]);
      if (pos < cap) out[(uint64_t) sg * stride + pos] = e & emask;
    }
    __syncthreads();
    for (uint32_t i = tid; i < W; i += BLOCK) {
      gcnt[i] += hist[i];
      hist[i] = 0;
    }
    if (tid == 0) *tile_n = 0;
    __syncthreads();
    if (!more) break;
  }

  uint32_t written = 0;
  for (uint32_t sgi = tid; sgi < W; sgi += BLOCK) {
    uint32_t c = gcnt[sgi];
    if (c > cap) { atomicOr(a.overflow, 1u); c = cap; }
    a.counts[(uint64_t) sgi * a.num_lists + list] = c;
    written += c;
  }
  for (int o = 16; o > 0; o >>= 1) written += __shfl_xor_sync(0xffffffffu, written, o);
  if (lane == 0 && written) atomicAdd(a.entry_total, (unsigned long long) written);
}

} // namespace psg
