// sieve_kernel.cuh -- the segment sieve kernel (sm_100a).
//
// One CTA sieves one wheel-30 segment at a time in shared memory and walks a
// contiguous stripe of segments (persistent grid), so per-prime state carries
// from one segment to the next instead of being recomputed. Per segment:
//   1. pre-sieve : AND of the pre-sieve patterns, 16 bytes per thread per
//                  step, read as aligned 128-bit loads from 16 pre-shifted
//                  copies of each pattern (L2-resident), stored with
//                  conflict-free 128-bit shared stores.
//   2. small     : warp-cooperative cross-off. One warp per prime (its
//                  remainder segLow mod p carried in a register); lane
//                  (j = lane&7, r = lane>>3) walks the multiples whose
//                  cofactor is in class kCofactor[j] (mod 30), every 4th
//                  one starting at phase r. Those multiples are p bytes
//                  apart, so the lane strides 4p bytes = p words and its
//                  bit (and byte-in-word) never changes: the inner loop is
//                  one shared atomicAnd per crossing.
//   3. medium    : one thread per prime, sequential wheel walk; each prime's
//                  (byte position, wheel index) is kept in shared memory
//                  between the segments of the stripe (primesieve's EratSmall/
//                  EratMedium carry the same pair per sieving prime).
//   4. big       : crossings streamed from the per-segment bucket lists
//                  that the bucket kernel wrote to HBM (4-byte entries).
//   5. count     : edge masking, __popc over the word and over shifted ANDs
//                  for the k-tuplet start masks, warp-shuffle reduction,
//                  one 64-bit atomicAdd per warp and kind at kernel end.
//
// Reference counterpart: ps_count, src/gpu/cuda/sieve.cu:157-320 (one
// block per segment, shared-memory sieve, smem atomicAnd cross-off, byte
// LUT count and a tree reduction into one u64 per segment).
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>
#include "wheel.hpp"

namespace psg {

// The dynamic shared-memory limit of a kernel is one attribute for the whole
// process, not per context: each context raises it to what the device allows
// (less the kernel's static shared memory) instead of setting its own size,
// so that a context with a smaller layout never lowers it under one with a
// larger layout.
template <typename Kernel>
inline cudaError_t allow_max_dynamic_smem(Kernel kernel, int device) {
  int optin = 0;
  cudaError_t e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  cudaFuncAttributes fa;
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kernel);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int) fa.sharedSizeBytes);
  return e;
}

constexpr int kMaxPresieveTables = 6;
constexpr int kMaxPresievePrimes = 24;

struct SieveArgs {
  uint64_t seg_low0;          // value base of segment 0 (multiple of 30)
  uint64_t lo, hi;            // inclusive range, lo >= 7
  uint64_t num_segments;
  uint32_t seg_bytes;         // multiple of 16
  uint32_t num_tables;
  const uint8_t* pat_base[kMaxPresieveTables];  // 16 shifted copies each
  uint32_t pat_period[kMaxPresieveTables];      // bytes
  uint32_t pat_stride[kMaxPresieveTables];      // bytes per shifted copy
  uint64_t pat_rcp[kMaxPresieveTables];         // floor((2^64-1)/period)
  uint32_t presieve_primes[kMaxPresievePrimes]; // restored in segment 0/1
  uint32_t num_presieve_primes;
  uint32_t presieve_max;
  const uint32_t* primes;     // sieving primes (> presieve_max), ascending
  const uint64_t* recip;      // floor((2^64-1)/p) per prime
  uint32_t n_small;           // primes[0, n_small): warp-cooperative
  uint32_t n_primes;          // primes[n_small, n_primes): thread per prime
                              // (their state fits the shared-memory area)
  uint32_t n_direct;          // primes[n_primes, n_direct): thread per prime,
                              // first multiple recomputed every segment
  // big primes via buckets (num_bucket_lists == 0: none)
  const uint32_t* bucket_entries;   // [segment][seg_stride] entries
  const uint32_t* bucket_counts;    // [segment][list] entries from the list's start
  const uint32_t* bucket_spill;     // [segment][list] entries at the list's top
  const uint32_t* bucket_list_off;  // [list] offset inside a segment region
  const uint32_t* bucket_list_cap;  // [list] capacity
  uint64_t bucket_seg_stride;       // entries per segment region
  uint32_t num_bucket_lists;        // lists per segment (0: no big primes)
  uint32_t wheel_tab[16];           // per class: bits, corr (wheel walk)
  uint32_t kinds;
  unsigned long long* counts;       // [6]
  uint8_t* bitmap_out;              // optional: the sieved segments of this launch
                                    // (edges masked), seg_bytes per segment
};

// x mod p for p < 2^32 with a precomputed rcp = floor((2^64-1)/p).
// q_est = mulhi(x, rcp) is at most 2 below floor(x/p) (Granlund-Montgomery
// style reciprocal estimate), so at most two corrections are needed.
__device__ __forceinline__ uint32_t mod_recip(uint64_t x, uint32_t p, uint64_t rcp) {
  uint64_t q = __umul64hi(x, rcp);
  uint64_t r = x - q * (uint64_t) p;
  if (r >= p) r -= p;
  if (r >= p) r -= p;
  return (uint32_t) r;
}

// Offset d (relative to x0 = segLow + 7) of the first multiple of p that is
// >= x0 and >= p*p, and the residue (mod 30) of its cofactor.
// Reference: first multiple > segLow + 6 with cofactor >= p,
// src/gpu/cuda/sieve.cu:69-99 and src/Wheel.hpp:50-89.
__device__ __forceinline__ void first_multiple(uint64_t segLow, uint32_t p, uint64_t rcp,
                                               uint64_t& d, uint32_t& c0) {
  const uint64_t x0 = segLow + 7;
  const uint64_t pp = (uint64_t) p * p;
  const uint32_t pm = p % 30u;
  if (x0 <= pp) {
    d = pp - x0;
    c0 = pm;
  } else {
    uint32_t r = mod_recip(x0, p, rcp);
    uint32_t dd = r ? p - r : 0u;
    d = dd;
    // x0 + d = p * c  ->  c == (7 + d) * p^-1 (mod 30)
    c0 = (((7u + dd % 30u) % 30u) * inverse_mod30(pm)) % 30u;
  }
}

__device__ __forceinline__ uint32_t cofactor_class(uint32_t j) {
  // kCofactor[j] = {1,7,11,13,17,19,23,29}[j], 5 bits each
  const uint64_t packed = 1ull | (7ull << 5) | (11ull << 10) | (13ull << 15) |
                          (17ull << 20) | (19ull << 25) | (23ull << 30) | (29ull << 35);
  return (uint32_t) ((packed >> (5 * j)) & 31u);
}

// Keep-mask of the byte whose values are base + {7..31} for the inclusive
// window [rlo, rhi] (all relative to segLow; no wrap-around).
__device__ __forceinline__ uint32_t byte_keep(uint64_t base, uint64_t rlo, uint64_t rhi) {
  uint32_t m = 0;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const uint32_t off = (j == 0) ? 7u : (j == 1) ? 11u : (j == 2) ? 13u : (j == 3) ? 17u
                       : (j == 4) ? 19u : (j == 5) ? 23u : (j == 6) ? 29u : 31u;
    const uint64_t v = base + off;
    if (v >= rlo && v <= rhi) m |= 1u << j;
  }
  return m;
}

template <bool ALL_KINDS>
__device__ __forceinline__ void count_word(uint32_t w, uint32_t (&c)[6]) {
  c[0] += __popc(w);
  if (ALL_KINDS) {
    const uint32_t t2 = w & (w >> 1);
    c[1] += __popc(t2 & kTwinStart);
    const uint32_t t3 = t2 & (w >> 2);
    c[2] += __popc(t3 & kTripStart);
    const uint32_t t4 = t3 & (w >> 3);
    c[3] += __popc(t4 & kQuadStart);
    const uint32_t t5 = t4 & (w >> 4);
    c[4] += __popc(t5 & kQuintStart);
    const uint32_t t6 = t5 & (w >> 5);
    c[5] += __popc(t6 & kSextStart);
  }
}

// ---- per-segment phases ---------------------------------------------------
// Shared by the range kernel below and the batch kernel (batch_kernel.cuh).
// `a` carries what is common to a launch (tables, sieving primes, segment
// size); prime-tier bounds, segment base and range edges are arguments.

constexpr int kSmallRegs = 2;                // small primes per lane kept in registers
constexpr uint32_t kMedFar = 0xffffffffu;  // medium state: next multiple not representable yet

// 1. pre-sieve: AND of the pattern tables, 16 bytes per thread per step.
template <int BLOCK>
__device__ __forceinline__ void phase_presieve(const SieveArgs& a, uint4* smem4, uint64_t segLow, uint32_t tid) {
  const uint32_t nchunks = a.seg_bytes >> 4;
  const uint64_t g0 = segLow / 30u;   // global byte index of byte 0
  uint32_t phase[kMaxPresieveTables], step[kMaxPresieveTables];
#pragma unroll
  for (int t = 0; t < kMaxPresieveTables; t++) {
    if (t < (int) a.num_tables) {
      const uint32_t P = a.pat_period[t];
      phase[t] = mod_recip(g0 + 16ull * tid, P, a.pat_rcp[t]);
      step[t] = (16u * BLOCK) % P;
    }
  }
  for (uint32_t c = tid; c < nchunks; c += BLOCK) {
    uint4 v = make_uint4(~0u, ~0u, ~0u, ~0u);
#pragma unroll
    for (int t = 0; t < kMaxPresieveTables; t++) {
      if (t < (int) a.num_tables) {
        const uint32_t ph = phase[t];
        const uint32_t k = ph & 15u;
        const uint4 pv = __ldg(reinterpret_cast<const uint4*>(
            a.pat_base[t] + (size_t) k * a.pat_stride[t] + (ph - k)));
        v.x &= pv.x; v.y &= pv.y; v.z &= pv.z; v.w &= pv.w;
        uint32_t np = ph + step[t];
        phase[t] = (np >= a.pat_period[t]) ? np - a.pat_period[t] : np;
      }
    }
    if (c == 0 && segLow <= a.presieve_max) {
      // The patterns also cleared the pre-sieve primes themselves;
      // put them back (reference: restore bytes, GpuTables.cpp:108-127).
      uint32_t w4[4] = { v.x, v.y, v.z, v.w };
      for (uint32_t i = 0; i < a.num_presieve_primes; i++) {
        const uint64_t q = a.presieve_primes[i];
        if (q < segLow + 7) continue;
        const uint64_t rel = q - segLow - 7;      // < 16*30
        const uint32_t byte = (uint32_t) (rel / 30u);
        if (byte >= 16) continue;
        const uint32_t bit = residue_to_bit((uint32_t) (q % 30u));
        w4[byte >> 2] |= 1u << (8 * (byte & 3) + bit);
      }
      v = make_uint4(w4[0], w4[1], w4[2], w4[3]);
    }
    smem4[c] = v;
  }
}

// Small primes of this warp, register resident: p, r = (segLow+7) mod p of
// the current segment, and span mod p to advance r by one segment.
template <int BLOCK>
__device__ __forceinline__ void small_setup(const SieveArgs& a, uint32_t n_small, uint64_t x0, bool active,
                                            uint32_t warp, uint32_t lane, uint32_t (&sp)[kSmallRegs],
                                            uint32_t (&sr)[kSmallRegs], uint32_t (&sdl)[kSmallRegs]) {
  constexpr uint32_t NWARPS = BLOCK / 32;
  const uint64_t span = (uint64_t) a.seg_bytes * 30u;
#pragma unroll
  for (int m = 0; m < kSmallRegs; m++) {
    const uint32_t idx = warp + NWARPS * (lane + 32u * m);
    sp[m] = 1; sr[m] = 0; sdl[m] = 0;
    if (idx < n_small && active) {
      const uint32_t p = a.primes[idx];
      sp[m] = p;
      sr[m] = mod_recip(x0, p, a.recip[idx]);
      sdl[m] = (uint32_t) (span % p);
    }
  }
}

__device__ __forceinline__ void small_advance(uint32_t (&sp)[kSmallRegs], uint32_t (&sr)[kSmallRegs],
                                              const uint32_t (&sdl)[kSmallRegs]) {
#pragma unroll
  for (int m = 0; m < kSmallRegs; m++) {
    const uint32_t nr = sr[m] + sdl[m];
    sr[m] = (nr >= sp[m]) ? nr - sp[m] : nr;
  }
}

// The progression w0, w0 + p, ... (< nwords) of one lane of a small prime.
// The 32 lanes of a warp step by the same p words, so the bank pattern of
// their first crossings repeats at every step; for primes below kSkewBelow
// (over 64 steps per lane) each lane therefore starts delta = (lane - w0)
// p^-1 (mod 32) steps in, where the word is == lane (mod 32) -- distinct
// banks for all 32 lanes, step after step -- and crosses the skipped start
// afterwards. (For larger primes the up to 31 extra steps of the warp's
// longest lane cost more than the conflicts: skewing all small primes,
// those below 1024 and those below 512 measured 22.1, 21.4 and 20.9 ms of
// sieve per pass on [1e15, 1e15+1e11], 21.6 unskewed.) p is odd,
// so p^-1 mod 32 exists: p (2 - p p), one Newton step from p, the inverse
// mod 8 of any odd p.
constexpr uint32_t kSkewBelow = 512;
__device__ __forceinline__ void small_walk(uint32_t* sieve32, uint32_t w0, uint32_t p, uint32_t nwords,
                                           uint32_t mask, uint32_t lane) {
  const uint32_t pinv = p * (2u - p * p);
  const uint32_t ws = w0 + (((lane - w0) * pinv) & 31u) * p;
  const uint32_t start = (p < kSkewBelow && ws < nwords) ? ws : w0;
  for (uint32_t w = start; w < nwords; w += p)
    atomicAnd(&sieve32[w], mask);
  for (uint32_t w = w0; w < start; w += p)
    atomicAnd(&sieve32[w], mask);
}

// 2. small primes: one warp per prime; lane (j = lane&7, r = lane>>3) walks
// the multiples with cofactor class j, every 4th from phase r (stride p words).
template <int BLOCK>
__device__ __forceinline__ void phase_small(const SieveArgs& a, uint32_t n_small, uint32_t* sieve32, uint64_t segLow,
                                            uint32_t warp, uint32_t lane, const uint32_t (&sp)[kSmallRegs],
                                            const uint32_t (&sr)[kSmallRegs]) {
  constexpr uint32_t NWARPS = BLOCK / 32;
  const uint32_t seg_bytes = a.seg_bytes;
  const uint32_t nwords = seg_bytes >> 2;
  const uint64_t span = (uint64_t) seg_bytes * 30u;
  const uint32_t j = lane & 7u;
  const uint32_t r = lane >> 3;
  const uint32_t Q = cofactor_class(j);
  const uint64_t x0 = segLow + 7;
#pragma unroll
  for (int m = 0; m < kSmallRegs; m++) {
    const uint32_t tbase = 32u * m;
    if (warp + NWARPS * tbase >= n_small) break;
    for (uint32_t l = 0; l < 32; l++) {
      const uint32_t idx = warp + NWARPS * (tbase + l);
      if (idx >= n_small) break;
      const uint32_t p = __shfl_sync(0xffffffffu, sp[m], l);
      const uint32_t rem = __shfl_sync(0xffffffffu, sr[m], l);
      const uint32_t pm = p % 30u;
      const uint64_t pp = (uint64_t) p * p;
      uint32_t b;
      if (x0 <= pp) {                   // the segment starts before p^2
        const uint64_t d = pp - x0;
        if (d >= span) continue;
        const uint32_t k = (Q >= pm) ? Q - pm : Q + 30u - pm;
        const uint64_t b64 = (d + (uint64_t) k * p) / 30u + (uint64_t) r * p;
        if (b64 >= seg_bytes) continue;
        b = (uint32_t) b64;
      } else {                          // register-resident primes (the first 2048) are
                                        // below 2^15: d + k p < 2^20, all in 32 bits
        const uint32_t dd = rem ? p - rem : 0u;
        const uint32_t c0 = (((7u + dd % 30u) % 30u) * inverse_mod30(pm)) % 30u;
        const uint32_t k = (Q >= c0) ? Q - c0 : Q + 30u - c0;
        b = (dd + k * p) / 30u + r * p;
      }
      if (b < seg_bytes) {
        const uint32_t bit = residue_to_bit((Q * pm) % 30u);
        const uint32_t mask = ~(1u << (bit + 8u * (b & 3u)));
        small_walk(sieve32, b >> 2, p, nwords, mask, lane);
      }
    }
  }
  // small primes beyond the register-resident ones
  for (uint32_t idx = warp + NWARPS * 32u * kSmallRegs; idx < n_small; idx += NWARPS) {
    const uint32_t p = a.primes[idx];
    uint64_t d; uint32_t c0;
    first_multiple(segLow, p, a.recip[idx], d, c0);
    if (d >= span) continue;
    const uint32_t pm = p % 30u;
    const uint32_t k = (Q >= c0) ? Q - c0 : Q + 30u - c0;
    const uint64_t b64 = (d + (uint64_t) k * p) / 30u + (uint64_t) r * p;
    if (b64 < seg_bytes) {
      const uint32_t b = (uint32_t) b64;
      const uint32_t bit = residue_to_bit((Q * pm) % 30u);
      const uint32_t mask = ~(1u << (bit + 8u * (b & 3u)));
      small_walk(sieve32, b >> 2, p, nwords, mask, lane);
    }
  }
}

// Medium primes primes[first, first + n): state (byte << 3 | wheel index)
// relative to the current segment, or kMedFar when the first multiple is
// still far away.
__device__ __forceinline__ uint32_t medium_state(uint64_t segLow, uint32_t p, uint64_t rcp) {
  uint64_t d; uint32_t c0;
  first_multiple(segLow, p, rcp, d, c0);
  const uint32_t j = first_class_ge(c0);
  const uint64_t b = (d + (uint64_t) (cofactor_class(j) - c0) * p) / 30u;
  return (b < (1ull << 29) - 1) ? (uint32_t) (b << 3) | j : kMedFar;
}

template <int BLOCK>
__device__ __forceinline__ void medium_setup(const SieveArgs& a, uint32_t first, uint32_t n, uint32_t* mstate,
                                             uint64_t segLow, uint32_t tid) {
  for (uint32_t i = tid; i < n; i += BLOCK)
    mstate[i] = medium_state(segLow, a.primes[first + i], a.recip[first + i]);
}

// One prime's sequential wheel walk from byte b (wheel index j) to the end
// of the segment; returns the byte past the segment where it stopped. Eight
// consecutive multiples (one wheel rotation) span exactly p bytes and end
// at the same wheel index, so while a whole rotation fits in the segment the
// walk applies the 8 crossings at offsets computed once, with masks that only
// rotate from one rotation to the next, and no per-step table lookups or
// bound checks. PARTIAL (medium primes, carried state): the last, partial
// rotation uses the same offsets with a bound check each; otherwise (direct
// primes, a few crossings per segment, for which the offsets do not pay) the
// rest goes step by step.
template <bool PARTIAL>
__device__ __forceinline__ uint32_t wheel_walk(uint32_t* sieve32, const uint32_t* wheel_tab, uint32_t p,
                                               uint32_t b, uint32_t& j, uint32_t seg_bytes) {
  const uint32_t pdiv30 = p / 30u;
  const uint32_t cls = residue_to_bit(p - 30u * pdiv30);
  const uint32_t bits = wheel_tab[2 * cls];
  const uint32_t corr = wheel_tab[2 * cls + 1];
  if (PARTIAL || p <= seg_bytes - b) {
    uint32_t off[8];                 // off[0] = 0
    uint32_t bitp = 0;               // bit of multiple k in bits 3k..3k+2
    uint32_t o = 0, jj = j;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const uint32_t sh = 3u * jj;
      off[k] = o;
      bitp |= ((bits >> sh) & 7u) << (3 * k);
      o += pdiv30 * ((kGapPacked >> sh) & 7u) + ((corr >> sh) & 7u);
      jj = (jj + 1u) & 7u;
    }
    // the cleared bit of multiple k moves by 8 (p mod 4) bits (mod 32) from
    // one rotation to the next: its inverted mask rotates
    uint32_t m[8];
#pragma unroll
    for (int k = 0; k < 8; k++) m[k] = ~(1u << (((bitp >> (3 * k)) & 7u) + 8u * ((b + off[k]) & 3u)));
    const uint32_t rot = 8u * (p & 3u);
    while (p <= seg_bytes - b) {     // b <= seg_bytes here
#pragma unroll
      for (int k = 0; k < 8; k++) {
        atomicAnd(&sieve32[(b + off[k]) >> 2], m[k]);
        m[k] = __funnelshift_l(m[k], m[k], rot);
      }
      b += p;
    }
    if constexpr (PARTIAL) {
      // the crossings of the last, partial rotation; the first multiple past
      // the segment is where the walk stops (the next rotation's first one,
      // of the same wheel index, when all 8 fit)
      uint32_t nb = b + p, jn = 0;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const uint32_t bk = b + off[k];
        if (bk >= seg_bytes) { nb = bk; jn = (uint32_t) k; break; }
        atomicAnd(&sieve32[bk >> 2], m[k]);
      }
      j = (j + jn) & 7u;
      return nb;
    }
  }
  if constexpr (!PARTIAL) {
    while (b < seg_bytes) {
      const uint32_t sh = 3u * j;
      atomicAnd(&sieve32[b >> 2], ~(1u << (((bits >> sh) & 7u) + 8u * (b & 3u))));
      b += pdiv30 * ((kGapPacked >> sh) & 7u) + ((corr >> sh) & 7u);
      j = (j + 1u) & 7u;
    }
  }
  return b;
}

// 3. medium primes: one thread per prime, carried wheel walk.
template <int BLOCK>
__device__ __forceinline__ void phase_medium(const SieveArgs& a, uint32_t first, uint32_t n, uint32_t* mstate,
                                             uint32_t* sieve32, const uint32_t* wheel_tab, uint64_t segLow,
                                             uint32_t tid) {
  const uint32_t seg_bytes = a.seg_bytes;
  // the primes of the next kMP iterations are loaded ahead (L2 latency)
  constexpr uint32_t kMP = 2;
  uint32_t pq[kMP];
#pragma unroll
  for (uint32_t u = 0; u < kMP; u++) pq[u] = (tid + u * BLOCK < n) ? a.primes[first + tid + u * BLOCK] : 0u;
  for (uint32_t i = tid; i < n; i += BLOCK) {
    const uint32_t inext = i + kMP * BLOCK;
    const uint32_t pn = (inext < n) ? a.primes[first + inext] : 0u;
    const uint32_t p = pq[0];
#pragma unroll
    for (uint32_t u = 0; u + 1 < kMP; u++) pq[u] = pq[u + 1];
    pq[kMP - 1] = pn;
    uint32_t st = mstate[i];
    if (st == kMedFar) st = medium_state(segLow, p, a.recip[first + i]);
    if (st != kMedFar) {
      uint32_t b = st >> 3;
      uint32_t j = st & 7u;
      // a prime above the segment length has under one rotation per
      // segment: the offsets do not pay for it, the step walk is cheaper
      if (b < seg_bytes)
        b = (p <= seg_bytes) ? wheel_walk<true>(sieve32, wheel_tab, p, b, j, seg_bytes)
                             : wheel_walk<false>(sieve32, wheel_tab, p, b, j, seg_bytes);
      const uint32_t nb = b - seg_bytes;
      st = (nb < (1u << 29) - 1u) ? (nb << 3) | j : kMedFar;
    }
    mstate[i] = st;
  }
}

// 3b. direct primes primes[first, end): one thread per prime, no carried
// state. Beyond what the shared state holds, a prime that still hits most
// segments is cheaper to locate again (one reciprocal multiply) than to
// route through the bucket lists.
template <int BLOCK>
__device__ __forceinline__ void phase_direct(const SieveArgs& a, uint32_t first, uint32_t end, uint32_t* sieve32,
                                             const uint32_t* wheel_tab, uint64_t segLow, uint32_t tid) {
  constexpr uint32_t kDU = 4;         // primes in flight per thread
  const uint32_t seg_bytes = a.seg_bytes;
  const uint64_t span = (uint64_t) seg_bytes * 30u;
  for (uint32_t i0 = first + tid; i0 < end; i0 += kDU * BLOCK) {
    uint32_t pv[kDU];
    uint64_t rv[kDU];
#pragma unroll
    for (uint32_t u = 0; u < kDU; u++) {
      const uint32_t i = i0 + u * BLOCK;
      pv[u] = (i < end) ? a.primes[i] : 0u;
      rv[u] = (i < end) ? a.recip[i] : 0ull;
    }
#pragma unroll
    for (uint32_t u = 0; u < kDU; u++) {
      const uint32_t p = pv[u];
      if (p == 0) continue;
      uint64_t d; uint32_t c0;
      first_multiple(segLow, p, rv[u], d, c0);
      if (d >= span) continue;
      uint32_t j = first_class_ge(c0);
      const uint32_t b = (uint32_t) ((d + (uint64_t) (cofactor_class(j) - c0) * p) / 30u);
      if (b >= seg_bytes) continue;
      wheel_walk<false>(sieve32, wheel_tab, p, b, j, seg_bytes);
    }
  }
}

// Bulk prefetch of [p, p + bytes) into L2 (TMA engine; p 16-byte aligned,
// bytes a multiple of 16). A hint: no completion to wait for.
__device__ __forceinline__ void prefetch_l2_bulk(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" :: "l"(p), "r"(bytes) : "memory");
}

// 4. big primes: the bucket lists of launch segment s. Warps take lists from
// a shared counter (lists differ in length); each lane applies 4 entries per
// 16-byte load (lists start 16-byte aligned), then the list's spills, if
// any, from the top of its capacity. An entry is byte << 3 | bit.
__device__ __forceinline__ void phase_buckets(const SieveArgs& a, uint64_t s, uint32_t* sieve32,
                                              uint32_t* list_next, uint32_t lane) {
  const uint32_t* cnt = a.bucket_counts + s * a.num_bucket_lists;
  const uint32_t* spill = a.bucket_spill + s * a.num_bucket_lists;
  const uint32_t* seg_entries = a.bucket_entries + s * a.bucket_seg_stride;
  for (;;) {
    uint32_t l = 0;
    if (lane == 0) l = atomicAdd(list_next, 1u);
    l = __shfl_sync(0xffffffffu, l, 0);
    if (l >= a.num_bucket_lists) break;
    // the list's length, spill count and place, loaded together
    const uint32_t n = __ldg(cnt + l);
    const uint32_t ns = __ldg(spill + l);
    const uint32_t cap = __ldg(a.bucket_list_cap + l);
    const uint32_t* e = seg_entries + __ldg(a.bucket_list_off + l);
    const uint32_t n4 = n & ~3u;
    // four 16-byte loads in flight per lane before the atomics that use them
    // (one load per iteration left the warps waiting on HBM latency); the
    // rest of the list beyond the first iteration is prefetched into L2 in
    // one request, so later iterations wait on L2, not HBM
    constexpr uint32_t kBU = 4;
    if (lane == 0 && n4 > 128 * kBU) prefetch_l2_bulk(e + 128 * kBU, 4u * (n4 - 128 * kBU));
    for (uint32_t x0 = 4 * lane; x0 < n4; x0 += 128 * kBU) {
      uint4 v4[kBU];
#pragma unroll
      for (uint32_t u = 0; u < kBU; u++)
        v4[u] = (x0 + 128 * u < n4) ? __ldg(reinterpret_cast<const uint4*>(e + x0 + 128 * u))
                                    : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
      for (uint32_t u = 0; u < kBU; u++) {
        if (x0 + 128 * u >= n4) break;         // past the list's whole quads
        const uint32_t v[4] = { v4[u].x, v4[u].y, v4[u].z, v4[u].w };
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const uint32_t bb = v[q] >> 3;       // entry: byte index << 3 | bit
          atomicAnd(&sieve32[bb >> 2], ~(1u << ((v[q] & 7u) + 8u * (bb & 3u))));
        }
      }
    }
    if (n4 + lane < n) {
      const uint32_t v = __ldg(e + n4 + lane);
      const uint32_t bb = v >> 3;
      atomicAnd(&sieve32[bb >> 2], ~(1u << ((v & 7u) + 8u * (bb & 3u))));
    }
    if (ns) {
      const uint32_t* top = e + cap - ns;
      for (uint32_t x = lane; x < ns; x += 32u) {
        const uint32_t v = __ldg(top + x);
        const uint32_t bb = v >> 3;
        atomicAnd(&sieve32[bb >> 2], ~(1u << ((v & 7u) + 8u * (bb & 3u))));
      }
    }
  }
}

// 5. mask the range edges [lo, hi] and count into acc; with bm set, also
// store the masked segment there (128-bit stores).
template <int BLOCK, bool ALL_KINDS>
__device__ __forceinline__ void phase_count(const uint4* smem4, uint32_t seg_bytes, uint64_t segLow,
                                            uint64_t lo, uint64_t hi, uint32_t tid, uint64_t (&acc)[6],
                                            uint4* bm = nullptr) {
  const uint32_t nchunks = seg_bytes >> 4;
  const uint64_t span = (uint64_t) seg_bytes * 30u;
  const uint64_t rhi = hi - segLow;                   // >= 7
  const uint64_t rlo = (lo > segLow) ? lo - segLow : 0;
  const bool full = (rlo <= 7) && (rhi >= span + 1);
  uint32_t c[6] = { 0, 0, 0, 0, 0, 0 };
  for (uint32_t ch = tid; ch < nchunks; ch += BLOCK) {
    uint4 v = smem4[ch];
    if (!full) {
      uint32_t w4[4] = { v.x, v.y, v.z, v.w };
#pragma unroll
      for (int q = 0; q < 4; q++) {
        uint32_t m = 0;
#pragma unroll
        for (int by = 0; by < 4; by++) {
          const uint64_t base = 30ull * (16ull * ch + 4u * q + by);
          m |= byte_keep(base, rlo, rhi) << (8 * by);
        }
        w4[q] &= m;
      }
      v = make_uint4(w4[0], w4[1], w4[2], w4[3]);
    }
    if (bm) bm[ch] = v;
    count_word<ALL_KINDS>(v.x, c);
    count_word<ALL_KINDS>(v.y, c);
    count_word<ALL_KINDS>(v.z, c);
    count_word<ALL_KINDS>(v.w, c);
  }
#pragma unroll
  for (int k = 0; k < 6; k++) acc[k] += c[k];
}

// Warp reduction of acc, one 64-bit atomic per warp and requested kind.
template <bool ALL_KINDS>
__device__ __forceinline__ void flush_counts(uint64_t (&acc)[6], uint32_t kinds, unsigned long long* out,
                                             uint32_t lane) {
#pragma unroll
  for (int k = 0; k < 6; k++) {
    if (!ALL_KINDS && k > 0) break;
    uint64_t v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0 && v && ((kinds >> k) & 1u))
      atomicAdd(&out[k], (unsigned long long) v);
    acc[k] = 0;
  }
}

// ---- the range kernel: one range, persistent grid of segment stripes -------
template <int BLOCK, bool ALL_KINDS>
__global__ void __launch_bounds__(BLOCK)
sieve_count_kernel(const __grid_constant__ SieveArgs a)
{
  extern __shared__ uint4 smem4[];
  uint32_t* const sieve32 = reinterpret_cast<uint32_t*>(smem4);
  uint32_t* const mstate = sieve32 + (a.seg_bytes >> 2);   // medium-prime state
  const uint32_t tid = threadIdx.x;
  const uint32_t lane = tid & 31u;
  const uint32_t warp = tid >> 5;
  const uint64_t span = (uint64_t) a.seg_bytes * 30u;
  const uint32_t n_med = a.n_primes - a.n_small;

  // contiguous stripe of segments
  const uint64_t per = (a.num_segments + gridDim.x - 1) / gridDim.x;
  const uint64_t s_begin = (uint64_t) blockIdx.x * per;
  const uint64_t s_end = (s_begin + per < a.num_segments) ? s_begin + per : a.num_segments;

  uint64_t acc[6] = { 0, 0, 0, 0, 0, 0 };

  __shared__ uint32_t wheel_tab[16];
  __shared__ uint32_t list_next;           // bucket list dispenser (per segment)
  if (tid < 16) wheel_tab[tid] = a.wheel_tab[tid];

  uint32_t sp[kSmallRegs], sr[kSmallRegs], sdl[kSmallRegs];
  small_setup<BLOCK>(a, a.n_small, a.seg_low0 + s_begin * span + 7, s_begin < s_end, warp, lane, sp, sr, sdl);
  if (s_begin < s_end) medium_setup<BLOCK>(a, a.n_small, n_med, mstate, a.seg_low0 + s_begin * span, tid);

  for (uint64_t s = s_begin; s < s_end; s++) {
    const uint64_t segLow = a.seg_low0 + s * span;
    if (tid == 0) list_next = 0;      // read after the next barrier
    phase_presieve<BLOCK>(a, smem4, segLow, tid);
    __syncthreads();
    phase_small<BLOCK>(a, a.n_small, sieve32, segLow, warp, lane, sp, sr);
    phase_medium<BLOCK>(a, a.n_small, n_med, mstate, sieve32, wheel_tab, segLow, tid);
    phase_direct<BLOCK>(a, a.n_primes, a.n_direct, sieve32, wheel_tab, segLow, tid);
    if (a.num_bucket_lists) phase_buckets(a, s, sieve32, &list_next, lane);
    __syncthreads();
    phase_count<BLOCK, ALL_KINDS>(smem4, a.seg_bytes, segLow, a.lo, a.hi, tid, acc,
                                  a.bitmap_out ? reinterpret_cast<uint4*>(a.bitmap_out + s * a.seg_bytes) : nullptr);
    small_advance(sp, sr, sdl);
    __syncthreads();
  }
  flush_counts<ALL_KINDS>(acc, a.kinds, a.counts, lane);
}

} // namespace psg
