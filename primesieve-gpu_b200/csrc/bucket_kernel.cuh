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
  uint32_t sqrt_x0;           // floor(sqrt(win_low + 6)): p <= sqrt_x0 <=> p*p < win_low + 7
  uint32_t win_segments;      // segments in this window (<= counters in smem)
  uint32_t seg_bytes;
  uint32_t seg_magic;         // floor(2^32 / seg_bytes) + 1 (segment index)
  uint32_t seg_shift;         // log2(seg_bytes) when it is a power of two
  uint32_t tile_steps;        // generate steps per warp between bin flushes
  uint32_t flush_at;          // thread walk: entries in the bins that trigger a flush
  uint32_t stagger_below;     // group walk: primes below this start staggered
  uint32_t wheel_tab[16];     // per class: bits, corr (wheel walk)
  const uint32_t* primes;
  const uint64_t* recip;
  const uint32_t* chunk_begin;  // [CTAs + 1] group-walk prime range per CTA
  const uint32_t* thread_chunk; // [CTAs + 1] thread-walk prime range per CTA
  const uint32_t* far_chunk;    // [CTAs + 1] range of primes above the window per CTA
  uint32_t num_lists;         // lists per segment, all kernels
  const uint32_t* list_off;   // [num_lists] entry offset inside a segment region
  const uint32_t* list_cap;   // [num_lists] capacity
  uint64_t seg_stride;        // entries per segment region
  uint32_t* entries;
  uint32_t* counts;           // [win_segments][num_lists] entries from the list's start
  uint32_t* spill;            // [win_segments][num_lists] entries at the list's top (spills)
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

// Binned prime-major fill. A warp takes 4 big primes at a time; lane
// (g = lane>>3, c = lane&7) walks the multiples of prime g whose cofactor is
// in wheel class c -- one arithmetic progression of stride p bytes with a
// fixed bit -- emitting one entry per step. An entry goes straight into its
// segment's bin in shared memory (kBinCap slots per segment, rank from one
// shared atomicAdd); an entry that finds its bin full goes to its HBM list
// at once, stored downward from the top of the list's capacity (rank from a
// per-segment spill counter), so nothing is ever dropped whatever the
// distribution and the list's main run stays whole quads. After tile_steps
// steps per warp the CTA copies the whole quads of every bin to the end of
// the main run with 16-byte stores, 4 lanes per bin; the 0-3 entries of a
// bin's last partial quad move to the front of the bin and wait for the
// next flush, and the CTA's final flush writes them as single entries. A
// list is thus its main run [0, counts) followed, at [cap - spill, cap), by
// its spills; the two overlap only if the list overflowed.
// Primes with at most ~32 multiples per class in a window (the CTA's
// thread_chunk range, above the window's byte length / 32) are walked one
// thread per prime through all 8 wheel classes (the medium tier's wheel
// walk), so that locating a prime costs one lane, not eight; they stream
// through shared memory in chunks of one prime per thread.
// (A one-prime-per-warp walk emitting 32 consecutive multiples per step with
// one rank atomic per segment run measured slower on B200: 42-47 ms against
// 38 ms per pass on [1e15, 1e15+1e11].)
constexpr uint32_t kBinCap = 32;          // bin slots per segment
constexpr uint32_t kBinStride = 36;       // 16-byte rows; bins 4 apart start 16 banks apart
static_assert(kBinCap <= 32 && kBinStride >= kBinCap + 4, "the flush moves at most two quads per lane");

// smem: thread-walk prime chunks rbuf[2][kChunk] (u64), pbuf[2][kChunk] |
//       bins[W][kBinStride] (16-byte aligned) |
//       cnt[W] (entries in the bin, plus spills since the last flush) |
//       gcnt[W] (entries in the HBM list's main run, a multiple of 4 until
//       the final flush) | gsp[W] (spilled entries at the list's top)
constexpr uint32_t kChunk = 1024;         // thread-walk primes per chunk (= threads)
constexpr size_t kChunkBytes = 2ull * kChunk * (8 + 4);
constexpr size_t kFillBytesPerSegment = (3 + kBinStride) * 4;
constexpr size_t fill_smem_bytes(uint32_t W) {
  return kChunkBytes + (size_t) W * kFillBytesPerSegment;
}

// 4- and 8-byte asynchronous global->shared copies (zero-filled when
// src_bytes is 0; the source address is then not read).
__device__ __forceinline__ void cp_async4(void* dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n"
               :: "r"((uint32_t) __cvta_generic_to_shared(dst)), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n"
               :: "r"((uint32_t) __cvta_generic_to_shared(dst)), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" :: "n"(N) : "memory"); }

template <int BLOCK, bool POW2>
__global__ void __launch_bounds__(BLOCK, 1)
bucket_fill_kernel(const __grid_constant__ BucketArgs a)
{
  static_assert(BLOCK == (int) kChunk, "one thread-walk prime per thread and chunk");
  constexpr uint32_t NWARPS = BLOCK / 32;
  extern __shared__ uint32_t smem_u32[];
  const uint32_t W = a.win_segments;
  uint64_t* const rbuf = reinterpret_cast<uint64_t*>(smem_u32);  // [2][kChunk]
  uint32_t* const pbuf = smem_u32 + 4 * kChunk;  // [2][kChunk]
  uint32_t* const bins = pbuf + 2 * kChunk;      // [W][kBinStride], byte offset 24 KiB
  uint32_t* const cnt = bins + W * kBinStride;   // [W]
  uint32_t* const gcnt = cnt + W;                // [W]
  uint32_t* const gsp = gcnt + W;                // [W]
  __shared__ uint32_t wheel_tab[16];
  __shared__ uint32_t s_round[3];                // thread walk: entries per round, 3 rotating slots
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  for (uint32_t i = tid; i < 3 * W; i += BLOCK) cnt[i] = 0;   // cnt, gcnt, gsp
  if (tid < 16) wheel_tab[tid] = a.wheel_tab[tid];
  if (tid < 3) s_round[tid] = 0;
  __syncthreads();

  const uint32_t list = blockIdx.x;
  const uint32_t cap = a.list_cap[list];
  uint32_t* const out = a.entries + a.list_off[list];
  const uint32_t win_bytes = W * a.seg_bytes;       // < 2^31 (host-checked)
  const uint32_t seg_bytes = a.seg_bytes;
  const uint32_t magic = a.seg_magic;
  const uint32_t shift = a.seg_shift;
  const uint64_t stride = a.seg_stride;
  const uint32_t lo = a.chunk_begin[blockIdx.x];
  const uint32_t hi = a.chunk_begin[blockIdx.x + 1];
  const uint32_t t_lo = a.thread_chunk[blockIdx.x];
  const uint32_t t_hi = a.thread_chunk[blockIdx.x + 1];
  const uint32_t f_lo = a.far_chunk[blockIdx.x];
  const uint32_t f_hi = a.far_chunk[blockIdx.x + 1];
  uint32_t rr = 0;                                // round slot (block-uniform)
  uint32_t in_bins = 0;                           // entries since the last flush (block-uniform)
  const uint32_t steps = a.tile_steps;
  constexpr uint32_t kFull = 0xffffffffu;
  constexpr uint32_t kDone = 0xffffffffu;
  const uint32_t g = lane >> 3;
  const uint32_t Q = cofactor_class(lane & 7u);

  // emit one entry into its segment's bin, or, the bin being full, straight
  // into the top of its HBM list
  auto put = [&](uint32_t sg, uint32_t r, uint32_t e) {
    if (r < kBinCap) {
      bins[sg * kBinStride + r] = e;
    } else {
      const uint32_t pos = atomicAdd(&gsp[sg], 1u);
      if (pos < cap) out[(uint64_t) sg * stride + (cap - 1u - pos)] = e;
    }
  };
  auto split_b = [&](uint32_t b, uint32_t& bo) -> uint32_t {
    if (POW2) { bo = b & (seg_bytes - 1u); return b >> shift; }
    return seg_of(b, seg_bytes, magic, bo);
  };
  // copy the whole quads of every bin to the end of its list's main run, 4
  // lanes per bin and 8 bins per warp step (all threads; the bins must be
  // complete, i.e. after a barrier). A bin holds at most 32 entries, so a
  // lane has at most two quads (entries 4j.. and 4j+16..): both are loaded
  // at once, predicated, before the stores -- the flush is latency-bound,
  // and a loop over the quads measured 5% slower for the whole fill. A
  // bin's last partial quad moves to the bin's front, or, on the CTA's final
  // flush, is written as single entries. The two bins of one 8-lane phase of
  // a 128-bit shared load are 4 apart, 16 banks apart with the 36-word
  // stride: conflict-free.
  auto flush = [&](bool last) {
    const uint32_t q = lane >> 2, j = lane & 3u;
    const uint32_t slot = (q >> 1) + 4u * (q & 1u);
    const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
    for (uint32_t s0 = warp * 8u; s0 < W; s0 += NWARPS * 8u) {   // warp-uniform trip count
      const uint32_t sg = s0 + slot;
      const bool valid = sg < W;
      const uint32_t n = valid ? min(cnt[sg], kBinCap) : 0u;
      const uint32_t base = valid ? gcnt[sg] : 0u;   // a multiple of 4
      const uint4* src = reinterpret_cast<const uint4*>(bins + sg * kBinStride);
      const uint4 v0 = 4u * j < n ? src[j] : zero;
      const uint4 v1 = 4u * j + 16u < n ? src[j + 4u] : zero;
      const uint32_t nq = n & ~3u, rem = n & 3u;     // entries in whole quads, and the rest
      const uint32_t room = base < cap ? cap - base : 0u;
      uint32_t* const dst = out + (uint64_t) sg * stride + base;
      if (4u * j + 4u <= nq && 4u * j + 4u <= room) reinterpret_cast<uint4*>(dst)[j] = v0;
      if (4u * j + 20u <= nq && 4u * j + 20u <= room) reinterpret_cast<uint4*>(dst)[j + 4u] = v1;
      __syncwarp();                                  // every lane has read its quads
      if (rem && (4u * j == nq || 4u * j + 16u == nq)) {   // this lane read the partial quad
        const uint4 tail = 4u * j == nq ? v0 : v1;
        uint32_t* const t = last ? dst + nq : bins + sg * kBinStride;
        if (!last || nq + rem <= room) {
          t[0] = tail.x;
          if (rem > 1u) t[1] = tail.y;
          if (rem > 2u) t[2] = tail.z;
        }
      }
      if (valid && j == 0) {
        gcnt[sg] = base + (last ? n : nq);
        cnt[sg] = last ? 0u : rem;
      }
    }
    __syncthreads();
  };

  // ---- phase 1: group walk over primes [lo, hi), tiles of `steps` steps
  {
    uint32_t b = kDone, p = 0, ebit = 0;    // this lane's progression
    uint32_t b0 = 0, bs = 0, end = 0;       // first multiple, start, current end (win_bytes, then bs)
    const float stagger = (float) (warp * 4u + g) / (float) (NWARPS * 4u);   // one offset per prime group
    // next multiple of the progression: up to the window's end, then from
    // the first multiple up to the start (b + p < 2^32: p, b < win_bytes)
    auto advance = [&](uint32_t x) -> uint32_t {
      const uint32_t nx = x + p;
      if (nx < end) return nx;
      if (end == win_bytes && b0 < bs) { end = bs; return b0; }
      return kDone;
    };
    uint32_t group = warp;                  // next group of 4 primes of this warp
    bool warp_done = lo >= hi;
    uint32_t p_nx = 0;                      // prefetched prime of the next group
    uint64_t r_nx = 0;
    {
      const uint32_t idx = lo + group * 4u + g;
      if (idx < hi) { p_nx = a.primes[idx]; r_nx = a.recip[idx]; }
    }
    for (;;) {
      for (uint32_t step = 0; step < steps && !warp_done; step++) {
        if (__ballot_sync(kFull, b != kDone) == 0) {
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
            if (b64 < win_bytes) {
              // primes with many multiples per window: start prime group
              // G (of 4 * 32 per CTA) about G/128 of the way through the
              // progression and wrap to its first multiple, so that the
              // CTA's warps (all on similar primes) emit into different
              // segments rather than together into the window's first ones
              // and past their bins' capacity
              b0 = (uint32_t) b64;
              b = b0;
              if (p < a.stagger_below) {
                const uint32_t ks = (uint32_t) ((float) (win_bytes - b0) * __frcp_rz((float) p) * stagger);
                const uint64_t bs64 = b64 + (uint64_t) ks * p;
                if (bs64 < win_bytes) b = (uint32_t) bs64;
              }
              end = win_bytes;
              bs = b;
            }
            ebit = residue_to_bit((Q * (p % 30u)) % 30u);
          }
        }
        if (b != kDone) {
          uint32_t bo;
          const uint32_t sg = split_b(b, bo);
          put(sg, atomicAdd(&cnt[sg], 1u), (bo << 3) | ebit);
          b = advance(b);
          if (b != kDone) {                 // two multiples per step: half the loop overhead
            const uint32_t sg2 = split_b(b, bo);
            put(sg2, atomicAdd(&cnt[sg2], 1u), (bo << 3) | ebit);
            b = advance(b);
          }
        }
      }
      const int more = __syncthreads_or(warp_done ? 0 : 1);
      flush(!more && t_lo >= t_hi && f_lo >= f_hi);   // the CTA's final flush writes the partial quads
      if (!more) break;
    }
  }

  // ---- phase 2: thread walk over primes [t_lo, t_hi), one prime per thread
  // and chunk; the chunks stream through shared memory (cp.async, double
  // buffered), the bins are flushed when they may be getting full
  if (t_lo < t_hi) {
    const uint32_t nchunk = (t_hi - t_lo + kChunk - 1) / kChunk;
    const uint32_t flush_at = a.flush_at;
    const float tstagger = (float) tid / (float) BLOCK;
    auto issue = [&](uint32_t k) {
      const uint32_t i = t_lo + k * kChunk + tid;
      const bool in = i < t_hi;
      const uint32_t src = in ? i : t_lo;         // a valid address even when zero-filling
      cp_async4(pbuf + (k & 1u) * kChunk + tid, a.primes + src, in ? 4u : 0u);
      cp_async8(rbuf + (k & 1u) * kChunk + tid, a.recip + src, in ? 8u : 0u);
      cp_async_commit();
    };
    issue(0);
    for (uint32_t k = 0; k < nchunk; k++) {
      if (k + 1 < nchunk) { issue(k + 1); cp_async_wait<1>(); }
      else cp_async_wait<0>();
      __syncthreads();                            // chunk k complete for every thread
      const uint32_t pc = pbuf[(k & 1u) * kChunk + tid];
      const uint64_t rc = rbuf[(k & 1u) * kChunk + tid];
      // this thread's walk: byte tb of the next multiple and its wheel index
      // j, running while tb < tend. A prime above half the window (at most
      // two wheel rotations, 16 multiples) is walked at once; a smaller one
      // starts about tid/1024 of the way through its rotations (p bytes
      // each) and wraps to its first multiple (tb0, j0) once, in rounds:
      // the CTA's threads then emit into different segments, not all into
      // the window's first ones.
      uint32_t tb = 0, tend = 0, tb0 = 0, tbs = 0, j = 0, j0 = 0, tpd = 0, tbits = 0, tcorr = 0;
      const uint32_t two_p = pc < (1u << 30) ? 2u * pc : (1u << 31);   // round length, saturated
      uint32_t emitted = 0;
      if (pc != 0) {
        uint64_t d; uint32_t c0;
        first_multiple(a.win_low, pc, rc, d, c0);
        j = first_class_ge(c0);
        const uint64_t b64 = (d + (uint64_t) (cofactor_class(j) - c0) * pc) / 30u;
        if (b64 < win_bytes) {
          tb = (uint32_t) b64;
          tpd = pc / 30u;
          const uint32_t cls = residue_to_bit(pc - 30u * tpd);
          tbits = wheel_tab[2 * cls];
          tcorr = wheel_tab[2 * cls + 1];
          if (pc > (win_bytes >> 1)) {
            do {
              uint32_t bo;
              const uint32_t sg = split_b(tb, bo);
              const uint32_t sh = 3u * j;
              put(sg, atomicAdd(&cnt[sg], 1u), (bo << 3) | ((tbits >> sh) & 7u));
              emitted++;
              // tb < 2^31 and the step < 2^30: no wrap
              tb += tpd * ((kGapPacked >> sh) & 7u) + ((tcorr >> sh) & 7u);
              j = (j + 1u) & 7u;
            } while (tb < win_bytes);
            tb = 0;                               // done (tend = 0)
          } else {
            tb0 = tb;
            j0 = j;
            const uint32_t q = (uint32_t) ((float) (win_bytes - tb0) * __frcp_rz((float) pc) * tstagger);
            const uint64_t bs64 = b64 + (uint64_t) q * pc;        // q whole rotations on
            if (bs64 < win_bytes) tb = (uint32_t) bs64;
            tbs = tb;
            tend = win_bytes;
          }
        }
      }
      // rounds of at most 16 multiples per thread, so that the bins are
      // flushed before they overflow however many multiples the primes have
      for (;;) {
        // a round ends after two wheel rotations (2p bytes, 16 multiples) or
        // at the end of the run; the wrap to the first multiple happens
        // between rounds
        const uint32_t rend = (tb >= tend) ? tb : (tend - tb > two_p) ? tb + two_p : tend;
        while (tb < rend) {
          uint32_t bo;
          const uint32_t sg = split_b(tb, bo);
          const uint32_t sh = 3u * j;
          put(sg, atomicAdd(&cnt[sg], 1u), (bo << 3) | ((tbits >> sh) & 7u));
          emitted++;
          // tb < 2^31 and the step < 2^30: no wrap
          tb += tpd * ((kGapPacked >> sh) & 7u) + ((tcorr >> sh) & 7u);
          j = (j + 1u) & 7u;
        }
        if (tb >= tend && tend == win_bytes && tb0 < tbs) { tb = tb0; j = j0; tend = tbs; }
        // round rr adds to slot rr % 3 and clears slot (rr + 1) % 3, which no
        // thread reads any more (its last reads were before the previous
        // barrier) and none adds to before the next barrier: after this
        // barrier every thread reads the same complete count, with no
        // second barrier
        emitted = __reduce_add_sync(kFull, emitted);
        if (lane == 0 && emitted) atomicAdd(&s_round[rr], emitted);
        if (tid == 0) s_round[rr == 2 ? 0 : rr + 1] = 0;
        const int more = __syncthreads_or(tb < tend ? 1 : 0);
        in_bins += s_round[rr];
        rr = rr == 2 ? 0 : rr + 1;
        const bool last = !more && k + 1 == nchunk && f_lo >= f_hi;
        if (in_bins >= flush_at || last) {
          flush(last);                            // ends with a barrier
          in_bins = 0;
        }
        if (!more) break;
        emitted = 0;
      }
    }
  }

  // ---- phase 3: primes above the window's byte length, [f_lo, f_hi): at
  // most eight multiples each in the window, so the per-prime staging and
  // the round bookkeeping of phase 2 would cost more than the walk. Each
  // thread takes kFU primes per step, loaded straight from global memory
  // (coalesced, the next step's loads in flight while this step walks) and
  // walks each at once; the CTA checks the bins once per step. (Eight primes
  // per step measured slower: register spills.)
  if (f_lo < f_hi) {
    constexpr uint32_t kFU = 4;
    const uint64_t x0 = a.win_low + 7u;
    uint32_t pn[kFU];
    uint64_t rn[kFU];
    auto load = [&](uint32_t base) {
#pragma unroll
      for (uint32_t u = 0; u < kFU; u++) {
        const uint32_t i = base + u * BLOCK + tid;
        pn[u] = i < f_hi ? __ldg(a.primes + i) : 0u;
        rn[u] = i < f_hi ? __ldg(a.recip + i) : 0ull;
      }
    };
    load(f_lo);
    for (uint32_t base = f_lo; base < f_hi; base += kFU * BLOCK) {
      uint32_t pc[kFU];
      uint64_t rc[kFU];
#pragma unroll
      for (uint32_t u = 0; u < kFU; u++) { pc[u] = pn[u]; rc[u] = rn[u]; }
      if (base + kFU * BLOCK < f_hi) load(base + kFU * BLOCK);
      uint32_t emitted = 0;
#pragma unroll
      for (uint32_t u = 0; u < kFU; u++) {          // unrolled: pc and rc stay in registers
        const uint32_t p = pc[u];
        if (p == 0) continue;
        // the first multiple's offset d from x0 as 30 * dq + dm and its
        // cofactor's residue c0 (first_multiple's cases, the p*p test by the
        // window's square root); then with p = 30 * tpd + pm and k the gap to
        // the first wheel class, byte = (d + k * p) / 30
        //   = dq + k * tpd + (dm + k * pm) / 30, all in 32 bits
        const uint32_t tpd = p / 30u;
        const uint32_t pm = p - 30u * tpd;
        uint32_t dq, dm, c0;
        if (p <= a.sqrt_x0) {
          const uint32_t r = mod_recip(x0, p, rc[u]);
          const uint32_t dd = r ? p - r : 0u;
          dq = dd / 30u;                          // < 2^28
          dm = dd - 30u * dq;
          const uint32_t t = dm < 23u ? dm + 7u : dm - 23u;   // (7 + d) mod 30
          c0 = (t * inverse_mod30(pm)) % 30u;
        } else {
          const uint64_t d = (uint64_t) p * p - x0;
          if (d >= 30ull * win_bytes) continue;   // p*p beyond the window
          dq = (uint32_t) (d / 30u);              // < win_bytes
          dm = (uint32_t) d - 30u * dq;
          c0 = pm;
        }
        uint32_t j = first_class_ge(c0);
        const uint32_t k = cofactor_class(j) - c0;   // < 30
        const uint32_t kt = k * tpd;                  // < p < 2^32
        if (kt >= win_bytes) continue;
        uint32_t tb = kt + dq + (dm + k * pm) / 30u;  // < 2^31 + 2^28 + 30
        if (tb >= win_bytes) continue;
        const uint32_t cls = residue_to_bit(pm);
        const uint32_t tbits = wheel_tab[2 * cls];
        const uint32_t tcorr = wheel_tab[2 * cls + 1];
        do {
          uint32_t bo;
          const uint32_t sg = split_b(tb, bo);
          const uint32_t sh = 3u * j;
          put(sg, atomicAdd(&cnt[sg], 1u), (bo << 3) | ((tbits >> sh) & 7u));
          emitted++;
          // tb < 2^31 and the step < 2^30: no wrap
          tb += tpd * ((kGapPacked >> sh) & 7u) + ((tcorr >> sh) & 7u);
          j = (j + 1u) & 7u;
        } while (tb < win_bytes);
      }
      // the round protocol of phase 2 (three rotating count slots, one barrier)
      emitted = __reduce_add_sync(kFull, emitted);
      if (lane == 0 && emitted) atomicAdd(&s_round[rr], emitted);
      if (tid == 0) s_round[rr == 2 ? 0 : rr + 1] = 0;
      __syncthreads();
      in_bins += s_round[rr];
      rr = rr == 2 ? 0 : rr + 1;
      const bool last = base + kFU * BLOCK >= f_hi;
      if (in_bins >= a.flush_at || last) {
        flush(last);                              // ends with a barrier
        in_bins = 0;
      }
    }
  }

  uint32_t written = 0;
  for (uint32_t sgi = tid; sgi < W; sgi += BLOCK) {
    uint32_t c = gcnt[sgi], sp = gsp[sgi];
    if ((uint64_t) c + sp > cap) {       // main run and spills met: recount
      atomicOr(a.overflow, 1u);
      c = min(c, cap);
      sp = min(sp, cap - c);
    }
    a.counts[(uint64_t) sgi * a.num_lists + list] = c;
    a.spill[(uint64_t) sgi * a.num_lists + list] = sp;
    written += c + sp;
  }
  for (int o = 16; o > 0; o >>= 1) written += __shfl_xor_sync(0xffffffffu, written, o);
  if (lane == 0 && written) atomicAdd(a.entry_total, (unsigned long long) written);
}

} // namespace psg
