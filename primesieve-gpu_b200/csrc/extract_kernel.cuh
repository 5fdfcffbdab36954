// extract_kernel.cuh -- sieved wheel-30 bitmap -> ascending list of primes.
//
// The reference extracts primes on the CPU (CountPrintPrimes.cpp:187-259,
// bit -> value through its bitValues table, LookupTables.cpp:35). Here the
// sieve kernel stores the masked segments and this kernel turns them into
// values on the device in two passes over blocks of kExtractBlockBytes:
// pass 0 writes each block's prime count; the host turns the counts into
// output offsets; pass 1 writes each block's primes in ascending order (one
// 16-byte chunk per thread, block-wide exclusive scan of the chunk counts).
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

namespace psg {

constexpr uint32_t kExtractThreads = 256;
constexpr uint32_t kExtractBlockBytes = 16 * kExtractThreads;   // 4 KiB

struct ExtractArgs {
  const uint8_t* bitmap;        // wheel-30 bytes, byte i = values base + 30 i + {7..31}
  uint64_t bytes;               // multiple of 16
  uint64_t base;                // multiple of 30
  uint32_t pass;                // 0: count, 1: emit
  uint32_t* block_counts;       // [blocks] (pass 0)
  const uint64_t* block_offsets;// [blocks] (pass 1)
  uint64_t* out;                // pass 1
};

__global__ void __launch_bounds__(kExtractThreads)
extract_kernel(const __grid_constant__ ExtractArgs a)
{
  __shared__ uint32_t wsum[kExtractThreads / 32];
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint64_t nblocks = (a.bytes + kExtractBlockBytes - 1) / kExtractBlockBytes;
  for (uint64_t blk = blockIdx.x; blk < nblocks; blk += gridDim.x) {
    const uint64_t off = blk * kExtractBlockBytes + 16ull * tid;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (off < a.bytes) v = *reinterpret_cast<const uint4*>(a.bitmap + off);
    const uint32_t c = __popc(v.x) + __popc(v.y) + __popc(v.z) + __popc(v.w);
    // block-wide exclusive scan of c
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t) o) incl += t;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t wbase = 0, total = 0;
    for (uint32_t w = 0; w < kExtractThreads / 32; w++) {
      if (w < warp) wbase += wsum[w];
      total += wsum[w];
    }
    if (a.pass == 0) {
      if (tid == 0) a.block_counts[blk] = total;
    } else {
      uint64_t pos = a.block_offsets[blk] + wbase + incl - c;
      const uint32_t w4[4] = { v.x, v.y, v.z, v.w };
#pragma unroll
      for (int q = 0; q < 4; q++) {
        uint32_t bits = w4[q];
        while (bits) {
          const uint32_t b = __ffs(bits) - 1u;
          bits &= bits - 1u;
          const uint64_t byte = off + 4u * q + (b >> 3);
          const uint32_t bv = b & 7u;
          const uint32_t ofs = (bv == 0) ? 7u : (bv == 1) ? 11u : (bv == 2) ? 13u : (bv == 3) ? 17u
                             : (bv == 4) ? 19u : (bv == 5) ? 23u : (bv == 6) ? 29u : 31u;
          a.out[pos++] = a.base + 30ull * byte + ofs;
        }
      }
    }
    __syncthreads();                  // wsum reused by the next block
  }
}

} // namespace psg
