// noalloc.cu -- psg_count_noalloc(): counting without any allocation.
//
// Some callers cannot allocate device memory at the moment they count:
// allocators' own callbacks (a cudaMalloc there re-enters the allocator),
// real-time loops that must not touch the allocator (a cudaMalloc can
// synchronise the device and take milliseconds), or embedders that give a
// library a fixed memory budget and account for every byte of it. For them
// this entry point runs the same segment-sieve kernel as
// psg_count(), but every piece of scratch it needs -- the sieving-prime
// table, its reciprocals and the six count accumulators -- lives in one
// file-scope static __device__ array of fixed size (kScratchBytes, about
// 270 KiB, held by every GPU that loads the library until the process
// exits). The caller passes the inputs (start, stop, kinds, stream) and the
// output (a device buffer of 6 uint64_t).
//
// Limits: stop <= 2^36, so that every sieving prime (<= 2^18) fits the
// table and the shared-memory wheel state of one CTA (no bucket storage is
// needed), and no pre-sieve tables are used.
#include "../../include/psgpu.h"
#include "sieve_kernel.cuh"
#include "wheel.hpp"

#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>

namespace psg {                                                   // capi.cpp
void set_last_error(const std::string& msg);
void set_last_error_nothrow(const char* msg) noexcept;
}

namespace {

constexpr uint64_t kMaxStop = 1ull << 36;
constexpr uint32_t kMaxPrime = 1u << 18;        // sqrt(kMaxStop)
constexpr uint32_t kMaxPrimes = 23040;          // > pi(2^18) = 23000
constexpr uint32_t kSegBytes = 131072;
constexpr int kBlock = 1024;
constexpr uint32_t kSmallLimit = 4096;

// Scratch layout: [recip: u64 x kMaxPrimes][counts: u64 x 8][primes: u32 x kMaxPrimes]
constexpr size_t kRecipOff = 0;
constexpr size_t kCountsOff = kRecipOff + 8ull * kMaxPrimes;
constexpr size_t kPrimesOff = kCountsOff + 8ull * 8;
constexpr size_t kScratchBytes = kPrimesOff + 4ull * kMaxPrimes;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Host copy of the sieving primes 7 <= p <= 2^18 (no heap: a fixed array,
// filled once per process by a plain odd-only sieve).
uint32_t g_host_primes[kMaxPrimes];
uint32_t g_host_nprimes = 0;

struct DeviceSetup {
  bool ready = false;
  unsigned char* scratch = nullptr;   // device address of g_scratch
  uint32_t grid = 0;
  uint32_t smem = 0;
  uint32_t state_cap = 0;
};
constexpr int kMaxDevices = 64;
DeviceSetup g_dev[kMaxDevices];
std::mutex g_mu;

__global__ void noalloc_recip_kernel(const uint32_t* __restrict__ p, uint64_t* __restrict__ r, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    r[i] = 0xffffffffffffffffull / p[i];
}

// Writes the six results (accumulators + the 2/3/5 table) to the caller.
__global__ void noalloc_finish_kernel(const unsigned long long* __restrict__ acc, uint64_t* __restrict__ out,
                                      uint32_t kinds, unsigned long long s0, unsigned long long s1,
                                      unsigned long long s2, unsigned long long s3,
                                      unsigned long long s4, unsigned long long s5) {
  const uint32_t k = threadIdx.x;
  if (k < 6) {
    const unsigned long long small = k == 0 ? s0 : k == 1 ? s1 : k == 2 ? s2 : k == 3 ? s3 : k == 4 ? s4 : s5;
    out[k] = ((kinds >> k) & 1u) ? acc[k] + small : 0ull;
  }
}

void host_primes_once() {
  if (g_host_nprimes) return;
  static unsigned char composite[kMaxPrime / 2 + 1];   // odd n -> composite[n / 2]
  for (uint32_t i = 3; (uint64_t) i * i <= kMaxPrime; i += 2)
    if (!composite[i / 2])
      for (uint32_t j = i * i; j <= kMaxPrime; j += 2 * i) composite[j / 2] = 1;
  uint32_t n = 0;
  for (uint32_t v = 7; v <= kMaxPrime; v += 2)
    if (!composite[v / 2]) g_host_primes[n++] = v;
  g_host_nprimes = n;
}

int fail(int status, const std::string& msg) {
  psg::set_last_error(msg);          // reported by psg_last_error()
  return status;
}

// Once per device, with that device current: find the array's device
// address (the host-side name is only a stand-in), fill the prime table and
// its reciprocals, and fix the launch geometry.
int setup_device(int dev, DeviceSetup& d) {
  host_primes_once();
  void* ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
  if (e != cudaSuccess) return fail(PSG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  unsigned char* base = static_cast<unsigned char*>(ptr);
  e = cudaMemcpy(base + kPrimesOff, g_host_primes, 4ull * g_host_nprimes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail(PSG_ERR_CUDA, std::string("cudaMemcpy: ") + cudaGetErrorString(e));
  noalloc_recip_kernel<<<64, 256>>>(reinterpret_cast<const uint32_t*>(base + kPrimesOff),
                                    reinterpret_cast<uint64_t*>(base + kRecipOff), g_host_nprimes);
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return fail(PSG_ERR_CUDA, std::string("reciprocal kernel: ") + cudaGetErrorString(e));

  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, dev);
  if (e != cudaSuccess) return fail(PSG_ERR_CUDA, std::string("cudaGetDeviceProperties: ") + cudaGetErrorString(e));
  uint32_t budget = (uint32_t) prop.sharedMemPerMultiprocessor;
  budget = budget > 1152u ? budget - 1152u : 0u;
  budget = std::min<uint32_t>(budget, (uint32_t) prop.sharedMemPerBlockOptin - 128u) & ~15u;
  if (budget < kSegBytes) return fail(PSG_ERR_NO_DEVICE, "device has too little shared memory");
  d.state_cap = (budget - kSegBytes) / 4u;
  d.smem = kSegBytes + 4u * d.state_cap;
  e = psg::allow_max_dynamic_smem(psg::sieve_count_kernel<kBlock, true>, dev);
  if (e == cudaSuccess) e = psg::allow_max_dynamic_smem(psg::sieve_count_kernel<kBlock, false>, dev);
  if (e != cudaSuccess) return fail(PSG_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  d.grid = (uint32_t) prop.multiProcessorCount;
  d.scratch = base;
  d.ready = true;
  return PSG_OK;
}

int count_noalloc(uint64_t start, uint64_t stop, uint32_t kinds, uint64_t* dev_counts, void* stream) {
  if (!dev_counts) return fail(PSG_ERR_ARG, "psg_count_noalloc: dev_counts is NULL");
  if (stop > kMaxStop)
    return fail(PSG_ERR_LIMIT, "psg_count_noalloc: stop must be <= 2^36 = 68719476736 (its sieving "
                               "primes live in a fixed table of the primes <= 2^18); use psg_count for larger stops");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(PSG_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(PSG_ERR_NO_DEVICE, "device index beyond the supported 64");
  DeviceSetup* d = &g_dev[dev];
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!d->ready) {
      const int rc = setup_device(dev, *d);
      if (rc) return rc;
    }
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  kinds &= 0x3fu;

  // the 2/3/5 table (primes and tuplets below 7), as psg_count
  unsigned long long small[6] = { 0, 0, 0, 0, 0, 0 };
  if (start <= stop && start <= 5) {
    struct T { uint64_t first, last; int kind; };
    static const T tab[8] = { { 2, 2, 0 }, { 3, 3, 0 }, { 5, 5, 0 }, { 3, 5, 1 },
                              { 5, 7, 1 }, { 5, 11, 2 }, { 5, 13, 3 }, { 5, 17, 4 } };
    for (const T& t : tab)
      if (t.first >= start && t.last <= stop) small[t.kind]++;
  }

  // the accumulators keep the previous call's counts: clear them first
  unsigned long long* acc = reinterpret_cast<unsigned long long*>(d->scratch + kCountsOff);
  e = cudaMemsetAsync(acc, 0, 8 * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return fail(PSG_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));

  if (start <= stop && stop >= 7 && kinds) {
    const uint64_t lo = std::max<uint64_t>(start, 7), hi = stop;
    uint32_t sq = (uint32_t) std::sqrt((double) hi);
    while ((uint64_t) sq * sq > hi) sq--;
    while ((uint64_t) (sq + 1) * (sq + 1) <= hi) sq++;
    const uint32_t n_total = (uint32_t) (std::upper_bound(g_host_primes, g_host_primes + g_host_nprimes, sq) - g_host_primes);
    const uint32_t n_small = std::min<uint32_t>(n_total, (uint32_t) (std::lower_bound(g_host_primes, g_host_primes + g_host_nprimes, kSmallLimit) - g_host_primes));
    if (n_total - n_small > d->state_cap)
      return fail(PSG_ERR_LIMIT, "psg_count_noalloc: sieving primes exceed this device's shared-memory state");
    const uint64_t span = (uint64_t) kSegBytes * 30u;
    psg::SieveArgs a;
    std::memset(&a, 0, sizeof a);
    a.seg_low0 = lo - ((lo - 7) % 30 + 7);
    a.lo = lo;
    a.hi = hi;
    a.num_segments = (hi - 7 - a.seg_low0) / span + 1;
    a.seg_bytes = kSegBytes;
    a.num_tables = 0;                  // no pre-sieve tables
    a.presieve_max = 5;
    a.primes = reinterpret_cast<const uint32_t*>(d->scratch + kPrimesOff);
    a.recip = reinterpret_cast<const uint64_t*>(d->scratch + kRecipOff);
    a.n_small = n_small;
    a.n_primes = n_total;
    for (uint32_t c = 0; c < 8; c++) {
      a.wheel_tab[2 * c] = psg::wheel_bits_packed(c);
      a.wheel_tab[2 * c + 1] = psg::wheel_corr_packed(c);
    }
    a.kinds = kinds;
    a.counts = acc;
    const uint32_t grid = (uint32_t) std::min<uint64_t>(d->grid, a.num_segments);
    if ((kinds & ~1u) != 0) psg::sieve_count_kernel<kBlock, true><<<grid, kBlock, d->smem, st>>>(a);
    else psg::sieve_count_kernel<kBlock, false><<<grid, kBlock, d->smem, st>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(PSG_ERR_CUDA, std::string("sieve kernel launch: ") + cudaGetErrorString(e));
  }
  noalloc_finish_kernel<<<1, 32, 0, st>>>(acc, dev_counts, kinds, small[0], small[1], small[2],
                                          small[3], small[4], small[5]);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(PSG_ERR_CUDA, std::string("finish kernel launch: ") + cudaGetErrorString(e));
  return PSG_OK;
}

} // namespace

// No C++ exception may unwind through the C boundary: a message that
// cannot be built (no host memory) or a mutex that cannot be taken becomes
// a status, as for every other psg_* entry point.
extern "C" int psg_count_noalloc(uint64_t start, uint64_t stop, uint32_t kinds,
                                 uint64_t* dev_counts, void* stream) {
  try {
    return count_noalloc(start, stop, kinds, dev_counts, stream);
  } catch (const std::bad_alloc&) {
    psg::set_last_error_nothrow("psg_count_noalloc: out of host memory");
    return PSG_ERR_NOMEM;
  } catch (...) {
    psg::set_last_error_nothrow("psg_count_noalloc: internal error");
    return PSG_ERR_INTERNAL;
  }
}
