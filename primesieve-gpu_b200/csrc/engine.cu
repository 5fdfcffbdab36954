// engine.cu -- host engine: tables, sieving primes, windows and launches.
#include "engine.hpp"
#include "sieve_kernel.cuh"
#include "bucket_kernel.cuh"
#include "primegen_kernel.cuh"
#include "../../include/psgpu.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

namespace psg {

uint32_t isqrt_u64(uint64_t x) {
  uint64_t r = (uint64_t) std::sqrt((double) x);
  while (r > 0 && (r > 0xffffffffull || r * r > x)) r--;
  while (r + 1 <= 0xffffffffull && (r + 1) * (r + 1) <= x) r++;
  return (uint32_t) r;
}

// The primes 2, 3, 5 and the k-tuplets containing them cannot be stored in
// the wheel-30 bit array; they are counted from this table when
// start <= 5 (reference src/gpu/GpuSieve.cpp:149-169,
// src/PrimeSieveClass.cpp:38-48).
void small_table(uint64_t start, uint64_t stop, uint32_t kinds, uint64_t out[6]) {
  struct T { uint64_t first, last; int kind; };
  static const T tab[8] = { { 2, 2, 0 }, { 3, 3, 0 }, { 5, 5, 0 }, { 3, 5, 1 },
                            { 5, 7, 1 }, { 5, 11, 2 }, { 5, 13, 3 }, { 5, 17, 4 } };
  if (start > 5) return;
  for (const T& t : tab)
    if (((kinds >> t.kind) & 1u) && t.first >= start && t.last <= stop) out[t.kind]++;
}

namespace {

constexpr int kBucketBlock = 1024;
constexpr double kSetupGroup = 8.0;     // fill-chunk cost of locating a group-walk prime (entries)
constexpr double kSetupThread = 4.0;    // ... of a thread-walk prime
constexpr double kSetupFar = 2.5;       // ... of a prime above the window (four per thread and step)
// Bucket fill bins: group-walk steps per warp between flushes (as a fill
// fraction of the bins) and the thread walk's flush threshold; group-walk
// primes with at least kStaggerMultiples multiples per class and window
// start staggered by prime group.
constexpr double kTileFill = 0.4;
constexpr double kFlushFill = 0.6;
constexpr uint64_t kStaggerMultiples = 16;

#define PSG_CUDA(call)                                                          \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      err = std::string(#call) + ": " + cudaGetErrorString(e_);                 \
      return PSG_ERR_CUDA;                                                      \
    }                                                                           \
  } while (0)


// Primes in (after, limit], limit < 2^32, by an odd-only segmented sieve.
void host_primes(uint32_t after, uint32_t limit, std::vector<uint32_t>& out) {
  if (limit <= after) return;
  const uint32_t r = isqrt_u64(limit);
  std::vector<uint8_t> small(r + 1, 0);
  std::vector<uint32_t> base;
  for (uint32_t i = 3; i <= r; i += 2) {
    if (small[i]) continue;
    base.push_back(i);
    for (uint64_t j = (uint64_t) i * i; j <= r; j += 2ull * i) small[j] = 1;
  }
  if (after < 2 && limit >= 2) out.push_back(2);
  const uint64_t SEG = 1u << 18;               // odd numbers per segment
  std::vector<uint8_t> seg(SEG);
  std::vector<uint64_t> next(base.size(), 0);
  uint64_t lo0 = std::max<uint64_t>(3, (uint64_t) after + 1) | 1ull;
  for (size_t k = 0; k < base.size(); k++) {
    const uint64_t p = base[k];
    uint64_t m = std::max<uint64_t>(p * p, (lo0 + p - 1) / p * p);
    if ((m & 1) == 0) m += p;
    next[k] = m;
  }
  for (uint64_t lo = lo0; lo <= limit; lo += 2 * SEG) {
    const uint64_t hi = std::min<uint64_t>(lo + 2 * SEG - 2, limit);
    const uint64_t cnt = (hi - lo) / 2 + 1;
    std::memset(seg.data(), 0, cnt);
    for (size_t k = 0; k < base.size(); k++) {
      const uint64_t p = base[k];
      if (p * p > hi) break;
      uint64_t m = next[k];
      for (; m <= hi; m += 2 * p) seg[(m - lo) >> 1] = 1;
      next[k] = m;
    }
    for (uint64_t i = 0; i < cnt; i++)
      if (!seg[i]) out.push_back((uint32_t) (lo + 2 * i));
  }
}

__global__ void recip_kernel(const uint32_t* __restrict__ p, uint64_t* __restrict__ r, size_t n) {
  for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n;
       i += (size_t) gridDim.x * blockDim.x)
    r[i] = 0xffffffffffffffffull / p[i];
}

__global__ void gather_kernel(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, size_t n, size_t stride) {
  for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
    dst[i] = src[i * stride];
}

__global__ void add_counts_kernel(unsigned long long* c, unsigned long long a0, unsigned long long a1,
                                  unsigned long long a2, unsigned long long a3,
                                  unsigned long long a4, unsigned long long a5) {
  if (threadIdx.x == 0) {
    c[0] += a0; c[1] += a1; c[2] += a2; c[3] += a3; c[4] += a4; c[5] += a5;
  }
}


template <int BLOCK>
void set_smem_attrs(int device) {
  allow_max_dynamic_smem(sieve_count_kernel<BLOCK, false>, device);
  allow_max_dynamic_smem(sieve_count_kernel<BLOCK, true>, device);
}

template <int BLOCK>
int occupancy(uint32_t bytes) {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sieve_count_kernel<BLOCK, true>, BLOCK, bytes);
  return n;
}

cudaError_t launch_sieve(uint32_t block, bool all, uint32_t grid, uint32_t smem,
                         cudaStream_t st, const SieveArgs& a) {
  switch (block) {
    case 256:
      if (all) sieve_count_kernel<256, true><<<grid, 256, smem, st>>>(a);
      else     sieve_count_kernel<256, false><<<grid, 256, smem, st>>>(a);
      break;
    case 1024:
      if (all) sieve_count_kernel<1024, true><<<grid, 1024, smem, st>>>(a);
      else     sieve_count_kernel<1024, false><<<grid, 1024, smem, st>>>(a);
      break;
    default:
      if (all) sieve_count_kernel<512, true><<<grid, 512, smem, st>>>(a);
      else     sieve_count_kernel<512, false><<<grid, 512, smem, st>>>(a);
      break;
  }
  return cudaGetLastError();
}

// Roofline probes of shared-memory atomicAnd, the operation the cross-off
// phases are made of. RANDOM: each thread walks its own odd word stride, so
// a warp's 32 addresses fall on banks at random (the access pattern of the
// medium, direct and bucket phases). CONFLICT_FREE: lane l always hits a
// word of bank l (word 32 k + l), one wavefront per warp instruction, the
// device's shared-atomic ceiling. Indices stay below kProbeWords.
constexpr uint32_t kProbeWords = 8192;    // 32 KiB of static shared memory
template <bool CONFLICT_FREE>
__global__ void __launch_bounds__(512) smem_atomic_probe_kernel(uint32_t iters, uint32_t* out) {
  __shared__ uint32_t s[kProbeWords];
  for (uint32_t i = threadIdx.x; i < kProbeWords; i += blockDim.x) s[i] = ~0u;
  __syncthreads();
  uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u;
  h ^= h >> 15; h *= 0x2c1b3c6du; h ^= h >> 12;
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t w, stride;
  if (CONFLICT_FREE) {
    w = (threadIdx.x >> 5) * 32u * 7u % kProbeWords + lane;     // row of this warp, bank = lane
    stride = 32u * 37u;                                         // whole rows: the bank stays
  } else {
    w = h % kProbeWords;
    stride = 2u * ((h >> 8) % 2048u) + 1u;                      // < kProbeWords
  }
  for (uint32_t it = 0; it < iters; it++) {
    atomicAnd(&s[w], ~(1u << (it & 31u)));
    w += stride;
    if (w >= kProbeWords) w -= kProbeWords;
  }
  __syncthreads();
  if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

template <bool CONFLICT_FREE>
double probe_rate(cudaStream_t st, int grid, uint32_t* out) {
  cudaEvent_t a, b;
  cudaEventCreate(&a); cudaEventCreate(&b);
  smem_atomic_probe_kernel<CONFLICT_FREE><<<grid, 512, 0, st>>>(64, out);
  const uint32_t iters = 8192;
  cudaEventRecord(a, st);
  smem_atomic_probe_kernel<CONFLICT_FREE><<<grid, 512, 0, st>>>(iters, out);
  cudaEventRecord(b, st);
  cudaEventSynchronize(b);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a); cudaEventDestroy(b);
  if (cudaGetLastError() != cudaSuccess || ms <= 0) return 0;
  return (double) grid * 512.0 * iters / (ms * 1e-3);
}

} // namespace

void Engine::measure_smem_atomic_rates(double& random_rate, double& conflict_free_rate) {
  random_rate = conflict_free_rate = 0;
  cudaSetDevice(device_);
  const int grid = prop_.multiProcessorCount * 2;
  uint32_t* out = nullptr;
  if (cudaMalloc(&out, grid * sizeof(uint32_t)) != cudaSuccess) { cudaGetLastError(); return; }
  random_rate = probe_rate<false>(stream_, grid, out);
  conflict_free_rate = probe_rate<true>(stream_, grid, out);
  cudaStreamSynchronize(stream_);
  cudaFree(out);
}

Engine::~Engine() {
  if (device_ < 0) return;
  cudaSetDevice(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  for (auto& t : timed_)
    for (auto& e : t.ev) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
  cudaFree(d_pat_);
  cudaFree(d_primes_);
  cudaFree(d_recip_);
  if (aux_stream_) cudaStreamSynchronize(aux_stream_);
  cudaFree(d_entries_);
  cudaFree(d_bcounts_);
  cudaFree(d_entries2_);
  cudaFree(d_bcounts2_);
  if (fork_event_) cudaEventDestroy(fork_event_);
  if (join_event_) cudaEventDestroy(join_event_);
  if (aux_stream_) cudaStreamDestroy(aux_stream_);
  for (auto& sl : slots_) cudaFree(sl.d_table);
  for (auto& g : stages_) {
    if (g.ev) cudaEventSynchronize(g.ev);
    if (g.h) cudaFreeHost(g.h);
    if (g.ev) cudaEventDestroy(g.ev);
  }
  cudaFree(d_overflow_);
  cudaFree(d_async_overflow_);
  cudaFree(d_entry_total_);
  cudaFree(d_counts_);
  cudaFree(d_batch_rows_);
  cudaFree(d_batch_ranges_);
  cudaFree(d_batch_items_);
  cudaFree(d_batch_queue_);
  if (h_counts_) cudaFreeHost(h_counts_);
  if (done_event_) cudaEventDestroy(done_event_);
  if (stream_) cudaStreamDestroy(stream_);
}

int Engine::init(int device, const EngineConfig& cfg, std::string& err) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    err = "no CUDA device found";
    return PSG_ERR_NO_DEVICE;
  }
  if (device < 0) {
    int best = 0, best_sm = -1;
    for (int i = 0; i < n; i++) {
      int sm = 0;
      cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, i);
      if (sm > best_sm) { best_sm = sm; best = i; }
    }
    device = best;
  }
  if (device >= n) {
    err = "GPU device index out of range";
    return PSG_ERR_NO_DEVICE;
  }
  device_ = device;
  cfg_ = cfg;
  PSG_CUDA(cudaSetDevice(device_));
  PSG_CUDA(cudaGetDeviceProperties(&prop_, device_));
  if (prop_.major < 10) {
    err = "this build contains sm_100a code only; device " + std::string(prop_.name) +
          " has compute capability " + std::to_string(prop_.major) + "." + std::to_string(prop_.minor);
    return PSG_ERR_NO_DEVICE;
  }
  PSG_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  PSG_CUDA(cudaStreamCreateWithFlags(&aux_stream_, cudaStreamNonBlocking));
  PSG_CUDA(cudaEventCreateWithFlags(&fork_event_, cudaEventDisableTiming));
  PSG_CUDA(cudaEventCreateWithFlags(&join_event_, cudaEventDisableTiming));
  PSG_CUDA(cudaEventCreateWithFlags(&done_event_, cudaEventDisableTiming));

  // ---- geometry ------------------------------------------------------------
  // Shared memory per CTA = sieve segment + medium-prime state. By default
  // one 1024-thread CTA per SM holds a 128 KiB segment and gives the rest of
  // the SM's shared memory to the carried medium-prime state.
  block_ = cfg.block ? cfg.block : 1024;
  if (block_ != 256 && block_ != 512 && block_ != 1024) {
    err = "block must be 256, 512 or 1024";
    return PSG_ERR_ARG;
  }
  const uint32_t target_ctas = cfg.ctas_per_sm ? cfg.ctas_per_sm : 1;
  const uint32_t smem_optin = (uint32_t) prop_.sharedMemPerBlockOptin;
  const uint32_t smem_sm = (uint32_t) prop_.sharedMemPerMultiprocessor;
  uint32_t budget = smem_sm / target_ctas;
  budget = (budget > 1024u + 128u) ? budget - 1024u - 128u : 0u;   // driver reserve + static smem
  budget = std::min(budget, smem_optin - 128u) & ~15u;
  seg_bytes_ = cfg.seg_bytes ? cfg.seg_bytes : 131072u;
  seg_bytes_ = std::min(seg_bytes_, budget);
  seg_bytes_ &= ~(16u * block_ - 1u);          // whole 16-byte chunks per thread
  if (seg_bytes_ < 16u * block_) {
    err = "segment too small for the block size";
    return PSG_ERR_ARG;
  }
  state_cap_ = (budget - seg_bytes_) / 4u;
  smem_dyn_ = seg_bytes_ + 4u * state_cap_;
  switch (block_) {
    case 256: set_smem_attrs<256>(device_); break;
    case 1024: set_smem_attrs<1024>(device_); break;
    default: set_smem_attrs<512>(device_); break;
  }
  int occ = block_ == 256 ? occupancy<256>(smem_dyn_)
          : block_ == 1024 ? occupancy<1024>(smem_dyn_) : occupancy<512>(smem_dyn_);
  if (occ < 1) {
    err = "sieve kernel cannot be resident with this segment/block size";
    return PSG_ERR_ARG;
  }
  occ = std::min<int>(occ, (int) target_ctas);
  grid_ = (uint32_t) (prop_.multiProcessorCount * occ);

  const uint64_t span = (uint64_t) seg_bytes_ * 30u;
  small_limit_ = cfg.small_limit ? cfg.small_limit : 4096u;
  small_auto_ = cfg.small_limit == 0;
  big_limit_ = cfg.big_limit ? cfg.big_limit : (uint32_t) std::min<uint64_t>(span / 10u, 0xffffffffull);
  if (big_limit_ < small_limit_) big_limit_ = small_limit_;
  window_ = cfg.window_segments ? cfg.window_segments : grid_ * 8u;
  lists_ = cfg.bucket_lists ? cfg.bucket_lists : (uint32_t) prop_.multiProcessorCount;
  // the bucket fill kernel keeps one bin per window segment in shared memory
  // and indexes a window with 32-bit byte offsets
  const size_t fill_smem_max = (size_t) prop_.sharedMemPerBlockOptin;
  window_ = std::min<uint32_t>(window_, (uint32_t) ((fill_smem_max - kChunkBytes) / kFillBytesPerSegment));
  window_ = std::min<uint32_t>(window_, (uint32_t) ((1ull << 31) / seg_bytes_));
  window_ = std::max<uint32_t>(window_, 1u);
  seg_pow2_ = (seg_bytes_ & (seg_bytes_ - 1u)) == 0;
  seg_shift_ = 0;
  while ((1u << seg_shift_) < seg_bytes_) seg_shift_++;
  allow_max_dynamic_smem(bucket_fill_kernel<kBucketBlock, true>, device_);
  allow_max_dynamic_smem(bucket_fill_kernel<kBucketBlock, false>, device_);
  allow_max_dynamic_smem(primegen_kernel<1024>, device_);
  cap_scale_ = cfg.list_capacity_pct ? (double) cfg.list_capacity_pct / 100.0 : 1.0;

  PSG_CUDA(cudaMalloc(&d_counts_, 6 * sizeof(unsigned long long)));
  PSG_CUDA(cudaMalloc(&d_batch_queue_, sizeof(uint32_t)));
  PSG_CUDA(cudaMalloc(&d_overflow_, sizeof(uint32_t)));
  PSG_CUDA(cudaMalloc(&d_async_overflow_, sizeof(uint32_t)));
  PSG_CUDA(cudaMemset(d_async_overflow_, 0, sizeof(uint32_t)));
  cur_overflow_ = d_overflow_;
  PSG_CUDA(cudaMalloc(&d_entry_total_, sizeof(unsigned long long)));
  PSG_CUDA(cudaMemset(d_entry_total_, 0, sizeof(unsigned long long)));
  PSG_CUDA(cudaMemset(d_overflow_, 0, sizeof(uint32_t)));
  PSG_CUDA(cudaMallocHost(&h_counts_, 8 * sizeof(unsigned long long)));

  if (cfg.presieve == 2) {          // 0 = default (on), 1 = on, 2 = off
    presieve_max_ = 5;
  } else {
    int rc = build_presieve(err);
    if (rc) return rc;
  }
  return PSG_OK;
}

// Pre-sieve pattern tables. A group's pattern has one byte per wheel-30 byte
// over one period (the product of the group's primes); a bit is cleared iff
// its value is a multiple of a group prime. Stored as 16 copies shifted by
// 0..15 bytes so that any 16 consecutive pattern bytes are one aligned
// 128-bit load. (Reference: 4-byte sliding windows,
// src/gpu/GpuTables.cpp:31-130; the groups here reach 59.)
int Engine::build_presieve(std::string& err) {
  groups_ = { { 7, 11, 13, 17 }, { 19, 23, 29, 31 }, { 37, 41, 43 }, { 47, 53, 59 } };
  size_t total = 0;
  pat_off_.clear(); pat_period_.clear(); pat_stride_.clear(); presieve_primes_.clear();
  for (auto& g : groups_) {
    uint64_t P = 1;
    for (uint32_t p : g) { P *= p; presieve_primes_.push_back(p); presieve_max_ = std::max(presieve_max_, p); }
    const uint32_t stride = (uint32_t) ((P + 15 + 15) & ~15ull);
    pat_off_.push_back(total);
    pat_period_.push_back((uint32_t) P);
    pat_stride_.push_back(stride);
    total += 16ull * stride;
  }
  std::vector<uint8_t> host(total, 0);
  for (size_t t = 0; t < groups_.size(); t++) {
    const uint32_t P = pat_period_[t];
    std::vector<uint8_t> pat(P, 0xff);
    for (uint32_t p : groups_[t]) {
      // multiples of p coprime to 30 inside [0, 30 P)
      for (uint64_t m = p; m < 30ull * P; m += 2ull * p) {
        if (m % 3 == 0 || m % 5 == 0) continue;
        const uint64_t byte = (m - 7) / 30;               // value 30*byte + off
        const uint32_t bit = residue_to_bit((uint32_t) (m % 30));
        pat[byte] &= (uint8_t) ~(1u << bit);
      }
    }
    for (uint32_t k = 0; k < 16; k++) {
      uint8_t* copy = host.data() + pat_off_[t] + (size_t) k * pat_stride_[t];
      for (uint32_t i = 0; i < pat_stride_[t]; i++) copy[i] = pat[(i + k) % P];
    }
  }
  PSG_CUDA(cudaMalloc(&d_pat_, total));
  PSG_CUDA(cudaMemcpy(d_pat_, host.data(), total, cudaMemcpyHostToDevice));
  return PSG_OK;
}

// Grow the device table d_primes_/d_recip_ to hold n primes (keeping the
// first keep entries).
int Engine::reserve_primes(size_t n, size_t keep, std::string& err) {
  if (n <= d_primes_cap_) return PSG_OK;
  uint32_t* np = nullptr; uint64_t* nr = nullptr;
  const size_t cap = std::max<size_t>(n, 1024);
  PSG_CUDA(cudaMalloc(&np, cap * sizeof(uint32_t)));
  PSG_CUDA(cudaMalloc(&nr, cap * sizeof(uint64_t)));
  if (keep) {
    PSG_CUDA(cudaMemcpyAsync(np, d_primes_, keep * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream_));
    PSG_CUDA(cudaMemcpyAsync(nr, d_recip_, keep * sizeof(uint64_t), cudaMemcpyDeviceToDevice, stream_));
  }
  PSG_CUDA(cudaStreamSynchronize(stream_));
  cudaFree(d_primes_); cudaFree(d_recip_);
  d_primes_ = np; d_recip_ = nr; d_primes_cap_ = cap;
  return PSG_OK;
}

// Sieving primes (presieve_max_, limit]. Up to kHostExact they are made on
// the host (exact host copy h_primes_, used for tier limits and bucket
// planning); beyond, on the device by primegen_kernel (two passes: count per
// segment, then write at the scanned offsets), with a 1-in-kSample host
// sample of the whole table for lookups and planning.
int Engine::ensure_primes(uint64_t limit, std::string& err) {
  if (limit <= primes_upto_ && d_primes_) return PSG_OK;
  // grow geometrically so repeated calls with rising stops stay cheap
  uint64_t target = std::max<uint64_t>(limit, std::min<uint64_t>(primes_upto_ * 2, 0xffffffffull));
  target = std::max<uint64_t>(target, 1u << 16);
  target = std::min<uint64_t>(target, 0xffffffffull);

  // ---- host part (exact): up to kHostExact
  if (primes_upto_ < kHostExact || !d_primes_) {
    const uint64_t htarget = std::min<uint64_t>(target, kHostExact);
    const uint32_t after = std::max<uint32_t>(presieve_max_, (uint32_t) primes_upto_);
    std::vector<uint32_t> more;
    host_primes(after, (uint32_t) htarget, more);
    const size_t old_n = n_dev_;
    const size_t n = old_n + more.size();
    int rc = reserve_primes(n, old_n, err);
    if (rc) return rc;
    h_primes_.insert(h_primes_.end(), more.begin(), more.end());
    if (n > old_n) {
      PSG_CUDA(cudaMemcpyAsync(d_primes_ + old_n, h_primes_.data() + old_n, (n - old_n) * sizeof(uint32_t),
                               cudaMemcpyHostToDevice, stream_));
      const size_t m = n - old_n;
      recip_kernel<<<(uint32_t) std::min<size_t>((m + 255) / 256, 4096), 256, 0, stream_>>>(d_primes_ + old_n, d_recip_ + old_n, m);
      PSG_CUDA(cudaGetLastError());
      PSG_CUDA(cudaStreamSynchronize(stream_));
    }
    n_dev_ = n;
    primes_upto_ = htarget;
  }

  // ---- device part: (primes_upto_, target]
  if (target > primes_upto_) {
    const uint64_t lo = primes_upto_ + 1, hi = target;
    // base primes 7 .. sqrt(hi) (<= 2^16): the pre-sieve primes + the head
    std::vector<uint32_t> base;
    const uint32_t r = isqrt_u64(hi);
    host_primes(6, std::min<uint32_t>(presieve_max_, r), base);
    for (uint32_t q : h_primes_) { if (q > r) break; base.push_back(q); }
    uint32_t n_small = 0;
    while (n_small < base.size() && base[n_small] < 1024u) n_small++;
    const uint32_t seg = 131072u;                       // primegen segment, 1024 threads
    const uint64_t span = (uint64_t) seg * 30u;
    const uint64_t seg_low0 = lo - ((lo - 7) % 30 + 7);
    const uint32_t nseg = (uint32_t) ((hi - 7 - seg_low0) / span + 1);
    uint32_t* d_base = nullptr; uint64_t* d_brecip = nullptr;
    uint32_t* d_cnt = nullptr; uint64_t* d_off = nullptr;
    auto cleanup = [&]() { cudaFree(d_base); cudaFree(d_brecip); cudaFree(d_cnt); cudaFree(d_off); };
    if (cudaMalloc(&d_base, base.size() * 4) != cudaSuccess || cudaMalloc(&d_brecip, base.size() * 8) != cudaSuccess ||
        cudaMalloc(&d_cnt, (size_t) nseg * 4) != cudaSuccess || cudaMalloc(&d_off, (size_t) nseg * 8) != cudaSuccess) {
      cudaGetLastError(); cleanup();
      err = "cannot allocate the prime generator's buffers";
      return PSG_ERR_NOMEM;
    }
    PrimeGenArgs g;
    std::memset(&g, 0, sizeof g);
    g.seg_low0 = seg_low0; g.lo = lo; g.hi = hi; g.num_segments = nseg; g.seg_bytes = seg;
    g.base = d_base; g.base_recip = d_brecip; g.n_base_small = n_small; g.n_base = (uint32_t) base.size();
    g.seg_counts = d_cnt; g.seg_offsets = d_off;
    for (uint32_t c = 0; c < 8; c++) { g.wheel_tab[2 * c] = wheel_bits_packed(c); g.wheel_tab[2 * c + 1] = wheel_corr_packed(c); }
    cudaError_t e = cudaMemcpyAsync(d_base, base.data(), base.size() * 4, cudaMemcpyHostToDevice, stream_);
    recip_kernel<<<64, 256, 0, stream_>>>(d_base, d_brecip, base.size());
    const uint32_t grid = std::min<uint32_t>(nseg, (uint32_t) prop_.multiProcessorCount);
    g.pass = 0;
    primegen_kernel<1024><<<grid, 1024, seg, stream_>>>(g);
    std::vector<uint32_t> cnt(nseg);
    std::vector<uint64_t> off(nseg);
    if (e == cudaSuccess) e = cudaMemcpyAsync(cnt.data(), d_cnt, (size_t) nseg * 4, cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) { cleanup(); err = std::string("prime generator (count): ") + cudaGetErrorString(e); return PSG_ERR_CUDA; }
    uint64_t total = 0;
    for (uint32_t i = 0; i < nseg; i++) { off[i] = total; total += cnt[i]; }
    const size_t old_n = n_dev_;
    int rc = reserve_primes(old_n + total, old_n, err);
    if (rc) { cleanup(); return rc; }
    e = cudaMemcpyAsync(d_off, off.data(), (size_t) nseg * 8, cudaMemcpyHostToDevice, stream_);
    g.pass = 1;
    g.out = d_primes_ + old_n;
    primegen_kernel<1024><<<grid, 1024, seg, stream_>>>(g);
    if (total)
      recip_kernel<<<(uint32_t) std::min<uint64_t>((total + 255) / 256, 4096), 256, 0, stream_>>>(d_primes_ + old_n, d_recip_ + old_n, total);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e == cudaSuccess) e = cudaGetLastError();
    cleanup();
    if (e != cudaSuccess) { err = std::string("prime generator (write): ") + cudaGetErrorString(e); return PSG_ERR_CUDA; }
    n_dev_ = old_n + total;
    primes_upto_ = target;
  }

  // ---- 1-in-kSample host sample of the whole table (gathered on the device)
  const size_t ns = (n_dev_ + kSample - 1) / kSample;
  h_sample_.resize(ns);
  if (ns) {
    uint32_t* d_s = nullptr;
    PSG_CUDA(cudaMalloc(&d_s, ns * sizeof(uint32_t)));
    gather_kernel<<<(uint32_t) std::min<size_t>((ns + 255) / 256, 4096), 256, 0, stream_>>>(d_primes_, d_s, ns, kSample);
    cudaError_t e = cudaMemcpyAsync(h_sample_.data(), d_s, ns * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    cudaFree(d_s);
    if (e != cudaSuccess) { err = std::string("prime sample: ") + cudaGetErrorString(e); return PSG_ERR_CUDA; }
  }
  // prefix of sum(1/p) per sample block: exact inside the host head, the
  // block's first (smallest) prime for all of a block beyond it (an upper
  // bound, which is what the bucket capacities need); per prime inside the
  // head
  if (h_inv_head_.size() != h_primes_.size() + 1) {
    h_inv_head_.assign(h_primes_.size() + 1, 0.0);
    for (size_t j = 0; j < h_primes_.size(); j++) h_inv_head_[j + 1] = h_inv_head_[j] + 1.0 / (double) h_primes_[j];
  }
  h_inv_block_.assign(ns + 1, 0.0);
  for (size_t k = 0; k < ns; k++) {
    const size_t j0 = k * kSample, j1 = std::min<size_t>(j0 + kSample, n_dev_);
    const size_t jh = std::min(std::max(j0, h_primes_.size()), j1);   // [j0, jh) in the head
    double v = (double) (j1 - jh) / (double) h_sample_[k];
    for (size_t j = j0; j < jh; j++) v += 1.0 / (double) h_primes_[j];
    h_inv_block_[k + 1] = h_inv_block_[k] + v;
  }
  return PSG_OK;
}

// Number of table primes <= v (strict = false) or < v (strict = true).
uint32_t Engine::count_primes_le(uint64_t v, bool strict) {
  const uint32_t x = (uint32_t) std::min<uint64_t>(v, 0xffffffffull);
  if (v <= kHostExact || v <= (h_primes_.empty() ? 0 : h_primes_.back())) {
    auto it = strict ? std::lower_bound(h_primes_.begin(), h_primes_.end(), x)
                     : std::upper_bound(h_primes_.begin(), h_primes_.end(), x);
    if (it != h_primes_.end() || n_dev_ == h_primes_.size()) return (uint32_t) (it - h_primes_.begin());
  }
  // beyond the exact head: locate the sample block, then fetch that block
  auto it = strict ? std::lower_bound(h_sample_.begin(), h_sample_.end(), x)
                   : std::upper_bound(h_sample_.begin(), h_sample_.end(), x);
  const size_t k = (size_t) (it - h_sample_.begin());
  if (k == 0) return 0;
  const size_t b0 = (k - 1) * kSample;
  const size_t b1 = std::min<size_t>(b0 + kSample, n_dev_);
  uint32_t blk[kSample];
  cudaMemcpy(blk, d_primes_ + b0, (b1 - b0) * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  auto jt = strict ? std::lower_bound(blk, blk + (b1 - b0), x) : std::upper_bound(blk, blk + (b1 - b0), x);
  return (uint32_t) (b0 + (size_t) (jt - blk));
}

// An upper bound of the number of table primes <= v from the host tables
// alone: exact inside the head, the end of v's sample block beyond it.
uint32_t Engine::count_primes_upper(uint64_t v) const {
  const uint32_t x = (uint32_t) std::min<uint64_t>(v, 0xffffffffull);
  if (!h_primes_.empty() && (x < h_primes_.back() || n_dev_ == h_primes_.size()))
    return (uint32_t) (std::upper_bound(h_primes_.begin(), h_primes_.end(), x) - h_primes_.begin());
  const size_t k = (size_t) (std::upper_bound(h_sample_.begin(), h_sample_.end(), x) - h_sample_.begin());
  return (uint32_t) std::min<size_t>(std::max<size_t>(k * kSample, h_primes_.size()), n_dev_);
}

// Number of table primes < v from the host tables alone: exact inside the
// head, rounded to a sample block beyond it (for splits that only steer
// work, never correctness).
uint32_t Engine::approx_count_below(uint64_t v) const {
  const uint32_t x = (uint32_t) std::min<uint64_t>(v, 0xffffffffull);
  if (!h_primes_.empty() && x <= h_primes_.back())
    return (uint32_t) (std::lower_bound(h_primes_.begin(), h_primes_.end(), x) - h_primes_.begin());
  const size_t k = (size_t) (std::lower_bound(h_sample_.begin(), h_sample_.end(), x) - h_sample_.begin());
  return (uint32_t) std::min<size_t>(std::max<size_t>(k * kSample, h_primes_.size()), n_dev_);
}

// Table prime i for planning: exact in the host head, else the smallest prime
// of its sample block (a slight underestimate).
double Engine::approx_prime(uint32_t i) const {
  if (i < h_primes_.size()) return (double) h_primes_[i];
  return (double) h_sample_[std::min<size_t>(i / kSample, h_sample_.size() - 1)];
}

// Sum of 1/p over table primes [0, i), same weights as h_inv_block_.
// O(1): the bucket planner's binary searches call it thousands of times per
// range.
double Engine::inv_prefix(uint32_t i) const {
  const size_t head = h_primes_.size();
  if (i <= head) return h_inv_head_[i];
  const size_t k = std::min<size_t>(i / kSample, h_inv_block_.size() - 1);
  const size_t j0 = k * kSample;
  double v = h_inv_block_[k];
  // [j0, i): exact inside the head, the block's smallest prime beyond it
  const size_t jh = std::min<size_t>(std::max(j0, head), i);
  if (jh > j0) v += h_inv_head_[jh] - h_inv_head_[j0];
  if (i > jh) v += (double) (i - jh) / (double) h_sample_[std::min(k, h_sample_.size() - 1)];
  return v;
}

int Engine::prepare(uint64_t stop, std::string& err) {
  PSG_CUDA(cudaSetDevice(device_));
  return ensure_primes(std::max<uint32_t>(isqrt_u64(stop), 7u), err);
}

int Engine::sieving_primes(uint64_t stop, size_t first, uint32_t* out, size_t n, size_t& total,
                           uint64_t& lo_excl, uint64_t& hi_incl, std::string& err) {
  int rc = prepare(stop, err);
  if (rc) return rc;
  total = n_dev_;
  lo_excl = presieve_max_;
  hi_incl = primes_upto_;
  if (first < n_dev_ && n) {
    const size_t m = std::min(n, n_dev_ - first);
    PSG_CUDA(cudaMemcpyAsync(out, d_primes_ + first, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
    PSG_CUDA(cudaStreamSynchronize(stream_));
  }
  return PSG_OK;
}

// Bucket lists for the big primes primes[first, last): one list per fill
// CTA and segment, the CTAs' prime chunks cut for equal expected work
// (setup + hits per window). Capacity = expected entries per segment +
// 6 sigma + 32 (x cap_scale_: grown after an overflow, or set below 1 by
// the list_capacity_pct knob). All lists of one segment are packed in one
// region.
int Engine::ensure_buckets(uint32_t first, uint32_t last, std::string& err) {
  if (plan_.last && first == plan_.first && last == plan_.last && d_entries_) return PSG_OK;
  const double span = (double) seg_bytes_ * 30.0;
  const double per_seg = span * (8.0 / 30.0);
  std::vector<uint32_t> off, cap, begin;
  uint64_t stride = 0;
  auto add_list = [&](double mu) {
    uint32_t ci = (uint32_t) std::ceil((mu + 6.0 * std::sqrt(mu) + 32.0) * cap_scale_);
    ci = std::max<uint32_t>((ci + 3u) & ~3u, 4u);
    off.push_back((uint32_t) stride);
    cap.push_back(ci);
    stride += ci;
  };
  const uint32_t nfill = last - first;
  uint32_t fill_ctas = 0;
  if (nfill) {
    fill_ctas = std::max<uint32_t>(1, std::min<uint32_t>(lists_, nfill));
    const double win_span = span * (8.0 / 30.0) * (double) window_;
    // per-window setup of a prime in entries: 8 lanes in the group walk,
    // one in the thread walk
    // Per-window cost of a prime in entry units: its setup (8 lanes in the
    // group walk, one in the thread walk) plus its entries. Group walk:
    // primes [first, t_end); thread walk: primes [t_end, last). Each range is
    // cut into fill_ctas chunks of equal cost (binary search on the monotone
    // cost over the 1/p prefix table); CTA c takes chunk c of both.
    const double setup_group = kSetupGroup, setup_thread = kSetupThread;
    const uint32_t t_end = std::min(std::max(approx_count_below(thread_limit(window_)), first), last);
    // primes above the window's byte length: at most eight multiples per
    // window (the threshold twice as high measured 1-2% slower at 1e18 and
    // near 2^64)
    const uint32_t f_end = std::min(std::max(approx_count_below(1ull * window_ * seg_bytes_ + 1), t_end), last);
    begin.assign(3 * (fill_ctas + 1), 0);
    const auto cut = [&](uint32_t from, uint32_t to, double setup, uint32_t* bounds) {
      const double s0 = inv_prefix(from);
      const auto cost = [&](uint32_t i) { return setup * (double) (i - from) + win_span * (inv_prefix(i) - s0); };
      const double total = cost(to);
      bounds[0] = from;
      bounds[fill_ctas] = to;
      for (uint32_t l = 1; l < fill_ctas; l++) {
        const double target = total * (double) l / (double) fill_ctas;
        uint32_t x = bounds[l - 1], y = to;      // smallest i in [x, y] with cost(i) >= target
        while (x < y) {
          const uint32_t m = x + (y - x) / 2;
          if (cost(m) >= target) y = m; else x = m + 1;
        }
        bounds[l] = x;
      }
    };
    cut(first, t_end, setup_group, begin.data());
    uint32_t* tchunk = begin.data() + fill_ctas + 1;
    cut(t_end, f_end, setup_thread, tchunk);
    uint32_t* fchunk = tchunk + fill_ctas + 1;
    cut(f_end, last, kSetupFar, fchunk);
    std::vector<double> mu(fill_ctas, 0.0);
    for (uint32_t c = 0; c < fill_ctas; c++)
      mu[c] = per_seg * (inv_prefix(begin[c + 1]) - inv_prefix(begin[c]) +
                         inv_prefix(tchunk[c + 1]) - inv_prefix(tchunk[c]) +
                         inv_prefix(fchunk[c + 1]) - inv_prefix(fchunk[c]));
    for (uint32_t c = 0; c < fill_ctas; c++) add_list(mu[c]);
  }
  const uint32_t lists = fill_ctas;
  if (stride > 0xffffffffull) { err = "bucket region too large"; return PSG_ERR_LIMIT; }

  const size_t need_entries = (size_t) stride * window_;
  const size_t need_counts = 2 * (size_t) lists * window_;   // counts, then spill counts
  // buffers grow only when no window can still be using them
  if (need_entries > entries_cap_ || need_counts > bcounts_cap_ || need_entries > entries2_cap_ ||
      need_counts > bcounts2_cap_)
    quiesce();
  if (need_entries > entries_cap_) {
    cudaFree(d_entries_); d_entries_ = nullptr; entries_cap_ = 0;
    if (cudaMalloc(&d_entries_, need_entries * sizeof(uint32_t)) != cudaSuccess) {
      cudaGetLastError();
      err = "cannot allocate " + std::to_string(need_entries * 4 >> 20) + " MiB of bucket storage";
      return PSG_ERR_NOMEM;
    }
    entries_cap_ = need_entries;
  }
  if (need_counts > bcounts_cap_) {
    cudaFree(d_bcounts_); d_bcounts_ = nullptr;
    PSG_CUDA(cudaMalloc(&d_bcounts_, need_counts * sizeof(uint32_t)));
    bcounts_cap_ = need_counts;
  }
  // a second set of lists lets consecutive windows overlap on two streams;
  // without the memory for it the windows run one after another
  if (need_entries > entries2_cap_ || need_counts > bcounts2_cap_) {
    cudaFree(d_entries2_); cudaFree(d_bcounts2_);
    d_entries2_ = nullptr; d_bcounts2_ = nullptr; entries2_cap_ = bcounts2_cap_ = 0;
    if (cudaMalloc(&d_entries2_, need_entries * sizeof(uint32_t)) == cudaSuccess &&
        cudaMalloc(&d_bcounts2_, need_counts * sizeof(uint32_t)) == cudaSuccess) {
      entries2_cap_ = need_entries;
      bcounts2_cap_ = need_counts;
    } else {
      cudaGetLastError();
      cudaFree(d_entries2_); cudaFree(d_bcounts2_);
      d_entries2_ = nullptr; d_bcounts2_ = nullptr;
    }
  }
  plan_.table.assign(off.begin(), off.end());
  plan_.table.insert(plan_.table.end(), cap.begin(), cap.end());
  if (fill_ctas) plan_.table.insert(plan_.table.end(), begin.begin(), begin.begin() + 3 * (fill_ctas + 1));
  plan_.first = first;
  plan_.last = last;
  plan_.geom.seg_stride = stride;
  plan_.geom.lists = lists;
  plan_.geom.fill_ctas = fill_ctas;
  plan_gen_++;
  return PSG_OK;
}

// The current plan's tables for list set `set`, uploaded on ws (the stream
// the set's windows run on, so after every earlier window that reads the
// set's copy) unless the set holds them already. The upload source is a
// pinned staging buffer that is reused only once its copy has run, so the
// host never waits for the device here.
int Engine::plan_to_slot(uint32_t set, cudaStream_t ws, std::string& err) {
  PlanSlot& sl = slots_[set];
  if (sl.gen == plan_gen_) return PSG_OK;
  const size_t n = plan_.table.size();
  // sized once for any plan of lists_ fill lists: growing
  // waits for every window in flight
  const size_t want = std::max<size_t>(n, 5 * (size_t) lists_ + 8);
  if (n > sl.cap) {
    if (sl.d_table) quiesce();        // the old table may still be read
    cudaFree(sl.d_table); sl.d_table = nullptr; sl.cap = 0;
    PSG_CUDA(cudaMalloc(&sl.d_table, want * sizeof(uint32_t)));
    sl.cap = want;
  }
  Stage& g = stages_[stage_next_];
  stage_next_ = (stage_next_ + 1) % kStages;
  if (g.used) PSG_CUDA(cudaEventSynchronize(g.ev));
  if (n > g.cap) {
    if (g.h) cudaFreeHost(g.h);
    g.h = nullptr; g.cap = 0;
    PSG_CUDA(cudaMallocHost(&g.h, want * sizeof(uint32_t)));
    g.cap = want;
  }
  if (!g.ev) PSG_CUDA(cudaEventCreateWithFlags(&g.ev, cudaEventDisableTiming));
  std::memcpy(g.h, plan_.table.data(), n * sizeof(uint32_t));
  PSG_CUDA(cudaMemcpyAsync(sl.d_table, g.h, n * sizeof(uint32_t), cudaMemcpyHostToDevice, ws));
  PSG_CUDA(cudaEventRecord(g.ev, ws));
  g.used = true;
  sl.gen = plan_gen_;
  sl.geom = plan_.geom;
  return PSG_OK;
}

// Wait for every window in flight (before bucket buffers are freed).
void Engine::quiesce() {
  cudaDeviceSynchronize();
}

void Engine::chain_begin(cudaStream_t st) {
  if (!aux_stream_ || profiling_) return;
  cudaEventRecord(fork_event_, st);
  cudaStreamWaitEvent(aux_stream_, fork_event_, 0);
  chain_ = true;
  parity_ = 0;
}

void Engine::chain_end(cudaStream_t st) {
  if (!chain_) return;
  cudaEventRecord(join_event_, aux_stream_);
  cudaStreamWaitEvent(st, join_event_, 0);
  chain_ = false;
}

void Engine::timed_begin(int which, cudaStream_t st) {
  timed_[which].launches++;
  if (!profiling_) return;
  cudaEvent_t a, b;
  cudaEventCreate(&a); cudaEventCreate(&b);
  cudaEventRecord(a, st);
  timed_[which].ev.emplace_back(a, b);
}

void Engine::timed_end(int which, cudaStream_t st) {
  if (!profiling_) return;
  cudaEventRecord(timed_[which].ev.back().second, st);
}

std::vector<KernelStat> Engine::kernel_stats() {
  std::vector<KernelStat> out;
  cudaSetDevice(device_);
  for (auto& t : timed_) {
    for (auto& e : t.ev) {
      cudaEventSynchronize(e.second);
      float ms = 0;
      cudaEventElapsedTime(&ms, e.first, e.second);
      t.ms += ms;
      cudaEventDestroy(e.first); cudaEventDestroy(e.second);
    }
    t.ev.clear();
    KernelStat k; k.name = t.name; k.launches = t.launches; k.ms = t.ms;
    out.push_back(k);
  }
  return out;
}

void Engine::reset_kernel_stats() {
  kernel_stats();
  for (auto& t : timed_) { t.launches = 0; t.ms = 0; }
}

// Bucket storage the windows of p need: per segment, every list's expected
// entries plus its margin (as ensure_buckets sizes them), times the window,
// for both list sets (consecutive windows overlap).
size_t Engine::bucket_bytes(const RangePlan& p) const {
  if (!p.buckets) return 0;
  const double per_seg = (double) seg_bytes_ * 30.0 * (8.0 / 30.0);
  const double total = per_seg * (inv_prefix(p.n_total) - inv_prefix(p.n_dir));
  const double lists = std::max<double>(1.0, std::min<double>(lists_, p.n_total - p.n_dir));
  const double mu = total / lists;
  const double stride = lists * (mu + 6.0 * std::sqrt(mu) + 36.0) * cap_scale_;
  return (size_t) (2.0 * stride * (double) window_ * 4.0);
}

// Launch-wide sieve arguments: segment size, pre-sieve tables, sieving
// primes and the wheel walk tables (range and tier fields zero).
void Engine::fill_common_args(SieveArgs& a) const {
  std::memset(&a, 0, sizeof a);
  a.seg_bytes = seg_bytes_;
  a.num_tables = (uint32_t) pat_period_.size();
  for (size_t t = 0; t < pat_period_.size(); t++) {
    a.pat_base[t] = d_pat_ + pat_off_[t];
    a.pat_period[t] = pat_period_[t];
    a.pat_stride[t] = pat_stride_[t];
    a.pat_rcp[t] = 0xffffffffffffffffull / pat_period_[t];
  }
  a.num_presieve_primes = (uint32_t) presieve_primes_.size();
  for (size_t i = 0; i < presieve_primes_.size() && i < (size_t) kMaxPresievePrimes; i++)
    a.presieve_primes[i] = presieve_primes_[i];
  a.presieve_max = presieve_max_;
  a.primes = d_primes_;
  a.recip = d_recip_;
  for (uint32_t c = 0; c < 8; c++) {
    a.wheel_tab[2 * c] = wheel_bits_packed(c);
    a.wheel_tab[2 * c + 1] = wheel_corr_packed(c);
  }
}

// Primes 1024..4096 cross off fewer times per instruction in the
// warp-cooperative tier, but as medium primes (one thread each, a few
// hundred crossings per segment) they cost fewer instructions in all; the
// longer threads then finish late, which the bucket phase's dynamically
// shared lists absorb when there are many. Measured per pass (1e11-integer
// ranges): 4096 best up to sqrt(stop) ~1e6, 2048 at ~3e6 (-0.7%), 1024 from
// ~1e7 (-1.7% at 1e14, -2.1% at 1e15, -1.3% at 1e18, -0.8% near 2^64);
// 512 and 768 slower everywhere.
uint32_t Engine::range_small_limit(uint64_t hi) const {
  if (!small_auto_) return small_limit_;
  const uint32_t sq = isqrt_u64(hi);
  return sq >= 8000000u ? 1024u : sq >= 2000000u ? 2048u : 4096u;
}

// Prime tiers and launch geometry of [lo, hi] (lo >= 7, lo <= hi).
int Engine::plan_range(uint64_t lo, uint64_t hi, RangePlan& p, std::string& err, uint32_t big_limit,
                       uint32_t small_limit) {
  const uint32_t big = big_limit ? big_limit : big_limit_;
  const uint64_t span = (uint64_t) seg_bytes_ * 30u;
  p.lo = lo;
  p.hi = hi;
  // byteRemainder (reference src/Erat.cpp:231-237, CudaBackend.cpp:457)
  p.seg_low0 = lo - ((lo - 7) % 30 + 7);
  p.nseg = (hi - 7 - p.seg_low0) / span + 1;
  const uint32_t sq = isqrt_u64(hi);
  int rc = ensure_primes(std::max<uint32_t>(sq, 7u), err);
  if (rc) return rc;
  const auto upto = [&](uint64_t v) { return count_primes_le(v, false); };
  const auto below = [&](uint64_t v) { return count_primes_le(v, true); };
  p.n_total = upto(sq);
  p.n_small = std::min(below(small_limit ? small_limit : range_small_limit(hi)), p.n_total);
  // medium primes must fit the shared-memory state area
  p.n_med = std::max(p.n_small, std::min({ below(big), p.n_total, p.n_small + state_cap_ }));
  // beyond the shared state and below big: direct tier (no state);
  // the rest go to buckets
  p.n_dir = std::max(p.n_med, std::min(below(big), p.n_total));
  p.buckets = p.n_dir < p.n_total;
  p.step = p.buckets ? window_ : (cfg_.segments_per_launch ? cfg_.segments_per_launch : p.nseg);
  return PSG_OK;
}

int Engine::run(uint64_t lo, uint64_t hi, uint32_t kinds, unsigned long long* dev_counts,
                cudaStream_t st, std::string& err) {
  RangePlan p;
  int rc = plan_range(lo, hi, p, err);
  if (rc) return rc;
  return run_windows(p, kinds, dev_counts, st, 0, p.windows(), err);
}

// Launches [w0, w0 + nw) of a planned range: one sieve launch per window of
// p.step segments, each preceded by its bucket fill when the range has big
// primes. Counts are added to dev_counts.
int Engine::run_windows(const RangePlan& p, uint32_t kinds, unsigned long long* dev_counts,
                        cudaStream_t st, uint64_t w0, uint64_t nw, std::string& err) {
  const uint64_t span = (uint64_t) seg_bytes_ * 30u;
  const uint64_t nseg = p.nseg, seg_low0 = p.seg_low0, step = p.step;
  const bool use_buckets = p.buckets;
  int rc;
  if (use_buckets) {
    rc = ensure_buckets(p.n_dir, p.n_total, err);
    if (rc) return rc;
  }

  SieveArgs a;
  fill_common_args(a);
  a.lo = p.lo; a.hi = p.hi;
  a.n_small = p.n_small;
  a.n_primes = p.n_med;
  a.n_direct = p.n_dir;
  a.kinds = kinds;
  a.counts = dev_counts;
  const bool all = (kinds & ~1u) != 0;

  const uint64_t s_first = w0 * step;
  const uint64_t s_last = std::min<uint64_t>(nseg, (w0 + nw) * step);
  // Two or more bucket windows (or any in a chain): alternate windows on st
  // with list set 0 and on the auxiliary stream with set 1, so that the fill
  // of one window can use the SMs the other window's kernels leave idle at
  // their tails. While profiling, windows run one after another so
  // that each kernel's CUDA-event time is its own.
  const bool two = use_buckets && d_entries2_ && aux_stream_ && !profiling_ &&
                   (chain_ || s_last - s_first > step);
  const bool fork = two && !chain_;
  if (!chain_) parity_ = 0;
  if (fork) {
    PSG_CUDA(cudaEventRecord(fork_event_, st));
    PSG_CUDA(cudaStreamWaitEvent(aux_stream_, fork_event_, 0));
  }
  for (uint64_t s0 = s_first; s0 < s_last; s0 += step) {
    const uint64_t ns = std::min<uint64_t>(step, nseg - s0);
    const uint64_t win_low = seg_low0 + s0 * span;
    const uint32_t set = two ? (parity_++ & 1u) : 0u;
    cudaStream_t ws = set ? aux_stream_ : st;
    uint32_t* const w_entries = set ? d_entries2_ : d_entries_;
    uint32_t* const w_counts = set ? d_bcounts2_ : d_bcounts_;
    a.seg_low0 = win_low;
    a.num_segments = ns;
    if (use_buckets) {
      rc = plan_to_slot(set, ws, err);
      if (rc) return rc;
      const PlanGeom& gm = slots_[set].geom;
      const uint32_t* const t_off = slots_[set].d_table;      // [lists] list offsets
      const uint32_t* const t_cap = t_off + gm.lists;        // [lists] capacities
      const uint32_t* const t_chunk = t_cap + gm.lists;      // fill chunk bounds
      if (gm.fill_ctas) {
        BucketArgs b;
        std::memset(&b, 0, sizeof b);
        b.win_low = win_low;
        b.sqrt_x0 = isqrt_u64(win_low + 6u);
        b.win_segments = (uint32_t) ns;
        b.seg_bytes = seg_bytes_;
        b.seg_magic = (uint32_t) ((1ull << 32) / seg_bytes_ + 1u);
        b.seg_shift = seg_shift_;
        // steps per tile (up to two entries per lane and step): with the
        // staggered starts spreading a tile's entries over the window, a bin
        // expects ~80% of its slots per tile (the overflow spills to the
        // list's top); the thread walk flushes at 60%
        b.tile_steps = std::max<uint32_t>(1u, (uint32_t) (kTileFill * kBinCap * (double) ns / kBucketBlock));
        b.flush_at = (uint32_t) (kFlushFill * kBinCap * (double) ns);
        b.stagger_below = (uint32_t) std::min<uint64_t>(((uint64_t) ns * seg_bytes_) / kStaggerMultiples, 0xffffffffull);
        for (uint32_t c = 0; c < 8; c++) {
          b.wheel_tab[2 * c] = wheel_bits_packed(c);
          b.wheel_tab[2 * c + 1] = wheel_corr_packed(c);
        }
        b.primes = d_primes_;
        b.recip = d_recip_;
        b.chunk_begin = t_chunk;
        b.thread_chunk = t_chunk + gm.fill_ctas + 1;
        b.far_chunk = t_chunk + 2 * (gm.fill_ctas + 1);
        b.num_lists = gm.lists;
        b.list_off = t_off;
        b.list_cap = t_cap;
        b.seg_stride = gm.seg_stride;
        b.entries = w_entries;
        b.counts = w_counts;
        b.spill = w_counts + (size_t) gm.lists * window_;
        b.overflow = cur_overflow_;
        b.entry_total = d_entry_total_;
        timed_begin(1, ws);
        if (seg_pow2_)
          bucket_fill_kernel<kBucketBlock, true><<<gm.fill_ctas, kBucketBlock, fill_smem_bytes((uint32_t) ns), ws>>>(b);
        else
          bucket_fill_kernel<kBucketBlock, false><<<gm.fill_ctas, kBucketBlock, fill_smem_bytes((uint32_t) ns), ws>>>(b);
        timed_end(1, ws);
        PSG_CUDA(cudaGetLastError());
      }
      a.bucket_entries = w_entries;
      a.bucket_counts = w_counts;
      a.bucket_spill = w_counts + (size_t) gm.lists * window_;
      a.bucket_list_off = t_off;
      a.bucket_list_cap = t_cap;
      a.bucket_seg_stride = gm.seg_stride;
      a.num_bucket_lists = gm.lists;
    }
    const uint32_t g = (uint32_t) std::min<uint64_t>(grid_, ns);
    a.bitmap_out = bitmap_out_ ? bitmap_out_ + (s0 - s_first) * seg_bytes_ : nullptr;
    timed_begin(0, ws);
    cudaError_t e = launch_sieve(block_, all, g, smem_dyn_, ws, a);
    timed_end(0, ws);
    if (e != cudaSuccess) {
      err = std::string("sieve kernel launch: ") + cudaGetErrorString(e);
      return PSG_ERR_CUDA;
    }
  }
  if (fork) {
    PSG_CUDA(cudaEventRecord(join_event_, aux_stream_));
    PSG_CUDA(cudaStreamWaitEvent(st, join_event_, 0));
  }
  return PSG_OK;
}

int Engine::count_ordered(uint64_t start, uint64_t stop, uint32_t kinds, unsigned long long* dev_counts,
                          cudaStream_t stream, uint32_t* flag, std::string& err) {
  PSG_CUDA(cudaSetDevice(device_));
  cudaStream_t st = stream ? stream : stream_;
  // The engine's scratch (bucket lists) is shared by all counts of this
  // context: order this count after the previous one, whatever stream that
  // one ran on.
  if (last_stream_ && last_stream_ != st) PSG_CUDA(cudaStreamWaitEvent(st, done_event_, 0));
  cur_overflow_ = flag;
  int rc = count_enqueue(start, stop, kinds, dev_counts, st, err);
  cur_overflow_ = d_overflow_;
  PSG_CUDA(cudaEventRecord(done_event_, st));
  last_stream_ = st;
  return rc;
}

// Asynchronous counts cannot recount on an overflow; their fill kernels
// raise a flag of their own, which only async_status reads and clears, so
// no synchronous path's reset of d_overflow_ can hide it.
int Engine::count_async(uint64_t start, uint64_t stop, uint32_t kinds,
                        unsigned long long* dev_counts, cudaStream_t stream, std::string& err) {
  async_pending_ = true;
  return count_ordered(start, stop, kinds, dev_counts, stream, d_async_overflow_, err);
}

int Engine::async_status(std::string& err) {
  PSG_CUDA(cudaSetDevice(device_));
  if (!async_pending_) return PSG_OK;
  PSG_CUDA(cudaEventSynchronize(done_event_));
  PSG_CUDA(cudaMemcpyAsync(h_counts_ + 7, d_async_overflow_, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
  PSG_CUDA(cudaMemsetAsync(d_async_overflow_, 0, sizeof(uint32_t), stream_));
  PSG_CUDA(cudaStreamSynchronize(stream_));
  async_pending_ = false;
  if ((uint32_t) (h_counts_[7] & 0xffffffffu)) {
    grow_bucket_lists();
    err = "a bucket list overflowed during an asynchronous count: its counts are too high; count again";
    return PSG_ERR_OVERFLOW;
  }
  return PSG_OK;
}

int Engine::count_enqueue(uint64_t start, uint64_t stop, uint32_t kinds,
                          unsigned long long* dev_counts, cudaStream_t st, std::string& err) {
  kinds &= 0x3fu;
  if (start > stop || kinds == 0) return PSG_OK;
  uint64_t tab[6] = { 0, 0, 0, 0, 0, 0 };
  small_table(start, stop, kinds, tab);
  if (tab[0] | tab[1] | tab[2] | tab[3] | tab[4]) {
    add_counts_kernel<<<1, 32, 0, st>>>(dev_counts, tab[0], tab[1], tab[2], tab[3], tab[4], tab[5]);
    PSG_CUDA(cudaGetLastError());
  }
  if (stop < 7) return PSG_OK;
  const uint64_t lo = std::max<uint64_t>(start, 7);
  return run(lo, stop, kinds, dev_counts, st, err);
}

int Engine::count(uint64_t start, uint64_t stop, uint32_t kinds, uint64_t counts[6], std::string& err) {
  for (int i = 0; i < 6; i++) counts[i] = 0;
  PSG_CUDA(cudaSetDevice(device_));
  kinds &= 0x3fu;
  if (start > stop || kinds == 0) return PSG_OK;
  for (int attempt = 0; attempt < 4; attempt++) {
    PSG_CUDA(cudaMemsetAsync(d_counts_, 0, 6 * sizeof(unsigned long long), stream_));
    PSG_CUDA(cudaMemsetAsync(d_overflow_, 0, sizeof(uint32_t), stream_));
    int rc = count_ordered(start, stop, kinds, d_counts_, stream_, d_overflow_, err);
    if (rc) return rc;
    PSG_CUDA(cudaMemcpyAsync(h_counts_, d_counts_, 6 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_));
    PSG_CUDA(cudaMemcpyAsync(h_counts_ + 6, d_overflow_, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
    PSG_CUDA(cudaStreamSynchronize(stream_));
    const uint32_t overflow = (uint32_t) (h_counts_[6] & 0xffffffffu);
    if (!overflow) {
      for (int i = 0; i < 6; i++) counts[i] = ((kinds >> i) & 1u) ? h_counts_[i] : 0;
      return PSG_OK;
    }
    // a bucket list overflowed: recount with larger lists
    overflow_retries_++;
    cap_scale_ *= 2.0;
    plan_.last = 0;
  }
  err = "bucket lists kept overflowing";
  return PSG_ERR_INTERNAL;
}

uint64_t Engine::bucket_entries() {
  unsigned long long v = 0;
  cudaSetDevice(device_);
  cudaStreamSynchronize(stream_);
  cudaMemcpy(&v, d_entry_total_, sizeof v, cudaMemcpyDeviceToHost);
  return v;
}

void Engine::reset_bucket_entries() {
  cudaSetDevice(device_);
  cudaMemset(d_entry_total_, 0, sizeof(unsigned long long));
}

std::string Engine::describe() const {
  char buf[512];
  std::snprintf(buf, sizeof buf,
                "[%d] CUDA: %s (compute %d.%d), %d SMs, %llu MiB, segment %u B x %u threads, grid %u",
                device_, prop_.name, prop_.major, prop_.minor, prop_.multiProcessorCount,
                (unsigned long long) (prop_.totalGlobalMem >> 20), seg_bytes_, block_, grid_);
  return buf;
}

} // namespace psg
