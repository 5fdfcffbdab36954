// extract.cu -- prime extraction and nth_prime on the GPU.
//
// generate_primes: the range path runs window by window with the sieve
// kernel storing its masked segments; extract_kernel turns each window's
// bitmap into ascending values (count pass, host scan, emit pass).
// nth_prime: exact GPU counts bracket the answer (an estimate from the
// logarithmic integral, then interpolation probes counted from the nearer
// bracket end), and the last bracket's bitmap is decoded on the host.
// Semantics follow primesieve's nth_prime (src/nthPrime.cpp:47-181): n > 0
// the nth prime > start, n = 0 as n = 1, n < 0 the |n|th prime < start, with
// the same error messages.
#include "engine.hpp"
#include "extract_kernel.cuh"
#include "../../include/psgpu.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace psg {

namespace {

#define PSG_CUDA(call)                                                          \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      err = std::string(#call) + ": " + cudaGetErrorString(e_);                 \
      return PSG_ERR_CUDA;                                                      \
    }                                                                           \
  } while (0)

constexpr uint64_t kMaxU64 = ~0ull;
constexpr uint64_t kPiOf2To64 = 425656284035217743ull;   // number of primes below 2^64
constexpr uint64_t kFinalSpan = 1ull << 27;               // bracket decoded from one bitmap

// li(x) = gamma + ln ln x + sum_{k>=1} (ln x)^k / (k k!)  (x > 1)
double log_integral(double x) {
  if (x <= 2.0) return 1.045;
  const double L = std::log(x);
  double term = 1.0, sum = 0.0;
  for (int k = 1; k < 200; k++) {
    term *= L / k;
    const double t = term / k;
    sum += t;
    if (t < 1e-17 * sum) break;
  }
  return 0.5772156649015329 + std::log(L) + sum;
}

// x with li(x) ~ k (Newton on li, li'(x) = 1/ln x)
double inverse_log_integral(double k) {
  if (k < 2.0) return 2.0;
  double x = k * std::log(k) + 2.0;
  for (int i = 0; i < 40; i++) {
    const double nx = x - (log_integral(x) - k) * std::log(x);
    if (!(nx > 2.0)) return 2.0;
    if (std::fabs(nx - x) < 0.5) { x = nx; break; }
    x = nx;
  }
  return x;
}

uint64_t clamp_u64(double v, uint64_t lo, uint64_t hi) {
  if (!(v > (double) lo)) return lo;
  if (v >= 1.8446744073709552e19) return hi;
  const uint64_t u = (uint64_t) v;
  return std::min(std::max(u, lo), hi);
}

const uint32_t kBitOffset[8] = { 7, 11, 13, 17, 19, 23, 29, 31 };

} // namespace

uint64_t Engine::count_range(uint64_t lo, uint64_t hi, std::string& err, int& rc) {
  uint64_t c[6];
  rc = count(lo, hi, 1u, c, err);
  return c[0];
}

int Engine::sieve_bitmap(uint64_t lo, uint64_t hi, uint64_t& seg_low0, std::vector<uint8_t>& bits,
                         std::string& err) {
  RangePlan p;
  int rc = plan_range(lo, hi, p, err);
  if (rc) return rc;
  seg_low0 = p.seg_low0;
  const size_t bytes = (size_t) p.nseg * seg_bytes_;
  uint8_t* d_bits = nullptr;
  if (cudaMalloc(&d_bits, bytes) != cudaSuccess) {
    cudaGetLastError();
    err = "cannot allocate the sieve bitmap";
    return PSG_ERR_NOMEM;
  }
  bits.resize(bytes);
  cudaError_t e = cudaSuccess;
  for (int attempt = 0; attempt < 4; attempt++) {
    uint32_t overflow = 0;
    bitmap_out_ = d_bits;
    e = cudaMemsetAsync(overflow_flag(), 0, sizeof(uint32_t), stream_);
    if (e == cudaSuccess) rc = run_windows(p, 1u, d_counts_, stream_, 0, p.windows(), err);
    bitmap_out_ = nullptr;
    if (e == cudaSuccess && rc == PSG_OK) e = cudaMemcpyAsync(bits.data(), d_bits, bytes, cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess && rc == PSG_OK) e = cudaMemcpyAsync(&overflow, overflow_flag(), sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (rc || e != cudaSuccess || !overflow) break;
    grow_bucket_lists();                      // a bucket list overflowed: sieve again
    if (attempt == 3) { err = "bucket lists kept overflowing"; rc = PSG_ERR_INTERNAL; }
  }
  cudaFree(d_bits);
  if (rc) return rc;
  if (e != cudaSuccess) { err = std::string("sieve bitmap: ") + cudaGetErrorString(e); return PSG_ERR_CUDA; }
  return PSG_OK;
}

int Engine::generate_primes(uint64_t start, uint64_t stop, std::vector<uint64_t>& out, std::string& err) {
  PSG_CUDA(cudaSetDevice(device_));
  if (start > stop) return PSG_OK;
  for (uint64_t q : { 2ull, 3ull, 5ull })
    if (q >= start && q <= stop) out.push_back(q);
  if (stop < 7) return PSG_OK;
  RangePlan p;
  int rc = plan_range(std::max<uint64_t>(start, 7), stop, p, err);
  if (rc) return rc;
  // launches of at most one bucket window each, so one window's bitmap is
  // all the device holds at a time
  p.step = std::min<uint64_t>(p.step, window_);
  const size_t win_bytes = (size_t) p.step * seg_bytes_;
  uint8_t* d_bits = nullptr;
  uint32_t* d_cnt = nullptr;
  uint64_t* d_off = nullptr;
  uint64_t* d_out = nullptr;
  size_t out_cap = 0;
  const size_t max_blocks = (win_bytes + kExtractBlockBytes - 1) / kExtractBlockBytes;
  auto cleanup = [&]() { cudaFree(d_bits); cudaFree(d_cnt); cudaFree(d_off); cudaFree(d_out); };
  if (cudaMalloc(&d_bits, win_bytes) != cudaSuccess || cudaMalloc(&d_cnt, max_blocks * 4) != cudaSuccess ||
      cudaMalloc(&d_off, max_blocks * 8) != cudaSuccess) {
    cudaGetLastError(); cleanup();
    err = "cannot allocate the prime extraction buffers";
    return PSG_ERR_NOMEM;
  }
  std::vector<uint32_t> cnt(max_blocks);
  std::vector<uint64_t> off(max_blocks);
  const uint64_t nwin = p.windows();
  for (uint64_t w = 0; w < nwin; w++) {
    const uint64_t s0 = w * p.step;
    const uint64_t ns = std::min<uint64_t>(p.step, p.nseg - s0);
    const uint64_t bytes = ns * seg_bytes_;
    const uint64_t nblocks = (bytes + kExtractBlockBytes - 1) / kExtractBlockBytes;
    for (int attempt = 0;; attempt++) {
      uint32_t overflow = 0;
      bitmap_out_ = d_bits;
      cudaError_t e = cudaMemsetAsync(overflow_flag(), 0, sizeof(uint32_t), stream_);
      if (e == cudaSuccess) rc = run_windows(p, 1u, d_counts_, stream_, w, 1, err);
      bitmap_out_ = nullptr;
      if (e == cudaSuccess && rc == PSG_OK)
        e = cudaMemcpyAsync(&overflow, overflow_flag(), sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_);
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
      if (rc) { cleanup(); return rc; }
      if (e != cudaSuccess) { cleanup(); err = std::string("prime extraction: ") + cudaGetErrorString(e); return PSG_ERR_CUDA; }
      if (!overflow) break;
      grow_bucket_lists();                    // a bucket list overflowed: sieve the window again
      if (attempt == 3) { cleanup(); err = "bucket lists kept overflowing"; return PSG_ERR_INTERNAL; }
    }
    ExtractArgs x;
    std::memset(&x, 0, sizeof x);
    x.bitmap = d_bits;
    x.bytes = bytes;
    x.base = p.seg_low0 + s0 * (uint64_t) seg_bytes_ * 30u;
    x.block_counts = d_cnt;
    x.block_offsets = d_off;
    const uint32_t grid = (uint32_t) std::min<uint64_t>(nblocks, 8ull * prop_.multiProcessorCount);
    x.pass = 0;
    extract_kernel<<<grid, kExtractThreads, 0, stream_>>>(x);
    cudaError_t e = cudaMemcpyAsync(cnt.data(), d_cnt, nblocks * 4, cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) { cleanup(); err = std::string("prime extraction: ") + cudaGetErrorString(e); return PSG_ERR_CUDA; }
    uint64_t total = 0;
    for (uint64_t i = 0; i < nblocks; i++) { off[i] = total; total += cnt[i]; }
    if (total == 0) continue;
    if (total > out_cap) {
      cudaFree(d_out);
      d_out = nullptr;
      out_cap = 0;
      if (cudaMalloc(&d_out, total * 8) != cudaSuccess) {
        cudaGetLastError(); cleanup();
        err = "cannot allocate the prime output buffer";
        return PSG_ERR_NOMEM;
      }
      out_cap = total;
    }
    x.pass = 1;
    x.out = d_out;
    e = cudaMemcpyAsync(d_off, off.data(), nblocks * 8, cudaMemcpyHostToDevice, stream_);
    extract_kernel<<<grid, kExtractThreads, 0, stream_>>>(x);
    const size_t old = out.size();
    out.resize(old + total);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out.data() + old, d_out, total * 8, cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) { cleanup(); err = std::string("prime extraction: ") + cudaGetErrorString(e); return PSG_ERR_CUDA; }
  }
  cleanup();
  return PSG_OK;
}

int Engine::nth_prime(int64_t n, uint64_t start, uint64_t& prime, std::string& err) {
  PSG_CUDA(cudaSetDevice(device_));
  prime = 0;
  int rc = PSG_OK;
  const bool down = n < 0;
  // |n| without overflow for INT64_MIN
  uint64_t k = down ? (uint64_t) (~n) + 1u : (uint64_t) n;
  if (down) {
    if (k >= start) { err = "nth_prime(n): abs(n) must be < start"; return PSG_ERR_ARG; }
    if (k > kPiOf2To64) { err = "nth_prime(n): abs(n) must be <= " + std::to_string(kPiOf2To64); return PSG_ERR_ARG; }
  } else {
    if (k == 0) k = 1;
    if (k > kPiOf2To64) { err = "nth_prime(n): n must be <= " + std::to_string(kPiOf2To64); return PSG_ERR_ARG; }
    if (start == kMaxU64) { err = "cannot generate primes > 2^64"; return PSG_ERR_LIMIT; }
  }
  // the primes below 7 are not in the bit arrays: count them on the host
  const auto count = [&](uint64_t a, uint64_t b) -> uint64_t {
    if (a > b) return 0;
    uint64_t c = 0;
    for (uint64_t q : { 2ull, 3ull, 5ull })
      if (q >= a && q <= b) c++;
    if (b < 7 || rc) return c;
    return c + count_range(std::max<uint64_t>(a, 7), b, err, rc);
  };
  // Bracket on the counting axis: upward, c(x) = pi[start+1, x], find the
  // smallest x with c(x) >= k; downward, c(x) = pi[x, start-1], find the
  // largest x with c(x) >= k. (a, ca) is on the short side, (b, cb) on the
  // reaching side; |b - a| shrinks until it fits one bitmap.
  const uint64_t origin = down ? start - 1 : start + 1;
  const double est_pi = log_integral((double) start);
  const double target = down ? est_pi - (double) k : est_pi + (double) k;
  const uint64_t guess = down ? clamp_u64(inverse_log_integral(target), 2, origin)
                              : clamp_u64(inverse_log_integral(target), origin, kMaxU64);
  // c(x) for a probe x, counted from the nearer known point
  uint64_t a = origin, ca = 0;          // c(a) < k (a is "just outside" for down: see below)
  bool have_a = false;                  // a/ca describe a point with c < k
  uint64_t b = 0, cb = 0;
  bool have_b = false;
  const auto c_full = [&](uint64_t x) { return down ? count(x, origin) : count(origin, x); };
  {
    const uint64_t c = c_full(guess);
    if (rc) return rc;
    if (c >= k) { b = guess; cb = c; have_b = true; } else { a = guess; ca = c; have_a = true; }
  }
  // extend outward until the bracket reaches k
  while (!have_b) {
    const double gap = std::log(std::max<double>((double) a, 8.0)) + 2.0;
    const double step = 1.25 * (double) (k - ca) * gap + 1e4;
    if (down) {
      const uint64_t nb = (a <= 2 + (uint64_t) step) ? 2 : a - (uint64_t) step;
      const uint64_t c = ca + count(nb, a - 1);
      if (rc) return rc;
      if (c >= k) { b = nb; cb = c; have_b = true; }
      else if (nb == 2) { err = "nth_prime(n): invalid n, nth prime < 2 is impossible!"; return PSG_ERR_ARG; }
      else { a = nb; ca = c; }
    } else {
      const uint64_t nb = (kMaxU64 - a <= (uint64_t) step) ? kMaxU64 : a + (uint64_t) step;
      const uint64_t c = ca + count(a + 1, nb);
      if (rc) return rc;
      if (c >= k) { b = nb; cb = c; have_b = true; }
      else if (nb == kMaxU64) { err = "cannot generate primes > 2^64"; return PSG_ERR_LIMIT; }
      else { a = nb; ca = c; }
    }
  }
  if (!have_a) { a = down ? origin + 1 : origin - 1; ca = 0; }   // c = 0 just past the origin
  // shrink: interpolate where c reaches k, count from the nearer end
  const auto dist = [&](uint64_t x, uint64_t y) { return x > y ? x - y : y - x; };
  for (int it = 0; dist(a, b) > kFinalSpan; it++) {
    const double frac = (double) (k - ca) / (double) std::max<uint64_t>(cb - ca, 1);
    double d = frac * (double) dist(a, b);
    if (it % 3 == 2) d = 0.5 * (double) dist(a, b);          // guaranteed halving now and then
    uint64_t off = (uint64_t) std::max(1.0, std::min(d, (double) dist(a, b) - 1.0));
    const uint64_t m = down ? a - off : a + off;
    uint64_t cm;
    if (off <= dist(a, b) / 2) cm = ca + (down ? count(m, a - 1) : count(a + 1, m));
    else cm = cb - (down ? count(b, m - 1) : count(m + 1, b));
    if (rc) return rc;
    if (cm >= k) { b = m; cb = cm; } else { a = m; ca = cm; }
  }
  // decode the last bracket: the (k - ca)-th prime walking away from a
  const uint64_t lo = down ? b : a + 1, hi = down ? a - 1 : b;
  std::vector<uint64_t> small;
  for (uint64_t q : { 2ull, 3ull, 5ull })
    if (q >= lo && q <= hi) small.push_back(q);
  std::vector<uint64_t> vals(small);
  if (hi >= 7) {
    uint64_t seg_low0 = 0;
    std::vector<uint8_t> bits;
    rc = sieve_bitmap(std::max<uint64_t>(lo, 7), hi, seg_low0, bits, err);
    if (rc) return rc;
    for (size_t i = 0; i < bits.size(); i++)
      for (uint32_t bt = 0; bt < 8; bt++)
        if ((bits[i] >> bt) & 1u) vals.push_back(seg_low0 + 30ull * i + kBitOffset[bt]);
  }
  const uint64_t need = k - ca;           // >= 1
  if (need > vals.size()) { err = "nth_prime: inconsistent counts"; return PSG_ERR_INTERNAL; }
  prime = down ? vals[vals.size() - need] : vals[need - 1];
  return PSG_OK;
}

} // namespace psg
