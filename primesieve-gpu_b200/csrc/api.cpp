// api.cpp -- primesieve-compatible C and C++ API over the psg_* ABI:
// counts, nth_prime and prime generation.
//
// Mirrors the reference's public counting API (src/api.cpp:48-118,
// src/api-c.cpp:143-225) and its GPU API (src/gpu/GpuSieve.cpp:184-365):
// one lazily created process-wide engine context, one process-wide mutex,
// knobs that recreate the context. Unlike the reference there is no CPU
// sieve behind it: every count runs on the GPU, and a GPU failure is an
// error (primesieve_error in C++, PRIMESIEVE_ERROR + errno = EDOM in C).
#include "../../include/primesieve.h"
#include "../../include/primesieve.hpp"
#include "../../include/primesieve/gpu.hpp"
#include "../../include/psgpu.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cerrno>
#include <iostream>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

std::mutex g_mutex;
int g_device = -1;
bool g_enabled = false;
psg_config g_config = {};
psg_context* g_ctx = nullptr;
std::string g_last_error;
int g_sieve_size = 0;     // CPU knob, reported back only
int g_num_threads = 0;    // CPU knob, reported back only

void reset_context_locked() {
  if (g_ctx) {
    psg_destroy(g_ctx);
    g_ctx = nullptr;
  }
}

// Engine for the selected device, created on first use (reference
// activeBackend(), src/gpu/GpuSieve.cpp:120-129). nullptr + g_last_error on
// failure.
psg_context* context_locked() {
  if (!g_ctx) {
    psg_context* c = nullptr;
    int rc = psg_init(g_device, &g_config, &c);
    if (rc != PSG_OK) {
      g_last_error = psg_last_error();
      if (g_last_error.empty()) g_last_error = psg_status_string(rc);
      return nullptr;
    }
    g_ctx = c;
  }
  return g_ctx;
}

// Count kinds `mask` of [start, stop]; throws primesieve_error on failure.
void count_locked(uint64_t start, uint64_t stop, uint32_t mask, uint64_t out[6]) {
  psg_context* c = context_locked();
  if (!c) throw primesieve::primesieve_error("GPU is not available: " + g_last_error);
  int rc = psg_count(c, start, stop, mask, out);
  if (rc != PSG_OK) {
    g_last_error = psg_last_error();
    // A failed context is rebuilt on the next call (reference
    // gpu_try_count resets the backend, src/gpu/GpuSieve.cpp:357-363).
    reset_context_locked();
    throw primesieve::primesieve_error("GPU count failed: " + g_last_error);
  }
}

uint64_t count_kind(uint64_t start, uint64_t stop, int kind) {
  std::lock_guard<std::mutex> lock(g_mutex);
  uint64_t out[6] = { 0, 0, 0, 0, 0, 0 };
  count_locked(start, stop, 1u << kind, out);
  return out[kind];
}

uint64_t c_count(const char* name, uint64_t start, uint64_t stop, int kind) {
  try {
    return count_kind(start, stop, kind);
  } catch (const std::exception& e) {
    std::cerr << name << ": " << e.what() << std::endl;
    errno = EDOM;
    return PRIMESIEVE_ERROR;
  }
}

// psg status -> primesieve_error with the engine's message (argument errors
// keep the reference's wording, e.g. "nth_prime(n): abs(n) must be < start")
[[noreturn]] void throw_status(int rc) {
  g_last_error = psg_last_error();
  if (rc == PSG_ERR_CUDA || rc == PSG_ERR_NO_DEVICE || rc == PSG_ERR_INTERNAL) reset_context_locked();
  throw primesieve::primesieve_error(g_last_error.empty() ? psg_status_string(rc) : g_last_error);
}

psg_context* require_context_locked() {
  psg_context* c = context_locked();
  if (!c) throw primesieve::primesieve_error("GPU is not available: " + g_last_error);
  return c;
}

void generate_locked(uint64_t start, uint64_t stop, std::vector<uint64_t>& out) {
  psg_context* c = require_context_locked();
  if (start > stop) return;
  // capacity: an upper bound of pi(stop) - pi(start) first, the exact count
  // if that was short
  const double x = std::max(100.0, (double) stop);
  size_t cap = (size_t) ((double) (stop - start) / (std::log(x) - 1.1) + 16.0);
  for (int attempt = 0; attempt < 2; attempt++) {
    const size_t old = out.size();
    out.resize(old + cap);
    size_t n = 0;
    const int rc = psg_generate_primes(c, start, stop, out.data() + old, cap, &n);
    if (rc == PSG_OK) { out.resize(old + n); return; }
    out.resize(old);
    if (rc != PSG_ERR_LIMIT) throw_status(rc);
    cap = n;
  }
  throw primesieve::primesieve_error("generate_primes: inconsistent prime count");
}

uint64_t nth_prime_locked(int64_t n, uint64_t start) {
  psg_context* c = require_context_locked();
  uint64_t p = 0;
  const int rc = psg_nth_prime(c, n, start, &p);
  if (rc != PSG_OK) throw_status(rc);
  return p;
}

template <typename T>
void* c_generate(const char* name, uint64_t start, uint64_t stop, uint64_t n, bool first_n, size_t* size) {
  try {
    std::vector<T> v;
    if (first_n) primesieve::generate_n_primes(n, start, &v);
    else primesieve::generate_primes(start, stop, &v);
    if (size) *size = v.size();
    if (v.empty()) return nullptr;
    T* out = static_cast<T*>(std::malloc(v.size() * sizeof(T)));
    if (!out) throw std::bad_alloc();
    std::copy(v.begin(), v.end(), out);
    return out;
  } catch (const std::exception& e) {
    if (size) *size = 0;
    std::cerr << name << ": " << e.what() << std::endl;
    errno = EDOM;
    return nullptr;
  }
}

void* c_generate_typed(const char* name, uint64_t start, uint64_t stop, uint64_t n, bool first_n,
                       size_t* size, int type) {
  switch (type) {
    case SHORT_PRIMES:     return c_generate<short>(name, start, stop, n, first_n, size);
    case USHORT_PRIMES:    return c_generate<unsigned short>(name, start, stop, n, first_n, size);
    case INT_PRIMES:       return c_generate<int>(name, start, stop, n, first_n, size);
    case UINT_PRIMES:      return c_generate<unsigned int>(name, start, stop, n, first_n, size);
    case LONG_PRIMES:      return c_generate<long>(name, start, stop, n, first_n, size);
    case ULONG_PRIMES:     return c_generate<unsigned long>(name, start, stop, n, first_n, size);
    case LONGLONG_PRIMES:  return c_generate<long long>(name, start, stop, n, first_n, size);
    case ULONGLONG_PRIMES: return c_generate<unsigned long long>(name, start, stop, n, first_n, size);
    case INT16_PRIMES:     return c_generate<int16_t>(name, start, stop, n, first_n, size);
    case UINT16_PRIMES:    return c_generate<uint16_t>(name, start, stop, n, first_n, size);
    case INT32_PRIMES:     return c_generate<int32_t>(name, start, stop, n, first_n, size);
    case UINT32_PRIMES:    return c_generate<uint32_t>(name, start, stop, n, first_n, size);
    case INT64_PRIMES:     return c_generate<int64_t>(name, start, stop, n, first_n, size);
    case UINT64_PRIMES:    return c_generate<uint64_t>(name, start, stop, n, first_n, size);
  }
  if (size) *size = 0;
  std::cerr << name << ": Invalid type parameter!" << std::endl;
  errno = EDOM;
  return nullptr;
}

int max_threads() {
  unsigned n = std::thread::hardware_concurrency();
  return n ? (int) n : 1;
}

} // namespace

// ---------------------------------------------------------------------------
// C++ API
// ---------------------------------------------------------------------------
namespace primesieve {

uint64_t count_primes(uint64_t start, uint64_t stop) { return count_kind(start, stop, 0); }
uint64_t count_twins(uint64_t start, uint64_t stop) { return count_kind(start, stop, 1); }
uint64_t count_triplets(uint64_t start, uint64_t stop) { return count_kind(start, stop, 2); }
uint64_t count_quadruplets(uint64_t start, uint64_t stop) { return count_kind(start, stop, 3); }
uint64_t count_quintuplets(uint64_t start, uint64_t stop) { return count_kind(start, stop, 4); }
uint64_t count_sextuplets(uint64_t start, uint64_t stop) { return count_kind(start, stop, 5); }

std::array<uint64_t, 6> count_all(uint64_t start, uint64_t stop) {
  std::lock_guard<std::mutex> lock(g_mutex);
  std::array<uint64_t, 6> out{};
  count_locked(start, stop, PSG_ALL_KINDS, out.data());
  return out;
}

uint64_t nth_prime(int64_t n, uint64_t start) {
  std::lock_guard<std::mutex> lock(g_mutex);
  return nth_prime_locked(n, start);
}

void generate_primes_u64(uint64_t start, uint64_t stop, std::vector<uint64_t>& out) {
  std::lock_guard<std::mutex> lock(g_mutex);
  generate_locked(start, stop, out);
}

void generate_n_primes_u64(uint64_t n, uint64_t start, std::vector<uint64_t>& out) {
  if (n == 0) return;
  std::lock_guard<std::mutex> lock(g_mutex);
  // the nth prime >= start is the nth prime > start - 1
  const uint64_t last = (start == 0) ? nth_prime_locked((int64_t) n, 0)
                                     : nth_prime_locked((int64_t) n, start - 1);
  generate_locked(start, last, out);
}

void check_element_type(const char* fn, int bits, bool is_signed, const char* name, uint64_t largest) {
  const uint64_t max = is_signed ? ((1ull << (bits - 1)) - 1) : (bits >= 64 ? ~0ull : (1ull << bits) - 1);
  if (largest > max)
    throw primesieve_error(std::string(fn) + ": " + name + " is too narrow for generating primes up to " +
                           std::to_string(largest));
}

uint64_t get_max_stop() { return ~(uint64_t) 0; }

int get_sieve_size() {
  std::lock_guard<std::mutex> lock(g_mutex);
  return g_sieve_size ? g_sieve_size : 256;
}

int get_num_threads() {
  std::lock_guard<std::mutex> lock(g_mutex);
  return g_num_threads ? g_num_threads : max_threads();
}

void set_sieve_size(int size) {
  std::lock_guard<std::mutex> lock(g_mutex);
  g_sieve_size = std::min(std::max(size, 16), 8192);     // reference src/api.cpp:174-177
}

void set_num_threads(int threads) {
  std::lock_guard<std::mutex> lock(g_mutex);
  g_num_threads = std::min(std::max(threads, 1), max_threads());
}

std::string primesieve_version() { return PRIMESIEVE_VERSION; }

// ---- GPU API ----------------------------------------------------------------

bool gpu_available() {
  std::lock_guard<std::mutex> lock(g_mutex);
  int n = 0;
  psg_device_count(&n);
  return n > 0;
}

std::vector<std::string> gpu_devices() {
  std::lock_guard<std::mutex> lock(g_mutex);
  int n = 0;
  psg_device_count(&n);
  std::vector<std::string> out;
  for (int i = 0; i < n; i++) {
    char buf[512];
    if (psg_device_describe(i, buf, sizeof buf) == PSG_OK) out.push_back(buf);
  }
  return out;
}

void set_gpu_device(int device) {
  std::lock_guard<std::mutex> lock(g_mutex);
  if (device != g_device) {
    g_device = device;
    reset_context_locked();
  }
}

int get_gpu_device() {
  std::lock_guard<std::mutex> lock(g_mutex);
  return g_device;
}

void set_gpu_enabled(bool enable) {
  std::lock_guard<std::mutex> lock(g_mutex);
  g_enabled = enable;
}

bool get_gpu_enabled() {
  std::lock_guard<std::mutex> lock(g_mutex);
  return g_enabled;
}

void set_gpu_sieve_size(int kilobytes) {
  std::lock_guard<std::mutex> lock(g_mutex);
  g_config.seg_bytes = kilobytes > 0 ? (uint32_t) kilobytes * 1024u : 0u;
  reset_context_locked();
}

void set_gpu_work_group_size(int size) {
  std::lock_guard<std::mutex> lock(g_mutex);
  g_config.block = size > 0 ? (uint32_t) size : 0u;
  reset_context_locked();
}

void set_gpu_segments_per_launch(int segments) {
  std::lock_guard<std::mutex> lock(g_mutex);
  g_config.segments_per_launch = segments > 0 ? (uint32_t) segments : 0u;
  reset_context_locked();
}

void set_gpu_presieve(bool enable) {
  std::lock_guard<std::mutex> lock(g_mutex);
  // psg_config: 0 = auto (on); 2 = explicitly off
  g_config.presieve = enable ? 1u : 2u;
  reset_context_locked();
}

std::string gpu_active_device() {
  std::lock_guard<std::mutex> lock(g_mutex);
  psg_context* c = context_locked();
  if (!c) return std::string();
  char buf[512];
  if (psg_describe(c, buf, sizeof buf) != PSG_OK) return std::string();
  return buf;
}

std::string gpu_last_error() {
  std::lock_guard<std::mutex> lock(g_mutex);
  return g_last_error;
}

bool gpu_worthwhile(uint64_t start, uint64_t stop) { return start <= stop; }

uint64_t gpu_count_primes(uint64_t start, uint64_t stop) { return count_kind(start, stop, 0); }
uint64_t gpu_count_twins(uint64_t start, uint64_t stop) { return count_kind(start, stop, 1); }
uint64_t gpu_count_triplets(uint64_t start, uint64_t stop) { return count_kind(start, stop, 2); }
uint64_t gpu_count_quadruplets(uint64_t start, uint64_t stop) { return count_kind(start, stop, 3); }
uint64_t gpu_count_quintuplets(uint64_t start, uint64_t stop) { return count_kind(start, stop, 4); }
uint64_t gpu_count_sextuplets(uint64_t start, uint64_t stop) { return count_kind(start, stop, 5); }

bool gpu_try_count(uint64_t start, uint64_t stop, int countType, uint64_t& result) {
  if (countType < 0 || countType > 5) return false;
  try {
    result = count_kind(start, stop, countType);
    return true;
  } catch (const std::exception&) {
    return false;
  }
}

} // namespace primesieve

// ---------------------------------------------------------------------------
// C API
// ---------------------------------------------------------------------------
extern "C" {

uint64_t primesieve_count_primes(uint64_t start, uint64_t stop) {
  return c_count("primesieve_count_primes", start, stop, 0);
}
uint64_t primesieve_count_twins(uint64_t start, uint64_t stop) {
  return c_count("primesieve_count_twins", start, stop, 1);
}
uint64_t primesieve_count_triplets(uint64_t start, uint64_t stop) {
  return c_count("primesieve_count_triplets", start, stop, 2);
}
uint64_t primesieve_count_quadruplets(uint64_t start, uint64_t stop) {
  return c_count("primesieve_count_quadruplets", start, stop, 3);
}
uint64_t primesieve_count_quintuplets(uint64_t start, uint64_t stop) {
  return c_count("primesieve_count_quintuplets", start, stop, 4);
}
uint64_t primesieve_count_sextuplets(uint64_t start, uint64_t stop) {
  return c_count("primesieve_count_sextuplets", start, stop, 5);
}

int primesieve_count_all(uint64_t start, uint64_t stop, uint64_t counts[6]) {
  try {
    if (!counts) throw primesieve::primesieve_error("counts is NULL");
    std::array<uint64_t, 6> r = primesieve::count_all(start, stop);
    for (int i = 0; i < 6; i++) counts[i] = r[i];
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "primesieve_count_all: " << e.what() << std::endl;
    errno = EDOM;
    return -1;
  }
}

void* primesieve_generate_primes(uint64_t start, uint64_t stop, size_t* size, int type) {
  return c_generate_typed("primesieve_generate_primes", start, stop, 0, false, size, type);
}

void* primesieve_generate_n_primes(uint64_t n, uint64_t start, int type) {
  return c_generate_typed("primesieve_generate_n_primes", start, 0, n, true, nullptr, type);
}

uint64_t primesieve_nth_prime(int64_t n, uint64_t start) {
  try {
    return primesieve::nth_prime(n, start);
  } catch (const std::exception& e) {
    std::cerr << "primesieve_nth_prime: " << e.what() << std::endl;
    errno = EDOM;
    return PRIMESIEVE_ERROR;
  }
}

void primesieve_free(void* primes) { std::free(primes); }

uint64_t primesieve_get_max_stop(void) { return primesieve::get_max_stop(); }
int primesieve_get_sieve_size(void) { return primesieve::get_sieve_size(); }
int primesieve_get_num_threads(void) { return primesieve::get_num_threads(); }
void primesieve_set_sieve_size(int size) { primesieve::set_sieve_size(size); }
void primesieve_set_num_threads(int threads) { primesieve::set_num_threads(threads); }
const char* primesieve_version(void) { return PRIMESIEVE_VERSION; }

} // extern "C"
