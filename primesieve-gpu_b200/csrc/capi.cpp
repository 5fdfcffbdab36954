// capi.cpp -- the extern "C" psg_* boundary over psg::Engine.
//
// Status codes in, no exceptions out; a thread-local message for the last
// failure. Each context serialises its own calls with a mutex (the reference
// serialises every GPU call with one global mutex, src/gpu/GpuSieve.cpp:27).
#include "../../include/psgpu.h"
#include "engine.hpp"
#include "server.hpp"

#include <cuda_runtime.h>
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <cstddef>
#include <exception>
#include <mutex>
#include <new>
#include <string>
#include <vector>

struct psg_context {
  psg::Engine engine;
  std::mutex mu;
};

struct psg_server {
  std::unique_ptr<psg::Server> srv;
};

namespace {

thread_local std::string t_last_error;

int fail(int status, const std::string& msg) {
  t_last_error = msg;
  return status;
}

psg::EngineConfig to_engine(const psg_config* c) {
  psg::EngineConfig e;
  if (!c) return e;
  e.seg_bytes = c->seg_bytes;
  e.block = c->block;
  e.ctas_per_sm = c->ctas_per_sm;
  e.small_limit = c->small_limit;
  e.big_limit = c->big_limit;
  e.window_segments = c->window_segments;
  e.bucket_lists = c->bucket_lists;
  e.presieve = c->presieve;
  e.segments_per_launch = c->segments_per_launch;
  e.list_capacity_pct = c->list_capacity_pct;
  return e;
}

// Sets the message without throwing: a message that cannot be stored (no
// host memory) leaves it empty.
void fail_nothrow(const char* msg) noexcept {
  try {
    t_last_error = msg;
  } catch (...) {
    t_last_error.clear();
  }
}

// Runs the body of a C entry point; no C++ exception (a failed host
// allocation, a thread that cannot start) may unwind through the C boundary,
// each becomes a status and a message.
template <typename F>
int guarded(F&& body) {
  try {
    return body();
  } catch (const std::bad_alloc&) {
    fail_nothrow("out of host memory");
    return PSG_ERR_NOMEM;
  } catch (const std::exception& e) {
    fail_nothrow("internal error: ");
    try { t_last_error += e.what(); } catch (...) {}
    return PSG_ERR_INTERNAL;
  } catch (...) {
    fail_nothrow("internal error: unknown exception");
    return PSG_ERR_INTERNAL;
  }
}

} // namespace

namespace psg {
// Lets other translation units of the library report through psg_last_error().
void set_last_error(const std::string& msg) { t_last_error = msg; }
void set_last_error_nothrow(const char* msg) noexcept { fail_nothrow(msg); }
}

extern "C" {

int psg_server_start(psg_context* ctx, const psg_server_config* cfg, psg_server** out) {
  return guarded([&]() -> int {
    if (!ctx || !out) return fail(PSG_ERR_ARG, "NULL argument");
    *out = nullptr;
    psg::ServerConfig c;
    if (cfg) {
      c.max_slots = cfg->max_slots;
      c.step_segments = cfg->step_segments;
      c.prime_limit = cfg->prime_limit;
      c.hbm_budget = cfg->hbm_budget;
    }
    std::unique_ptr<psg_server> s(new (std::nothrow) psg_server{ std::make_unique<psg::Server>(ctx->engine, ctx->mu) });
    if (!s) return fail(PSG_ERR_NOMEM, "out of host memory");
    std::string err;
    int rc = s->srv->start(c, err);
    if (rc) return fail(rc, err);
    *out = s.release();
    return PSG_OK;
  });
}

int psg_server_submit(psg_server* s, uint64_t start, uint64_t stop, uint32_t kinds, uint64_t* id) {
  return guarded([&]() -> int {
    if (!s || !id) return fail(PSG_ERR_ARG, "NULL argument");
    std::string err;
    int rc = s->srv->submit(start, stop, kinds, *id, err);
    return rc ? fail(rc, err) : PSG_OK;
  });
}

int psg_server_wait(psg_server* s, uint64_t id, uint64_t counts[6], double* latency_seconds) {
  return guarded([&]() -> int {
    if (!s) return fail(PSG_ERR_ARG, "NULL argument");
    std::string err;
    int rc = s->srv->wait(id, counts, latency_seconds, err);
    return rc ? fail(rc, err) : PSG_OK;
  });
}

int psg_server_replay(psg_server* s, const psg_range* requests, const double* arrival_seconds,
                      size_t n, uint64_t* counts, double* latency_seconds) {
  return guarded([&]() -> int {
    if (!s || (n && (!requests || !arrival_seconds))) return fail(PSG_ERR_ARG, "NULL argument");
    for (size_t i = 1; i < n; i++)
      if (arrival_seconds[i] < arrival_seconds[i - 1]) return fail(PSG_ERR_ARG, "arrival times must ascend");
    std::string err;
    int rc = s->srv->replay(reinterpret_cast<const psg::RangeQuery*>(requests), arrival_seconds, n, counts,
                            latency_seconds, err);
    return rc ? fail(rc, err) : PSG_OK;
  });
}

int psg_server_get_stats(psg_server* s, psg_server_stats* out) {
  return guarded([&]() -> int {
    if (!s || !out) return fail(PSG_ERR_ARG, "NULL argument");
    const psg::ServerStats st = s->srv->stats();
    out->submitted = st.submitted;
    out->completed = st.completed;
    out->refused = st.refused;
    out->steps = st.steps;
    out->bucket_requests = st.bucket_requests;
    out->batch_requests = st.batch_requests;
    out->integers = st.integers;
    out->gpu_busy_seconds = st.gpu_busy_seconds;
    return PSG_OK;
  });
}

int psg_server_inject_failure(psg_server* s, uint32_t nth, int status) {
  return guarded([&]() -> int {
    if (!s || status == PSG_OK) return fail(PSG_ERR_ARG, "NULL server or status PSG_OK");
    s->srv->inject_failure(nth, status);
    return PSG_OK;
  });
}

void psg_server_stop(psg_server* s) {
  if (!s) return;
  try {
    s->srv->stop();
  } catch (...) {
  }
  delete s;
}

const char* psg_version(void) { return "primesieve-b200 1.0 (primesieve 12.16 count API)"; }

const char* psg_last_error(void) { return t_last_error.c_str(); }

const char* psg_status_string(int s) {
  switch (s) {
    case PSG_OK: return "ok";
    case PSG_ERR_ARG: return "invalid argument";
    case PSG_ERR_NO_DEVICE: return "no usable CUDA device";
    case PSG_ERR_CUDA: return "CUDA error";
    case PSG_ERR_NOMEM: return "out of memory";
    case PSG_ERR_LIMIT: return "request beyond a supported limit";
    case PSG_ERR_INTERNAL: return "internal error";
    case PSG_ERR_TIMEOUT: return "timed out";
    case PSG_ERR_CLOSED: return "closed";
    case PSG_ERR_OVERFLOW: return "bucket list overflow in an asynchronous count";
    default: return "unknown status";
  }
}

int psg_device_count(int* count) {
  return guarded([&]() -> int {
    if (!count) return fail(PSG_ERR_ARG, "count is NULL");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
      cudaGetLastError();
      *count = 0;
      return PSG_OK;      // no driver / no device: zero devices
    }
    *count = n;
    return PSG_OK;
  });
}

int psg_device_describe(int index, char* buf, size_t len) {
  return guarded([&]() -> int {
    if (!buf || len == 0) return fail(PSG_ERR_ARG, "buffer is NULL");
    int n = 0;
    psg_device_count(&n);
    if (index < 0 || index >= n) return fail(PSG_ERR_NO_DEVICE, "GPU device index out of range");
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, index) != cudaSuccess) {
      cudaGetLastError();
      return fail(PSG_ERR_CUDA, "cudaGetDeviceProperties failed");
    }
    std::snprintf(buf, len,
                  "[%d] CUDA: %s (CUDA compute %d.%d)\n"
                  "      %d compute units, %d MHz, %llu MiB global, %llu KiB local, max work-group %d",
                  index, p.name, p.major, p.minor, p.multiProcessorCount, p.clockRate / 1000,
                  (unsigned long long) (p.totalGlobalMem >> 20),
                  (unsigned long long) (p.sharedMemPerBlockOptin >> 10), p.maxThreadsPerBlock);
    return PSG_OK;
  });
}

int psg_init(int device, const psg_config* cfg, psg_context** out) {
  return guarded([&]() -> int {
    if (!out) return fail(PSG_ERR_ARG, "out is NULL");
    *out = nullptr;
    std::unique_ptr<psg_context> ctx(new (std::nothrow) psg_context());
    if (!ctx) return fail(PSG_ERR_NOMEM, "cannot allocate context");
    std::string err;
    int rc = ctx->engine.init(device, to_engine(cfg), err);
    if (rc) return fail(rc, err);
    *out = ctx.release();
    return PSG_OK;
  });
}

void psg_destroy(psg_context* ctx) { delete ctx; }

int psg_get_config(const psg_context* ctx, psg_config* out) {
  return guarded([&]() -> int {
    if (!ctx || !out) return fail(PSG_ERR_ARG, "NULL argument");
    const psg::EngineConfig& c = ctx->engine.config();
    std::memset(out, 0, sizeof *out);
    out->seg_bytes = ctx->engine.seg_bytes();
    out->block = ctx->engine.block();
    out->ctas_per_sm = ctx->engine.grid() / (uint32_t) ctx->engine.props().multiProcessorCount;
    out->small_limit = c.small_limit;
    out->big_limit = c.big_limit;
    out->window_segments = c.window_segments;
    out->bucket_lists = c.bucket_lists;
    out->presieve = c.presieve;
    out->segments_per_launch = c.segments_per_launch;
    out->list_capacity_pct = c.list_capacity_pct;
    return PSG_OK;
  });
}

int psg_describe(const psg_context* ctx, char* buf, size_t len) {
  return guarded([&]() -> int {
    if (!ctx || !buf || !len) return fail(PSG_ERR_ARG, "NULL argument");
    std::snprintf(buf, len, "%s", ctx->engine.describe().c_str());
    return PSG_OK;
  });
}

int psg_count(psg_context* ctx, uint64_t start, uint64_t stop, uint32_t kinds, uint64_t counts[6]) {
  return guarded([&]() -> int {
    if (!ctx || !counts) return fail(PSG_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    std::string err;
    int rc = ctx->engine.count(start, stop, kinds, counts, err);
    return rc ? fail(rc, err) : PSG_OK;
  });
}

int psg_count_async(psg_context* ctx, uint64_t start, uint64_t stop, uint32_t kinds,
                    uint64_t* dev_counts, void* stream) {
  return guarded([&]() -> int {
    if (!ctx || !dev_counts) return fail(PSG_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    std::string err;
    int rc = ctx->engine.count_async(start, stop, kinds, reinterpret_cast<unsigned long long*>(dev_counts),
                                     static_cast<cudaStream_t>(stream), err);
    return rc ? fail(rc, err) : PSG_OK;
  });
}

int psg_count_async_status(psg_context* ctx) {
  return guarded([&]() -> int {
    if (!ctx) return fail(PSG_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    std::string err;
    int rc = ctx->engine.async_status(err);
    return rc ? fail(rc, err) : PSG_OK;
  });
}

int psg_count_batch(psg_context* ctx, const psg_range* ranges, size_t n, uint64_t* counts) {
  return guarded([&]() -> int {
    if (!ctx || (n && (!ranges || !counts))) return fail(PSG_ERR_ARG, "NULL argument");
    static_assert(sizeof(psg_range) == sizeof(psg::RangeQuery) &&
                  offsetof(psg_range, start) == offsetof(psg::RangeQuery, start) &&
                  offsetof(psg_range, stop) == offsetof(psg::RangeQuery, stop) &&
                  offsetof(psg_range, kinds) == offsetof(psg::RangeQuery, kinds), "psg_range layout");
    std::lock_guard<std::mutex> lock(ctx->mu);
    std::string err;
    int rc = ctx->engine.count_batch(reinterpret_cast<const psg::RangeQuery*>(ranges), n, counts, err);
    return rc ? fail(rc, err) : PSG_OK;
  });
}

int psg_generate_primes(psg_context* ctx, uint64_t start, uint64_t stop, uint64_t* out, size_t capacity,
                        size_t* count) {
  return guarded([&]() -> int {
    if (!ctx || !count || (capacity && !out)) return fail(PSG_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    std::string err;
    std::vector<uint64_t> v;
    int rc = ctx->engine.generate_primes(start, stop, v, err);
    if (rc) return fail(rc, err);
    *count = v.size();
    std::copy(v.begin(), v.begin() + std::min(v.size(), capacity), out);
    if (capacity < v.size())
      return fail(PSG_ERR_LIMIT, "output capacity " + std::to_string(capacity) + " < " + std::to_string(v.size()) + " primes");
    return PSG_OK;
  });
}

int psg_nth_prime(psg_context* ctx, int64_t n, uint64_t start, uint64_t* prime) {
  return guarded([&]() -> int {
    if (!ctx || !prime) return fail(PSG_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    std::string err;
    int rc = ctx->engine.nth_prime(n, start, *prime, err);
    return rc ? fail(rc, err) : PSG_OK;
  });
}

int psg_autotune_batch(psg_context* ctx, const psg_range* ranges, size_t n, double budget_seconds,
                       psg_tune_class* report, size_t cap, size_t* count) {
  return guarded([&]() -> int {
    if (!ctx || (n && !ranges) || (cap && !report)) return fail(PSG_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    std::string err;
    std::vector<psg::TuneReport> rep;
    int rc = ctx->engine.autotune_batch(reinterpret_cast<const psg::RangeQuery*>(ranges), n, budget_seconds, rep, err);
    if (rc) return fail(rc, err);
    if (count) *count = rep.size();
    for (size_t i = 0; i < rep.size() && i < cap; i++) {
      psg_tune_class& o = report[i];
      o.range_class = rep[i].cls;
      o.sample_ranges = (uint32_t) rep[i].sample_ranges;
      o.sample_integers = rep[i].sample_integers;
      o.direct_budget = rep[i].chosen.direct_budget;
      o.big_limit = rep[i].chosen.big_limit;
      o.stripe = rep[i].chosen.stripe;
      o.small_limit = rep[i].chosen.small_limit;
      o.reserved = 0;
      o.best_seconds = rep[i].best_seconds;
      o.default_seconds = rep[i].default_seconds;
    }
    return PSG_OK;
  });
}

int psg_prepare(psg_context* ctx, uint64_t stop) {
  return guarded([&]() -> int {
    if (!ctx) return fail(PSG_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    std::string err;
    int rc = ctx->engine.prepare(stop, err);
    return rc ? fail(rc, err) : PSG_OK;
  });
}

int psg_sieving_primes(psg_context* ctx, uint64_t stop, size_t first, uint32_t* out, size_t n,
                       size_t* total, uint64_t* lo_excl, uint64_t* hi_incl) {
  return guarded([&]() -> int {
    if (!ctx || !total || (n && !out)) return fail(PSG_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    std::string err;
    size_t t = 0;
    uint64_t lo = 0, hi = 0;
    int rc = ctx->engine.sieving_primes(stop, first, out, n, t, lo, hi, err);
    if (rc) return fail(rc, err);
    *total = t;
    if (lo_excl) *lo_excl = lo;
    if (hi_incl) *hi_incl = hi;
    return PSG_OK;
  });
}

int psg_set_profiling(psg_context* ctx, int on) {
  return guarded([&]() -> int {
    if (!ctx) return fail(PSG_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->engine.set_profiling(on != 0);
    return PSG_OK;
  });
}

int psg_kernel_stats(psg_context* ctx, const char** names, uint64_t* launches, double* ms,
                     size_t cap, size_t* n) {
  return guarded([&]() -> int {
    if (!ctx || !n) return fail(PSG_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    std::vector<psg::KernelStat> st = ctx->engine.kernel_stats();
    *n = st.size();
    for (size_t i = 0; i < st.size() && i < cap; i++) {
      if (names) names[i] = st[i].name;
      if (launches) launches[i] = st[i].launches;
      if (ms) ms[i] = st[i].ms;
    }
    return PSG_OK;
  });
}

int psg_bucket_entries(psg_context* ctx, uint64_t* total, int reset) {
  return guarded([&]() -> int {
    if (!ctx || !total) return fail(PSG_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    *total = ctx->engine.bucket_entries();
    if (reset) ctx->engine.reset_bucket_entries();
    return PSG_OK;
  });
}

int psg_measure_smem_atomic_rate(psg_context* ctx, double* random_addr, double* conflict_free) {
  return guarded([&]() -> int {
    if (!ctx || !random_addr) return fail(PSG_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    double r = 0, c = 0;
    ctx->engine.measure_smem_atomic_rates(r, c);
    *random_addr = r;
    if (conflict_free) *conflict_free = c;
    return (r > 0 && c > 0) ? PSG_OK : fail(PSG_ERR_CUDA, "probe kernel failed");
  });
}

int psg_reset_kernel_stats(psg_context* ctx) {
  return guarded([&]() -> int {
    if (!ctx) return fail(PSG_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->engine.reset_kernel_stats();
    return PSG_OK;
  });
}

} // extern "C"
