/*
 * psgpu.h -- the C ABI of the B200 prime / k-tuplet counting engine.
 *
 * This is the thin boundary the host layers (the primesieve-compatible C and
 * C++ APIs, the CLI, and foreign-language bindings) call. Plain C types only:
 * integers, pointers, sizes and an opaque context handle. Every function
 * returns a psg_status; on failure a message is available from
 * psg_last_error() (thread-local). Nothing here throws.
 *
 * Reference interfaces each entry point replaces (paths inside the reference
 * project):
 *   psg_count            GpuBackend::count(lo, hi, countType)
 *                        src/gpu/GpuBackend.hpp:66-69 and countOnGpu()
 *                        src/gpu/GpuSieve.cpp:131-176 (incl. the 2/3/5 table),
 *                        widened to all six counts in one pass.
 *   psg_count_batch      no counterpart (the reference counts one range per
 *                        call: src/api.cpp:48-118).
 *   psg_init / psg_destroy  CudaBackend::init / ~CudaBackend
 *                        src/gpu/cuda/CudaBackend.cpp:222-344, :114-123.
 *   psg_device_count / psg_device_describe  listDevices(), DeviceInfo::describe()
 *                        src/gpu/GpuSieve.cpp:43-72.
 *   psg_config fields    GpuConfig src/gpu/GpuBackend.hpp:45-58 and the
 *                        set_gpu_* knobs include/primesieve/gpu.hpp:48-53.
 *   psg_get_config / psg_describe  GpuBackend::sieveBytes(), workGroupSize(),
 *                        device() src/gpu/GpuBackend.hpp:64, :72-73 and
 *                        gpu_active_device() include/primesieve/gpu.hpp:57.
 *   psg_last_error       gpu_last_error() include/primesieve/gpu.hpp:60
 *                        (here per thread; psg_status_string has no
 *                        counterpart: the reference throws primesieve_error).
 *   psg_version          primesieve_version() include/primesieve.h:243.
 *   psg_generate_primes, psg_nth_prime, psg_sieving_primes  cited at their
 *                        declarations below.
 *   psg_count_async, psg_count_async_status, psg_prepare,
 *   psg_autotune_batch, psg_server_*, the
 *   profiling calls and psg_count_noalloc  no counterpart (the reference
 *                        counts one range per synchronous call,
 *                        src/api.cpp:48-118, and has no device-side API).
 */
#ifndef PSGPU_H
#define PSGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  PSG_OK = 0,
  PSG_ERR_ARG = 1,        /* invalid argument (e.g. start > stop where not allowed) */
  PSG_ERR_NO_DEVICE = 2,  /* no usable CUDA device / bad device index */
  PSG_ERR_CUDA = 3,       /* a CUDA runtime call failed */
  PSG_ERR_NOMEM = 4,      /* device or host allocation failed */
  PSG_ERR_LIMIT = 5,      /* request beyond a documented maximum */
  PSG_ERR_INTERNAL = 6,   /* internal consistency check failed */
  PSG_ERR_TIMEOUT = 7,    /* a bounded wait gave up */
  PSG_ERR_CLOSED = 8,     /* the server / queue has been shut down */
  PSG_ERR_OVERFLOW = 9    /* an asynchronous count dropped bucket entries: recount */
} psg_status;

/* Count kinds: bit i of a kinds mask selects counts[i]. */
enum {
  PSG_PRIMES = 1u << 0,
  PSG_TWINS = 1u << 1,
  PSG_TRIPLETS = 1u << 2,
  PSG_QUADRUPLETS = 1u << 3,
  PSG_QUINTUPLETS = 1u << 4,
  PSG_SEXTUPLETS = 1u << 5,
  PSG_ALL_KINDS = 0x3fu
};

typedef struct psg_context psg_context;

/* Tuning knobs; 0 means "auto". Mirrors GpuConfig plus the big-prime and
 * batching parameters this engine adds. */
typedef struct {
  uint32_t seg_bytes;          /* shared-memory sieve segment per CTA (bytes) */
  uint32_t block;              /* threads per CTA: 256, 512 or 1024 */
  uint32_t ctas_per_sm;        /* resident sieve CTAs per SM */
  uint32_t small_limit;        /* sieving primes below: one warp per prime (0: per range,
                                  4096, 2048 or 1024 as sqrt(stop) grows past 2e6 and 8e6) */
  uint32_t big_limit;          /* sieving primes from: bucket sieve */
  uint32_t window_segments;    /* segments per bucket window */
  uint32_t bucket_lists;       /* bucket lists per segment */
  uint32_t presieve;           /* pre-sieve with pattern tables: 0 = default (on), 1 = on, 2 = off */
  uint32_t segments_per_launch;/* cap on segments per launch (reference knob) */
  uint32_t list_capacity_pct;  /* bucket-list capacity in % of the engine's estimate
                                  (0 = 100); values below 100 make lists overflow, for
                                  tests of the overflow handling */
} psg_config;

/* A [start, stop] range and the kinds wanted for it (batch API). */
typedef struct {
  uint64_t start;
  uint64_t stop;
  uint32_t kinds;
  uint32_t reserved;
} psg_range;

/* ---- devices ------------------------------------------------------------ */
int psg_device_count(int* count);
/* One human-readable line for device `index`. */
int psg_device_describe(int index, char* buf, size_t len);

/* ---- context ------------------------------------------------------------ */
/* device < 0 picks the device with the most SMs. cfg may be NULL. */
int psg_init(int device, const psg_config* cfg, psg_context** out);
/* Stop every server started on ctx (psg_server_stop) before destroying it:
 * a server's worker thread uses the context. */
void psg_destroy(psg_context* ctx);
/* The configuration actually in use (autotuned values filled in). */
int psg_get_config(const psg_context* ctx, psg_config* out);
int psg_describe(const psg_context* ctx, char* buf, size_t len);

/* ---- counting ----------------------------------------------------------- */
/* Count primes and/or k-tuplets in [start, stop] (0 <= start, stop <= 2^64-1).
 * counts[i] receives the count of kind i if bit i of kinds is set, else 0.
 * start > stop gives all zeros. Synchronous. */
int psg_count(psg_context* ctx, uint64_t start, uint64_t stop, uint32_t kinds,
              uint64_t counts[6]);

/* Asynchronous variant: ADDS the counts to dev_counts (device memory,
 * 6 x uint64_t) on `stream` (a cudaStream_t, NULL = the context's stream).
 * The 2/3/5 table is included. Host-side preparation (the sieving-prime
 * table for sqrt(stop)) happens before return. Unlike psg_count it cannot
 * recount when a bucket list overflows (the lists are sized for their
 * expected length plus 6 sigma plus 32 entries): an overflow drops entries,
 * so the counts written are too high. The kernels record it in the
 * context, and psg_count_async_status() reports it: call it before
 * trusting asynchronous counts. */
int psg_count_async(psg_context* ctx, uint64_t start, uint64_t stop, uint32_t kinds,
                    uint64_t* dev_counts, void* stream);

/* Waits for every count enqueued on the context so far and reports whether
 * the psg_count_async calls since the previous status call were exact:
 * PSG_OK, or PSG_ERR_OVERFLOW if a bucket list of one of them overflowed
 * (its counts are too high; the lists have grown, so counting again gives
 * the exact values). Clears the recorded state. No reference counterpart:
 * the reference's GPU count is synchronous and surfaces every failure of
 * its launch (src/gpu/GpuSieve.cpp:341-365). */
int psg_count_async_status(psg_context* ctx);

/* Count n ranges; counts is n x 6 (row i for ranges[i]). */
int psg_count_batch(psg_context* ctx, const psg_range* ranges, size_t n,
                    uint64_t* counts);

/* The primes in [start, stop], ascending. Replaces the reference's CPU prime
 * extraction (src/CountPrintPrimes.cpp:187-259, store_primes in
 * include/primesieve/StorePrimes.hpp): the GPU sieve keeps its segments as
 * bitmaps and a GPU kernel turns them into values. *count gets the number
 * of primes; up to `capacity` of them are written to out (host memory);
 * PSG_ERR_LIMIT when capacity < *count (nothing is lost: call again). */
int psg_generate_primes(psg_context* ctx, uint64_t start, uint64_t stop,
                        uint64_t* out, size_t capacity, size_t* count);

/* primesieve's nth_prime(n, start) (src/nthPrime.cpp:47-181): n > 0 the nth
 * prime > start, n = 0 the first prime > start, n < 0 the |n|th prime
 * < start. Exact GPU counts locate it; the last bracket is sieved as a
 * bitmap. Errors (PSG_ERR_ARG / PSG_ERR_LIMIT) carry the reference's
 * messages. */
int psg_nth_prime(psg_context* ctx, int64_t n, uint64_t start, uint64_t* prime);

/* Batch autotuner (no reference counterpart). Range classes are the decimal
 * lengths of stop; for every class present in `ranges` a seeded sample of
 * its ranges is counted under candidate parameters -- the batch-kernel vs
 * bucket-path budget, the direct-tier extent of bucket-path ranges, the
 * stripe length of work items, then the small/medium sieving-prime
 * threshold -- and the fastest are kept in the context for
 * psg_count_batch and the server. Stops after about budget_seconds. One
 * report row per tuned class (up to cap rows; *count = rows). */
typedef struct {
  int32_t range_class;         /* decimal digits of stop - 1 */
  uint32_t sample_ranges;
  double sample_integers;
  double direct_budget;        /* chosen: segments x primes past the shared state */
  uint32_t big_limit;          /* chosen: direct tier below this prime (bucket-path ranges) */
  uint32_t stripe;             /* chosen: segments per work item */
  double best_seconds;         /* sample time with the chosen parameters */
  double default_seconds;      /* sample time with the defaults */
  uint32_t small_limit;        /* chosen: warp-cooperative tier below this prime (0: default) */
  uint32_t reserved;
} psg_tune_class;

int psg_autotune_batch(psg_context* ctx, const psg_range* ranges, size_t n, double budget_seconds,
                       psg_tune_class* report, size_t cap, size_t* count);

/* Build the sieving-prime table up to sqrt(stop) ahead of time. */
int psg_prepare(psg_context* ctx, uint64_t stop);

/* The device sieving-prime table, for tests and diagnostics. Replaces the
 * reference's CPU generate_primes(7, sqrt(hi)) and upload
 * (src/gpu/cuda/CudaBackend.cpp:346-388): psg_prepare(stop), then entries
 * [first, first + n) of the table (clipped to its length) are copied to out
 * (host). *total = the table's length; it holds, ascending, the primes p
 * with *lo_excl < p <= *hi_incl (the pre-sieve primes are not in it; the
 * table may reach beyond sqrt(stop), it grows geometrically). */
int psg_sieving_primes(psg_context* ctx, uint64_t stop, size_t first, uint32_t* out, size_t n,
                       size_t* total, uint64_t* lo_excl, uint64_t* hi_incl);

/* ---- diagnostics -------------------------------------------------------- */
const char* psg_last_error(void);
const char* psg_status_string(int status);

/* Per-kernel CUDA-event timing of this context's launches. */
int psg_set_profiling(psg_context* ctx, int on);
/* Fills up to `cap` entries: name (static string), launches, total ms.
 * *n receives the number of kernels. */
int psg_kernel_stats(psg_context* ctx, const char** names, uint64_t* launches,
                     double* ms, size_t cap, size_t* n);
int psg_reset_kernel_stats(psg_context* ctx);
/* Bucket-sieve entries written (4 bytes each) since the last reset; waits for
 * the context's stream. reset != 0 zeroes the counter afterwards. */
int psg_bucket_entries(psg_context* ctx, uint64_t* total, int reset);
/* Roofline denominators of the cross-off phases, measured on this device
 * (atomics/s): shared-memory atomicAnd at random addresses (a warp's lanes
 * on banks at random, as in the medium, direct and bucket phases) and
 * conflict-free (every lane on its own bank: the ceiling). conflict_free
 * may be NULL. */
int psg_measure_smem_atomic_rate(psg_context* ctx, double* random_addr, double* conflict_free);

/* Count without allocating anything (no reference counterpart: the
 * reference always allocates through its backend). For callers that cannot
 * allocate device memory when they count: an allocator's own callbacks (a
 * cudaMalloc there re-enters the allocator), real-time loops (a cudaMalloc
 * can synchronise the device), embedders with a fixed memory budget. Same result
 * as psg_count(), written (overwritten) to dev_counts, a device buffer of 6
 * uint64_t, on `stream` (a cudaStream_t; NULL = the legacy default stream).
 * Runs on the current device; no context is needed.
 *   Limit: stop <= 2^36 (PSG_ERR_LIMIT beyond). No cudaMalloc or cudaFree:
 *   the sieving primes <= 2^18, their reciprocals and the count accumulators
 *   live in one fixed static device array of about 270 KiB that every GPU
 *   loading the library keeps until the process exits.
 *   The first call on a device sets that array up synchronously (symbol
 *   lookup, table copy, one kernel); make it before any stream capture.
 *   All calls share the array, so calls that overlap on the GPU (different
 *   streams, different host threads) race; serialise them. */
int psg_count_noalloc(uint64_t start, uint64_t stop, uint32_t kinds,
                      uint64_t* dev_counts, void* stream);

/* ---- request server: continuous batching -------------------------------
 * No reference counterpart (the reference answers one count per call,
 * src/api.cpp:48-118). A worker thread owns the context's GPU and runs it in
 * steps: each step admits waiting requests into free device slots, runs one
 * launch of the persistent batch kernel over segment stripes taken
 * round-robin from the admitted requests plus up to two bucket windows of
 * the oldest long high request, and completes the requests whose last piece ran.
 * Requests that arrive meanwhile join the next step. The sieving-prime table
 * stays resident (up to prime_limit, 2^32 by default: every 64-bit stop).
 * A request whose bucket storage would exceed the HBM budget is refused
 * with PSG_ERR_NOMEM. The context must outlive the server; other calls on
 * the context wait for the current step. */
typedef struct psg_server psg_server;

typedef struct {
  uint32_t max_slots;          /* requests on the device at once; 0 = 4096 */
  uint32_t step_segments;      /* batch-kernel segments per step; 0 = auto */
  uint64_t prime_limit;        /* resident sieving primes up to; 0 = 2^32 - 1 */
  uint64_t hbm_budget;         /* bytes of bucket storage allowed; 0 = 80% of free HBM */
} psg_server_config;

typedef struct {
  uint64_t submitted, completed, refused, steps;
  uint64_t bucket_requests;    /* admitted on the windowed bucket path */
  uint64_t batch_requests;     /* admitted on the persistent batch kernel */
  double integers;             /* integers of completed requests */
  double gpu_busy_seconds;     /* wall time spent in steps */
} psg_server_stats;

int psg_server_start(psg_context* ctx, const psg_server_config* cfg, psg_server** out);
/* Queue a count of [start, stop] (kinds mask); *id names it for wait. */
int psg_server_submit(psg_server* s, uint64_t start, uint64_t stop, uint32_t kinds, uint64_t* id);
/* Block until request id is done: counts[6] and its latency (seconds from
 * submit to completion). Returns the request's status. Each id is collected
 * by one wait: a second wait for it, concurrent or later, fails with
 * PSG_ERR_ARG. */
int psg_server_wait(psg_server* s, uint64_t id, uint64_t counts[6], double* latency_seconds);
/* Load replay: submits requests[i] at arrival_seconds[i] after the call
 * (ascending), waits for all; counts is n x 6, latency from the scheduled
 * arrival. */
int psg_server_replay(psg_server* s, const psg_range* requests, const double* arrival_seconds,
                      size_t n, uint64_t* counts, double* latency_seconds);
int psg_server_get_stats(psg_server* s, psg_server_stats* out);
/* For tests of the failure handling, on the host (no reference counterpart):
 * the nth request the worker plans from now on (nth >= 1; 0 cancels) makes
 * its step fail with `status`, as a failed CUDA call at that point would.
 * Every request of that step, planned or not, completes with `status`. */
int psg_server_inject_failure(psg_server* s, uint32_t nth, int status);
/* Stops the worker (requests still queued fail with PSG_ERR_CLOSED). */
void psg_server_stop(psg_server* s);

/* The library version string. */
const char* psg_version(void);

#ifdef __cplusplus
}
#endif

#endif
