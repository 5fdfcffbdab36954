/*
 * primesieve.h -- primesieve-compatible C API of the B200 counting engine.
 *
 * Drop-in for the counting subset of the reference's C API
 * (include/primesieve.h:130-233, implementation src/api-c.cpp:143-225).
 * Every count runs on the GPU (no CPU fallback, no minimum range). On error
 * the functions print a message to stderr, set errno to EDOM and return
 * PRIMESIEVE_ERROR, exactly like the reference.
 *
 * Prime generation (primesieve_generate_primes, primesieve_generate_n_primes)
 * and primesieve_nth_prime are declared below too; they run on the GPU as
 * well (the sieve keeps its segments as bitmaps, a kernel turns them into
 * values). The iterator, printing and the RiemannR functions are not part
 * of this library.
 */
#ifndef PRIMESIEVE_H
#define PRIMESIEVE_H

#define PRIMESIEVE_VERSION "12.16"
#define PRIMESIEVE_VERSION_MAJOR 12
#define PRIMESIEVE_VERSION_MINOR 16

#include <stddef.h>
#include <stdint.h>

/* Returned by the uint64_t functions on error (reference include/primesieve.h:31). */
#define PRIMESIEVE_ERROR ((uint64_t) ~((uint64_t) 0))

#ifdef __cplusplus
extern "C" {
#endif

/* Element types of primesieve_generate_primes() / _generate_n_primes()
 * (same names and values as the reference, include/primesieve.h:37-66). */
enum {
  SHORT_PRIMES,
  USHORT_PRIMES,
  INT_PRIMES,
  UINT_PRIMES,
  LONG_PRIMES,
  ULONG_PRIMES,
  LONGLONG_PRIMES,
  ULONGLONG_PRIMES,
  INT16_PRIMES,
  UINT16_PRIMES,
  INT32_PRIMES,
  UINT32_PRIMES,
  INT64_PRIMES,
  UINT64_PRIMES
};

/* The primes inside [start, stop] as a malloc'd array of `type` elements
 * (free with primesieve_free); *size = number of primes. NULL, *size = 0 and
 * errno = EDOM on error (reference include/primesieve.h:68-81,
 * src/api-c.cpp). The primes are extracted on the GPU. */
void* primesieve_generate_primes(uint64_t start, uint64_t stop, size_t* size, int type);

/* The first n primes >= start (reference include/primesieve.h:83-96). */
void* primesieve_generate_n_primes(uint64_t n, uint64_t start, int type);

/* n > 0: the nth prime > start; n = 0: the first prime > start; n < 0: the
 * |n|th prime < start (reference include/primesieve.h:98-115). Located with
 * exact GPU counts. PRIMESIEVE_ERROR + errno = EDOM on error. */
uint64_t primesieve_nth_prime(int64_t n, uint64_t start);

/* Frees an array of primesieve_generate_primes / _generate_n_primes. */
void primesieve_free(void* primes);

/* Count the primes / prime k-tuplets inside [start, stop], stop <= 2^64-1.
 * Reference: include/primesieve.h:130-170, src/api-c.cpp:143-225. */
uint64_t primesieve_count_primes(uint64_t start, uint64_t stop);
uint64_t primesieve_count_twins(uint64_t start, uint64_t stop);
uint64_t primesieve_count_triplets(uint64_t start, uint64_t stop);
uint64_t primesieve_count_quadruplets(uint64_t start, uint64_t stop);
uint64_t primesieve_count_quintuplets(uint64_t start, uint64_t stop);
uint64_t primesieve_count_sextuplets(uint64_t start, uint64_t stop);

/* All six counts of [start, stop] from one sieve pass (no reference
 * counterpart: the reference counts one kind per GPU pass,
 * src/app/main.cpp:158-160). counts[i] = primes, twins, ..., sextuplets.
 * Returns 0, or -1 on error (message on stderr, errno = EDOM). */
int primesieve_count_all(uint64_t start, uint64_t stop, uint64_t counts[6]);

/* 2^64-1 (reference src/api.cpp:169-172). */
uint64_t primesieve_get_max_stop(void);

/* CPU tuning knobs of the reference (include/primesieve.h:205-233). They are
 * accepted and reported back but do not influence the GPU sieve. */
int primesieve_get_sieve_size(void);
int primesieve_get_num_threads(void);
void primesieve_set_sieve_size(int sieve_size);
void primesieve_set_num_threads(int num_threads);

/* "12.16" (the API version this library implements). */
const char* primesieve_version(void);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif
