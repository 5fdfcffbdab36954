/*
 * oracle.h -- CPU restatement of the reference's prime / k-tuplet counting
 * path. TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the CPU
 * baseline leg of bench.py may call this; the product never does.
 *
 * Two independent counters:
 *   oracle_count_plain  a plain segmented byte-array sieve of Eratosthenes
 *                       (one byte per integer) that counts primes and the
 *                       k-tuplet patterns by their definitions.
 *   oracle_count_wheel  the reference's own algorithm, restated: wheel-30 bit
 *                       array (bit b of byte i = segLow + 30 i +
 *                       {7,11,13,17,19,23,29,31}[b]), segments starting at
 *                       lo - byteRemainder(lo), per-byte k-tuplet lookup,
 *                       range masks at the edges and the 2/3/5 table.
 *
 * counts[i] for i = 0..5: primes, twins, triplets, quadruplets, quintuplets,
 * sextuplets. kinds_mask bit i selects counts[i]; unselected entries are 0.
 */
#ifndef PSG_ORACLE_H
#define PSG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Returns 0 on success, -1 on a bad argument or allocation failure. */
int oracle_count_plain(uint64_t start, uint64_t stop, uint32_t kinds_mask,
                       uint64_t counts[6]);

int oracle_count_wheel(uint64_t start, uint64_t stop, uint32_t sieve_bytes,
                       uint32_t kinds_mask, uint64_t counts[6]);

/* All primes p with lo <= p <= hi (hi < 2^32), written to out (capacity cap).
 * Returns the number of primes, or -1 if cap is too small. */
int64_t oracle_primes_u32(uint32_t lo, uint32_t hi, uint32_t* out, size_t cap);

/* Byte-wise k-tuplet lookup table for kind k (1..5), derived from the tuplet
 * definitions; k = 0 gives the popcount table. */
void oracle_ktuplet_table(int kind, uint8_t table[256]);

#ifdef __cplusplus
}
#endif

#endif
