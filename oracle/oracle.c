/*
 * oracle.c -- CPU restatement of the reference's counting path.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the shipped library links, loads or
 * calls this file; it is the checker that the GPU results are compared with.
 *
 * Reference anchors (paths inside the reference project):
 *   - wheel-30 bit layout: src/gpu/GpuWheel.hpp:4-6 (bit b of byte i stands for
 *     segmentLow + i*30 + {7,11,13,17,19,23,29,31}[b]); CPU twin
 *     src/Erat.cpp:231-237 (byteRemainder, classes 7..36).
 *   - first segment low: src/gpu/cuda/CudaBackend.cpp:457.
 *   - first multiple of a sieving prime above segmentLow + 6, cofactor coprime
 *     to 30 and >= p: src/gpu/cuda/sieve.cu:69-99, src/Wheel.hpp:50-89.
 *   - range masking of the edge words: src/gpu/cuda/sieve.cu:119-139 (CPU:
 *     src/Erat.cpp:30-48 unsetSmaller / unsetLarger).
 *   - per-byte k-tuplet counting: src/gpu/GpuTables.cpp:132-168,
 *     src/CountPrintPrimes.cpp:33-41 (bitmasks) and :162-184.
 *   - the primes 2, 3, 5 and the tuplets that contain them:
 *     src/gpu/GpuSieve.cpp:149-169, src/PrimeSieveClass.cpp:38-48.
 */
#include "oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* Offsets of the 8 bits of a wheel-30 byte relative to 30*i. */
static const uint32_t kBitOffset[8] = { 7, 11, 13, 17, 19, 23, 29, 31 };

/* k-tuplet patterns as offsets from the smallest member
 * (src/CountPrintPrimes.cpp:33-41 lists the same patterns as byte masks). */
typedef struct { int n; uint32_t off[6]; } pattern_t;
static const pattern_t kPatterns[6][2] = {
  { { 1, { 0 } },                 { 0, { 0 } } },                  /* prime */
  { { 2, { 0, 2 } },              { 0, { 0 } } },                  /* twins */
  { { 3, { 0, 2, 6 } },           { 3, { 0, 4, 6 } } },            /* triplets */
  { { 4, { 0, 2, 6, 8 } },        { 0, { 0 } } },                  /* quadruplets */
  { { 5, { 0, 2, 6, 8, 12 } },    { 5, { 0, 4, 6, 10, 12 } } },    /* quintuplets */
  { { 6, { 0, 4, 6, 10, 12, 16 } }, { 0, { 0 } } }                 /* sextuplets */
};

/* ------------------------------------------------------------------ */
/* Sieving primes (cached; plain odd-only sieve, segmented)            */
/* ------------------------------------------------------------------ */

static pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;
static uint32_t* g_primes = NULL;   /* all primes <= g_limit */
static size_t g_nprimes = 0;
static uint64_t g_limit = 0;

static uint32_t isqrt64(uint64_t x)
{
  uint64_t r = 0;
  for (int b = 31; b >= 0; b--) {
    uint64_t t = r | (1ull << b);
    if (t * t <= x && t <= 0xffffffffull)
      r = t;
  }
  return (uint32_t) r;
}

/* Make sure g_primes holds every prime <= limit (limit < 2^32). */
static int ensure_primes(uint64_t limit)
{
  if (limit <= g_limit && g_primes)
    return 0;
  if (limit < 1024)
    limit = 1024;
  /* base primes up to sqrt(limit) with a tiny sieve */
  uint32_t r = isqrt64(limit) + 1;
  uint8_t* small = (uint8_t*) calloc(r + 1, 1);
  uint32_t* base = (uint32_t*) malloc(sizeof(uint32_t) * (r / 2 + 16));
  if (!small || !base) { free(small); free(base); return -1; }
  size_t nb = 0;
  for (uint32_t i = 2; i <= r; i++) {
    if (small[i]) continue;
    base[nb++] = i;
    for (uint64_t j = (uint64_t) i * i; j <= r; j += i) small[j] = 1;
  }
  free(small);

  /* pi(x) < 1.26 x / ln x; be generous */
  size_t cap = (size_t) (limit / 8 + 1024);
  if (limit > 100000) {
    double lx = 0; { double x = (double) limit; double l = 0; while (x > 2.718281828) { x /= 2.718281828; l += 1; } lx = l; }
    cap = (size_t) (1.3 * (double) limit / (lx > 1 ? lx : 1)) + 1024;
  }
  uint32_t* out = (uint32_t*) malloc(sizeof(uint32_t) * cap);
  if (!out) { free(base); return -1; }
  size_t n = 0;
  out[n++] = 2;

  /* odd-only segmented sieve over [3, limit] */
  const uint64_t SEG = 1u << 20;          /* odd numbers per segment */
  uint8_t* seg = (uint8_t*) malloc(SEG);
  if (!seg) { free(base); free(out); return -1; }
  for (uint64_t lo = 3; lo <= limit; lo += 2 * SEG) {
    uint64_t hi = lo + 2 * SEG - 2;        /* last odd in segment */
    if (hi > limit) hi = (limit % 2) ? limit : limit - 1;
    uint64_t cnt = (hi - lo) / 2 + 1;
    memset(seg, 0, cnt);
    for (size_t k = 1; k < nb; k++) {      /* skip 2 */
      uint64_t p = base[k];
      if (p * p > hi) break;
      uint64_t m = (lo + p - 1) / p * p;
      if (m < p * p) m = p * p;
      if (m % 2 == 0) m += p;
      for (; m <= hi; m += 2 * p) seg[(m - lo) / 2] = 1;
    }
    for (uint64_t i = 0; i < cnt; i++)
      if (!seg[i]) {
        if (n == cap) { free(seg); free(base); free(out); return -1; }
        out[n++] = (uint32_t) (lo + 2 * i);
      }
  }
  free(seg);
  free(base);
  free(g_primes);
  g_primes = out;
  g_nprimes = n;
  g_limit = limit;
  return 0;
}

int64_t oracle_primes_u32(uint32_t lo, uint32_t hi, uint32_t* out, size_t cap)
{
  pthread_mutex_lock(&g_lock);
  if (ensure_primes(hi) != 0) { pthread_mutex_unlock(&g_lock); return -1; }
  size_t n = 0;
  for (size_t i = 0; i < g_nprimes && g_primes[i] <= hi; i++) {
    if (g_primes[i] < lo) continue;
    if (n == cap) { pthread_mutex_unlock(&g_lock); return -1; }
    out[n++] = g_primes[i];
  }
  pthread_mutex_unlock(&g_lock);
  return (int64_t) n;
}

/* ------------------------------------------------------------------ */
/* k-tuplet byte tables derived from the definitions                   */
/* ------------------------------------------------------------------ */

/* Byte mask of a pattern whose smallest member sits on bit b, or 0 when the
 * pattern does not fit inside one byte (then it can never occur there: all
 * admissible k-tuplets >= 7 fit in one byte, src/gpu/cuda/sieve.cu:308-309). */
static unsigned pattern_mask(const pattern_t* pt, int b)
{
  unsigned mask = 0;
  for (int m = 0; m < pt->n; m++) {
    uint32_t v = kBitOffset[b] + pt->off[m];
    int bit = -1;
    for (int j = 0; j < 8; j++) if (kBitOffset[j] == v) bit = j;
    if (bit < 0) return 0;
    mask |= 1u << bit;
  }
  return mask;
}

void oracle_ktuplet_table(int kind, uint8_t table[256])
{
  for (unsigned x = 0; x < 256; x++) {
    unsigned c = 0;
    if (kind == 0) {
      for (int b = 0; b < 8; b++) c += (x >> b) & 1u;
    } else {
      for (int v = 0; v < 2; v++) {
        const pattern_t* pt = &kPatterns[kind][v];
        if (pt->n == 0) continue;
        for (int b = 0; b < 8; b++) {
          unsigned m = pattern_mask(pt, b);
          if (m && (x & m) == m) c++;
        }
      }
    }
    table[x] = (uint8_t) c;
  }
}

/* ------------------------------------------------------------------ */
/* The 2/3/5 table (src/gpu/GpuSieve.cpp:149-169)                      */
/* ------------------------------------------------------------------ */

static void add_small_table(uint64_t start, uint64_t stop, uint32_t kinds, uint64_t counts[6])
{
  /* tuplets with a member below 7, as (first, last, kind) */
  static const uint64_t small[8][3] = {
    { 2, 2, 0 }, { 3, 3, 0 }, { 5, 5, 0 },
    { 3, 5, 1 }, { 5, 7, 1 }, { 5, 11, 2 }, { 5, 13, 3 }, { 5, 17, 4 }
  };
  if (start > 5)
    return;
  for (int i = 0; i < 8; i++) {
    int k = (int) small[i][2];
    if ((kinds >> k) & 1u)
      if (small[i][0] >= start && small[i][1] <= stop)
        counts[k]++;
  }
}

/* ------------------------------------------------------------------ */
/* Wheel-30 restatement (src/gpu/cuda/CudaBackend.cpp:443-491 with     */
/* the per-segment body of src/gpu/cuda/sieve.cu:157-320)              */
/* ------------------------------------------------------------------ */

/* index of residue v (mod 30, classes 7..31 where 1 is written as 31) */
static int bit_of_residue(uint32_t r)
{
  for (int j = 0; j < 8; j++) if (kBitOffset[j] == r) return j;
  return -1;
}

int oracle_count_wheel(uint64_t start, uint64_t stop, uint32_t sieve_bytes,
                       uint32_t kinds, uint64_t counts[6])
{
  for (int i = 0; i < 6; i++) counts[i] = 0;
  if (sieve_bytes == 0 || start > stop)
    return start > stop ? 0 : -1;

  add_small_table(start, stop, kinds, counts);
  if (stop < 7)
    return 0;

  uint64_t lo = start < 7 ? 7 : start;
  uint64_t hi = stop;
  uint32_t sq = isqrt64(hi);

  pthread_mutex_lock(&g_lock);
  int rc = ensure_primes(sq < 7 ? 7 : sq);
  const uint32_t* primes = g_primes;
  size_t np = g_nprimes;
  pthread_mutex_unlock(&g_lock);
  if (rc != 0) return -1;

  uint8_t tab[6][256];
  for (int k = 0; k < 6; k++) oracle_ktuplet_table(k, tab[k]);

  uint8_t* sieve = (uint8_t*) malloc(sieve_bytes);
  if (!sieve) return -1;

  const uint64_t span = (uint64_t) sieve_bytes * 30;
  /* byteRemainder: src/Erat.cpp:231-237; firstSegLow: CudaBackend.cpp:457 */
  uint64_t segLow = lo - ((lo - 7) % 30 + 7);

  for (;;) {
    memset(sieve, 0xff, sieve_bytes);
    /* last value representable in this segment */
    u128 segTop = (u128) segLow + span + 1;
    for (size_t i = 0; i < np; i++) {
      uint64_t p = primes[i];
      if (p < 7) continue;
      if ((u128) p * p > hi) break;
      /* first multiple m = p*q > segLow + 6 with q >= p and gcd(q, 30) = 1 */
      uint64_t low = segLow + 6;
      u128 q = (u128) (low / p) + 1;
      if (q < p) q = p;
      while ((uint64_t) (q % 2) == 0 || (uint64_t) (q % 3) == 0 || (uint64_t) (q % 5) == 0) q++;
      for (u128 m = (u128) p * q; m <= segTop && m <= hi; ) {
        uint64_t d = (uint64_t) (m - segLow);       /* >= 7 */
        uint64_t byte = (d - 7) / 30;
        if (byte >= sieve_bytes) break;
        int bit = bit_of_residue((uint32_t) ((d - 7) % 30 + 7));
        sieve[byte] &= (uint8_t) ~(1u << bit);
        /* next cofactor coprime to 30 */
        do { q++; } while ((uint64_t) (q % 2) == 0 || (uint64_t) (q % 3) == 0 || (uint64_t) (q % 5) == 0);
        m = (u128) p * q;
      }
    }
    /* mask values outside [lo, hi] and count */
    for (uint32_t i = 0; i < sieve_bytes; i++) {
      uint8_t b = sieve[i];
      if (!b) continue;
      u128 base = (u128) segLow + (u128) i * 30;
      if (base + 7 < lo || base + 31 > hi) {
        uint8_t keep = 0;
        for (int j = 0; j < 8; j++) {
          u128 v = base + kBitOffset[j];
          if (v >= lo && v <= hi) keep |= (uint8_t) (1u << j);
        }
        b &= keep;
      }
      for (int k = 0; k < 6; k++)
        if ((kinds >> k) & 1u) counts[k] += tab[k][b];
    }
    /* next segment (stop when the next one would start beyond hi) */
    if ((u128) segLow + span + 7 > hi) break;
    segLow += span;
  }
  free(sieve);
  return 0;
}

/* ------------------------------------------------------------------ */
/* Plain byte-array sieve, tuplets counted from their definitions       */
/* ------------------------------------------------------------------ */

int oracle_count_plain(uint64_t start, uint64_t stop, uint32_t kinds, uint64_t counts[6])
{
  for (int i = 0; i < 6; i++) counts[i] = 0;
  if (start > stop)
    return 0;
  uint32_t sq = isqrt64(stop);
  pthread_mutex_lock(&g_lock);
  int rc = ensure_primes(sq < 7 ? 7 : sq);
  const uint32_t* primes = g_primes;
  size_t np = g_nprimes;
  pthread_mutex_unlock(&g_lock);
  if (rc != 0) return -1;

  const uint64_t CHUNK = 1u << 20;
  const uint64_t LOOK = 16;
  uint8_t* isp = (uint8_t*) malloc(CHUNK + LOOK + 1);
  if (!isp) return -1;

  for (u128 a = start; a <= stop; a += CHUNK) {
    uint64_t a64 = (uint64_t) a;
    /* window [a, w_end] holds the chunk plus the look-ahead */
    u128 w_end = a + CHUNK + LOOK - 1;
    if (w_end > stop) w_end = stop;
    uint64_t wlen = (uint64_t) (w_end - a) + 1;
    memset(isp, 1, wlen);
    for (uint64_t i = 0; i < wlen; i++)
      if (a64 + i < 2) isp[i] = 0;
    for (size_t k = 0; k < np; k++) {
      uint64_t p = primes[k];
      if ((u128) p * p > w_end) break;
      u128 m = ((u128) a64 + p - 1) / p * p;
      if (m < (u128) p * p) m = (u128) p * p;
      for (; m <= w_end; m += p) isp[(uint64_t) (m - a)] = 0;
    }
    uint64_t chunk_len = wlen < CHUNK ? wlen : CHUNK;
    for (uint64_t i = 0; i < chunk_len; i++) {
      if (!isp[i]) continue;
      for (int k = 0; k < 6; k++) {
        if (!((kinds >> k) & 1u)) continue;
        for (int v = 0; v < 2; v++) {
          const pattern_t* pt = &kPatterns[k][v];
          if (pt->n == 0) continue;
          int ok = 1;
          for (int m = 1; m < pt->n && ok; m++) {
            uint64_t j = i + pt->off[m];
            if (j >= wlen) ok = 0;           /* member beyond stop */
            else if (!isp[j]) ok = 0;
          }
          if (ok) counts[k]++;
        }
      }
    }
  }
  free(isp);
  return 0;
}
