// wheel.hpp -- wheel-30 facts shared by the host engine and the kernels.
//
// Bit layout (must match the reference so that k-tuplet byte masks and the
// CPU/GPU counts agree): bit b of sieve byte i stands for the value
//     segLow + 30*i + {7, 11, 13, 17, 19, 23, 29, 31}[b]
// with segLow a multiple of 30 (reference src/gpu/GpuWheel.hpp:4-6,
// src/Erat.cpp:231-237). A value v == 1 (mod 30) therefore lives in the
// byte *before* the one a naive v/30 picks, as "segLow + 31".
//
// Everything below is derived arithmetic, packed into integer constants so
// that device code reads it from registers instead of divergent memory.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define PSG_HD __host__ __device__ __forceinline__
#else
#define PSG_HD inline
#endif

namespace psg {

// Value offsets of the 8 bits of a byte.
constexpr uint32_t kBitValue[8] = { 7, 11, 13, 17, 19, 23, 29, 31 };

// Cofactor classes q (mod 30) with gcd(q, 30) = 1, in increasing order.
constexpr uint32_t kCofactor[8] = { 1, 7, 11, 13, 17, 19, 23, 29 };

// Number of values covered by one sieve byte.
constexpr uint32_t kNumbersPerByte = 30;

// ---- packed lookup helpers ----------------------------------------------

// residue r (mod 30, coprime to 30) -> bit index; 3 bits per residue.
constexpr uint64_t res2bit_packed(int part) {
  uint64_t v = 0;
  for (int r = 0; r < 30; r++) {
    int bit = 0;
    for (int j = 0; j < 8; j++)
      if (kBitValue[j] % 30 == (uint32_t) r) bit = j;
    if (r / 20 == part) v |= (uint64_t) bit << (3 * (r % 20));
  }
  return v;
}
constexpr uint64_t kRes2Bit0 = res2bit_packed(0);   // residues 0..19
constexpr uint64_t kRes2Bit1 = res2bit_packed(1);   // residues 20..29

PSG_HD uint32_t residue_to_bit(uint32_t r) {
  return (uint32_t) ((r < 20 ? (kRes2Bit0 >> (3 * r)) : (kRes2Bit1 >> (3 * (r - 20)))) & 7u);
}

// inverse of r (mod 30) for r coprime to 30; 5 bits per residue.
constexpr uint64_t inv30_packed(int part) {
  uint64_t v = 0;
  for (int r = 0; r < 30; r++) {
    int inv = 0;
    for (int x = 1; x < 30; x++)
      if ((r * x) % 30 == 1) inv = x;
    if (r / 12 == part) v |= (uint64_t) inv << (5 * (r % 12));
  }
  return v;
}
constexpr uint64_t kInv30_0 = inv30_packed(0);      // residues 0..11
constexpr uint64_t kInv30_1 = inv30_packed(1);      // residues 12..23
constexpr uint64_t kInv30_2 = inv30_packed(2);      // residues 24..29

PSG_HD uint32_t inverse_mod30(uint32_t r) {
  uint64_t w = r < 12 ? kInv30_0 : (r < 24 ? kInv30_1 : kInv30_2);
  return (uint32_t) ((w >> (5 * (r % 12))) & 31u);
}

// ---- wheel walk tables ----------------------------------------------------
// Walking the multiples p*q of a sieving prime p in increasing order, the
// cofactor q steps through the classes kCofactor[j] with gaps
// {6,4,2,4,2,4,6,2}. With p = 30*pdiv30 + pm, the byte index of the next
// multiple grows by pdiv30*gap_j + corr_j(pm), and its bit is bit_j(pm).
// Both depend only on the class of pm (8 classes, indexed by
// residue_to_bit(pm)); they are packed 3 bits per j.
constexpr uint32_t kGapPacked = 6u | (4u << 3) | (2u << 6) | (4u << 9) | (2u << 12) |
                                (4u << 15) | (6u << 18) | (2u << 21);

constexpr uint32_t value_offset_of_residue(uint32_t r) { return r < 7 ? r + 30 : r; }

constexpr uint32_t class_residue(uint32_t c) { return c == 7 ? 1u : kBitValue[c]; }

constexpr uint32_t bit_of_residue_c(uint32_t r) {
  uint32_t b = 0;
  for (uint32_t j = 0; j < 8; j++) if (kBitValue[j] % 30 == r) b = j;
  return b;
}

constexpr uint32_t wheel_bits_packed(uint32_t c) {
  uint32_t v = 0;
  for (uint32_t j = 0; j < 8; j++)
    v |= bit_of_residue_c((class_residue(c) * kCofactor[j]) % 30) << (3 * j);
  return v;
}

constexpr uint32_t wheel_corr_packed(uint32_t c) {
  uint32_t v = 0;
  const uint32_t pm = class_residue(c);
  for (uint32_t j = 0; j < 8; j++) {
    const uint32_t gap = (kGapPacked >> (3 * j)) & 7u;
    const uint32_t vj = value_offset_of_residue((pm * kCofactor[j]) % 30);
    const uint32_t vn = value_offset_of_residue((pm * kCofactor[(j + 1) & 7]) % 30);
    v |= ((vj + pm * gap - vn) / 30) << (3 * j);
  }
  return v;
}

// c0 (cofactor residue 0..29) -> first class j with kCofactor[j] >= c0.
constexpr uint64_t first_class_packed(int part) {
  uint64_t v = 0;
  for (int c = 0; c < 30; c++) {
    int j = 0;
    while (kCofactor[j] < (uint32_t) c) j++;
    if (c / 20 == part) v |= (uint64_t) j << (3 * (c % 20));
  }
  return v;
}
constexpr uint64_t kFirstClass0 = first_class_packed(0);
constexpr uint64_t kFirstClass1 = first_class_packed(1);

PSG_HD uint32_t first_class_ge(uint32_t c0) {
  return (uint32_t) ((c0 < 20 ? (kFirstClass0 >> (3 * c0)) : (kFirstClass1 >> (3 * (c0 - 20)))) & 7u);
}

// ---- count kinds --------------------------------------------------------
enum : uint32_t {
  kPrimes = 0, kTwins = 1, kTriplets = 2, kQuadruplets = 3,
  kQuintuplets = 4, kSextuplets = 5, kNumKinds = 6
};

// k-tuplet bit masks inside one byte, derived from the pattern offsets
// (twins p,p+2; triplets p,p+2,p+6 | p,p+4,p+6; quadruplets p,p+2,p+6,p+8;
// quintuplets p,p+2,p+6,p+8,p+12 | p,p+4,p+6,p+10,p+12; sextuplets
// p,p+4,p+6,p+10,p+12,p+16). In this layout every admissible k-tuplet
// >= 7 occupies consecutive bits of one byte, so a tuplet whose first
// member is bit b is "bits b..b+k-1 all set". The word-wide counters below
// test that with shifted ANDs; the per-byte start masks are
//   twins       bits {1,3,6}    -> 0x4A per byte
//   triplets    bits {0,1,2,3}  -> 0x0F per byte
//   quadruplets bit  {1}        -> 0x02 per byte
//   quintuplets bits {0,1}      -> 0x03 per byte
//   sextuplets  bit  {0}        -> 0x01 per byte
// (reference bitmasks: src/CountPrintPrimes.cpp:33-41).
constexpr uint32_t kTwinStart   = 0x4A4A4A4Au;
constexpr uint32_t kTripStart   = 0x0F0F0F0Fu;
constexpr uint32_t kQuadStart   = 0x02020202u;
constexpr uint32_t kQuintStart  = 0x03030303u;
constexpr uint32_t kSextStart   = 0x01010101u;

} // namespace psg
