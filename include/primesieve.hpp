/// primesieve.hpp -- primesieve-compatible C++ counting API of the B200 engine.
///
/// Drop-in for the counting subset of the reference's C++ API
/// (include/primesieve.hpp:102-198, implementation src/api.cpp:48-118).
/// All counts run on the GPU; failures throw primesieve_error.
#ifndef PRIMESIEVE_HPP
#define PRIMESIEVE_HPP

#define PRIMESIEVE_VERSION "12.16"
#define PRIMESIEVE_VERSION_MAJOR 12
#define PRIMESIEVE_VERSION_MINOR 16

#include <primesieve/primesieve_error.hpp>

#include <stdint.h>
#include <array>
#include <string>

namespace primesieve {

uint64_t count_primes(uint64_t start, uint64_t stop);
uint64_t count_twins(uint64_t start, uint64_t stop);
uint64_t count_triplets(uint64_t start, uint64_t stop);
uint64_t count_quadruplets(uint64_t start, uint64_t stop);
uint64_t count_quintuplets(uint64_t start, uint64_t stop);
uint64_t count_sextuplets(uint64_t start, uint64_t stop);

/// All six counts from one sieve pass (no reference counterpart).
std::array<uint64_t, 6> count_all(uint64_t start, uint64_t stop);

uint64_t get_max_stop();
int get_sieve_size();
int get_num_threads();
void set_sieve_size(int sieve_size);
void set_num_threads(int num_threads);
std::string primesieve_version();

} // namespace primesieve

#endif
