/// primesieve.hpp -- primesieve-compatible C++ API of the B200 engine.
///
/// Drop-in for the counting, nth-prime and prime-generation parts of the
/// reference's C++ API (include/primesieve.hpp:28-198, implementation
/// src/api.cpp:48-118). Everything runs on the GPU; failures throw
/// primesieve_error.
#ifndef PRIMESIEVE_HPP
#define PRIMESIEVE_HPP

#define PRIMESIEVE_VERSION "12.16"
#define PRIMESIEVE_VERSION_MAJOR 12
#define PRIMESIEVE_VERSION_MINOR 16

#include <primesieve/primesieve_error.hpp>

#include <stdint.h>
#include <array>
#include <string>
#include <vector>

namespace primesieve {

/// n > 0: the nth prime > start; n = 0: the first prime > start; n < 0: the
/// |n|th prime < start (reference include/primesieve.hpp:76-89).
uint64_t nth_prime(int64_t n, uint64_t start = 0);

/// The primes inside [start, stop] appended to out, extracted on the GPU
/// (the element-type templates below convert from it).
void generate_primes_u64(uint64_t start, uint64_t stop, std::vector<uint64_t>& out);
/// The first n primes >= start appended to out.
void generate_n_primes_u64(uint64_t n, uint64_t start, std::vector<uint64_t>& out);
/// Throws primesieve_error when `largest` does not fit the element type
/// `bits`/`is_signed` (the reference's "is too narrow" check).
void check_element_type(const char* fn, int bits, bool is_signed, const char* name, uint64_t largest);

namespace detail {
template <typename V> constexpr const char* type_name() { return "Type"; }
template <> constexpr const char* type_name<int16_t>() { return "int16_t"; }
template <> constexpr const char* type_name<uint16_t>() { return "uint16_t"; }
template <> constexpr const char* type_name<int32_t>() { return "int32_t"; }
template <> constexpr const char* type_name<uint32_t>() { return "uint32_t"; }
template <> constexpr const char* type_name<int64_t>() { return "int64_t"; }
template <> constexpr const char* type_name<uint64_t>() { return "uint64_t"; }
template <typename vect>
void check(const char* fn, uint64_t largest) {
  using V = typename vect::value_type;
  check_element_type(fn, (int) (8 * sizeof(V)), V(-1) < V(0), type_name<V>(), largest);
}
template <typename vect>
void append(const std::vector<uint64_t>& v, vect& primes) {
  using V = typename vect::value_type;
  primes.reserve(primes.size() + v.size());
  for (uint64_t p : v) primes.push_back((V) p);
}
} // namespace detail

/// Appends the primes inside [start, stop] (reference include/primesieve.hpp:40-49).
template <typename vect>
inline void generate_primes(uint64_t start, uint64_t stop, vect* primes) {
  if (!primes || start > stop) return;
  detail::check<vect>("store_primes()", stop);
  std::vector<uint64_t> v;
  generate_primes_u64(start, stop, v);
  detail::append(v, *primes);
}

/// Appends the primes <= stop.
template <typename vect>
inline void generate_primes(uint64_t stop, vect* primes) { generate_primes(0, stop, primes); }

/// Appends the first n primes >= start (reference include/primesieve.hpp:51-71).
template <typename vect>
inline void generate_n_primes(uint64_t n, uint64_t start, vect* primes) {
  if (!primes || n == 0) return;
  std::vector<uint64_t> v;
  generate_n_primes_u64(n, start, v);
  detail::check<vect>("store_n_primes()", v.empty() ? 0 : v.back());
  detail::append(v, *primes);
}

/// Appends the first n primes.
template <typename vect>
inline void generate_n_primes(uint64_t n, vect* primes) { generate_n_primes(n, 0, primes); }

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
