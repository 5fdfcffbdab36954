// Exercises the primesieve-compatible C++ API (include/primesieve.hpp,
// include/primesieve/gpu.hpp) the way test/gpu_count.cpp in the reference
// does; prints one line per check so the Python test can compare it.
#include <primesieve.hpp>
#include <primesieve/gpu.hpp>

#include <cstdio>
#include <cstdlib>

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const uint64_t a = std::strtoull(argv[1], nullptr, 10);
  const uint64_t b = std::strtoull(argv[2], nullptr, 10);
  if (!primesieve::gpu_available()) { std::printf("no gpu\n"); return 3; }
  std::printf("devices %zu\n", primesieve::gpu_devices().size());
  std::printf("active %d\n", primesieve::gpu_active_device().empty() ? 0 : 1);
  std::printf("count %llu %llu %llu %llu %llu %llu\n",
              (unsigned long long) primesieve::count_primes(a, b),
              (unsigned long long) primesieve::count_twins(a, b),
              (unsigned long long) primesieve::count_triplets(a, b),
              (unsigned long long) primesieve::count_quadruplets(a, b),
              (unsigned long long) primesieve::count_quintuplets(a, b),
              (unsigned long long) primesieve::count_sextuplets(a, b));
  std::printf("gpu %llu %llu %llu %llu %llu %llu\n",
              (unsigned long long) primesieve::gpu_count_primes(a, b),
              (unsigned long long) primesieve::gpu_count_twins(a, b),
              (unsigned long long) primesieve::gpu_count_triplets(a, b),
              (unsigned long long) primesieve::gpu_count_quadruplets(a, b),
              (unsigned long long) primesieve::gpu_count_quintuplets(a, b),
              (unsigned long long) primesieve::gpu_count_sextuplets(a, b));
  auto all = primesieve::count_all(a, b);
  std::printf("all %llu %llu %llu %llu %llu %llu\n",
              (unsigned long long) all[0], (unsigned long long) all[1], (unsigned long long) all[2],
              (unsigned long long) all[3], (unsigned long long) all[4], (unsigned long long) all[5]);
  // knobs recreate the engine; results must not change
  primesieve::set_gpu_sieve_size(32);
  primesieve::set_gpu_work_group_size(256);
  primesieve::set_gpu_presieve(false);
  uint64_t r = 0;
  bool ok = primesieve::gpu_try_count(a, b, 0, r);
  std::printf("knobs %d %llu\n", ok ? 1 : 0, (unsigned long long) r);
  primesieve::set_gpu_sieve_size(0);
  primesieve::set_gpu_work_group_size(0);
  primesieve::set_gpu_presieve(true);
  std::printf("worthwhile %d %d\n", primesieve::gpu_worthwhile(a, b) ? 1 : 0,
              primesieve::gpu_worthwhile(b + 1, b) ? 1 : 0);
  return 0;
}
