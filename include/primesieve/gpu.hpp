/// gpu.hpp -- the GPU API of the reference (include/primesieve/gpu.hpp:31-81,
/// implementation src/gpu/GpuSieve.cpp:184-365), B200 edition.
///
/// Differences, by design: every count runs on the GPU (there is no CPU
/// sieve in this library), so there is no minimum range (gpu_worthwhile()
/// is true for any non-empty range) and gpu_try_count() only reports GPU
/// failures. All functions serialise on one process-wide mutex, like the
/// reference.
#ifndef PRIMESIEVE_GPU_HPP
#define PRIMESIEVE_GPU_HPP

#include <stdint.h>
#include <string>
#include <vector>

namespace primesieve {

bool gpu_available();
std::vector<std::string> gpu_devices();

/// -1 selects the device with the most SMs. Takes effect on the next call.
void set_gpu_device(int deviceIndex);
int get_gpu_device();

/// Kept for API compatibility; counting always uses the GPU.
void set_gpu_enabled(bool enable);
bool get_gpu_enabled();

/// Tuning knobs (0 = auto). Each one recreates the engine on the next call.
void set_gpu_sieve_size(int kilobytes);        // shared-memory segment per CTA
void set_gpu_work_group_size(int size);        // threads per CTA: 256, 512, 1024
void set_gpu_segments_per_launch(int segments);
void set_gpu_presieve(bool enable);

std::string gpu_active_device();
std::string gpu_last_error();
bool gpu_worthwhile(uint64_t start, uint64_t stop);

uint64_t gpu_count_primes(uint64_t start, uint64_t stop);
uint64_t gpu_count_twins(uint64_t start, uint64_t stop);
uint64_t gpu_count_triplets(uint64_t start, uint64_t stop);
uint64_t gpu_count_quadruplets(uint64_t start, uint64_t stop);
uint64_t gpu_count_quintuplets(uint64_t start, uint64_t stop);
uint64_t gpu_count_sextuplets(uint64_t start, uint64_t stop);

/// countType 0..5 = primes..sextuplets. Returns false (and records
/// gpu_last_error()) when the GPU count failed.
bool gpu_try_count(uint64_t start, uint64_t stop, int countType, uint64_t& result);

} // namespace primesieve

#endif
