// engine.hpp -- host side of the B200 counting engine.
//
// An Engine owns one CUDA device context's worth of state: a stream, the
// pre-sieve pattern tables, the sieving-prime table (+ reciprocals), the
// bucket storage of the big-prime sieve and the count accumulators. It is
// the replacement of the reference's CudaBackend (src/gpu/cuda/CudaBackend.cpp)
// behind the GpuBackend::count(lo, hi, countType) contract
// (src/gpu/GpuBackend.hpp:66-69), extended to all six counts in one pass.
#pragma once
#include <stdint.h>
#include <string>
#include <vector>
#include <mutex>
#include <cuda_runtime.h>
#include "batch_types.hpp"

namespace psg {

struct EngineConfig {
  uint32_t seg_bytes = 0;        // shared-memory segment per CTA; 0 = auto
  uint32_t block = 0;            // threads per CTA (256/512/1024); 0 = auto
  uint32_t ctas_per_sm = 0;      // resident sieve CTAs per SM; 0 = max
  uint32_t small_limit = 0;      // primes below: warp-cooperative; 0 = auto
  uint32_t big_limit = 0;        // primes from: bucket sieve; 0 = auto
  uint32_t window_segments = 0;  // segments per bucket window; 0 = auto
  uint32_t bucket_lists = 0;     // lists (bucket CTAs) per segment; 0 = auto
  uint32_t presieve = 0;         // pre-sieve tables: 0 = default (on), 1 = on, 2 = off
  uint32_t segments_per_launch = 0; // cap on segments per sieve launch; 0 = auto
  uint32_t list_capacity_pct = 0; // bucket-list capacity, % of the estimate (0 = 100)
};

// One range of a batch; same layout as psg_range (include/psgpu.h).
struct RangeQuery {
  uint64_t start, stop;
  uint32_t kinds, reserved;
};

struct SieveArgs;
struct BatchArgs;

// floor(sqrt(x))
uint32_t isqrt_u64(uint64_t x);
// The primes 2, 3, 5 and the k-tuplets containing them (not representable
// in the wheel-30 bit array): counts added to out[kind] when start <= 5.
void small_table(uint64_t start, uint64_t stop, uint32_t kinds, uint64_t out[6]);

// Batch parameters of one range class (ranges whose stop has the same
// number of decimal digits), set by Engine::autotune_batch.
struct BatchClassParams {
  double direct_budget = 1e8;   // segments x primes past the shared state: batch kernel up to this
  uint32_t big_limit = 0;       // bucket-path ranges: direct tier below this prime (0: engine default)
  uint32_t stripe = 8;          // segments per batch-kernel work item
  uint32_t small_limit = 0;     // warp-cooperative tier below this prime (0: engine default)
};
constexpr int kBatchClasses = 21;   // stop < 10^20

struct TuneReport {
  int cls;                      // decimal digits of stop - 1
  size_t sample_ranges;
  double sample_integers;
  BatchClassParams chosen;
  double best_seconds, default_seconds;
};

// Bucket fill: primes above the window's byte length / kThreadWalkDiv take
// the thread walk (one thread per prime), the rest the group walk (8 lanes
// per prime, one per wheel class).
constexpr uint32_t kThreadWalkDiv = 32;

// Prime tiers and launch geometry of one range [lo, hi] (lo >= 7):
// primes [0, n_small) warp-cooperative, [n_small, n_med) carried state,
// [n_med, n_dir) direct, [n_dir, n_total) bucket lists; sieve launches of
// `step` segments.
struct RangePlan {
  uint64_t lo = 0, hi = 0, seg_low0 = 0, nseg = 0, step = 1;
  uint32_t n_small = 0, n_med = 0, n_dir = 0, n_total = 0;
  bool buckets = false;
  uint64_t windows() const { return (nseg + step - 1) / step; }
};

struct KernelStat {
  const char* name;
  uint64_t launches = 0;
  double ms = 0.0;
};

class Engine {
public:
  Engine() = default;
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  // Returns 0 or a psg status code; err gets a message.
  int init(int device, const EngineConfig& cfg, std::string& err);

  // Count the requested kinds (bit i of kinds = counts[i]) in [start, stop].
  // Results are added to dev_counts (device, 6 x u64) on `stream`
  // (nullptr: the engine's stream). No host synchronisation.
  int count_async(uint64_t start, uint64_t stop, uint32_t kinds,
                  unsigned long long* dev_counts, cudaStream_t stream, std::string& err);

  // Waits for every count issued so far; PSG_ERR_OVERFLOW if a bucket list
  // of a count_async since the last call overflowed (entries dropped: those
  // counts are too high), after growing the lists. Clears the record.
  int async_status(std::string& err);

  // Synchronous host-result version (counts[6] overwritten).
  int count(uint64_t start, uint64_t stop, uint32_t kinds, uint64_t counts[6], std::string& err);

  // Count n ranges (out is n x 6, row i for q[i]) with the persistent batch
  // kernel; ranges that need the bucket tier run through the range path.
  int count_batch(const RangeQuery* q, size_t n, uint64_t* out, std::string& err);
  // Classes of the last batch: ranges in the persistent kernel, ranges on
  // the windowed bucket path, work items.
  size_t batch_direct_ranges() const { return batch_direct_ranges_; }
  size_t batch_bucket_ranges() const { return batch_bucket_ranges_; }
  size_t batch_items() const { return batch_items_; }

  // Tiers of [lo, hi] (lo >= 7) and launches of its windows [w0, w0 + nw);
  // counts added to dev_counts on st. Bucket windows alternate between two
  // list sets (set 0 on st, set 1 on the auxiliary stream), each with its
  // own copy of the range's list tables; between chain_begin and chain_end
  // the alternation continues from one call to the next, so that windows
  // of consecutive ranges overlap too (the caller orders everything the
  // ranges share before chain_begin and reads results after chain_end).
  // The range kernel's warp-cooperative tier for a range ending at hi: the
  // config's small_limit, else by the bucket primes' share of the work.
  uint32_t range_small_limit(uint64_t hi) const;
  int plan_range(uint64_t lo, uint64_t hi, RangePlan& p, std::string& err, uint32_t big_limit = 0,
                 uint32_t small_limit = 0);
  int run_windows(const RangePlan& p, uint32_t kinds, unsigned long long* dev_counts,
                  cudaStream_t st, uint64_t w0, uint64_t nw, std::string& err);
  void chain_begin(cudaStream_t st);
  void chain_end(cudaStream_t st);

  // Batch-kernel building blocks (also used by the request server):
  // tiers of [lo, hi] for the persistent kernel (false: needs the bucket
  // path), its stripes as work items, and one launch over device items.
  bool batch_range(uint64_t lo, uint64_t hi, uint32_t kinds, BatchRange& r, double& seg_cost);
  // Per range class, time a sample of the batch's ranges of that class under
  // candidate parameters and keep the fastest (wall-clock budget in seconds).
  int autotune_batch(const RangeQuery* q, size_t n, double budget_s, std::vector<TuneReport>& report,
                     std::string& err);
  const BatchClassParams& batch_params(uint64_t stop) const { return batch_tune_[batch_class(stop)]; }
  static int batch_class(uint64_t stop);
  uint64_t range_segments(const BatchRange& r) const;
  uint64_t append_stripes(uint32_t k, const BatchRange& r, double seg_cost, uint64_t s0, uint64_t max_seg,
                          std::vector<BatchItem>& items, std::vector<double>& cost, uint32_t stripe = 0) const;
  static void sort_items(std::vector<BatchItem>& items, const std::vector<double>& cost);
  int launch_items(const BatchRange* d_ranges, const BatchItem* d_items, uint32_t n_items,
                   unsigned long long* d_rows, uint32_t* d_queue, cudaStream_t st, std::string& err);
  // Bucket-list overflow flag (device) and the response to it: lists grow
  // and the next windows are planned again.
  uint32_t* overflow_flag() { return d_overflow_; }
  void grow_bucket_lists() { overflow_retries_++; cap_scale_ *= 2.0; plan_.last = 0; }
  // Estimated bucket storage of a planned range (bytes).
  size_t bucket_bytes(const RangePlan& p) const;

  // Primes in [start, stop], ascending (sieve segments kept as bitmaps and
  // turned into values on the device). Appended to out.
  int generate_primes(uint64_t start, uint64_t stop, std::vector<uint64_t>& out, std::string& err);
  // primesieve's nth_prime(n, start): n > 0 the nth prime > start, n = 0 as
  // n = 1, n < 0 the |n|th prime < start.
  int nth_prime(int64_t n, uint64_t start, uint64_t& prime, std::string& err);

  // Make sure the sieving-prime table covers sqrt(stop) (host work + upload).
  int prepare(uint64_t stop, std::string& err);
  // prepare(stop), then entries [first, first + n) of the device table (clipped)
  // into host out; total = its length, and it holds the primes p with
  // lo_excl < p <= hi_incl.
  int sieving_primes(uint64_t stop, size_t first, uint32_t* out, size_t n, size_t& total,
                     uint64_t& lo_excl, uint64_t& hi_incl, std::string& err);

  int device() const { return device_; }
  const cudaDeviceProp& props() const { return prop_; }
  cudaStream_t stream() const { return stream_; }
  const EngineConfig& config() const { return cfg_; }
  uint32_t seg_bytes() const { return seg_bytes_; }
  uint32_t block() const { return block_; }
  uint32_t grid() const { return grid_; }
  // integers covered by one bucket window
  uint64_t window_span() const { return (uint64_t) window_ * seg_bytes_ * 30u; }
  std::string describe() const;

  // Per-kernel CUDA-event timing (off by default).
  void set_profiling(bool on) { profiling_ = on; }
  std::vector<KernelStat> kernel_stats();
  void reset_kernel_stats();
  uint64_t overflow_retries() const { return overflow_retries_; }
  // Bucket entries written since the last reset (device counter; syncs).
  uint64_t bucket_entries();
  void reset_bucket_entries();
  // Measured shared-memory atomicAnd rates (atomics/s), the roofline
  // denominators of the cross-off phases: random addresses (bank conflicts
  // as in the medium, direct and bucket phases) and conflict-free (every
  // lane on its own bank: the ceiling).
  void measure_smem_atomic_rates(double& random_rate, double& conflict_free_rate);

private:
  int build_presieve(std::string& err);
  int ensure_primes(uint64_t limit, std::string& err);
  int reserve_primes(size_t n, size_t keep, std::string& err);
  uint32_t count_primes_le(uint64_t v, bool strict);
  uint32_t count_primes_upper(uint64_t v) const;   // >= table primes <= v, no device read
  void fill_common_args(SieveArgs& a) const;
  cudaError_t launch_batch(const BatchArgs& b, cudaStream_t st);
  double approx_prime(uint32_t i) const;
  double inv_prefix(uint32_t i) const;   // ~ sum of 1/p over table primes [0, i)
  uint32_t approx_count_below(uint64_t v) const;
  // big primes from this value on have at most ~8 kThreadWalkDiv multiples
  // in a window of w segments: the fill kernel walks them one lane per prime
  // (one first-multiple setup instead of eight)
  uint64_t thread_limit(uint32_t w) const { return (uint64_t) w * seg_bytes_ / kThreadWalkDiv; }
  int ensure_buckets(uint32_t first_big, uint32_t last_big, std::string& err);
  int plan_to_slot(uint32_t set, cudaStream_t ws, std::string& err);
  void quiesce();
  int run(uint64_t lo, uint64_t hi, uint32_t kinds, unsigned long long* dev_counts,
          cudaStream_t st, std::string& err);
  // bitmap of [lo, hi] (lo >= 7) into host bytes, from segment base seg_low0
  int sieve_bitmap(uint64_t lo, uint64_t hi, uint64_t& seg_low0, std::vector<uint8_t>& bits, std::string& err);
  uint64_t count_range(uint64_t lo, uint64_t hi, std::string& err, int& rc);
  int count_enqueue(uint64_t start, uint64_t stop, uint32_t kinds,
                    unsigned long long* dev_counts, cudaStream_t st, std::string& err);
  // count_enqueue after everything issued before, on stream (nullptr: the
  // engine's stream); its fill kernels report overflow to `flag`
  int count_ordered(uint64_t start, uint64_t stop, uint32_t kinds, unsigned long long* dev_counts,
                    cudaStream_t stream, uint32_t* flag, std::string& err);
  void timed_begin(int which, cudaStream_t st);
  void timed_end(int which, cudaStream_t st);

  int device_ = -1;
  cudaDeviceProp prop_{};
  cudaStream_t stream_ = nullptr;
  cudaStream_t last_stream_ = nullptr;
  cudaEvent_t done_event_ = nullptr;
  EngineConfig cfg_;
  uint32_t seg_bytes_ = 0, block_ = 0, grid_ = 0, bucket_block_ = 256;
  uint32_t small_limit_ = 0, big_limit_ = 0, window_ = 0, lists_ = 0;
  bool small_auto_ = true;        // small_limit_ not set by the config: chosen per range
  uint32_t state_cap_ = 0, smem_dyn_ = 0, seg_shift_ = 0;
  bool seg_pow2_ = true;

  // pre-sieve tables
  std::vector<std::vector<uint32_t>> groups_;
  uint8_t* d_pat_ = nullptr;
  std::vector<size_t> pat_off_;
  std::vector<uint32_t> pat_period_, pat_stride_;
  std::vector<uint32_t> presieve_primes_;
  uint32_t presieve_max_ = 0;

  // sieving primes > presieve_max_, ascending: all on the device (n_dev_);
  // exact host copy up to kHostExact, 1-in-kSample host sample of all
  static constexpr uint64_t kHostExact = 1ull << 24;
  static constexpr size_t kSample = 256;
  std::vector<uint32_t> h_primes_;
  std::vector<uint32_t> h_sample_;
  std::vector<double> h_inv_block_;      // [blocks + 1] prefix of sum(1/p) per sample block
  std::vector<double> h_inv_head_;       // [head + 1] prefix of sum(1/p) over the exact head
  size_t n_dev_ = 0;
  uint64_t primes_upto_ = 0;
  uint32_t* d_primes_ = nullptr;
  uint64_t* d_recip_ = nullptr;
  size_t d_primes_cap_ = 0;

  // bucket storage
  uint32_t* d_entries_ = nullptr;
  size_t entries_cap_ = 0;
  uint32_t* d_bcounts_ = nullptr;
  size_t bcounts_cap_ = 0;
  uint32_t* d_entries2_ = nullptr;       // second list set (windows on the auxiliary stream)
  uint32_t* d_bcounts2_ = nullptr;
  size_t entries2_cap_ = 0, bcounts2_cap_ = 0;
  cudaStream_t aux_stream_ = nullptr;    // windows of list set 1
  cudaEvent_t fork_event_ = nullptr, join_event_ = nullptr;
  // Bucket plan of the current big primes [first, last) (host): geometry and
  // one u32 table [lists offsets | lists capacities | 3 (fill_ctas + 1)
  // fill chunk bounds: group walk, thread walk, primes above the window];
  // gen changes with every new plan.
  struct PlanGeom {
    uint64_t seg_stride = 0;              // entries per segment region
    uint32_t lists = 0, fill_ctas = 0;
  };
  struct BucketPlan {
    uint32_t first = 0, last = 0;            // last == 0: none
    PlanGeom geom;
    std::vector<uint32_t> table;
  };
  BucketPlan plan_;
  uint64_t plan_gen_ = 0;
  // device copy of a plan per list set, uploaded on the set's stream
  struct PlanSlot {
    uint64_t gen = 0;                      // plan_gen_ of the table it holds (0: none)
    PlanGeom geom;
    uint32_t* d_table = nullptr;
    size_t cap = 0;
  };
  PlanSlot slots_[2];
  // pinned upload sources, reused round robin once their copy has run
  struct Stage {
    uint32_t* h = nullptr;
    size_t cap = 0;
    cudaEvent_t ev = nullptr;
    bool used = false;
  };
  static constexpr int kStages = 8;
  Stage stages_[kStages];
  int stage_next_ = 0;
  bool chain_ = false;                     // window sets alternate across run_windows calls
  bool batch_smem_set_ = false;            // persistent kernel's shared-memory limit raised
  uint32_t parity_ = 0;                    // next window's list set (bit 0)
  double cap_scale_ = 1.0;
  uint32_t* d_overflow_ = nullptr;         // overflow flag of synchronous paths (reset per use)
  uint32_t* d_async_overflow_ = nullptr;   // sticky flag of count_async, read by async_status
  uint32_t* cur_overflow_ = nullptr;       // the flag the next fill launches report to
  bool async_pending_ = false;             // count_async issued since the last async_status
  unsigned long long* d_entry_total_ = nullptr;
  uint64_t overflow_retries_ = 0;

  unsigned long long* d_counts_ = nullptr;
  unsigned long long* h_counts_ = nullptr;   // pinned
  uint8_t* bitmap_out_ = nullptr;            // set while run_windows stores bitmaps

  // batch storage
  unsigned long long* d_batch_rows_ = nullptr;
  size_t batch_rows_cap_ = 0;
  BatchRange* d_batch_ranges_ = nullptr;
  size_t batch_ranges_cap_ = 0;
  BatchItem* d_batch_items_ = nullptr;
  size_t batch_items_cap_ = 0;
  uint32_t* d_batch_queue_ = nullptr;
  std::vector<unsigned long long> h_batch_rows_;
  size_t batch_direct_ranges_ = 0, batch_bucket_ranges_ = 0, batch_items_ = 0;
  BatchClassParams batch_tune_[kBatchClasses];

  // profiling
  bool profiling_ = false;
  // launches are always counted; CUDA-event times only while profiling
  struct Timed { const char* name; std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev; uint64_t launches = 0; double ms = 0; };
  Timed timed_[3] = { { "sieve_count_kernel", {}, 0, 0 }, { "bucket_fill_kernel", {}, 0, 0 },
                      { "batch_sieve_kernel", {}, 0, 0 } };
};

} // namespace psg
