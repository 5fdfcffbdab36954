// batch.cu -- Engine::count_batch: many ranges in one persistent launch.
//
// Plan (host, once per batch):
//  * 2/3/5 table per range on the host, as in count();
//  * one sieving-prime table for the largest stop;
//  * per range its prime tiers (small / medium with carried state / direct)
//    and its class: a range whose primes beyond the shared state are few
//    enough for its length (segments x such primes <= the direct budget of
//    its range class) is sieved entirely by the persistent batch kernel;
//    longer ranges with many big primes run through the windowed bucket path;
//  * direct ranges are cut into stripes of <= `stripe` segments (the medium
//    state is set up once per stripe), ordered most expensive first, and
//    served to the persistent grid from a device counter.
// The ranges' rows are accumulated on the device and read back once.
#include "engine.hpp"
#include "batch_kernel.cuh"
#include "../../include/psgpu.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

namespace psg {

namespace {


#define PSG_CUDA(call)                                                          \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      err = std::string(#call) + ": " + cudaGetErrorString(e_);                 \
      return PSG_ERR_CUDA;                                                      \
    }                                                                           \
  } while (0)

template <typename T>
int grow(T*& ptr, size_t& cap, size_t n, std::string& err) {
  if (n <= cap) return PSG_OK;
  const size_t c = std::max<size_t>(n, 2 * cap);
  cudaFree(ptr);
  ptr = nullptr;
  cap = 0;
  if (cudaMalloc(&ptr, c * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    err = "cannot allocate " + std::to_string(c * sizeof(T)) + " bytes of batch storage";
    return PSG_ERR_NOMEM;
  }
  cap = c;
  return PSG_OK;
}

} // namespace

uint64_t Engine::range_segments(const BatchRange& r) const {
  return (r.hi - 7 - r.seg_low0) / ((uint64_t) seg_bytes_ * 30u) + 1;
}

// Batch-kernel tiers of [lo, hi] (lo >= 7); false when the range has so many
// primes beyond the shared state for its length that the bucket path is
// cheaper. seg_cost: relative cost of one of its segments.
bool Engine::batch_range(uint64_t lo, uint64_t hi, uint32_t kinds, BatchRange& r, double& seg_cost) {
  const uint64_t span = (uint64_t) seg_bytes_ * 30u;
  const uint32_t small = batch_params(hi).small_limit ? batch_params(hi).small_limit : small_limit_;
  const uint32_t n_small_all = count_primes_le(small, true);           // inside the exact head
  const uint64_t seg_low0 = lo - ((lo - 7) % 30 + 7);
  const uint64_t nseg = (hi - 7 - seg_low0) / span + 1;
  const uint32_t n_total = count_primes_upper(isqrt_u64(hi));
  const uint32_t n_small = std::min(n_small_all, n_total);
  const uint32_t n_med = std::max(n_small, std::min(n_total, n_small_all + state_cap_));
  const double direct = (double) (n_total - n_med);
  if (direct > 0 && (direct * (double) nseg > batch_params(hi).direct_budget || nseg >= (1ull << 32))) return false;
  r.seg_low0 = seg_low0;
  r.lo = lo;
  r.hi = hi;
  r.n_small = n_small;
  r.n_med_end = n_med;
  r.n_end = n_total;
  r.kinds = kinds;
  // sieve work + one reciprocal per direct prime
  seg_cost = 1.0 + direct / 2.0e4;
  return true;
}

// Stripes of <= `stripe` segments (0: the range class's) of range `k` from segment s0 on, at most
// max_seg segments in all; returns the segment after the last one taken.
uint64_t Engine::append_stripes(uint32_t k, const BatchRange& r, double seg_cost, uint64_t s0, uint64_t max_seg,
                                std::vector<BatchItem>& items, std::vector<double>& cost, uint32_t stripe) const {
  const uint64_t nseg = range_segments(r);
  const uint32_t len_max = stripe ? stripe : batch_params(r.hi).stripe;
  const uint64_t nst = (nseg + len_max - 1) / len_max;
  const uint64_t len = (nseg + nst - 1) / nst;
  uint64_t taken = 0;
  while (s0 < nseg && taken < max_seg) {
    BatchItem it;
    it.range = k;
    it.seg0 = (uint32_t) s0;
    it.nseg = (uint32_t) std::min<uint64_t>(len, nseg - s0);
    it.pad = 0;
    items.push_back(it);
    cost.push_back(seg_cost * it.nseg);
    s0 += it.nseg;
    taken += it.nseg;
  }
  return s0;
}

void Engine::sort_items(std::vector<BatchItem>& items, const std::vector<double>& cost) {
  std::vector<uint32_t> order(items.size());
  for (size_t i = 0; i < order.size(); i++) order[i] = (uint32_t) i;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return cost[x] > cost[y]; });
  std::vector<BatchItem> sorted(items.size());
  for (size_t i = 0; i < order.size(); i++) sorted[i] = items[order[i]];
  items.swap(sorted);
}

// The persistent batch kernel over n_items device items (queue zeroed here).
int Engine::launch_items(const BatchRange* d_ranges, const BatchItem* d_items, uint32_t n_items,
                         unsigned long long* d_rows, uint32_t* d_queue, cudaStream_t st, std::string& err) {
  if (n_items == 0) return PSG_OK;
  PSG_CUDA(cudaMemsetAsync(d_queue, 0, sizeof(uint32_t), st));
  BatchArgs b;
  std::memset(&b, 0, sizeof b);
  fill_common_args(b.common);
  b.ranges = d_ranges;
  b.items = d_items;
  b.num_items = n_items;
  b.queue = d_queue;
  b.counts = d_rows;
  timed_begin(2, st);
  cudaError_t e = launch_batch(b, st);
  timed_end(2, st);
  if (e != cudaSuccess) { err = std::string("batch kernel launch: ") + cudaGetErrorString(e); return PSG_ERR_CUDA; }
  return PSG_OK;
}

constexpr double kTuneSampleIntegers = 2e12;   // autotuner objective size per class
constexpr double kTuneMargin = 0.03;           // a candidate must beat the defaults by this

int Engine::batch_class(uint64_t stop) {
  int d = 0;
  for (uint64_t v = stop; v >= 10; v /= 10) d++;
  return std::min(d, kBatchClasses - 1);
}

// Autotuner. Range class = decimal digits of stop. For every class present
// in q: its ranges (all of them up to ~2e12 integers, else a selection by
// length rank that keeps the longest) are counted once to warm up, then
// timed under each candidate (direct budget x direct-tier extent, then the
// small/medium threshold halved and doubled from the best of those); the
// class keeps the fastest if it beats the defaults by more than 3%. (Small samples
// under-fill the persistent grid and mislead the choice.)
// Candidates are tried in order until budget_s is used up; the defaults
// stay where nothing was timed.
int Engine::autotune_batch(const RangeQuery* q, size_t n, double budget_s, std::vector<TuneReport>& report,
                           std::string& err) {
  using Clock = std::chrono::steady_clock;
  const Clock::time_point t_start = Clock::now();
  const auto elapsed = [&]() { return std::chrono::duration<double>(Clock::now() - t_start).count(); };
  std::vector<std::vector<size_t>> by_class(kBatchClasses);
  for (size_t i = 0; i < n; i++)
    if (q[i].start <= q[i].stop && (q[i].kinds & 0x3fu) && q[i].stop >= 7)
      by_class[batch_class(q[i].stop)].push_back(i);
  const uint64_t span = (uint64_t) seg_bytes_ * 30u;
  const uint32_t big_candidates[2] = { big_limit_, (uint32_t) std::min<uint64_t>(span / 4, 0xffffffffull) };
  const double budgets[3] = { 1e7, 1e8, 1e9 };
  const uint32_t stripes[1] = { 8 };
  const uint32_t small_candidates[2] = { small_limit_ / 2, small_limit_ * 2 };
  std::vector<uint64_t> rows;
  int rc = PSG_OK;
  for (int c = 0; c < kBatchClasses && elapsed() < budget_s; c++) {
    std::vector<size_t>& idx = by_class[c];
    if (idx.size() < 4) continue;
    // objective: the class's own ranges (all of them up to ~kTuneSampleIntegers,
    // else an evenly spaced selection by length rank that keeps the longest)
    std::sort(idx.begin(), idx.end(), [&](size_t x, size_t y) {
      return q[x].stop - q[x].start > q[y].stop - q[y].start;
    });
    std::vector<RangeQuery> sample;
    double ints = 0, total = 0;
    for (size_t j : idx) total += (double) (q[j].stop - q[j].start) + 1.0;
    const size_t stride = total <= kTuneSampleIntegers ? 1 : std::max<size_t>(1, (size_t) (total / kTuneSampleIntegers));
    for (size_t j = 0; j < idx.size(); j += stride) {
      sample.push_back(q[idx[j]]);
      ints += (double) (q[idx[j]].stop - q[idx[j]].start) + 1.0;
    }
    rows.assign(6 * sample.size(), 0);
    const BatchClassParams keep = batch_tune_[c];
    TuneReport rep{};
    rep.cls = c;
    rep.sample_ranges = sample.size();
    rep.sample_integers = ints;
    rep.best_seconds = 1e30;
    rep.default_seconds = 0;
    BatchClassParams best = keep;
    bool first = true;
    bool over = false;
    const auto time_candidate = [&](const BatchClassParams& cand, double& sec) -> int {
      batch_tune_[c] = cand;
      int r = PSG_OK;
      if (first && (r = count_batch(sample.data(), sample.size(), rows.data(), err))) return r;   // warm-up
      first = false;
      const Clock::time_point t0 = Clock::now();
      if ((r = count_batch(sample.data(), sample.size(), rows.data(), err))) return r;
      sec = std::chrono::duration<double>(Clock::now() - t0).count();
      return PSG_OK;
    };
    // stage 1: batch-kernel budget x direct-tier extent of bucket-path ranges
    for (double db : budgets)
      for (uint32_t bl : big_candidates)
        for (uint32_t st : stripes) {
          if (!first && elapsed() > budget_s) { over = true; break; }
          BatchClassParams cand;
          cand.direct_budget = db;
          cand.big_limit = bl;
          cand.stripe = st;
          double sec = 0;
          if ((rc = time_candidate(cand, sec))) return rc;
          if (db == 1e8 && bl == big_limit_ && st == 8) rep.default_seconds = sec;
          if (sec < rep.best_seconds) { rep.best_seconds = sec; best = cand; }
        }
    // stage 2, from the best of stage 1: the small/medium threshold (the
    // primes below it are crossed off warp-cooperatively, the rest by the
    // carried wheel walk)
    for (uint32_t sl : small_candidates) {
      if (over || elapsed() > budget_s) break;
      BatchClassParams cand = best;
      cand.small_limit = sl;
      double sec = 0;
      if ((rc = time_candidate(cand, sec))) return rc;
      if (sec < rep.best_seconds) { rep.best_seconds = sec; best = cand; }
    }
    // keep the defaults unless a candidate wins clearly (timing noise)
    if (rep.default_seconds > 0 && rep.best_seconds > (1.0 - kTuneMargin) * rep.default_seconds) {
      best = keep;
      rep.best_seconds = rep.default_seconds;
    }
    batch_tune_[c] = best;
    rep.chosen = best;
    report.push_back(rep);
  }
  return PSG_OK;
}

int Engine::count_batch(const RangeQuery* q, size_t n, uint64_t* out, std::string& err) {
  PSG_CUDA(cudaSetDevice(device_));
  std::fill(out, out + 6 * n, 0ull);
  // the engine's scratch is shared with counts queued on other streams
  if (last_stream_ && last_stream_ != stream_) PSG_CUDA(cudaStreamWaitEvent(stream_, done_event_, 0));
  if (n == 0) return PSG_OK;

  // ---- 1. host part of every range, largest stop
  std::vector<uint64_t> lo(n, 0), hi(n, 0);
  std::vector<uint32_t> kinds(n, 0);
  uint64_t max_hi = 0;
  for (size_t i = 0; i < n; i++) {
    const uint32_t k = q[i].kinds & 0x3fu;
    if (q[i].start > q[i].stop || k == 0) continue;
    uint64_t tab[6] = { 0, 0, 0, 0, 0, 0 };
    small_table(q[i].start, q[i].stop, k, tab);
    for (int j = 0; j < 6; j++) out[6 * i + j] += tab[j];
    if (q[i].stop < 7) continue;
    lo[i] = std::max<uint64_t>(q[i].start, 7);
    hi[i] = q[i].stop;
    kinds[i] = k;
    max_hi = std::max(max_hi, hi[i]);
  }
  if (max_hi == 0) return PSG_OK;
  int rc = ensure_primes(std::max<uint32_t>(isqrt_u64(max_hi), 7u), err);
  if (rc) return rc;

  // ---- 2. tiers and class of every range
  std::vector<BatchRange> br;
  std::vector<size_t> br_index;             // batch range -> query
  std::vector<size_t> bucket_ranges;        // queries for the windowed path
  std::vector<double> seg_cost;             // per batch range: cost of one segment
  for (size_t i = 0; i < n; i++) {
    if (!kinds[i]) continue;
    BatchRange r;
    double c = 0;
    if (!batch_range(lo[i], hi[i], kinds[i], r, c)) {
      bucket_ranges.push_back(i);
      continue;
    }
    br.push_back(r);
    br_index.push_back(i);
    seg_cost.push_back(c);
  }

  // ---- 3. work items: stripes of <= kStripe segments, most expensive first
  std::vector<BatchItem> items;
  std::vector<double> item_cost;
  for (size_t k = 0; k < br.size(); k++)
    append_stripes((uint32_t) k, br[k], seg_cost[k], 0, ~0ull, items, item_cost);
  sort_items(items, item_cost);
  batch_direct_ranges_ = br.size();
  batch_bucket_ranges_ = bucket_ranges.size();
  batch_items_ = items.size();

  // ---- 4. device rows: direct ranges first, then bucket ranges
  const size_t rows = br.size() + bucket_ranges.size();
  if ((rc = grow(d_batch_rows_, batch_rows_cap_, 6 * rows, err))) return rc;
  if ((rc = grow(d_batch_ranges_, batch_ranges_cap_, std::max<size_t>(br.size(), 1), err))) return rc;
  if ((rc = grow(d_batch_items_, batch_items_cap_, std::max<size_t>(items.size(), 1), err))) return rc;
  h_batch_rows_.resize(6 * rows);
  PSG_CUDA(cudaMemsetAsync(d_batch_rows_, 0, 6 * rows * sizeof(unsigned long long), stream_));
  PSG_CUDA(cudaMemsetAsync(d_overflow_, 0, sizeof(uint32_t), stream_));

  // The bucket ranges' windows alternate between the two list sets across
  // ranges (one range's fill overlaps the previous one's sieve), and the
  // first ones may start on the auxiliary stream while the persistent kernel
  // still drains: the chain starts after the row reset, before that launch.
  struct Chain {
    Engine* e; cudaStream_t st;
    ~Chain() { e->chain_end(st); }
  } chain{ this, stream_ };
  if (!bucket_ranges.empty()) chain_begin(stream_);
  if (!items.empty()) {
    PSG_CUDA(cudaMemcpyAsync(d_batch_ranges_, br.data(), br.size() * sizeof(BatchRange), cudaMemcpyHostToDevice, stream_));
    PSG_CUDA(cudaMemcpyAsync(d_batch_items_, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice, stream_));
    rc = launch_items(d_batch_ranges_, d_batch_items_, (uint32_t) items.size(), d_batch_rows_,
                      d_batch_queue_, stream_, err);
    if (rc) return rc;
  }
  for (size_t j = 0; j < bucket_ranges.size(); j++) {
    const size_t i = bucket_ranges[j];
    RangePlan p;
    rc = plan_range(lo[i], hi[i], p, err, batch_params(hi[i]).big_limit, batch_params(hi[i]).small_limit);
    if (rc) return rc;
    rc = run_windows(p, kinds[i], d_batch_rows_ + 6 * (br.size() + j), stream_, 0, p.windows(), err);
    if (rc) return rc;
  }
  chain_end(stream_);

  // ---- 5. results
  uint32_t overflow = 0;
  PSG_CUDA(cudaMemcpyAsync(h_batch_rows_.data(), d_batch_rows_, 6 * rows * sizeof(unsigned long long),
                           cudaMemcpyDeviceToHost, stream_));
  PSG_CUDA(cudaMemcpyAsync(&overflow, d_overflow_, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
  PSG_CUDA(cudaStreamSynchronize(stream_));
  for (size_t k = 0; k < br.size(); k++)
    for (int j = 0; j < 6; j++) out[6 * br_index[k] + j] += h_batch_rows_[6 * k + j];
  for (size_t j = 0; j < bucket_ranges.size(); j++) {
    const size_t i = bucket_ranges[j];
    if (overflow) {
      // some bucket list overflowed: recount these ranges one by one
      // (count() grows the lists until nothing overflows)
      uint64_t c[6];
      rc = count(lo[i], hi[i], kinds[i], c, err);
      if (rc) return rc;
      for (int k = 0; k < 6; k++) out[6 * i + k] += c[k];
    } else {
      for (int k = 0; k < 6; k++) out[6 * i + k] += h_batch_rows_[6 * (br.size() + j) + k];
    }
  }
  PSG_CUDA(cudaEventRecord(done_event_, stream_));
  last_stream_ = stream_;
  return PSG_OK;
}

cudaError_t Engine::launch_batch(const BatchArgs& b, cudaStream_t st) {
  static_assert(sizeof(BatchArgs) < 4000, "kernel parameter space");
  switch (block_) {
    case 256:
      if (!batch_smem_set_) allow_max_dynamic_smem(batch_sieve_kernel<256>, device_);
      batch_sieve_kernel<256><<<grid_, 256, smem_dyn_, st>>>(b);
      break;
    case 1024:
      if (!batch_smem_set_) allow_max_dynamic_smem(batch_sieve_kernel<1024>, device_);
      batch_sieve_kernel<1024><<<grid_, 1024, smem_dyn_, st>>>(b);
      break;
    default:
      if (!batch_smem_set_) allow_max_dynamic_smem(batch_sieve_kernel<512>, device_);
      batch_sieve_kernel<512><<<grid_, 512, smem_dyn_, st>>>(b);
      break;
  }
  batch_smem_set_ = true;                 // the limit only ever rises (see allow_max_dynamic_smem)
  return cudaGetLastError();
}

} // namespace psg
