// server.cpp -- request server with continuous batching (see server.hpp).
#include "server.hpp"
#include "../../include/psgpu.h"

#include <algorithm>
#include <cstring>

namespace psg {

namespace {

#define SRV_CUDA(call)                                                          \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      err = std::string(#call) + ": " + cudaGetErrorString(e_);                 \
      return PSG_ERR_CUDA;                                                      \
    }                                                                           \
  } while (0)

constexpr uint32_t kDefaultSlots = 4096;
// batch-kernel requests cost at most this many plain segments' work per
// segment (~1.7 ms on one SM); costlier ones take the bucket path
constexpr double kMaxSegCost = 16.0;
// bucket windows per step: with batch-class work waiting, and without
constexpr uint64_t kStepWindowsBusy = 2, kStepWindowsIdle = 4;

} // namespace

Server::~Server() { stop(); }

int Server::start(const ServerConfig& cfg, std::string& err) {
  if (started_) { err = "server already started"; return PSG_ERR_ARG; }
  cfg_ = cfg;
  if (!cfg_.max_slots) cfg_.max_slots = kDefaultSlots;
  if (!cfg_.step_segments) cfg_.step_segments = eng_.grid() * 16u;
  if (!cfg_.prime_limit) cfg_.prime_limit = 0xffffffffull;
  {
    std::lock_guard<std::mutex> g(eng_mu_);
    // whatever a failed start allocated is freed before it returns
    struct Undo {
      Server* s; bool armed = true;
      ~Undo() { if (armed) s->release(); }
    } undo{ this };
    SRV_CUDA(cudaSetDevice(eng_.device()));
    // resident sieving-prime table: every stop up to prime_limit^2
    const uint64_t lim = std::min<uint64_t>(cfg_.prime_limit, 0xffffffffull);
    const uint64_t stop = lim >= 0xffffffffull ? ~0ull : lim * lim;
    int rc = eng_.prepare(stop, err);
    if (rc) return rc;
    size_t free_b = 0, total_b = 0;
    SRV_CUDA(cudaMemGetInfo(&free_b, &total_b));
    hbm_budget_ = cfg_.hbm_budget ? (size_t) cfg_.hbm_budget : (size_t) (0.8 * (double) free_b);
    // warm-up: one full bucket window at the top of the table's reach (the
    // largest bucket storage any request can need, so the lists never grow
    // -- which waits for all work in flight -- while requests are served)
    // and one small range through the persistent kernel, so that no
    // request pays for buffer growth or a kernel's first launch
    {
      uint64_t c[6];
      const uint64_t span = std::min<uint64_t>(eng_.window_span(), stop - 7);
      rc = eng_.count(stop - span + 1, stop, 0x3f, c, err);
      const RangeQuery q{ 1000000000ull, 1001000000ull, 0x3f, 0 };
      uint64_t row[6];
      if (rc == PSG_OK) rc = eng_.count_batch(&q, 1, row, err);
      if (rc) return rc;
    }
    const size_t slots = cfg_.max_slots;
    st_ = eng_.stream();
    SRV_CUDA(cudaMalloc(&d_ranges_, slots * sizeof(BatchRange)));
    SRV_CUDA(cudaMalloc(&d_rows_, slots * 6 * sizeof(unsigned long long)));
    SRV_CUDA(cudaMallocHost(&h_rows_, slots * 6 * sizeof(unsigned long long)));
    SRV_CUDA(cudaMalloc(&d_queue_, sizeof(uint32_t)));
    SRV_CUDA(cudaMallocHost(&h_flag_, sizeof(uint32_t)));
    undo.armed = false;
  }
  free_slots_.clear();
  for (int s = (int) cfg_.max_slots - 1; s >= 0; s--) free_slots_.push_back(s);
  stop_ = false;
  try {
    worker_ = std::thread([this] { loop(); });
  } catch (...) {
    std::lock_guard<std::mutex> g(eng_mu_);
    free_slots_.clear();
    release();
    throw;
  }
  {
    std::lock_guard<std::mutex> lk(mu_);
    started_ = true;
  }
  return PSG_OK;
}

void Server::stop() {
  if (!started_) return;
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_work_.notify_all();
  worker_.join();
  started_ = false;
  std::lock_guard<std::mutex> g(eng_mu_);
  release();
}

void Server::release() {
  cudaSetDevice(eng_.device());
  if (st_) cudaStreamSynchronize(st_);
  cudaFree(d_ranges_); cudaFree(d_rows_); cudaFree(d_items_); cudaFree(d_queue_);
  if (h_rows_) cudaFreeHost(h_rows_);
  if (h_flag_) cudaFreeHost(h_flag_);
  d_ranges_ = nullptr; d_rows_ = nullptr; d_items_ = nullptr; d_queue_ = nullptr;
  h_rows_ = nullptr; h_flag_ = nullptr;
  items_cap_ = 0;
}

int Server::submit(uint64_t start, uint64_t stop, uint32_t kinds, uint64_t& id, std::string& err) {
  auto r = std::make_unique<Request>();
  r->start = start;
  r->stop = stop;
  r->kinds = kinds & 0x3fu;
  r->t_submit = Clock::now();
  const bool trivial = start > stop || r->kinds == 0 || stop < 7;
  if (start <= stop && r->kinds) small_table(start, stop, r->kinds, r->small);
  std::lock_guard<std::mutex> lk(mu_);
  if (!started_ || stop_) { err = "server is not running"; return PSG_ERR_CLOSED; }
  id = r->id = next_id_++;
  stats_.submitted++;
  Request* p = r.get();
  reqs_.emplace(id, std::move(r));
  if (trivial) {
    std::memcpy(p->counts, p->small, sizeof p->counts);
    p->done = true;
    p->t_done = Clock::now();
    stats_.completed++;
    return PSG_OK;
  }
  pending_.push_back(p);
  cv_work_.notify_one();
  return PSG_OK;
}

int Server::wait(uint64_t id, uint64_t counts[6], double* latency_s, std::string& err) {
  std::unique_lock<std::mutex> lk(mu_);
  auto it = reqs_.find(id);
  if (it == reqs_.end()) { err = "unknown request id " + std::to_string(id); return PSG_ERR_ARG; }
  Request* r = it->second.get();
  if (r->claimed) { err = "request " + std::to_string(id) + " is already being waited for"; return PSG_ERR_ARG; }
  r->claimed = true;
  cv_done_.wait(lk, [&] { return r->done; });
  if (counts) std::memcpy(counts, r->counts, 6 * sizeof(uint64_t));
  if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
  const int status = r->status;
  if (status) err = r->err;
  reqs_.erase(it);
  return status;
}

int Server::replay(const RangeQuery* q, const double* arrival_s, size_t n, uint64_t* counts,
                   double* latency_s, std::string& err) {
  std::vector<uint64_t> ids(n, 0);
  const Clock::time_point t0 = Clock::now();
  const auto due = [&](size_t i) {
    return t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrival_s[i]));
  };
  int rc = PSG_OK;
  size_t sent = 0;
  for (; sent < n; sent++) {
    std::this_thread::sleep_until(due(sent));
    rc = submit(q[sent].start, q[sent].stop, q[sent].kinds, ids[sent], err);
    if (rc) break;
    std::lock_guard<std::mutex> lk(mu_);
    auto it = reqs_.find(ids[sent]);
    if (it != reqs_.end()) it->second->claimed = true;
  }
  for (size_t i = 0; i < sent; i++) {
    double lat = 0;
    std::unique_lock<std::mutex> lk(mu_);
    auto it = reqs_.find(ids[i]);
    if (it == reqs_.end()) {              // collected by a wait() of its own
      if (rc == PSG_OK) { rc = PSG_ERR_ARG; err = "request " + std::to_string(ids[i]) + " was collected elsewhere"; }
      continue;
    }
    Request* r = it->second.get();
    cv_done_.wait(lk, [&] { return r->done; });
    // latency from the scheduled arrival, so a late submission is not hidden
    lat = std::chrono::duration<double>(r->t_done - due(i)).count();
    if (counts) std::memcpy(counts + 6 * i, r->counts, 6 * sizeof(uint64_t));
    if (latency_s) latency_s[i] = lat;
    if (r->status && rc == PSG_OK) { rc = r->status; err = r->err; }
    reqs_.erase(it);
  }
  return rc;
}

void Server::inject_failure(uint32_t nth, int status) {
  std::lock_guard<std::mutex> lk(mu_);
  inject_countdown_ = nth;
  inject_status_ = status;
}

ServerStats Server::stats() {
  std::lock_guard<std::mutex> lk(mu_);
  return stats_;
}

void Server::finish(Request* r, int status, const std::string& err) {
  std::lock_guard<std::mutex> lk(mu_);
  r->status = status;
  r->err = err;
  r->done = true;
  r->t_done = Clock::now();
  if (status == PSG_OK) {
    stats_.completed++;
    stats_.integers += (double) (r->stop - std::max<uint64_t>(r->start, 0) + 1);
  } else {
    stats_.refused++;
  }
  cv_done_.notify_all();
}

void Server::loop() {
  for (;;) {
    std::vector<Request*> admitted;
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_work_.wait(lk, [&] { return stop_ || !pending_.empty() || !active_.empty(); });
      if (stop_) {
        std::vector<Request*> left(pending_.begin(), pending_.end());
        pending_.clear();
        lk.unlock();
        left.insert(left.end(), active_.begin(), active_.end());
        active_.clear();
        for (Request* r : left) finish(r, PSG_ERR_CLOSED, "server stopped");
        return;
      }
      // free_slots_ and active_ belong to the worker thread (start() fills
      // free_slots_ before the worker exists); mu_ guards only pending_ here
      while (!pending_.empty() && !free_slots_.empty()) {
        Request* r = pending_.front();
        pending_.pop_front();
        r->slot = free_slots_.back();
        free_slots_.pop_back();
        admitted.push_back(r);
      }
    }
    std::string err;
    const Clock::time_point t = Clock::now();
    const int rc = step(admitted, err);
    {
      std::lock_guard<std::mutex> lk(mu_);
      stats_.steps++;
      stats_.gpu_busy_seconds += std::chrono::duration<double>(Clock::now() - t).count();
    }
    if (rc) {
      // a failed step leaves the rows unreliable: fail what is in flight,
      // and the requests admitted in this step that it did not get to plan
      // (refused ones are already finished and nulled out of `admitted`)
      for (Request* r : admitted)
        if (r && !r->planned) { free_slots_.push_back(r->slot); finish(r, rc, err); }
      for (Request* r : active_) { free_slots_.push_back(r->slot); finish(r, rc, err); }
      active_.clear();
    }
  }
}

int Server::step(std::vector<Request*>& admitted, std::string& err) {
  std::lock_guard<std::mutex> g(eng_mu_);
  SRV_CUDA(cudaSetDevice(eng_.device()));

  // ---- plan the newly admitted requests
  for (Request*& r : admitted) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (inject_countdown_ && --inject_countdown_ == 0) {
        err = "injected failure (psg_server_inject_failure)";
        return inject_status_;
      }
    }
    const uint64_t lo = std::max<uint64_t>(r->start, 7), hi = r->stop;
    // batch class unless the range needs the bucket path, or its segments
    // are so costly (many direct-tier primes, each located again per
    // segment on one SM) that the bucket path, which locates every prime
    // once per window across all SMs, answers sooner
    if (eng_.batch_range(lo, hi, r->kinds, r->br, r->seg_cost) && r->seg_cost <= kMaxSegCost) {
      r->bucket = false;
      r->nseg = eng_.range_segments(r->br);
      r->next_seg = 0;
      SRV_CUDA(cudaMemcpyAsync(d_ranges_ + r->slot, &r->br, sizeof(BatchRange), cudaMemcpyHostToDevice, st_));
      std::lock_guard<std::mutex> lk(mu_);
      stats_.batch_requests++;
    } else {
      int rc = eng_.plan_range(lo, hi, r->plan, err, eng_.batch_params(hi).big_limit,
                               eng_.batch_params(hi).small_limit);
      if (rc == PSG_OK && eng_.bucket_bytes(r->plan) > hbm_budget_) {
        rc = PSG_ERR_NOMEM;
        err = "bucket storage of [" + std::to_string(r->start) + ", " + std::to_string(r->stop) +
              "] exceeds the HBM budget of the server";
      }
      if (rc) {
        free_slots_.push_back(r->slot);
        Request* done = r;
        r = nullptr;                 // a waiter may free it once it is finished
        finish(done, rc, err);
        err.clear();
        continue;
      }
      r->bucket = true;
      r->nwin = r->plan.windows();
      r->next_win = 0;
      std::lock_guard<std::mutex> lk(mu_);
      stats_.bucket_requests++;
    }
    SRV_CUDA(cudaMemsetAsync(d_rows_ + 6ull * r->slot, 0, 6 * sizeof(unsigned long long), st_));
    r->planned = true;
    active_.push_back(r);
  }
  if (active_.empty()) return PSG_OK;

  // ---- batch-kernel work: one stripe per request per round, oldest first
  std::vector<BatchItem> items;
  std::vector<double> cost;
  int64_t budget = cfg_.step_segments;
  for (bool any = true; any && budget > 0;) {
    any = false;
    for (Request* r : active_) {
      if (r->bucket || r->next_seg >= r->nseg) continue;
      const size_t before = items.size();
      r->next_seg = eng_.append_stripes((uint32_t) r->slot, r->br, r->seg_cost, r->next_seg, 1, items, cost);
      for (size_t i = before; i < items.size(); i++) budget -= items[i].nseg;
      any = true;
      if (budget <= 0) break;
    }
  }
  Engine::sort_items(items, cost);

  // ---- bucket-class windows: requests with the fewest windows left first
  // (short requests do not queue behind long ones), the oldest request at
  // least one window per step; their windows chain across requests, so one
  // window's fill overlaps the previous one's sieve, and the chain starts
  // before the persistent launch, so the first windows can take the SMs its
  // tail leaves idle
  std::vector<std::pair<Request*, uint64_t>> wplan;
  {
    std::vector<Request*> cand;
    for (Request* r : active_)
      if (r->bucket && r->next_win < r->nwin) cand.push_back(r);
    if (!cand.empty()) {
      Request* oldest = cand.front();
      std::stable_sort(cand.begin(), cand.end(), [](const Request* x, const Request* y) {
        return x->nwin - x->next_win < y->nwin - y->next_win;
      });
      uint64_t left = items.empty() ? kStepWindowsIdle : kStepWindowsBusy;
      bool has_oldest = false;
      for (Request* r : cand) {
        if (left == 0) break;
        const uint64_t nw = std::min<uint64_t>(left, r->nwin - r->next_win);
        wplan.emplace_back(r, nw);
        left -= nw;
        has_oldest = has_oldest || r == oldest;
      }
      if (!has_oldest) wplan.emplace_back(oldest, 1);
      SRV_CUDA(cudaMemsetAsync(eng_.overflow_flag(), 0, sizeof(uint32_t), st_));
      eng_.chain_begin(st_);
    }
  }
  struct Chain {
    Engine& e; cudaStream_t st;
    ~Chain() { e.chain_end(st); }
  } chain{ eng_, st_ };

  if (!items.empty()) {
    if (items.size() > items_cap_) {
      cudaFree(d_items_);
      d_items_ = nullptr;
      items_cap_ = 0;
      SRV_CUDA(cudaMalloc(&d_items_, 2 * items.size() * sizeof(BatchItem)));
      items_cap_ = 2 * items.size();
    }
    SRV_CUDA(cudaMemcpyAsync(d_items_, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice, st_));
    int rc = eng_.launch_items(d_ranges_, d_items_, (uint32_t) items.size(), d_rows_, d_queue_, st_, err);
    if (rc) return rc;
  }

  std::vector<Request*> ran;
  for (auto& w : wplan) {
    Request* r = w.first;
    const int rc = eng_.run_windows(r->plan, r->kinds, d_rows_ + 6ull * r->slot, st_, r->next_win, w.second, err);
    if (rc) return rc;
    r->next_win += w.second;
    ran.push_back(r);
  }
  eng_.chain_end(st_);
  if (!wplan.empty())
    SRV_CUDA(cudaMemcpyAsync(h_flag_, eng_.overflow_flag(), sizeof(uint32_t), cudaMemcpyDeviceToHost, st_));

  // ---- read back and complete
  int top = 0;
  for (Request* r : active_) top = std::max(top, r->slot + 1);
  SRV_CUDA(cudaMemcpyAsync(h_rows_, d_rows_, (size_t) top * 6 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st_));
  SRV_CUDA(cudaStreamSynchronize(st_));
  if (!ran.empty() && *h_flag_) {
    // a bucket list of one of this step's windows overflowed: grow the lists
    // and count those requests again from their first windows
    eng_.grow_bucket_lists();
    for (Request* r : ran) {
      r->next_win = 0;
      SRV_CUDA(cudaMemsetAsync(d_rows_ + 6ull * r->slot, 0, 6 * sizeof(unsigned long long), st_));
    }
  }
  std::vector<Request*> still;
  for (Request* r : active_) {
    const bool complete = r->bucket ? r->next_win >= r->nwin : r->next_seg >= r->nseg;
    if (!complete) { still.push_back(r); continue; }
    for (int k = 0; k < 6; k++) r->counts[k] = r->small[k] + h_rows_[6 * r->slot + k];
    free_slots_.push_back(r->slot);
    finish(r, PSG_OK, std::string());
  }
  active_.swap(still);
  return PSG_OK;
}

} // namespace psg
