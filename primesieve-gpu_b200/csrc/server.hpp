// server.hpp -- request server with continuous batching.
//
// The reference answers one count per call (src/api.cpp:48-118); a service
// built on it would run requests one after another. Here a worker thread
// owns the engine and runs it in steps. Every step it
//   1. admits waiting requests into free device slots (a request whose
//      bucket storage would exceed the HBM budget is refused),
//   2. takes segment stripes round-robin from the admitted batch-class
//      requests (up to a segment budget) and runs them in one launch of the
//      persistent batch kernel, and up to two windows of the oldest
//      bucket-class request on the windowed path,
//   3. reads back the rows of the requests whose last piece ran and
//      completes them.
// Requests that arrive while a step is on the GPU join the next step, so
// small queries are not held behind large ones, and the sieving-prime table
// (up to the configured limit, 2^32 by default: every 64-bit stop) stays
// resident on the device.
#pragma once
#include <stdint.h>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.hpp"

namespace psg {

struct ServerConfig {
  uint32_t max_slots = 0;        // requests on the device at once (0: 4096)
  uint32_t step_segments = 0;    // batch-kernel segments per step (0: grid x 16)
  uint64_t prime_limit = 0;      // resident sieving-prime table (0: 2^32 - 1)
  uint64_t hbm_budget = 0;       // bytes of bucket storage allowed (0: 80% of free HBM)
};

struct ServerStats {
  uint64_t submitted = 0, completed = 0, refused = 0, steps = 0;
  uint64_t bucket_requests = 0, batch_requests = 0;
  double integers = 0;           // integers of completed requests
  double gpu_busy_seconds = 0;   // wall time of steps
};

class Server {
public:
  Server(Engine& engine, std::mutex& engine_mu) : eng_(engine), eng_mu_(engine_mu) {}
  ~Server();
  int start(const ServerConfig& cfg, std::string& err);
  void stop();

  // Queue a count of [start, stop]; id identifies it for wait().
  int submit(uint64_t start, uint64_t stop, uint32_t kinds, uint64_t& id, std::string& err);
  // Block until request id is done; counts overwritten, latency = done - submit.
  // Each id is collected once: a second wait() for it fails with PSG_ERR_ARG.
  int wait(uint64_t id, uint64_t counts[6], double* latency_s, std::string& err);
  // Submit q[i] at arrival_s[i] seconds after the call (one thread paces the
  // arrivals), wait for all; latency[i] from the scheduled arrival.
  int replay(const RangeQuery* q, const double* arrival_s, size_t n, uint64_t* counts,
             double* latency_s, std::string& err);
  ServerStats stats();
  // Tests of the failure handling: the nth request planned from now on
  // (nth >= 1; 0 cancels) makes its step fail with `status` at that point,
  // as a failed CUDA call there would.
  void inject_failure(uint32_t nth, int status);

private:
  using Clock = std::chrono::steady_clock;
  struct Request {
    uint64_t id = 0;
    uint64_t start = 0, stop = 0;
    uint32_t kinds = 0;
    uint64_t small[6] = { 0, 0, 0, 0, 0, 0 };   // 2/3/5 table (host)
    Clock::time_point t_submit, t_done;
    bool done = false;
    bool claimed = false;                       // a wait() (or replay) collects it
    int status = 0;
    std::string err;
    uint64_t counts[6] = { 0, 0, 0, 0, 0, 0 };
    // worker-only state
    bool planned = false, bucket = false;
    int slot = -1;
    BatchRange br{};
    double seg_cost = 0;
    uint64_t nseg = 0, next_seg = 0;            // batch class
    RangePlan plan;
    uint64_t nwin = 0, next_win = 0;            // bucket class
  };

  void loop();
  void release();                  // free the device and pinned buffers (engine mutex held)
  int step(std::vector<Request*>& admitted, std::string& err);
  void finish(Request* r, int status, const std::string& err);

  Engine& eng_;
  std::mutex& eng_mu_;
  ServerConfig cfg_;
  std::thread worker_;
  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  bool stop_ = false, started_ = false;
  uint64_t next_id_ = 1;
  std::deque<Request*> pending_;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs_;
  ServerStats stats_;
  uint32_t inject_countdown_ = 0;   // guarded by mu_
  int inject_status_ = 0;

  // worker-only
  std::vector<Request*> active_;
  std::vector<int> free_slots_;
  size_t hbm_budget_ = 0;
  cudaStream_t st_ = nullptr;
  BatchRange* d_ranges_ = nullptr;            // [slot]
  BatchItem* d_items_ = nullptr;
  size_t items_cap_ = 0;
  unsigned long long* d_rows_ = nullptr;      // [slot][6]
  unsigned long long* h_rows_ = nullptr;      // pinned
  uint32_t* d_queue_ = nullptr;
  uint32_t* h_flag_ = nullptr;                // pinned overflow flag
};

} // namespace psg
