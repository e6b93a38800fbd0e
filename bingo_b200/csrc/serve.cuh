// Serving state shared by the serving kernel and its host scheduler.
#pragma once
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <list>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/bingo.h"
#include "common.cuh"
#include "engine.cuh"

namespace bingo {

constexpr uint32_t kServeMaxJobs = 4096;  // job ring capacity (power of two)
constexpr size_t kPinBytes = 64u << 20;    // pinned staging ring for publish copies

// Control block in device memory: written by the host (stream-ordered
// copies), polled by the serving kernel.
struct ServeCtl {
  volatile uint32_t published_jobs;  // job sequence numbers [0, published_jobs) are visible
  volatile uint32_t drain;           // exit once every published walk is claimed and finished
  volatile uint32_t stop;            // exit now
  uint32_t pad;
};

// Device-resident serving state. Walks are claimed per job: claim[slot]
// holds (job sequence number << 32) | walks handed out, opened by the warp
// that moves head_job onto that job, and taken 32 at a time by fetch-add
// (a tag that does not match the job asked for means "not open yet").
struct ServeDevState {
  uint32_t head_job;  // lowest job sequence number that may still have unclaimed walks
  uint32_t closing;   // set by the first warp that exits idle; every warp then exits (reset per launch)
  unsigned long long claim[kServeMaxJobs];
  uint32_t done[kServeMaxJobs];  // finished walks per ring slot
};

class Server {
 public:
  Server(Engine& eng, const bingo_serve_config& cfg);
  ~Server();
  uint64_t submit_walk(const bingo_walk_job& J);
  uint64_t submit_update(int kind, const uint32_t* a, const uint32_t* b, const uint32_t* c, uint64_t k,
                         uint32_t* out_slots);
  bool poll(uint64_t ticket, bingo_serve_status* out);
  bool wait(uint64_t ticket, uint64_t timeout_us, bingo_serve_status* out);
  void stats(uint64_t* completed, uint64_t* version);
  void metrics(bingo_serve_metrics* out);

 private:
  struct Request;
  struct InFlight;
  struct Ticket {
    int kind = 0;
    int done = 0;
    int status = 0;
    uint64_t version = 0, submit_ns = 0, done_ns = 0;
  };
  struct Region {
    size_t off, bytes;
    bool freed;
  };

  uint64_t enqueue(Request&& r);
  void finish_ticket(uint64_t ticket, int status, uint64_t version);
  bool alloc_region(size_t bytes, size_t* off);
  void release_region(size_t off);
  bool kernel_running();
  void launch_kernel();
  void push_ctl();
  bool step();
  void loop();

  Engine& eng_;
  bingo_serve_config cfg_;
  cudaStream_t kstream_ = nullptr, cstream_ = nullptr, rstream_ = nullptr;  // kernel, publish, results
  char* pin_ = nullptr;  // pinned staging ring
  size_t pin_head_ = 0;
  std::vector<cudaEvent_t> event_pool_;
  ServeCtl ctl_;             // host shadow
  ServeCtl* d_ctl_ = nullptr;
  volatile unsigned long long* done_seq_ = nullptr;
  unsigned long long* d_done_seq_ = nullptr;
  DevBuf jobs_, state_, budget_, ctlbuf_;
  bool launched_ = false;

  // scheduler-thread state
  std::list<InFlight> inflight_;
  std::set<uint32_t> retired_;
  std::deque<Region> regions_;
  size_t head_ = 0, tail_ = 0;
  uint32_t published_jobs_ = 0, oldest_ = 0;
  uint64_t version_ = 0;
  bingo_serve_metrics m_{};  // scheduler counters (guarded by mu_ when read)
  uint64_t drain_since_ = 0, drain_retired_ = 0;
  // The update batch enqueued on the engine's stream and not yet seen
  // complete (at most one; upd_ev_ marks its end, and every later walk
  // launch waits for it on the device).
  bool upd_pending_ = false;
  uint64_t upd_ticket_ = 0, upd_version_ = 0, upd_t0_ = 0;
  int upd_status_ = 0;
  cudaEvent_t upd_ev_ = nullptr;
  bool upd_recorded_ = false;

  // shared with submitters
  std::mutex mu_;
  std::condition_variable cv_, cv_done_;
  std::deque<Request> queue_;
  std::unordered_map<uint64_t, Ticket> tickets_;
  uint64_t next_ticket_ = 0;
  bool quit_ = false;
  std::string fatal_;
  std::thread thread_;
};

}  // namespace bingo
