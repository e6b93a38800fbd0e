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

#include "../../include/bingo.h"
#include "common.cuh"
#include "engine.cuh"

namespace bingo {

constexpr uint32_t kServeMaxJobs = 4096;  // job ring capacity (power of two)

// Control block in mapped pinned host memory: written by the host, polled
// by the serving kernel.
struct ServeCtl {
  volatile unsigned long long published_items;  // walk items [0, published_items) are claimable
  volatile uint32_t published_jobs;             // job sequence numbers [0, published_jobs) are visible
  volatile uint32_t oldest_job;                 // lowest sequence number not yet retired
  volatile uint32_t drain;                      // exit once every published item is finished
  volatile uint32_t stop;                       // exit now
};

// Device-resident serving state.
struct ServeDevState {
  unsigned long long next_item;  // next unclaimed walk item
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
  bool step();
  void loop();

  Engine& eng_;
  bingo_serve_config cfg_;
  cudaStream_t kstream_ = nullptr, cstream_ = nullptr;
  ServeCtl* ctl_ = nullptr;
  ServeCtl* d_ctl_ = nullptr;
  volatile unsigned long long* done_seq_ = nullptr;
  unsigned long long* d_done_seq_ = nullptr;
  DevBuf jobs_, base_, state_, budget_;
  bool launched_ = false;

  // scheduler-thread state
  std::list<InFlight> inflight_;
  std::set<uint32_t> retired_;
  std::deque<Region> regions_;
  size_t head_ = 0, tail_ = 0;
  uint32_t published_jobs_ = 0, oldest_ = 0;
  unsigned long long published_items_ = 0;
  uint64_t version_ = 0;

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
