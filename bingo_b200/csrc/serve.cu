// Serving: continuous batching of walk queries with interleaved update batches.
//
// Walk queries are admitted into a running persistent kernel as ring slots
// and output memory free up; their walks mix with the walks of every other
// admitted query on the device. Update batches commit between walk epochs:
// a query sees the graph after exactly the updates submitted before it
// (FIFO versioning), so its result equals the result of running it alone on
// that graph version (walks are keyed by (walk, step, trial, job) only).
//
// Device side: k_serve polls a control block in mapped pinned host memory
// with a bounded, backed-off spin and exits after an idle limit (the host
// relaunches it when work arrives). Items are claimed with a CAS bounded by
// the published item count; each lane copies its job's descriptor into
// shared memory through L2 (ring slots are reused while the kernel runs, and
// L1 is not coherent); the lane that finishes a job's last walk fences and
// writes the job's sequence number + 1 to a completion word in mapped memory.
//
// Host side: a scheduler thread admits queries in submission order (HBM
// budget for outputs and starts, ring capacity), applies updates after the
// walks before them have finished, copies finished outputs to the caller's
// buffers and records submit-to-ready latency.
#include <atomic>
#include <chrono>
#include <cstring>
#include <vector>

#include "engine.cuh"
#include "serve.cuh"
#include "walk.cuh"

namespace bingo {

namespace {

constexpr int kServeBlock = 256;

__global__ void __launch_bounds__(kServeBlock, 4)
    k_serve(WalkView W, const WalkJobDev* __restrict__ jobs, const unsigned long long* __restrict__ base,
            ServeCtl* ctl, ServeDevState* st, volatile unsigned long long* done_seq, uint32_t idle_limit) {
  __shared__ __align__(16) int32_t obuf[kServeBlock][8];
  __shared__ __align__(16) WalkJobDev jc[kServeBlock];
  const int lane = threadIdx.x & 31;
  WalkJobDev& J = jc[threadIdx.x];
  LaneWalk s;
  RowStage o{kNoSec, 0};
  uint32_t moves = 0, jseq = 0, idle_iters = 0;
  unsigned long long wb = 0, we = 0;
  bool active = false;

  auto finish = [&]() {
    __threadfence();  // this lane's row writes before the completion count
    const uint32_t slot = jseq & (kServeMaxJobs - 1);
    if (atomicAdd(&st->done[slot], 1u) + 1 == (uint32_t)J.n) {
      __threadfence_system();
      done_seq[slot] = (unsigned long long)jseq + 1;
    }
  };

  for (;;) {
    uint32_t idle = __ballot_sync(kFull, !active);
    while (idle) {
      if (wb >= we) {
        unsigned long long cur = 0, got = 0;
        if (lane == 0) {
          cur = *reinterpret_cast<volatile unsigned long long*>(&st->next_item);
          const unsigned long long pub = ctl->published_items;
          while (cur < pub) {
            const unsigned long long take = min((unsigned long long)32, pub - cur);
            const unsigned long long old = atomicCAS(&st->next_item, cur, cur + take);
            if (old == cur) {
              got = take;
              break;
            }
            cur = old;
          }
        }
        cur = __shfl_sync(kFull, cur, 0);
        got = __shfl_sync(kFull, got, 0);
        if (!got) break;
        wb = cur;
        we = cur + got;
      }
      const uint32_t take = (uint32_t)min((unsigned long long)__popc(idle), we - wb);
      const uint32_t rank = __popc(idle & lanemask_lt());
      if (!active && rank < take) {
        const unsigned long long item = wb + rank;
        uint32_t lo = ctl->oldest_job, hi = ctl->published_jobs;
        while (hi - lo > 1) {
          const uint32_t mid = lo + ((hi - lo) >> 1);
          if (__ldcg(base + (mid & (kServeMaxJobs - 1))) <= item)
            lo = mid;
          else
            hi = mid;
        }
        jseq = lo;
        const uint32_t slot = lo & (kServeMaxJobs - 1);
        const int4* src = reinterpret_cast<const int4*>(jobs + slot);
        int4* dst = reinterpret_cast<int4*>(&J);
#pragma unroll
        for (int t = 0; t < (int)(sizeof(WalkJobDev) / 16); ++t) dst[t] = __ldcg(src + t);
        const uint32_t i = (uint32_t)(item - __ldcg(base + slot));
        active = begin_any(W, J, i, s, o, obuf, moves);
        if (!active) finish();
      }
      wb += take;
      idle = __ballot_sync(kFull, !active);
    }
    if (!__any_sync(kFull, active)) {
      int quit = 0;
      if (lane == 0) {
        const unsigned long long nx = *reinterpret_cast<volatile unsigned long long*>(&st->next_item);
        quit = (ctl->drain && nx >= ctl->published_items) || ctl->stop;
      }
      quit = __shfl_sync(kFull, quit, 0);
      if (quit || ++idle_iters > idle_limit) break;
      __nanosleep(1000);
      continue;
    }
    idle_iters = 0;
    if (active) {
      active = advance_any(W, J, s, o, obuf, moves);
      if (!active) finish();
    }
  }
  add_steps(W, moves);
}

uint64_t now_ns() {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

}  // namespace

// ---------------------------------------------------------------------------
struct Server::Request {
  uint64_t ticket;
  int kind;  // 0 walk, 1 insert, 2 delete
  bingo_walk_job job;
  std::vector<uint32_t> a, b, c;  // starts (walk) or batch columns
  uint32_t* out_slots = nullptr;
};

struct Server::InFlight {
  uint64_t ticket;
  uint32_t seq;
  size_t off, bytes;    // output-budget region
  int32_t* dev_out;
  int32_t* host_out;
  size_t out_bytes;
  bool copying = false;
  cudaEvent_t ev = nullptr;
};

Server::Server(Engine& eng, const bingo_serve_config& cfg) : eng_(eng), cfg_(cfg) {
  if (cfg_.max_jobs == 0 || cfg_.max_jobs > kServeMaxJobs) cfg_.max_jobs = kServeMaxJobs;
  if (!cfg_.output_budget_bytes) cfg_.output_budget_bytes = 1ull << 30;
  if (!cfg_.max_update_batch) cfg_.max_update_batch = 1u << 20;
  if (!cfg_.idle_timeout_us) cfg_.idle_timeout_us = 2000;
  cuda_check(cudaStreamCreateWithFlags(&kstream_, cudaStreamNonBlocking), "serve stream");
  cuda_check(cudaStreamCreateWithFlags(&cstream_, cudaStreamNonBlocking), "serve copy stream");
  cuda_check(cudaHostAlloc((void**)&ctl_, sizeof(ServeCtl), cudaHostAllocMapped), "serve control block");
  cuda_check(cudaHostAlloc((void**)&done_seq_, kServeMaxJobs * sizeof(unsigned long long), cudaHostAllocMapped),
             "serve completion words");
  std::memset((void*)ctl_, 0, sizeof(ServeCtl));
  std::memset((void*)done_seq_, 0, kServeMaxJobs * sizeof(unsigned long long));
  cuda_check(cudaHostGetDevicePointer((void**)&d_ctl_, (void*)ctl_, 0), "serve control block");
  cuda_check(cudaHostGetDevicePointer((void**)&d_done_seq_, (void*)done_seq_, 0), "serve completion words");
  jobs_.ensure(kServeMaxJobs * sizeof(WalkJobDev), "serve job ring");
  base_.ensure(kServeMaxJobs * sizeof(unsigned long long), "serve job ring");
  state_.ensure(sizeof(ServeDevState), "serve state");
  cuda_check(cudaMemset(state_.p, 0, sizeof(ServeDevState)), "serve state");
  budget_.ensure(cfg_.output_budget_bytes, "serve output budget");
  eng_.prepare_batches(cfg_.max_update_batch);
  thread_ = std::thread([this] { loop(); });
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    quit_ = true;
  }
  cv_.notify_all();
  if (thread_.joinable()) thread_.join();
  cudaStreamSynchronize(kstream_);
  cudaStreamSynchronize(cstream_);
  for (auto& f : inflight_)
    if (f.ev) cudaEventDestroy(f.ev);
  jobs_.release(), base_.release(), state_.release(), budget_.release();
  cudaFreeHost((void*)ctl_);
  cudaFreeHost((void*)done_seq_);
  cudaStreamDestroy(kstream_);
  cudaStreamDestroy(cstream_);
}

uint64_t Server::submit_walk(const bingo_walk_job& J) {
  if (J.app < 0 || J.app > 3) throw Error(BINGO_ERR_INVALID_ARGUMENT, "unknown app");
  if (J.app != BINGO_SAMPLING && J.length == 0) throw Error(BINGO_ERR_INVALID_ARGUMENT, "length must be >= 1");
  if (!J.n_starts) throw Error(BINGO_ERR_INVALID_ARGUMENT, "empty query");
  if (!J.out) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null output");
  if (J.n_starts >= (1ull << 31)) throw Error(BINGO_ERR_UNSUPPORTED, "query too large");
  const uint64_t per = J.app == BINGO_SAMPLING ? 1 : J.length;
  const uint64_t need = ((J.n_starts * per * 4 + 31) & ~31ull) + ((J.n_starts * 4 + 31) & ~31ull);
  if (need > cfg_.output_budget_bytes)
    throw Error(BINGO_ERR_CAPACITY, "query needs more device memory than the serving budget");
  eng_.check_walk_job(J);
  Request r;
  r.kind = 0;
  r.job = J;
  if (J.starts) {
    r.a.resize(J.n_starts);
    cuda_check(cudaMemcpy(r.a.data(), J.starts, J.n_starts * 4, cudaMemcpyDefault), "copy starts");
    for (uint32_t v : r.a)
      if (v >= eng_.n()) throw Error(BINGO_ERR_OUT_OF_RANGE, "start id >= n");
  } else if ((uint64_t)J.first + J.n_starts > eng_.n()) {
    throw Error(BINGO_ERR_OUT_OF_RANGE, "start range exceeds n");
  }
  return enqueue(std::move(r));
}

uint64_t Server::submit_update(int kind, const uint32_t* a, const uint32_t* b, const uint32_t* c, uint64_t k,
                               uint32_t* out_slots) {
  if (kind != BINGO_OP_INSERT && kind != BINGO_OP_DELETE) throw Error(BINGO_ERR_INVALID_ARGUMENT, "bad update kind");
  if (k && (!a || !b || (kind == BINGO_OP_INSERT && !c))) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null batch array");
  Request r;
  r.kind = kind;
  r.a.resize(k), r.b.resize(k);
  if (k) {
    cuda_check(cudaMemcpy(r.a.data(), a, k * 4, cudaMemcpyDefault), "copy batch");
    cuda_check(cudaMemcpy(r.b.data(), b, k * 4, cudaMemcpyDefault), "copy batch");
    if (kind == BINGO_OP_INSERT) {
      r.c.resize(k);
      cuda_check(cudaMemcpy(r.c.data(), c, k * 4, cudaMemcpyDefault), "copy batch");
    }
  }
  r.out_slots = out_slots;
  return enqueue(std::move(r));
}

uint64_t Server::enqueue(Request&& r) {
  std::lock_guard<std::mutex> lk(mu_);
  if (quit_) throw Error(BINGO_ERR_INVALID_ARGUMENT, "server is stopping");
  r.ticket = ++next_ticket_;
  Ticket& t = tickets_[r.ticket];
  t.submit_ns = now_ns();
  t.kind = r.kind;
  queue_.push_back(std::move(r));
  cv_.notify_all();
  return queue_.back().ticket;
}

bool Server::poll(uint64_t ticket, bingo_serve_status* out) {
  std::lock_guard<std::mutex> lk(mu_);
  auto it = tickets_.find(ticket);
  if (it == tickets_.end()) throw Error(BINGO_ERR_INVALID_ARGUMENT, "unknown ticket");
  const Ticket& t = it->second;
  if (out) {
    std::memset(out, 0, sizeof *out);
    out->done = t.done;
    out->status = t.status;
    out->version = t.version;
    out->latency_ns = t.done ? t.done_ns - t.submit_ns : 0;
    out->kind = t.kind;
  }
  return t.done;
}

bool Server::wait(uint64_t ticket, uint64_t timeout_us, bingo_serve_status* out) {
  std::unique_lock<std::mutex> lk(mu_);
  auto done = [&] {
    auto it = tickets_.find(ticket);
    return it == tickets_.end() || it->second.done;
  };
  if (!cv_done_.wait_for(lk, std::chrono::microseconds(timeout_us), done)) {
    lk.unlock();
    poll(ticket, out);
    return false;
  }
  lk.unlock();
  return poll(ticket, out);
}

void Server::finish_ticket(uint64_t ticket, int status, uint64_t version) {
  std::lock_guard<std::mutex> lk(mu_);
  Ticket& t = tickets_[ticket];
  t.done = 1;
  t.status = status;
  t.version = version;
  t.done_ns = now_ns();
  cv_done_.notify_all();
}

// Output-budget ring: regions are handed out in admission order and
// reclaimed from the oldest once they are released.
bool Server::alloc_region(size_t bytes, size_t* off) {
  const size_t cap = budget_.bytes;
  if (regions_.empty()) head_ = tail_ = 0;
  if (head_ >= tail_ || regions_.empty()) {
    if (head_ + bytes <= cap) {
      *off = head_;
    } else if (bytes <= tail_ || (regions_.empty() && bytes <= cap)) {
      *off = 0;
    } else {
      return false;
    }
  } else {
    if (head_ + bytes <= tail_)
      *off = head_;
    else
      return false;
  }
  head_ = *off + bytes;
  regions_.push_back({*off, bytes, false});
  return true;
}

void Server::release_region(size_t off) {
  for (auto& r : regions_)
    if (r.off == off) r.freed = true;
  while (!regions_.empty() && regions_.front().freed) regions_.pop_front();
  tail_ = regions_.empty() ? 0 : regions_.front().off;
  if (regions_.empty()) head_ = 0;
}

bool Server::kernel_running() {
  if (!launched_) return false;
  const cudaError_t q = cudaStreamQuery(kstream_);
  if (q == cudaErrorNotReady) return true;
  if (q != cudaSuccess) throw Error(BINGO_ERR_CUDA, std::string("serving kernel: ") + cudaGetErrorString(q));
  launched_ = false;
  return false;
}

void Server::launch_kernel() {
  if (kernel_running()) return;
  int sms = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_serve, kServeBlock, 0) != cudaSuccess || per_sm <= 0) {
    cudaGetLastError();
    per_sm = 2;
  }
  const uint32_t idle_limit = cfg_.idle_timeout_us;  // ~1 us per idle iteration
  k_serve<<<sms * per_sm, kServeBlock, 0, kstream_>>>(eng_.walk_view(), jobs_.as<WalkJobDev>(),
                                                       base_.as<unsigned long long>(), d_ctl_,
                                                       state_.as<ServeDevState>(), d_done_seq_, idle_limit);
  cuda_check(cudaGetLastError(), "serving kernel launch");
  eng_.count_launch();
  launched_ = true;
}

// One pass of the scheduler; returns true if anything progressed.
bool Server::step() {
  bool progress = false;
  // ---- completions (in any order), copies, retirement (in order)
  for (auto& f : inflight_) {
    if (!f.copying && done_seq_[f.seq & (kServeMaxJobs - 1)] == (unsigned long long)f.seq + 1) {
      cuda_check(cudaMemcpyAsync(f.host_out, f.dev_out, f.out_bytes, cudaMemcpyDefault, cstream_), "result copy");
      cuda_check(cudaEventCreateWithFlags(&f.ev, cudaEventDisableTiming), "event");
      cuda_check(cudaEventRecord(f.ev, cstream_), "event");
      f.copying = true;
      progress = true;
    }
  }
  for (auto it = inflight_.begin(); it != inflight_.end();) {
    if (it->copying && cudaEventQuery(it->ev) == cudaSuccess) {
      cudaEventDestroy(it->ev);
      finish_ticket(it->ticket, BINGO_OK, version_);
      release_region(it->off);
      retired_.insert(it->seq);
      it = inflight_.erase(it);
      progress = true;
    } else {
      ++it;
    }
  }
  while (retired_.count(oldest_)) {
    retired_.erase(oldest_);
    ++oldest_;
    ctl_->oldest_job = oldest_;
  }
  // ---- admission in submission order
  for (;;) {
    Request* r = nullptr;
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (queue_.empty()) break;
      r = &queue_.front();
    }
    if (r->kind == 0) {
      const bingo_walk_job& J = r->job;
      if (published_jobs_ - oldest_ >= cfg_.max_jobs) break;
      const uint64_t per = J.app == BINGO_SAMPLING ? 1 : J.length;
      const size_t out_bytes = J.n_starts * per * 4;
      const size_t ob = (out_bytes + 31) & ~(size_t)31, sb = r->a.empty() ? 0 : ((J.n_starts * 4 + 31) & ~31ull);
      size_t off = 0;
      if (!alloc_region(ob + sb, &off)) break;
      int32_t* dev_out = reinterpret_cast<int32_t*>(budget_.as<char>() + off);
      uint32_t* dev_starts = sb ? reinterpret_cast<uint32_t*>(budget_.as<char>() + off + ob) : nullptr;
      const uint32_t seq = published_jobs_;
      const uint32_t slot = seq & (kServeMaxJobs - 1);
      WalkJobDev D = eng_.make_job(J);
      D.out = dev_out;
      D.starts = dev_starts;
      const unsigned long long b0 = published_items_;
      if (dev_starts)
        cuda_check(cudaMemcpyAsync(dev_starts, r->a.data(), J.n_starts * 4, cudaMemcpyHostToDevice, cstream_),
                   "starts H2D");
      cuda_check(cudaMemcpyAsync(jobs_.as<WalkJobDev>() + slot, &D, sizeof D, cudaMemcpyHostToDevice, cstream_),
                 "job H2D");
      cuda_check(cudaMemcpyAsync(base_.as<unsigned long long>() + slot, &b0, 8, cudaMemcpyHostToDevice, cstream_),
                 "job H2D");
      cuda_check(cudaMemsetAsync(&state_.as<ServeDevState>()->done[slot], 0, 4, cstream_), "job reset");
      cuda_check(cudaStreamSynchronize(cstream_), "job publish");
      done_seq_[slot] = 0;
      published_items_ += J.n_starts;
      ++published_jobs_;
      std::atomic_thread_fence(std::memory_order_seq_cst);
      ctl_->published_items = published_items_;
      ctl_->published_jobs = published_jobs_;
      std::atomic_thread_fence(std::memory_order_seq_cst);
      inflight_.push_back(InFlight{r->ticket, seq, off, ob + sb, dev_out, J.out, out_bytes});
      {
        std::lock_guard<std::mutex> lk(mu_);
        tickets_[r->ticket].version = version_;
        queue_.pop_front();
      }
      launch_kernel();
      progress = true;
    } else {
      // An update waits for every walk admitted before it, then commits.
      if (!inflight_.empty() || oldest_ != published_jobs_) {
        ctl_->drain = 1;
        break;
      }
      ctl_->drain = 1;
      if (kernel_running()) break;
      int st = BINGO_OK;
      try {
        const uint64_t k = r->a.size();
        for (uint64_t o = 0; o < k; o += cfg_.max_update_batch) {
          const uint64_t len = std::min<uint64_t>(cfg_.max_update_batch, k - o);
          if (r->kind == BINGO_OP_INSERT)
            eng_.insert(r->a.data() + o, r->b.data() + o, r->c.data() + o, len,
                        r->out_slots ? r->out_slots + o : nullptr);
          else
            eng_.erase(r->a.data() + o, r->b.data() + o, len);
        }
      } catch (const Error& e) {
        st = e.status;
      }
      ++version_;
      ctl_->drain = 0;
      const uint64_t t = r->ticket;
      {
        std::lock_guard<std::mutex> lk(mu_);
        queue_.pop_front();
      }
      finish_ticket(t, st, version_);
      progress = true;
    }
  }
  // Keep a kernel alive while admitted walks are unfinished.
  if (!inflight_.empty() && !kernel_running()) {
    bool pending = false;
    for (auto& f : inflight_) pending |= !f.copying;
    if (pending) launch_kernel();
  }
  return progress;
}

void Server::loop() {
  cudaSetDevice(eng_.device());
  for (;;) {
    bool progress = false;
    try {
      progress = step();
    } catch (const Error& e) {
      std::lock_guard<std::mutex> lk(mu_);
      fatal_ = e.what();
      for (auto& r : queue_) {
        Ticket& t = tickets_[r.ticket];
        t.done = 1, t.status = e.status, t.done_ns = now_ns();
      }
      queue_.clear();
      for (auto& f : inflight_) {
        Ticket& t = tickets_[f.ticket];
        t.done = 1, t.status = e.status, t.done_ns = now_ns();
      }
      inflight_.clear();
      cv_done_.notify_all();
      quit_ = true;
    }
    std::unique_lock<std::mutex> lk(mu_);
    const bool idle = queue_.empty() && inflight_.empty();
    if (quit_ && idle) break;
    if (!progress) {
      if (idle)
        cv_.wait_for(lk, std::chrono::milliseconds(5));
      else {
        lk.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(10));
      }
    }
  }
  ctl_->stop = 1;
  cudaStreamSynchronize(kstream_);
}

void Server::stats(uint64_t* completed, uint64_t* version) {
  std::lock_guard<std::mutex> lk(mu_);
  uint64_t c = 0;
  for (auto& kv : tickets_) c += kv.second.done;
  *completed = c;
  *version = version_;
}

}  // namespace bingo
