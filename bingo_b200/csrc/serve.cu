// Serving: continuous batching of walk queries with interleaved update batches.
//
// Walk queries are admitted into a running persistent kernel as ring slots
// and output memory free up; their walks mix with the walks of every other
// admitted query on the device. Update batches commit between walk epochs:
// a query sees the graph after exactly the updates submitted before it
// (FIFO versioning), so its result equals the result of running it alone on
// that graph version (walks are keyed by (walk, step, trial, job) only).
//
// Device side: k_serve polls a control block in device memory (the host
// publishes with stream-ordered copies: a job's descriptor lands before the
// count that exposes it) with a bounded, exponentially backed-off spin and
// closes as a whole after an idle time limit (the host relaunches it when
// work arrives).
// Walks are claimed 32 at a time by fetch-add on a per-job counter tagged
// with the job's sequence number (no compare-and-swap loop across thousands
// of warps); each lane copies its job's descriptor into shared memory
// through L2 (ring slots are reused while the kernel runs, and
// L1 is not coherent); the lane that finishes a job's last walk fences and
// writes the job's sequence number + 1 to a completion word in mapped memory.
//
// Host side: a scheduler thread admits queries in submission order (HBM
// budget for outputs and starts, ring capacity), commits updates once the
// walks before them have finished on the device, copies finished outputs to
// the caller's buffers and records submit-to-ready latency. An update batch
// is enqueued on the engine's stream without a host wait; an event marks its
// end, the next walk-kernel launch waits for that event on the device, and
// the update's ticket completes when the scheduler sees the event.
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
constexpr uint32_t kPollSteps = 8;
constexpr uint32_t kSpinPasses = 20000;  // scheduler passes polled without sleeping

// Lane 0 of a warp: take up to 32 walks of the oldest job that has any left.
// Returns the count taken (0: none now); *none_left is set when every
// published job is fully handed out.
__device__ __forceinline__ uint32_t claim_walks(const WalkJobDev* __restrict__ jobs, const ServeCtl* ctl,
                                                ServeDevState* st, volatile unsigned long long* err_word,
                                                uint32_t* job, uint32_t* first, bool* none_left) {
  volatile ServeDevState* vs = st;
  *none_left = false;
  for (int tries = 0; tries < 4; ++tries) {
    const uint32_t h = vs->head_job;
    const uint32_t pj = ctl->published_jobs;
    if ((int32_t)(pj - h) <= 0) {
      *none_left = true;
      return 0;
    }
    const uint32_t slot = h & (kServeMaxJobs - 1);
    const unsigned long long old = atomicAdd(&st->claim[slot], 32ull);
    if ((uint32_t)(old >> 32) != h) return 0;  // its predecessor's advancer has not opened it yet
    const uint32_t c = (uint32_t)old;
    const unsigned long long n = __ldcg(&jobs[slot].n);
    if (__ldcg(&jobs[slot].seq) != h) {  // the slot was reused under a claim: never expected
      *err_word = 1;
      __threadfence_system();
      return 0;
    }
    if (c < n) {
      *job = h;
      *first = c;
      return (uint32_t)min(32ull, n - c);
    }
    // Exhausted: move head_job past it and open the next job's counter.
    if (atomicCAS(&st->head_job, h, h + 1) == h)
      atomicExch(&st->claim[(h + 1) & (kServeMaxJobs - 1)], (unsigned long long)(h + 1) << 32);
  }
  return 0;
}

__global__ void __launch_bounds__(kServeBlock, 4)
    k_serve(WalkView W, const WalkJobDev* __restrict__ jobs, const ServeCtl* ctl, ServeDevState* st,
            volatile unsigned long long* done_seq, volatile unsigned long long* err_word, uint32_t idle_us) {
  __shared__ __align__(16) int32_t obuf[kServeBlock][8];
  __shared__ __align__(16) WalkJobDev jc[kServeBlock];
  const int lane = threadIdx.x & 31;
  WalkJobDev& J = jc[threadIdx.x];
  LaneWalk s;
  RowStage o{kNoSec, 0};
  uint32_t moves = 0, jseq = 0, nap = 256, poll_in = 0;
  s.trials = 0, s.probes = 0;
  unsigned long long idle_ns = 0;
  uint32_t wj = 0, wb = 0, we = 0;  // this warp's claimed range: walks [wb, we) of job wj
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
    // A warp that still has walks in flight asks for more only when half its
    // lanes are idle or every kPollSteps steps.
    const bool may_claim = idle == kFull || __popc(idle) >= 16 || poll_in == 0;
    poll_in = poll_in ? poll_in - 1 : kPollSteps;
    int none_left = 0;
    while (idle) {
      if (wb >= we) {
        if (!may_claim) break;
        uint32_t cj = 0, cb = 0, got = 0;
        // A closing kernel takes no new walks (its warps finish the walks
        // they hold and exit; the host relaunches a full grid for the rest).
        if (lane == 0 && !reinterpret_cast<volatile ServeDevState*>(st)->closing) {
          bool nl = false;
          got = claim_walks(jobs, ctl, st, err_word, &cj, &cb, &nl);
          none_left = nl;
        }
        got = __shfl_sync(kFull, got, 0);
        if (!got) {
          none_left = __shfl_sync(kFull, none_left, 0);
          break;
        }
        wj = __shfl_sync(kFull, cj, 0);
        wb = __shfl_sync(kFull, cb, 0);
        we = wb + got;
      }
      const uint32_t take = min((uint32_t)__popc(idle), we - wb);
      const uint32_t rank = __popc(idle & lanemask_lt());
      if (!active && rank < take) {
        jseq = wj;
        const int4* src = reinterpret_cast<const int4*>(jobs + (wj & (kServeMaxJobs - 1)));
        int4* dst = reinterpret_cast<int4*>(&J);
#pragma unroll
        for (int t = 0; t < (int)(sizeof(WalkJobDev) / 16); ++t) dst[t] = __ldcg(src + t);
        active = begin_any(W, J, wb + rank, s, o, obuf, moves);
        if (!active) finish();
      }
      wb += take;
      idle = __ballot_sync(kFull, !active);
    }
    if (!__any_sync(kFull, active)) {
      // Idle warp (its last claim attempt just ran): exit on drain, stop or a
      // closing kernel; after the idle limit, close the whole kernel (only
      // while nothing is unclaimed), so the host never sees a kernel that
      // runs on with a few warps left.
      int quit = 0;
      if (lane == 0) {
        volatile ServeDevState* vs = st;
        quit = (ctl->drain && none_left) || ctl->stop || vs->closing;
        if (!quit && none_left && idle_ns > (unsigned long long)idle_us * 1000) {
          atomicExch(&st->closing, 1u);
          quit = 1;
        }
      }
      quit = __shfl_sync(kFull, quit, 0);
      if (quit) break;
      __nanosleep(nap);
      idle_ns += nap;
      nap = min(nap * 2, 16384u);
      continue;
    }
    nap = 256;
    idle_ns = 0;
    if (active) {
      active = advance_any(W, J, s, o, obuf, moves);
      if (!active) finish();
    }
  }
  add_steps(W, moves);
  add_n2v(W, s);
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
  uint64_t admit_ns = 0, device_done_ns = 0;
};

Server::Server(Engine& eng, const bingo_serve_config& cfg) : eng_(eng), cfg_(cfg) {
  if (cfg_.max_jobs == 0 || cfg_.max_jobs > kServeMaxJobs) cfg_.max_jobs = kServeMaxJobs;
  if (!cfg_.output_budget_bytes) cfg_.output_budget_bytes = 1ull << 30;
  if (!cfg_.max_update_batch) cfg_.max_update_batch = 1u << 20;
  if (!cfg_.idle_timeout_us) cfg_.idle_timeout_us = 2000;
  cuda_check(cudaStreamCreateWithFlags(&kstream_, cudaStreamNonBlocking), "serve stream");
  cuda_check(cudaStreamCreateWithFlags(&cstream_, cudaStreamNonBlocking), "serve publish stream");
  cuda_check(cudaStreamCreateWithFlags(&rstream_, cudaStreamNonBlocking), "serve result stream");
  cuda_check(cudaHostAlloc((void**)&pin_, kPinBytes, cudaHostAllocDefault), "serve staging");
  cuda_check(cudaHostAlloc((void**)&done_seq_, (kServeMaxJobs + 1) * sizeof(unsigned long long), cudaHostAllocMapped),
             "serve completion words");
  std::memset((void*)done_seq_, 0, (kServeMaxJobs + 1) * sizeof(unsigned long long));
  cuda_check(cudaHostGetDevicePointer((void**)&d_done_seq_, (void*)done_seq_, 0), "serve completion words");
  ctlbuf_.ensure(sizeof(ServeCtl), "serve control block");
  d_ctl_ = ctlbuf_.as<ServeCtl>();
  std::memset(&ctl_, 0, sizeof ctl_);
  cuda_check(cudaMemcpy(d_ctl_, &ctl_, sizeof ctl_, cudaMemcpyHostToDevice), "serve control block");
  jobs_.ensure(kServeMaxJobs * sizeof(WalkJobDev), "serve job ring");
  state_.ensure(sizeof(ServeDevState), "serve state");
  cuda_check(cudaMemset(state_.p, 0, sizeof(ServeDevState)), "serve state");
  budget_.ensure(cfg_.output_budget_bytes, "serve output budget");
  eng_.prepare_batches(cfg_.max_update_batch);
  cuda_check(cudaEventCreateWithFlags(&upd_ev_, cudaEventDisableTiming), "serve update event");
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
  cudaStreamSynchronize(rstream_);
  cudaStreamSynchronize(eng_.stream());
  eng_.set_defer_sync(false);
  if (upd_ev_) cudaEventDestroy(upd_ev_);
  for (auto& f : inflight_)
    if (f.ev) cudaEventDestroy(f.ev);
  for (cudaEvent_t e : event_pool_) cudaEventDestroy(e);
  cudaFreeHost(pin_);
  jobs_.release(), state_.release(), budget_.release(), ctlbuf_.release();
  cudaFreeHost((void*)done_seq_);
  cudaStreamDestroy(kstream_);
  cudaStreamDestroy(cstream_);
  cudaStreamDestroy(rstream_);
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
    if (is_device_ptr(J.starts))
      cuda_check(cudaMemcpy(r.a.data(), J.starts, J.n_starts * 4, cudaMemcpyDeviceToHost), "copy starts");
    else
      std::memcpy(r.a.data(), J.starts, J.n_starts * 4);
    for (uint32_t v : r.a)
      if (v >= eng_.n()) throw Error(BINGO_ERR_OUT_OF_RANGE, "start id >= n");
  } else if ((uint64_t)J.first + J.n_starts > eng_.n()) {
    throw Error(BINGO_ERR_OUT_OF_RANGE, "start range exceeds n");
  }
  return enqueue(std::move(r));
}

uint64_t Server::submit_update(int kind, const uint32_t* a, const uint32_t* b, const uint32_t* c, uint64_t k,
                               uint32_t* out_slots) {
  if (kind != BINGO_OP_INSERT && kind != BINGO_OP_DELETE && kind != BINGO_OP_DELETE_PAIRS)
    throw Error(BINGO_ERR_INVALID_ARGUMENT, "bad update kind");
  if (k && (!a || !b || (kind == BINGO_OP_INSERT && !c))) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null batch array");
  Request r;
  r.kind = kind;
  auto grab = [&](std::vector<uint32_t>& dst, const uint32_t* src) {
    dst.resize(k);
    if (is_device_ptr(src))
      cuda_check(cudaMemcpy(dst.data(), src, k * 4, cudaMemcpyDeviceToHost), "copy batch");
    else
      std::memcpy(dst.data(), src, k * 4);
  };
  if (k) {
    grab(r.a, a);
    grab(r.b, b);
    if (kind == BINGO_OP_INSERT) grab(r.c, c);
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
    out->ready_ns = t.done ? t.done_ns : 0;
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
  // Walks read the graph only after the last update batch has applied.
  if (upd_recorded_) cuda_check(cudaStreamWaitEvent(kstream_, upd_ev_, 0), "serve launch after update");
  cuda_check(cudaMemsetAsync(&state_.as<ServeDevState>()->closing, 0, 4, kstream_), "serve launch");
  k_serve<<<sms * per_sm, kServeBlock, 0, kstream_>>>(eng_.walk_view(), jobs_.as<WalkJobDev>(), d_ctl_,
                                                       state_.as<ServeDevState>(), d_done_seq_,
                                                       d_done_seq_ + kServeMaxJobs, cfg_.idle_timeout_us);
  cuda_check(cudaGetLastError(), "serving kernel launch");
  eng_.count_launch();
  {
    std::lock_guard<std::mutex> lk(mu_);
    ++m_.walk_kernel_launches;
  }
  launched_ = true;
}

// One pass of the scheduler; returns true if anything progressed.
bool Server::step() {
  bool progress = false;
  const uint64_t t_begin = now_ns();
  // ---- completions (in any order), copies, retirement (in order)
  for (auto& f : inflight_) {
    if (!f.copying && done_seq_[f.seq & (kServeMaxJobs - 1)] == (unsigned long long)f.seq + 1) {
      cuda_check(cudaMemcpyAsync(f.host_out, f.dev_out, f.out_bytes, cudaMemcpyDefault, rstream_), "result copy");
      if (event_pool_.empty()) {
        cudaEvent_t e;
        cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        event_pool_.push_back(e);
      }
      f.ev = event_pool_.back();
      event_pool_.pop_back();
      cuda_check(cudaEventRecord(f.ev, rstream_), "event");
      f.copying = true;
      f.device_done_ns = now_ns();
      progress = true;
    }
  }
  for (auto it = inflight_.begin(); it != inflight_.end();) {
    if (it->copying && cudaEventQuery(it->ev) == cudaSuccess) {
      event_pool_.push_back(it->ev);
      it->ev = nullptr;
      {
        std::lock_guard<std::mutex> lk(mu_);
        const uint64_t t = now_ns();
        m_.device_ns += it->device_done_ns - it->admit_ns;
        m_.copy_ns += t - it->device_done_ns;
      }
      finish_ticket(it->ticket, BINGO_OK, version_);
      release_region(it->off);
      retired_.insert(it->seq);
      it = inflight_.erase(it);
      progress = true;
    } else {
      ++it;
    }
  }
  if (upd_pending_) {
    const cudaError_t q = cudaEventQuery(upd_ev_);
    if (q == cudaSuccess) {
      // Device-reported problems of the batch (skipped deletes) read here;
      // nothing else runs on the engine's stream meanwhile.
      const int dev_st = eng_.sync();
      const int st = upd_status_ ? upd_status_ : dev_st;
      {
        std::lock_guard<std::mutex> lk(mu_);
        m_.update_ns += now_ns() - upd_t0_;
      }
      upd_pending_ = false;
      finish_ticket(upd_ticket_, st, upd_version_);
      progress = true;
    } else if (q != cudaErrorNotReady) {
      throw Error(BINGO_ERR_CUDA, std::string("serving update: ") + cudaGetErrorString(q));
    }
  }
  const uint64_t t_completed = now_ns();
  if (done_seq_[kServeMaxJobs]) throw Error(BINGO_ERR_CUDA, "serving kernel met a reused job slot");
  while (retired_.count(oldest_)) {
    retired_.erase(oldest_);
    ++oldest_;
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
      const uint64_t t_adm = now_ns();
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
      // Publish sources go through the pinned staging ring so the copies are
      // asynchronous; the ring restarts once the publish stream has drained.
      const size_t need_pin = sizeof(WalkJobDev) + 64 + (dev_starts ? J.n_starts * 4 : 0);
      if (pin_head_ + need_pin > kPinBytes) {
        cuda_check(cudaStreamSynchronize(cstream_), "staging wrap");
        pin_head_ = 0;
      }
      WalkJobDev* hD = reinterpret_cast<WalkJobDev*>(pin_ + pin_head_);
      *hD = eng_.make_job(J);
      hD->out = dev_out;
      hD->starts = dev_starts;
      hD->seq = seq;
      pin_head_ += (sizeof(WalkJobDev) + 63) & ~(size_t)63;
      if (dev_starts) {
        uint32_t* hs = reinterpret_cast<uint32_t*>(pin_ + pin_head_);
        std::memcpy(hs, r->a.data(), J.n_starts * 4);
        pin_head_ += (J.n_starts * 4 + 63) & ~(size_t)63;
        cuda_check(cudaMemcpyAsync(dev_starts, hs, J.n_starts * 4, cudaMemcpyHostToDevice, cstream_), "starts H2D");
      }
      cuda_check(cudaMemcpyAsync(jobs_.as<WalkJobDev>() + slot, hD, sizeof(WalkJobDev), cudaMemcpyHostToDevice,
                                 cstream_),
                 "job H2D");
      cuda_check(cudaMemsetAsync(&state_.as<ServeDevState>()->done[slot], 0, 4, cstream_), "job reset");
      done_seq_[slot] = 0;
      ++published_jobs_;
      ctl_.published_jobs = published_jobs_;
      push_ctl();  // ordered after the descriptor copies on the same stream
      inflight_.push_back(InFlight{r->ticket, seq, off, ob + sb, dev_out, J.out, out_bytes});
      inflight_.back().admit_ns = t_adm;
      {
        std::lock_guard<std::mutex> lk(mu_);
        tickets_[r->ticket].version = version_;
        m_.queue_ns += t_adm - tickets_[r->ticket].submit_ns;
        queue_.pop_front();
      }
      launch_kernel();
      progress = true;
      {
        std::lock_guard<std::mutex> lk(mu_);
        m_.admit_ns += now_ns() - t_adm;
        m_.max_inflight = std::max<uint64_t>(m_.max_inflight, inflight_.size());
      }
    } else {
      // An update waits until every walk admitted before it has finished on
      // the device (their result copies may still run: they read query
      // outputs, not the graph) and the previous update's ticket is done,
      // then is enqueued on the engine's stream; walks admitted after it
      // launch behind its event.
      if (!ctl_.drain) {
        ctl_.drain = 1;
        push_ctl();
        drain_since_ = now_ns();
        drain_retired_ = 0;
      }
      bool walks_done = true;
      for (const auto& f : inflight_) walks_done = walks_done && f.copying;
      if (!walks_done || upd_pending_) break;
      if (!drain_retired_) drain_retired_ = now_ns();
      if (kernel_running()) break;
      const uint64_t t_upd = now_ns();
      const NvtxRange nvtx_("bingo serve update");
      int st = BINGO_OK;
      const uint64_t k = r->a.size();
      eng_.set_defer_sync(true);
      for (uint64_t o = 0; o < k; o += cfg_.max_update_batch) {
        const uint64_t len = std::min<uint64_t>(cfg_.max_update_batch, k - o);
        try {
          if (r->kind == BINGO_OP_INSERT)
            eng_.insert(r->a.data() + o, r->b.data() + o, r->c.data() + o, len,
                        r->out_slots ? r->out_slots + o : nullptr);
          else if (r->kind == BINGO_OP_DELETE_PAIRS)  // chunks see earlier chunks' deletes: same slots
            eng_.erase_pairs(r->a.data() + o, r->b.data() + o, len);
          else
            eng_.erase(r->a.data() + o, r->b.data() + o, len);
        } catch (const Error& e) {
          st = e.status;
          // Skipped deletes are reported after the rest of the batch applies;
          // any other error ends the batch.
          if (st != BINGO_ERR_INVALID_SLOT) break;
        }
      }
      eng_.set_defer_sync(false);
      cuda_check(cudaEventRecord(upd_ev_, eng_.stream()), "serve update event");
      upd_recorded_ = true;
      ++version_;
      upd_pending_ = true;
      upd_ticket_ = r->ticket;
      upd_version_ = version_;
      upd_status_ = st;
      upd_t0_ = t_upd;
      ctl_.drain = 0;
      push_ctl();
      {
        std::lock_guard<std::mutex> lk(mu_);
        m_.drain_wait_ns += t_upd - drain_since_;
        m_.drain_inflight_ns += drain_retired_ - drain_since_;
        queue_.pop_front();
      }
      progress = true;
    }
  }
  {
    std::lock_guard<std::mutex> lk(mu_);
    m_.complete_ns += t_completed - t_begin;
    ++m_.scheduler_passes;
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
  uint32_t quiet = 0;  // passes in a row without progress while work is in flight
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
      if (upd_pending_) {
        Ticket& t = tickets_[upd_ticket_];
        t.done = 1, t.status = e.status, t.done_ns = now_ns();
        upd_pending_ = false;
      }
      eng_.set_defer_sync(false);
      cv_done_.notify_all();
      quit_ = true;
    }
    std::unique_lock<std::mutex> lk(mu_);
    const bool idle = queue_.empty() && inflight_.empty() && !upd_pending_;
    if (quit_ && idle) break;
    if (progress) {
      quiet = 0;
    } else if (idle) {
      quiet = 0;
      cv_.wait_for(lk, std::chrono::milliseconds(5));
    } else {
      // Work in flight: poll without sleeping for a while (a timed sleep
      // costs tens of microseconds of timer slack on every hop of a
      // request), then back off to short sleeps.
      lk.unlock();
      if (++quiet < kSpinPasses)
        std::this_thread::yield();
      else
        std::this_thread::sleep_for(std::chrono::microseconds(10));
    }
  }
  ctl_.stop = 1;
  try {
    push_ctl();
  } catch (...) {
  }
  cudaStreamSynchronize(cstream_);
  cudaStreamSynchronize(kstream_);
}

// Copies the host shadow of the control block to the device (stream order
// keeps it after the job descriptors it exposes; pageable source, so the
// shadow may change once the call returns).
void Server::push_ctl() {
  if (pin_head_ + 64 > kPinBytes) {
    cuda_check(cudaStreamSynchronize(cstream_), "staging wrap");
    pin_head_ = 0;
  }
  void* h = pin_ + pin_head_;
  std::memcpy(h, (const void*)&ctl_, sizeof ctl_);
  pin_head_ += 64;
  cuda_check(cudaMemcpyAsync(d_ctl_, h, sizeof ctl_, cudaMemcpyHostToDevice, cstream_), "serve control");
}

void Server::metrics(bingo_serve_metrics* out) {
  std::lock_guard<std::mutex> lk(mu_);
  *out = m_;
  out->submitted = next_ticket_;
  uint64_t c = 0;
  for (auto& kv : tickets_) c += kv.second.done;
  out->completed = c;
}

void Server::stats(uint64_t* completed, uint64_t* version) {
  std::lock_guard<std::mutex> lk(mu_);
  uint64_t c = 0;
  for (auto& kv : tickets_) c += kv.second.done;
  *completed = c;
  *version = version_;
}

}  // namespace bingo
