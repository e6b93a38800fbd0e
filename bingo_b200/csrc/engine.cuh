// Host-side engine behind the C ABI: owns the device graph store, the
// staging buffers and the per-batch pipelines (group by vertex, plan, reserve,
// apply) and launches the walk kernels.
#pragma once
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/bingo.h"
#include "common.cuh"
#include "walk.cuh"

namespace bingo {

// Error carrying a bingo_status across the engine; the C ABI turns it into
// the return code and bingo_last_error().
struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void cuda_check(cudaError_t e, const char* what);

// NVTX range over one public operation, for Nsight timelines (a no-op when
// no tool is attached; the NVTX v3 header needs no library).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Device buffer that grows by reallocation (contents not preserved).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  void ensure(size_t want, const char* what);
  void release();
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

class Server;

// Launch and batching knobs (bingo_tuning); none changes any result.
struct Tuning {
  uint32_t walk_chunk = 0;          // 0 = each walk kernel's default (walk_default_chunk)
  uint32_t walk_blocks_per_sm = 0;  // 0 = each walk kernel's default (walk_default_bps)
  uint32_t walk_split = 0;
  uint32_t walk_order = 1;
  uint32_t update_chunk = 0;  // 0 = whole batch
  uint32_t apply_blocks_per_sm = 8;
};

// A device copy of the graph store (the update knobs are timed on the live
// graph and undone from it).
struct StateCopy {
  DevBuf vrec, meta, gdesc, gs;
  DevBuf arena[kArenas];
  unsigned long long top[kArenas] = {};
  void release();
};

class Engine {
 public:
  explicit Engine(const bingo_config& cfg);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  void load(const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t m, uint32_t n);
  void insert(const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t k, uint32_t* out_slots);
  void load_f32(const uint32_t* src, const uint32_t* dst, const float* w, uint64_t m, uint32_t n);
  void insert_f32(const uint32_t* src, const uint32_t* dst, const float* w, uint64_t k, uint32_t* out_slots);
  void erase(const uint32_t* u, const uint32_t* slot, uint64_t k);
  void erase_pairs(const uint32_t* u, const uint32_t* v, uint64_t k);
  void walk(const bingo_walk_job* jobs, uint32_t n_jobs, uint32_t mode);
  void walk_noalloc(const bingo_walk_job* jobs, uint32_t n_jobs);
  void run(const bingo_op* ops, uint32_t n_ops, uint32_t flags);
  int sync();  // returns a bingo_status
  void set_stream(void* s);
  void stats(bingo_stats* out);
  void dump_sizes(uint64_t sizes[3]);
  void dump(uint32_t* ecnt, uint32_t* live, uint32_t* ev, uint32_t* ew, uint32_t* gcnt, uint32_t* mslot,
            uint32_t* mv, uint32_t* mbp, uint32_t* am, uint64_t* athr, uint64_t* aT, uint8_t* aown,
            uint8_t* aalias);
  void philox_batch(const uint32_t* ctr4, uint64_t count, uint64_t key, uint32_t* out4);
  void save(const char* path);
  void restore(const char* path);
  void check(bingo_check_report* out);  // throws BINGO_ERR_CORRUPT after filling *out
  const Tuning& tuning() const { return tuning_; }
  void set_tuning(const Tuning& t);
  void autotune(const bingo_tune_request& req, bingo_tune_report* out);

  std::string last_error;
  cudaStream_t stream() const { return stream_; }

  // serving
  void serve_start(const bingo_serve_config& cfg);
  void serve_stop();
  Server* server() const { return server_.get(); }
  void require_idle() const;  // throws BINGO_ERR_BUSY while serving
  // used by the serving scheduler
  WalkView walk_view() const { return wview(); }
  WalkJobDev make_job(const bingo_walk_job& J) const;
  void check_walk_job(const bingo_walk_job& J) const;
  void prepare_batches(uint64_t k) { ensure_batch_scratch(k); }
  // The serving scheduler enqueues update batches without a host wait per
  // call (it polls an event instead); device-reported errors then surface
  // through sync().
  void set_defer_sync(bool on) { defer_sync_ = on; }
  void count_launch() { ++launches_; }
  uint32_t n() const { return n_; }
  int device() const { return cfg_.device; }

 private:
  bingo_config cfg_;
  cudaStream_t own_stream_ = nullptr, stream_ = nullptr;
  bool loaded_ = false;
  bool defer_sync_ = false;
  uint32_t n_ = 0;

  // store
  DevBuf vrec_, meta_, gdesc_;
  DevBuf arena_[kArenas];
  DevBuf gs_;  // per member, its slot's back-pointer index for the group (parallel to the member arena)
  unsigned long long* d_top_ = nullptr;  // [kArenas]
  unsigned long long cap_[kArenas] = {};
  uint32_t* d_err_ = nullptr;            // [0] ErrBit sticky, [1] rejected deletes
  uint32_t* h_err_ = nullptr;            // pinned mirror
  unsigned long long* h_top_ = nullptr;  // pinned mirror of d_top_
  // Insert plan read-back (totals, status, tops) through mapped host memory,
  // written by a kernel: no copy-engine transfer that could queue behind a
  // large result copy.
  volatile unsigned long long* h_plan_ = nullptr;
  unsigned long long* d_plan_ = nullptr;
  cudaEvent_t slots_ev_ = nullptr;  // host-bound slot ids copied out (asynchronous handles)
  bool slots_busy_ = false;
  unsigned long long* d_steps_ = nullptr;  // produced walk steps since create
  unsigned long long launches_ = 0;        // hand-written kernels launched since create

  // per-batch scratch
  DevBuf in_a_, in_b_, in_c_, key_s_, perm_, iota_, sa_, sb_, head_, seg_, nseg_, need_, scan_, base_, ctl_,
      slots_, cub_tmp_;
  DevBuf pair_key_, pair_key_s_, pair_slot_;  // delete-by-pair translation
  DevBuf fw_in_, fw_fixed_;                   // float weights: staged input, 16.16 fixed point
  DevBuf check_buf_, check_big_;              // store check: totals, large-vertex list
  uint64_t iota_n_ = 0;
  int group_cluster_ = -1;  // -1 not yet probed, else the group_cluster_ok() bits
  // walk scratch
  DevBuf jobs_, prefix_, queue_, wstart_;
  // Host-bound walk outputs: two device staging buffers used in turn; each
  // is copied out on xstream_ (asynchronous handles), so one call's copy-out
  // overlaps the next call's kernels. copy_ev_[k] marks buffer k's copy done.
  DevBuf wout_[2];
  cudaStream_t xstream_ = nullptr;
  cudaEvent_t walk_ev_[2] = {nullptr, nullptr}, copy_ev_[2] = {nullptr, nullptr};
  bool wout_busy_[2] = {false, false};
  int wout_next_ = 0;
  // programs
  DevBuf prog_jobs_, prog_prefix_, prog_queue_;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t graph_exec_ = nullptr;
  uint64_t graph_sig_ = 0, graph_launches_ = 0;
  uint64_t arena_gen_ = 0;  // bumped whenever an arena or the vertex arrays are reallocated
  std::unique_ptr<Server> server_;
  Tuning tuning_;

  StoreView view() const;
  WalkView wview() const;
  void ensure_batch_scratch(uint64_t k);
  const uint32_t* stage(const uint32_t* p, uint64_t k, DevBuf& buf, const char* what);
  // Stable grouping of a batch by `key` into key_s_/perm_/sa_/sb_/seg_/nseg_,
  // with the batch status word zeroed and the batch validated (`insert`: the
  // destinations too, and the weights are nonzero).
  void group_by_vertex(const uint32_t* key, const uint32_t* a, const uint32_t* b, uint64_t k, bool insert);
  int group_cluster_ok();  // which cluster sizes of the grouping kernel can run here (bit 0: 8, bit 1: 16)
  void run_insert(uint64_t k, uint32_t* dev_out_slots, bool load_mode, uint64_t m_hint);
  void wait_plan();  // until k_totals has published the insert plan
  unsigned long long* plan_needs(const StoreView& S, uint64_t k, uint32_t ks, volatile unsigned long long* publish,
                                 int reserve);
  void enqueue_insert(const uint32_t* a, const uint32_t* b, const uint32_t* c, uint64_t k, uint32_t* out_slots);
  void enqueue_delete(const uint32_t* u, const uint32_t* slot, uint64_t k);
  void ensure_headroom(uint64_t k_insert_total);
  void drop_graph();
  void alloc_arenas(const unsigned long long need[kArenas]);
  void grow_arena(int a, unsigned long long min_cap);
  void read_tops();
  void finish_call();
  void require_loaded() const;
  void insert_one(const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t k, uint32_t* out_slots);
  void erase_one(const uint32_t* u, const uint32_t* slot, uint64_t k);
  const uint32_t* fixed_weights(const float* w, uint64_t k);
  void ensure_pair_scratch(uint64_t k);
  void translate_pairs(const uint32_t* du, const uint32_t* dv, uint64_t k);
  void check_batch_on_device(const uint32_t* a, const uint32_t* b, const uint32_t* w, uint64_t k);
  void check_store(bingo_check_report* out);
  bool save_state(StateCopy& c);
  void restore_state(const StateCopy& c);
};

bool is_device_ptr(const void* p);
void probe_gather(cudaStream_t st, uint64_t table_bytes, double out[3]);

}  // namespace bingo
