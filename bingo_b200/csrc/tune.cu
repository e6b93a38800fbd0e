// Autotuner: picks the launch and batching knobs (Tuning) by timing the
// caller's own sample workload on the live graph.
//
// Walk knobs are timed on the job set through the batched walk path; walks
// do not change the graph, and no knob changes any walk, so the outputs are
// simply rewritten. Update knobs are timed by applying the sample batch and
// then restoring the store from a device copy taken before the first trial,
// so the graph is the same when the call returns.
//
// Search: one coordinate pass in a fixed order (walk_chunk, walk_split,
// walk_order, walk_blocks_per_sm, a second look at walk_chunk around the
// pick, then update_chunk and apply_blocks_per_sm). A candidate replaces the
// current choice only when its median wall time is at least 1 % lower, so
// noise does not move the knobs.
#include <algorithm>
#include <chrono>
#include <vector>

#include "engine.cuh"

namespace bingo {

namespace {

double median(std::vector<double> v) {
  std::sort(v.begin(), v.end());
  const size_t m = v.size() / 2;
  return v.size() % 2 ? v[m] : 0.5 * (v[m - 1] + v[m]);
}

}  // namespace

void Engine::autotune(const bingo_tune_request& R, bingo_tune_report* out) {
  const NvtxRange nvtx_("bingo autotune");
  require_loaded();
  require_idle();
  if (!R.n_jobs && !R.n_ins && !R.n_del) throw Error(BINGO_ERR_INVALID_ARGUMENT, "empty tuning request");
  if (R.n_jobs && !R.jobs) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null job array");
  const int reps = R.repeats ? (int)std::min<uint32_t>(R.repeats, 64) : 3;
  const Tuning start = tuning_;
  Tuning best = tuning_;
  uint32_t cand = 0;

  auto wall_ms = [&](auto&& fn) {
    cuda_check(cudaStreamSynchronize(stream_), "tune");
    const auto t0 = std::chrono::steady_clock::now();
    fn();
    const int st = sync();
    if (st) throw Error(st, last_error);
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  };

  double walk_start = -1, walk_best = -1;
  if (R.n_jobs) {
    auto time_walks = [&](const Tuning& t) {
      tuning_ = t;
      std::vector<double> v;
      for (int r = 0; r <= reps; ++r) {
        const double ms = wall_ms([&] { walk(R.jobs, R.n_jobs, BINGO_WALK_BATCHED); });
        if (r) v.push_back(ms);  // the first run warms up
      }
      ++cand;
      return median(v);
    };
    auto try_knob = [&](uint32_t Tuning::*f, const std::vector<uint32_t>& vals) {
      for (uint32_t x : vals) {
        if (best.*f == x) continue;
        Tuning t = best;
        t.*f = x;
        const double ms = time_walks(t);
        if (ms < walk_best * 0.99) walk_best = ms, best = t;
      }
    };
    try {
      walk_start = walk_best = time_walks(best);
      try_knob(&Tuning::walk_chunk, {8, 16, 32, 64, 128, 256});
      bool mixed = false;
      for (uint32_t j = 1; j < R.n_jobs; ++j) mixed |= R.jobs[j].app != R.jobs[0].app;
      if (mixed) try_knob(&Tuning::walk_split, {0, 1});
      if (R.n_jobs > 1) try_knob(&Tuning::walk_order, {1, 0});
      try_knob(&Tuning::walk_blocks_per_sm, {0, 6, 4, 3, 2});
      std::vector<uint32_t> around;  // 0 (each kernel's default) has no neighbours
      if (best.walk_chunk > 1) around.push_back(best.walk_chunk / 2);
      if (best.walk_chunk && best.walk_chunk < 1024) around.push_back(best.walk_chunk * 2);
      try_knob(&Tuning::walk_chunk, around);
    } catch (...) {
      tuning_ = start;
      throw;
    }
  }

  double upd_start = -1, upd_best = -1;
  if (R.n_ins || R.n_del) {
    if ((R.n_ins && (!R.ins_src || !R.ins_dst || !R.ins_w)) || (R.n_del && (!R.del_u || !R.del_slot)))
      throw Error(BINGO_ERR_INVALID_ARGUMENT, "null update array");
    StateCopy snap;
    if (save_state(snap)) {
      auto time_updates = [&](const Tuning& t) {
        tuning_ = t;
        std::vector<double> v;
        for (int r = 0; r <= reps; ++r) {
          restore_state(snap);
          const double ms = wall_ms([&] {
            if (R.n_ins) insert(R.ins_src, R.ins_dst, R.ins_w, R.n_ins, nullptr);
            if (R.n_del) erase(R.del_u, R.del_slot, R.n_del);
          });
          if (r) v.push_back(ms);
        }
        ++cand;
        return median(v);
      };
      auto try_knob = [&](uint32_t Tuning::*f, const std::vector<uint32_t>& vals) {
        for (uint32_t x : vals) {
          if (best.*f == x) continue;
          Tuning t = best;
          t.*f = x;
          const double ms = time_updates(t);
          if (ms < upd_best * 0.99) upd_best = ms, best = t;
        }
      };
      try {
        upd_start = upd_best = time_updates(best);
        const uint64_t kmax = std::max(R.n_ins, R.n_del);
        std::vector<uint32_t> chunks{0};
        for (uint64_t c = kmax / 2; c >= 16384 && chunks.size() < 4; c /= 2) chunks.push_back((uint32_t)c);
        try_knob(&Tuning::update_chunk, chunks);
        try_knob(&Tuning::apply_blocks_per_sm, {8, 4, 16, 32});
        restore_state(snap);
      } catch (...) {
        tuning_ = start;
        try {
          restore_state(snap);
        } catch (...) {
        }
        snap.release();
        throw;
      }
      snap.release();
    }
  }

  tuning_ = best;
  if (out) {
    *out = bingo_tune_report{};
    out->best.walk_chunk = best.walk_chunk;
    out->best.walk_blocks_per_sm = best.walk_blocks_per_sm;
    out->best.walk_split = best.walk_split;
    out->best.walk_order = best.walk_order;
    out->best.update_chunk = best.update_chunk;
    out->best.apply_blocks_per_sm = best.apply_blocks_per_sm;
    out->walk_ms_start = walk_start;
    out->walk_ms_best = walk_best;
    out->update_ms_start = upd_start;
    out->update_ms_best = upd_best;
    out->candidates = cand;
  }
}

}  // namespace bingo
