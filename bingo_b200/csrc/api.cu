// extern "C" boundary: every entry point catches engine errors and returns a
// bingo_status; the message stays readable through bingo_last_error().
#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "../../include/bingo.h"
#include "engine.cuh"
#include "serve.cuh"

struct bingo_handle {
  bingo::Engine* eng = nullptr;
  int device = 0;
};

namespace {

thread_local std::string g_create_error;

// busy_ok: the call is allowed while the handle is serving.
template <class F>
int guarded(bingo_handle* h, F&& f, bool busy_ok = false) {
  if (!h || !h->eng) return BINGO_ERR_INVALID_ARGUMENT;
  if (!busy_ok && h->eng->server()) {
    h->eng->last_error = "the handle is serving (bingo_serve_stop first)";
    return BINGO_ERR_BUSY;
  }
  try {
    if (cudaSetDevice(h->device) != cudaSuccess) {
      cudaGetLastError();
      h->eng->last_error = "cudaSetDevice failed";
      return BINGO_ERR_CUDA;
    }
    h->eng->last_error.clear();
    f(*h->eng);
    return BINGO_OK;
  } catch (const bingo::Error& e) {
    h->eng->last_error = e.what();
    return e.status;
  } catch (const std::bad_alloc&) {
    h->eng->last_error = "host allocation failed";
    return BINGO_ERR_CAPACITY;
  } catch (const std::exception& e) {
    h->eng->last_error = e.what();
    return BINGO_ERR_CUDA;
  }
}

}  // namespace

extern "C" {

void bingo_config_init(bingo_config* cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof *cfg);
  cfg->device = 0;
  cfg->node2vec = 1;
  cfg->synchronous = 1;
  cfg->arena_factor = 2.0;
  cfg->arena_bytes = 0;
}

int bingo_create(const bingo_config* cfg, bingo_handle** out) {
  if (!out) return BINGO_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  bingo_config c;
  bingo_config_init(&c);
  if (cfg) c = *cfg;
  if (c.weight_mode != BINGO_WEIGHTS_U32 && c.weight_mode != BINGO_WEIGHTS_F32) {
    g_create_error = "unknown weight_mode";
    return BINGO_ERR_INVALID_ARGUMENT;
  }
  try {
    bingo_handle* h = new bingo_handle;
    h->device = c.device;
    try {
      h->eng = new bingo::Engine(c);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    g_create_error.clear();
    return BINGO_OK;
  } catch (const bingo::Error& e) {
    g_create_error = e.what();
    return e.status;
  } catch (const std::exception& e) {
    g_create_error = e.what();
    return BINGO_ERR_CUDA;
  }
}

int bingo_destroy(bingo_handle* h) {
  // A serving handle finishes its submitted requests first (engine destructor).
  if (!h) return BINGO_ERR_INVALID_ARGUMENT;
  cudaSetDevice(h->device);
  delete h->eng;
  delete h;
  return BINGO_OK;
}

const char* bingo_last_error(const bingo_handle* h) {
  if (!h || !h->eng) return g_create_error.c_str();
  return h->eng->last_error.c_str();
}

int bingo_load_edges(bingo_handle* h, const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t m,
                     uint32_t n) {
  return guarded(h, [&](bingo::Engine& e) { e.load(src, dst, w, m, n); });
}

int bingo_insert_batch(bingo_handle* h, const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t k,
                       uint32_t* out_slots) {
  return guarded(h, [&](bingo::Engine& e) { e.insert(src, dst, w, k, out_slots); });
}

int bingo_delete_batch(bingo_handle* h, const uint32_t* u, const uint32_t* slot, uint64_t k) {
  return guarded(h, [&](bingo::Engine& e) { e.erase(u, slot, k); });
}

int bingo_load_edges_f32(bingo_handle* h, const uint32_t* src, const uint32_t* dst, const float* w, uint64_t m,
                         uint32_t n) {
  return guarded(h, [&](bingo::Engine& e) { e.load_f32(src, dst, w, m, n); });
}

int bingo_insert_batch_f32(bingo_handle* h, const uint32_t* src, const uint32_t* dst, const float* w, uint64_t k,
                           uint32_t* out_slots) {
  return guarded(h, [&](bingo::Engine& e) { e.insert_f32(src, dst, w, k, out_slots); });
}

uint64_t bingo_weights_to_fixed16(const float* w, uint64_t k, uint32_t* out) {
  uint64_t bad = 0;
  for (uint64_t i = 0; i < k; ++i) {
    const float x = w[i];
    uint32_t q = 0;
    if (x > 0.0f && x < 65536.0f) q = (uint32_t)std::nearbyint(x * 65536.0f);  // default mode: half to even
    bad += q == 0;
    out[i] = q;
  }
  return bad;
}

int bingo_delete_pairs(bingo_handle* h, const uint32_t* u, const uint32_t* v, uint64_t k) {
  return guarded(h, [&](bingo::Engine& e) { e.erase_pairs(u, v, k); });
}

int bingo_walk(bingo_handle* h, const bingo_walk_job* jobs, uint32_t n_jobs, uint32_t mode) {
  return guarded(h, [&](bingo::Engine& e) { e.walk(jobs, n_jobs, mode); });
}

int bingo_walk_noalloc(bingo_handle* h, const bingo_walk_job* jobs, uint32_t n_jobs) {
  return guarded(h, [&](bingo::Engine& e) { e.walk_noalloc(jobs, n_jobs); });
}

int bingo_run(bingo_handle* h, const bingo_op* ops, uint32_t n_ops, uint32_t flags) {
  return guarded(h, [&](bingo::Engine& e) { e.run(ops, n_ops, flags); });
}

int bingo_sync(bingo_handle* h) {
  int st = BINGO_OK;
  const int g = guarded(h, [&](bingo::Engine& e) { st = e.sync(); });
  return g ? g : st;
}

int bingo_set_stream(bingo_handle* h, void* stream) {
  return guarded(h, [&](bingo::Engine& e) { e.set_stream(stream); });
}

int bingo_get_stats(bingo_handle* h, bingo_stats* out) {
  if (!out) return BINGO_ERR_INVALID_ARGUMENT;
  return guarded(h, [&](bingo::Engine& e) { e.stats(out); }, true);
}

int bingo_save(bingo_handle* h, const char* path) {
  return guarded(h, [&](bingo::Engine& e) { e.save(path); });
}

int bingo_restore(bingo_handle* h, const char* path) {
  return guarded(h, [&](bingo::Engine& e) { e.restore(path); });
}

int bingo_check(bingo_handle* h, bingo_check_report* out) {
  if (!out) return BINGO_ERR_INVALID_ARGUMENT;
  return guarded(h, [&](bingo::Engine& e) { e.check(out); });
}

int bingo_get_tuning(bingo_handle* h, bingo_tuning* out) {
  if (!out) return BINGO_ERR_INVALID_ARGUMENT;
  return guarded(
      h,
      [&](bingo::Engine& e) {
        const bingo::Tuning& t = e.tuning();
        *out = bingo_tuning{};
        out->walk_chunk = t.walk_chunk;
        out->walk_blocks_per_sm = t.walk_blocks_per_sm;
        out->walk_split = t.walk_split;
        out->walk_order = t.walk_order;
        out->update_chunk = t.update_chunk;
        out->apply_blocks_per_sm = t.apply_blocks_per_sm;
      },
      true);
}

int bingo_set_tuning(bingo_handle* h, const bingo_tuning* in) {
  if (!in) return BINGO_ERR_INVALID_ARGUMENT;
  return guarded(h, [&](bingo::Engine& e) {
    bingo::Tuning t;
    t.walk_chunk = in->walk_chunk;
    t.walk_blocks_per_sm = in->walk_blocks_per_sm;
    t.walk_split = in->walk_split;
    t.walk_order = in->walk_order;
    t.update_chunk = in->update_chunk;
    t.apply_blocks_per_sm = in->apply_blocks_per_sm;
    e.set_tuning(t);
  });
}

int bingo_autotune(bingo_handle* h, const bingo_tune_request* req, bingo_tune_report* out) {
  if (!req) return BINGO_ERR_INVALID_ARGUMENT;
  return guarded(h, [&](bingo::Engine& e) { e.autotune(*req, out); });
}

int bingo_serve_start(bingo_handle* h, const bingo_serve_config* cfg) {
  bingo_serve_config c{};
  if (cfg) c = *cfg;
  return guarded(h, [&](bingo::Engine& e) { e.serve_start(c); });
}

int bingo_serve_submit_walk(bingo_handle* h, const bingo_walk_job* job, uint64_t* ticket) {
  if (!job || !ticket) return BINGO_ERR_INVALID_ARGUMENT;
  return guarded(
      h,
      [&](bingo::Engine& e) {
        if (!e.server()) throw bingo::Error(BINGO_ERR_INVALID_ARGUMENT, "not serving");
        *ticket = e.server()->submit_walk(*job);
      },
      true);
}

int bingo_serve_submit_update(bingo_handle* h, int32_t kind, const uint32_t* a, const uint32_t* b,
                              const uint32_t* c, uint64_t k, uint32_t* out_slots, uint64_t* ticket) {
  if (!ticket) return BINGO_ERR_INVALID_ARGUMENT;
  return guarded(
      h,
      [&](bingo::Engine& e) {
        if (!e.server()) throw bingo::Error(BINGO_ERR_INVALID_ARGUMENT, "not serving");
        *ticket = e.server()->submit_update(kind, a, b, c, k, out_slots);
      },
      true);
}

int bingo_serve_poll(bingo_handle* h, uint64_t ticket, bingo_serve_status* out) {
  return guarded(
      h,
      [&](bingo::Engine& e) {
        if (!e.server()) throw bingo::Error(BINGO_ERR_INVALID_ARGUMENT, "not serving");
        e.server()->poll(ticket, out);
      },
      true);
}

int bingo_serve_wait(bingo_handle* h, uint64_t ticket, uint64_t timeout_us, bingo_serve_status* out) {
  int st = BINGO_OK;
  const int g = guarded(
      h,
      [&](bingo::Engine& e) {
        if (!e.server()) throw bingo::Error(BINGO_ERR_INVALID_ARGUMENT, "not serving");
        if (!e.server()->wait(ticket, timeout_us, out)) st = BINGO_ERR_TIMEOUT;
      },
      true);
  return g ? g : st;
}

int bingo_serve_get_metrics(bingo_handle* h, bingo_serve_metrics* out) {
  if (!out) return BINGO_ERR_INVALID_ARGUMENT;
  return guarded(
      h,
      [&](bingo::Engine& e) {
        if (!e.server()) throw bingo::Error(BINGO_ERR_INVALID_ARGUMENT, "not serving");
        e.server()->metrics(out);
      },
      true);
}

int bingo_serve_stop(bingo_handle* h) {
  return guarded(h, [&](bingo::Engine& e) { e.serve_stop(); }, true);
}

int bingo_dump_sizes(bingo_handle* h, uint64_t sizes[3]) {
  if (!sizes) return BINGO_ERR_INVALID_ARGUMENT;
  return guarded(h, [&](bingo::Engine& e) { e.dump_sizes(sizes); });
}

int bingo_dump_state(bingo_handle* h, uint32_t* ecnt, uint32_t* live, uint32_t* ev, uint32_t* ew, uint32_t* gcnt,
                     uint32_t* mslot, uint32_t* mv, uint32_t* mbp, uint32_t* am, uint64_t* athr, uint64_t* aT,
                     uint8_t* aown, uint8_t* aalias) {
  return guarded(h, [&](bingo::Engine& e) {
    e.dump(ecnt, live, ev, ew, gcnt, mslot, mv, mbp, am, athr, aT, aown, aalias);
  });
}

int bingo_probe_gather(bingo_handle* h, uint64_t table_bytes, double out[3]) {
  if (!out || table_bytes < (1u << 20)) return BINGO_ERR_INVALID_ARGUMENT;
  return guarded(h, [&](bingo::Engine& e) { bingo::probe_gather(e.stream(), table_bytes, out); });
}

int bingo_philox(bingo_handle* h, const uint32_t* ctr4, uint64_t count, uint64_t key, uint32_t* out4) {
  return guarded(h, [&](bingo::Engine& e) { e.philox_batch(ctr4, count, key, out4); });
}

}  // extern "C"
