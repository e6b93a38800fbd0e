// bingo_driver: the reference's experiment driver (src/main.cpp, src/apps.cu
// instance(), include/graph.cuh loadGraph / insertGraph / deleteGraph /
// randomWalk) rewritten over the C ABI of libbingo.so.
//
//   bingo_driver [d|n|p|s] [-g edge_list | -r scale] [-i|-d|-m] [-b batch]
//                [-l len] [-k iterations] [-s seed] [-o] [-f] [-c]
//
// d / n / p / s: DeepWalk, node2vec, PPR, one-hop sampling (default d).
// -g: a "u v" edge-list file (the reference reads ../dataset/<name>);
// -r: an R-MAT graph of that scale instead (edge factor 16), for machines
//     without the datasets. Load weights follow the reference driver:
//     trunc(bias(outdeg(v))) + 1, bias = d or d^0.3 for n > 1e7.
// -i / -d / -m: insert-only, delete-only or mixed updates (mixed halves the
//     batch, as the reference does); default mixed.
// -b: batch size (default 100000); -l: walk length (default 80); -k:
//     iterations of {update, walk} (default 10); -s: seed; -o: print the
//     first 10 walks; -f: float weights (the reference's wtype::Float: the
//     integer weight plus a random hundredth, inserts too); -c: run the
//     store check (bingo_check) after the load and after every iteration's
//     updates, outside the timed regions, and stop on the first failure.
//
// Updates follow the reference: an insert batch copies random existing
// (u, v) pairs (parallel edges allowed) and a delete batch removes random
// live edges by (u, slot); the slot ids come back from bingo_insert_batch.
// One difference: the reference's insert weight bias(d[v]) can be 0, which
// this engine rejects, so inserts use the load formula bias(d[v]) + 1.
//
// Prints the reference's three summary lines on stderr and one JSON line
// with rates on stdout.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/bingo.h"
#include "../../include/bingo_gen.h"

namespace {

struct Rng {  // splitmix64
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  uint64_t below(uint64_t n) { return next() % n; }
};

struct EdgeData {  // the reference's EdgeData (include/type.h): slot -1 = deleted
  uint32_t u, v;
  int64_t slot;
};

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void check(bingo_handle* h, int st, const char* what) {
  if (st == BINGO_OK) return;
  std::fprintf(stderr, "bingo_driver: %s failed with status %d (%s)\n", what, st,
               bingo_last_error(h) ? bingo_last_error(h) : "");
  std::exit(2);
}

}  // namespace

int main(int argc, char** argv) {
  int app = BINGO_DEEPWALK;
  char utp = 'm';
  std::string graph_file;
  int scale = 0;
  uint64_t batch = 100000, iters = 10, seed = 1;
  uint32_t len = 80;
  bool print_paths = false, float_w = false, store_check = false;
  int pos = 1;
  if (pos < argc && argv[pos][0] != '-') {
    switch (argv[pos][0]) {
      case 'n': app = BINGO_NODE2VEC; break;
      case 'p': app = BINGO_PPR; break;
      case 's': app = BINGO_SAMPLING; break;
      default: app = BINGO_DEEPWALK; break;
    }
    ++pos;
  }
  for (; pos < argc; ++pos) {
    const std::string a = argv[pos];
    auto val = [&]() -> const char* {
      if (pos + 1 >= argc) {
        std::fprintf(stderr, "bingo_driver: %s needs a value\n", a.c_str());
        std::exit(1);
      }
      return argv[++pos];
    };
    if (a == "-g") graph_file = val();
    else if (a == "-r") scale = std::atoi(val());
    else if (a == "-i" || a == "-d" || a == "-m") utp = a[1];
    else if (a == "-b") batch = std::strtoull(val(), nullptr, 10);
    else if (a == "-l") len = (uint32_t)std::atoi(val());
    else if (a == "-k") iters = std::strtoull(val(), nullptr, 10);
    else if (a == "-s") seed = std::strtoull(val(), nullptr, 10);
    else if (a == "-o") print_paths = true;
    else if (a == "-f") float_w = true;
    else if (a == "-c") store_check = true;
    else {
      std::fprintf(stderr, "bingo_driver: unknown option %s\n", a.c_str());
      return 1;
    }
  }
  if (graph_file.empty() && !scale) scale = 16;
  if (utp == 'm') batch >>= 1;

  // ---- load (the reference's loadGraph)
  std::vector<uint32_t> src, dst;
  uint32_t n = 0;
  if (!graph_file.empty()) {
    uint64_t m = 0;
    int rc = bingo_edge_list_read(graph_file.c_str(), nullptr, nullptr, 0, &m, &n);
    if (rc == 0) {
      src.resize(m), dst.resize(m);
      rc = bingo_edge_list_read(graph_file.c_str(), src.data(), dst.data(), m, &m, &n);
    }
    if (rc) {
      std::fprintf(stderr, "bingo_driver: cannot read %s (code %d)\n", graph_file.c_str(), rc);
      return 1;
    }
    std::fprintf(stderr, "Graph dataset: %s.\n", graph_file.c_str());
  } else {
    const uint64_t cap = 16ull << scale;
    src.resize(cap), dst.resize(cap);
    const uint64_t m = bingo_gen_rmat((uint32_t)scale, 16, 0.57, 0.19, 0.19, seed, src.data(), dst.data());
    src.resize(m), dst.resize(m);
    n = 1u << scale;
    std::fprintf(stderr, "Graph dataset: R-MAT scale %d.\n", scale);
  }
  const uint64_t m = src.size();
  std::fprintf(stderr, "Edge number: %llu.\n", (unsigned long long)m);
  std::vector<uint32_t> w(m);
  if (bingo_driver_weights(BINGO_DRIVER_AUTO, src.data(), dst.data(), m, n, w.data())) {
    std::fprintf(stderr, "bingo_driver: bad edge list\n");
    return 1;
  }
  std::vector<uint32_t> deg(n, 0);  // d[]: slots per vertex as the reference tracks them (never decremented)
  for (uint64_t i = 0; i < m; ++i) ++deg[src[i]];
  const bool pow03 = n > 1e7;
  auto insert_weight = [&](uint32_t v) {
    const float b = pow03 ? (float)std::pow((double)deg[v], 0.3) : (float)deg[v];
    return (uint32_t)(b + 1.0f);
  };
  Rng rng{seed * 0x2545F4914F6CDD1Dull + 7};
  auto frac = [&]() { return (float)rng.below(100) * 0.01f; };

  bingo_config cfg;
  bingo_config_init(&cfg);
  cfg.node2vec = app == BINGO_NODE2VEC;  // the reference builds the hash only for node2vec
  cfg.weight_mode = float_w ? BINGO_WEIGHTS_F32 : BINGO_WEIGHTS_U32;
  bingo_handle* h = nullptr;
  if (int st = bingo_create(&cfg, &h)) {
    std::fprintf(stderr, "bingo_driver: create failed with status %d (%s)\n", st,
                 bingo_last_error(nullptr) ? bingo_last_error(nullptr) : "");
    return 2;
  }
  const double t_total0 = now_s();
  if (float_w) {
    std::vector<float> wf(m);
    for (uint64_t i = 0; i < m; ++i) wf[i] = (float)(w[i] - 1) + frac();  // d[v] + rd(100) * .01
    for (uint64_t i = 0; i < m; ++i) wf[i] = wf[i] > 0.0f ? wf[i] : 0.01f;  // the engine rejects 0
    check(h, bingo_load_edges_f32(h, src.data(), dst.data(), wf.data(), m, n), "load");
  } else {
    check(h, bingo_load_edges(h, src.data(), dst.data(), w.data(), m, n), "load");
  }
  uint64_t checks = 0;
  auto check_store = [&](const char* when) {
    if (!store_check) return;
    bingo_check_report rep;
    const int rc = bingo_check(h, &rep);
    if (rc != BINGO_OK) {
      std::fprintf(stderr, "bingo_driver: store check after %s failed (status %d): %llu bad vertices, first %u, "
                   "kinds %u\n", when, rc, (unsigned long long)rep.bad_vertices, rep.first_bad, rep.kinds);
      std::exit(3);
    }
    ++checks;
  };
  check_store("the load");
  std::vector<EdgeData> edges(m);
  {
    std::vector<uint32_t> next_slot(n, 0);
    for (uint64_t i = 0; i < m; ++i) edges[i] = EdgeData{src[i], dst[i], (int64_t)next_slot[src[i]]++};
  }
  uint64_t live = m;

  // ---- the reference's instance(): iterations of {insert, delete, walk}
  const uint64_t n_walks = app == BINGO_SAMPLING ? std::min<uint64_t>(batch ? batch : 1, n) : n;
  const uint64_t per = app == BINGO_SAMPLING ? 1 : len;
  std::vector<int32_t> rows(n_walks * per);
  std::vector<uint32_t> a(batch), b(batch), c(batch), slots(batch);
  std::vector<float> cf(batch);
  double t_walk = 0, t_update = 0;
  uint64_t steps0 = 0, updates = 0;
  bingo_stats st;
  check(h, bingo_get_stats(h, &st), "stats");
  steps0 = st.walk_steps;
  const double t_eval0 = now_s();
  for (uint64_t it = 0; it < iters; ++it) {
    if (batch && (utp == 'm' || utp == 'i')) {
      for (uint64_t i = 0; i < batch; ++i) {  // insertGraph: copies of random existing pairs
        const EdgeData& e = edges[rng.below(edges.size())];
        a[i] = e.u, b[i] = e.v;
        c[i] = insert_weight(e.v);
        cf[i] = (float)deg[e.v] + frac();
        if (!(cf[i] > 0.0f)) cf[i] = 0.01f;
        ++deg[e.u];
      }
      const double t0 = now_s();
      if (float_w)
        check(h, bingo_insert_batch_f32(h, a.data(), b.data(), cf.data(), batch, slots.data()), "insert");
      else
        check(h, bingo_insert_batch(h, a.data(), b.data(), c.data(), batch, slots.data()), "insert");
      t_update += now_s() - t0;
      for (uint64_t i = 0; i < batch; ++i) edges.push_back(EdgeData{a[i], b[i], (int64_t)slots[i]});
      live += batch;
      updates += batch;
    }
    if (batch && (utp == 'm' || utp == 'd') && live >= batch) {
      for (uint64_t i = 0; i < batch; ++i) {  // deleteGraph: random live edges by (u, slot)
        uint64_t p = rng.below(edges.size());
        while (edges[p].slot < 0) p = rng.below(edges.size());
        a[i] = edges[p].u, b[i] = (uint32_t)edges[p].slot;
        edges[p].slot = -1;  // d[u] stays: the reference's d[] counts slots, not live edges
      }
      const double t0 = now_s();
      check(h, bingo_delete_batch(h, a.data(), b.data(), batch), "delete");
      t_update += now_s() - t0;
      live -= batch;
      updates += batch;
    }
    check_store("an update iteration");
    bingo_walk_job j;
    std::memset(&j, 0, sizeof j);
    j.app = app;
    j.length = len;
    j.n_starts = n_walks;
    j.first = 0;
    j.job_id = (uint32_t)it;
    j.seed = seed + it;
    j.p = 0.5, j.q = 2.0, j.stop_prob = 0.0125;  // the reference's P, Q, TP (include/api.h:9-10, :21)
    j.out = rows.data();
    const double t0 = now_s();
    check(h, bingo_walk(h, &j, 1, BINGO_WALK_PLAIN), "walk");
    t_walk += now_s() - t0;
  }
  const double t_eval = now_s() - t_eval0;
  check(h, bingo_get_stats(h, &st), "stats");
  const uint64_t steps = st.walk_steps - steps0;
  std::fprintf(stderr, "Random walk in %.6f s.\n", t_walk);
  std::fprintf(stderr, "Evaluation time: %.6f s.\n", t_eval);
  std::fprintf(stderr, "Memory Consumption: %.3f GB.\n", (double)(st.arena_bytes + st.scratch_bytes) / (1ull << 30));
  if (print_paths)
    for (uint64_t i = 0; i < std::min<uint64_t>(10, n_walks); ++i) {
      for (uint64_t k = 0; k < per; ++k) std::printf("%d ", rows[i * per + k]);
      std::printf("\n");
    }
  std::printf(
      "{\"app\": %d, \"n\": %u, \"m\": %llu, \"iterations\": %llu, \"batch\": %llu, \"walk_s\": %.6f, "
      "\"update_s\": %.6f, \"eval_s\": %.6f, \"walk_steps\": %llu, \"walk_steps_per_s\": %.1f, "
      "\"edge_updates_per_s\": %.1f, \"live_edges\": %llu, \"store_checks\": %llu, \"total_s\": %.6f}\n",
      app, n, (unsigned long long)m, (unsigned long long)iters, (unsigned long long)batch, t_walk, t_update,
      t_eval, (unsigned long long)steps, t_walk > 0 ? steps / t_walk : 0.0, t_update > 0 ? updates / t_update : 0.0,
      (unsigned long long)st.live_edges, (unsigned long long)checks, now_s() - t_total0);
  bingo_destroy(h);
  return 0;
}
