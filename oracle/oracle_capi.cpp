// C entry points over the CPU oracle (bingo_oracle.hpp) for the Python test
// harness and the CPU baseline leg of bench.py. TEST INFRASTRUCTURE ONLY: the
// product library never links this file.
#include <cstdint>
#include <cstring>

#include "bingo_oracle.hpp"

using oracle::ExactGraph;
using oracle::RefGraph;

extern "C" {

// ----- primitives ----------------------------------------------------------
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  oracle::U4 r = oracle::philox4x32_10(oracle::U4{ctr[0], ctr[1], ctr[2], ctr[3]}, key[0], key[1]);
  out[0] = r.x, out[1] = r.y, out[2] = r.z, out[3] = r.w;
}

int orc_alias_build(const uint64_t mass[32], uint64_t* thr, uint64_t* T, uint8_t* own, uint8_t* alias) {
  oracle::AliasSlot s[32];
  int m = oracle::build_exact_alias(mass, s);
  for (int j = 0; j < m; ++j) thr[j] = s[j].thr, T[j] = s[j].T, own[j] = s[j].own, alias[j] = s[j].alias;
  return m;
}

void orc_walk_thresholds(double p, double q, double stop, uint64_t out[4], double* excess) {
  oracle::WalkThresholds t = oracle::walk_thresholds(p, q, stop);
  out[0] = t.ret, out[1] = t.in, out[2] = t.out, out[3] = t.stop;
  if (excess) *excess = t.ret_excess;
}

// ----- exact graph ---------------------------------------------------------
void* orc_new(uint32_t n) { return new ExactGraph(n); }
void orc_free(void* g) { delete (ExactGraph*)g; }

void orc_load(void* g, const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t m) {
  ((ExactGraph*)g)->load(src, dst, w, m);
}
void orc_insert(void* g, const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t k, uint32_t* out_slots) {
  ((ExactGraph*)g)->insert(src, dst, w, k, out_slots);
}
uint64_t orc_delete(void* g, const uint32_t* u, const uint32_t* slot, uint64_t k) {
  return ((ExactGraph*)g)->erase(u, slot, k);
}
uint64_t orc_delete_pairs(void* g, const uint32_t* u, const uint32_t* v, uint64_t k, uint32_t* slots_out) {
  return ((ExactGraph*)g)->erase_pairs(u, v, k, slots_out);
}
void orc_walk(void* g, int app, uint32_t L, const uint32_t* starts, uint64_t n_starts, uint64_t seed, uint32_t job,
              double p, double q, double stop, uint32_t flags, int32_t* out) {
  ((const ExactGraph*)g)->walk(app, L, starts, n_starts, seed, job, p, q, stop, flags, out);
}
// DeepWalk / PPR (no tail flag) with several walks per thread in flight:
// the same rows as orc_walk, faster (the timed CPU baseline).
void orc_walk_interleaved(void* g, int app, uint32_t L, const uint32_t* starts, uint64_t n_starts, uint64_t seed,
                          uint32_t job, double stop, int32_t* out) {
  ((const ExactGraph*)g)->walk_interleaved(app, L, starts, n_starts, seed, job, stop, out);
}
int orc_has_edge(void* g, uint32_t u, uint32_t v) {
  const ExactGraph* G = (const ExactGraph*)g;
  return G->adj_has(G->vx[u], v);
}

// sizes[0] = total slots, sizes[1] = total members, sizes[2] = total alias slots
void orc_dump_sizes(void* g, uint64_t sizes[3]) {
  const ExactGraph* G = (const ExactGraph*)g;
  uint64_t s = 0, mem = 0, a = 0;
  for (const auto& X : G->vx) {
    s += X.ev.size();
    for (int k = 0; k < 32; ++k) mem += X.gsize(k);
    a += X.m;
  }
  sizes[0] = s, sizes[1] = mem, sizes[2] = a;
}

// Dump in the layout shared with bingo_dump_state(): per vertex ecnt/live/m,
// slots (v, w) by vertex, gcnt[n*32], members (slot, v, back-pointer) by
// (vertex, bit), alias slots (thr, T, own bit, alias bit) by vertex.
void orc_dump(void* g, uint32_t* ecnt, uint32_t* live, uint32_t* ev, uint32_t* ew, uint32_t* gcnt, uint32_t* mslot,
              uint32_t* mv, uint32_t* mbp, uint32_t* am, uint64_t* athr, uint64_t* aT, uint8_t* aown, uint8_t* aalias) {
  const ExactGraph* G = (const ExactGraph*)g;
  uint64_t s = 0, mem = 0, a = 0;
  for (uint32_t u = 0; u < G->n; ++u) {
    const auto& X = G->vx[u];
    ecnt[u] = (uint32_t)X.ev.size();
    live[u] = X.live;
    for (size_t i = 0; i < X.ev.size(); ++i, ++s) ev[s] = X.ev[i], ew[s] = X.ew[i];
    for (int k = 0; k < 32; ++k) {
      gcnt[(uint64_t)u * 32 + k] = (uint32_t)X.gsize(k);
      const ExactGraph::Group* G = X.gptr(k);
      for (size_t p = 0; G && p < G->slot.size(); ++p, ++mem) {
        const uint32_t sl = G->slot[p];
        mslot[mem] = sl;
        mv[mem] = G->v[p];
        mbp[mem] = X.bp[X.ebp[sl] + ExactGraph::rank_of(X.ew[sl], k)];
      }
    }
    am[u] = (uint32_t)X.m;
    for (int j = 0; j < X.m; ++j, ++a)
      athr[a] = X.alias[j].thr, aT[a] = X.alias[j].T, aown[a] = X.alias[j].own, aalias[a] = X.alias[j].alias;
  }
}

// ----- reference-literal graph ---------------------------------------------
void* orl_new(uint32_t n, float rate) { return new RefGraph(n, rate); }
void orl_free(void* g) { delete (RefGraph*)g; }
void orl_load(void* g, const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t m) {
  ((RefGraph*)g)->load(src, dst, w, m);
}
void orl_insert(void* g, const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t k) {
  ((RefGraph*)g)->insert(src, dst, w, k);
}
void orl_delete(void* g, const uint32_t* u, const uint32_t* slot, uint64_t k) { ((RefGraph*)g)->erase(u, slot, k); }

// sizes: [0] slots, [1] sum LOGT, [2] sum BITS, [3] members, [4] alias entries
void orl_dump_sizes(void* g, uint64_t sizes[5]) {
  const RefGraph* G = (const RefGraph*)g;
  uint64_t z[5] = {0, 0, 0, 0, 0};
  for (const auto& N : G->nd) {
    z[0] += N.ev.size();
    z[1] += N.LOGT;
    z[2] += N.BITS;
    for (const auto& gr : N.group) z[3] += gr.size();
    z[4] += N.alias.size();
  }
  std::memcpy(sizes, z, sizeof z);
}

// Dump in the layout the reference harness writes (oracle/ref_harness.cu).
void orl_dump(void* g, int32_t* logt, int32_t* bits, int32_t* sz, uint32_t* ecnt, uint32_t* asz, uint32_t* ev,
              float* ew, int8_t* grouptp, float* num, uint32_t* gsz, uint32_t* members, int32_t* midx, float* ap,
              int8_t* aa, int8_t* ab) {
  const RefGraph* G = (const RefGraph*)g;
  uint64_t s = 0, l = 0, b = 0, mem = 0, a = 0;
  for (uint32_t u = 0; u < G->n; ++u) {
    const auto& N = G->nd[u];
    logt[u] = N.LOGT, bits[u] = N.BITS, sz[u] = N.SZ, ecnt[u] = (uint32_t)N.ev.size();
    for (size_t i = 0; i < N.ev.size(); ++i, ++s) ev[s] = N.ev[i], ew[s] = N.ew[i];
    for (int j = 0; j < N.LOGT; ++j, ++l) grouptp[l] = N.groupTP[j], num[l] = N.num[j];
    for (int gi = 0; gi < N.BITS; ++gi, ++b) {
      gsz[b] = (uint32_t)N.group[gi].size();
      for (uint32_t sl : N.group[gi]) {
        members[mem] = sl;
        midx[mem] = N.idx[gi][sl];
        ++mem;
      }
    }
    asz[u] = (uint32_t)N.alias.size();
    for (const auto& e : N.alias) ap[a] = e.p, aa[a] = e.a, ab[a] = e.b, ++a;
  }
}

void orl_implied_probs(void* g, uint32_t u, double out[32]) {
  const RefGraph* G = (const RefGraph*)g;
  RefGraph::implied_probs(G->nd[u], out);
}

}  // extern "C"
