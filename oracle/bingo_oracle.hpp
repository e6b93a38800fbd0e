// CPU oracle for the Bingo radix bias-factorization walk engine.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product library links, calls or
// ships this code; it is the checker that the CUDA path is compared against,
// and (compiled with OpenMP) the multithreaded CPU baseline timed beside it.
//
// Two restatements live here.
//
// 1. RefGraph - the reference's per-vertex NodeData state machine, restated
//    line by line from the reference sources (ids in this file are 0-based;
//    the reference shifts them by one and keeps vertex 0 as a scratch counter):
//      classification   include/operation.cuh:57-73 (RATE, dense = MAXLOG)
//      LOGT / capacity  include/operation.cuh:39-56, :163-166 (ORIGINAL=16)
//      build            include/operation.cuh:82-90 (stable bucket by u),
//                       include/Bingo.cuh:159-181
//      float alias      include/Bingo.cuh:111-158 (EPS=1e-3, api.h:5)
//      insert           include/operation.cuh:144-147 (stable_sort by u),
//                       include/Bingo.cuh:182-198
//      delete           include/operation.cuh:198-218, include/Bingo.cuh:199-218
//    Masses are float, weights are float-held integers, only bits below the
//    build-time LOGT are tracked, and only "sparse" bits keep member lists -
//    exactly the reference's limits.
//
// 2. ExactGraph - the integer semantics the CUDA path implements: every bit
//    group keeps a member list (append on insert, swap-remove on delete, the
//    same discipline as include/Bingo.cuh:182-218), integer masses
//    cnt_k * 2^k, an integer Vose alias table, Philox4x32-10 draws keyed by
//    (walk, step, trial, job), and DeepWalk / PPR / node2vec / one-hop
//    sampling walks following include/operation.cuh:252-368, :407-430.
//    For every bit the reference keeps a list for, the member sequence is
//    identical to RefGraph's; tests assert that.
#pragma once
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <map>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------------------
// Philox4x32-10, restated from Salmon, Moraes, Dror and Shaw, "Parallel random
// numbers: as easy as 1, 2, 3" (SC'11): two 32x32->64 multiplies per round,
// Weyl key schedule, ten rounds.
struct U4 {
  uint32_t x, y, z, w;
};

inline U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    c = U4{(uint32_t)(p1 >> 32) ^ c.y ^ k0, (uint32_t)p1,
           (uint32_t)(p0 >> 32) ^ c.w ^ k1, (uint32_t)p0};
  }
  return c;
}

inline uint32_t mulhi32(uint32_t a, uint32_t b) {
  return (uint32_t)(((uint64_t)a * b) >> 32);
}
inline uint64_t mulhi64(uint64_t a, uint64_t b) {
  return (uint64_t)(((unsigned __int128)a * b) >> 64);
}

// ---------------------------------------------------------------------------
// Integer alias table over the nonzero bit groups of one vertex.
//
// Slot j belongs to the j-th nonzero group in ascending bit order. With m
// slots and total mass T, group j's scaled mass is s_j = mass_j * m and every
// slot holds exactly T scaled units. Pairing: repeatedly take the lowest
// "small" (s < T) and the lowest "large" (s >= T) slot; the small slot keeps
// thr = s_small and aliases the large one, whose residual drops by
// T - s_small. Leftover slots hold exactly T (thr = T, alias = self). The
// table is therefore a pure function of the masses.
struct AliasSlot {
  uint64_t thr, T;
  uint8_t own, alias;  // bit indices
};

// mass[k] = cnt_k << k. Returns m and fills slots[0..m).
inline int build_exact_alias(const uint64_t mass[32], AliasSlot slots[32]) {
  int bit_of[32];
  int m = 0;
  unsigned __int128 T = 0;
  for (int k = 0; k < 32; ++k)
    if (mass[k]) {
      bit_of[m++] = k;
      T += mass[k];
    }
  if (!m) return 0;
  const uint64_t T64 = (uint64_t)T;  // callers keep the live weight sum < 2^64
  unsigned __int128 s[32];
  uint32_t small = 0, large = 0;
  for (int j = 0; j < m; ++j) {
    s[j] = (unsigned __int128)mass[bit_of[j]] * (unsigned)m;
    if (s[j] < T)
      small |= 1u << j;
    else
      large |= 1u << j;
  }
  int alias_of[32];
  uint64_t thr[32];
  while (small && large) {
    const int a = __builtin_ctz(small), b = __builtin_ctz(large);
    thr[a] = (uint64_t)s[a];
    alias_of[a] = b;
    small &= ~(1u << a);
    s[b] -= (unsigned __int128)(T64 - (uint64_t)s[a]);
    if (s[b] < T) {
      large &= ~(1u << b);
      small |= 1u << b;
    }
  }
  // With exact arithmetic every leftover slot holds exactly T.
  for (uint32_t r = large | small; r; r &= r - 1) {
    const int j = __builtin_ctz(r);
    thr[j] = T64;
    alias_of[j] = j;
  }
  for (int j = 0; j < m; ++j)
    slots[j] = AliasSlot{thr[j], T64, (uint8_t)bit_of[j], (uint8_t)bit_of[alias_of[j]]};
  return m;
}

// ---------------------------------------------------------------------------
// Walk parameters shared with the CUDA path. Thresholds are 33-bit integers:
// a 32-bit draw u passes when (uint64)u < thr, so thr = 2^32 always passes.
enum App : int { APP_DEEPWALK = 0, APP_NODE2VEC = 1, APP_PPR = 2, APP_SAMPLING = 3 };
enum : uint32_t { WALK_PPR_TAIL = 1u };  // PPR keeps walking past the last slot
constexpr uint32_t kMaxNode2vecTrials = 1u << 16;
constexpr uint32_t kMaxPprSteps = 1u << 20;

inline uint64_t prob_threshold(double p) {
  if (!(p > 0.0)) return 0;
  if (p >= 1.0) return 1ull << 32;
  double t = std::floor(std::ldexp(p, 32));
  return t >= 4294967296.0 ? (1ull << 32) : (uint64_t)t;
}

// node2vec weights: 1/p for returning to the previous vertex, 1 for a
// neighbour of it, 1/q otherwise. Proposals are accepted against the envelope
// am = max(1, 1/q); when 1/p exceeds it, the excess mass (1/p / am - 1) x
// w(cur -> prev) becomes a separate region that returns to the previous
// vertex directly (the "outlier" treatment of KnightKing, Yang et al.,
// SOSP'19), so a large 1/p does not inflate the rejection rate.
struct WalkThresholds {
  uint64_t ret, in, out, stop;
  double ret_excess;  // 0 when 1/p fits under the envelope
};

inline WalkThresholds walk_thresholds(double p, double q, double stop) {
  WalkThresholds t{};
  const double wr = 1.0 / p, wi = 1.0, wo = 1.0 / q;
  const double am = std::max(wi, wo);
  const double rr = wr / am;
  t.ret = prob_threshold(rr);
  t.ret_excess = rr > 1.0 ? rr - 1.0 : 0.0;
  t.in = prob_threshold(wi / am);
  t.out = prob_threshold(wo / am);
  t.stop = prob_threshold(stop);
  return t;
}

// Probability threshold of the return region at a step: D / (T + D) with
// D = excess x w(cur -> prev), T = total live weight at cur.
inline uint64_t region_threshold(double excess, uint64_t wp, uint64_t T) {
  if (!(excess > 0.0) || !wp) return 0;
  const double D = excess * (double)wp;
  return prob_threshold(D / ((double)T + D));
}

// ---------------------------------------------------------------------------
// ExactGraph: the integer semantics of the CUDA path.
struct ExactGraph {
  struct Group {
    std::vector<uint32_t> slot;  // member slot ids, list order
    std::vector<uint32_t> v;     // member neighbour ids, same order
  };
  struct Vertex {
    std::vector<uint32_t> ev, ew, ebp;  // per slot: neighbour, weight (0 = tombstone), bp run start
    std::vector<uint32_t> bp;           // back-pointer pool: position of (slot, bit) in its group
    std::vector<Group> gl;              // groups that ever held a member
    int8_t gi[32];                      // bit -> index into gl, -1 = none
    uint32_t live = 0;
    int m = 0;
    AliasSlot alias[32];
    std::unordered_map<uint32_t, std::pair<uint32_t, uint64_t>> adj;  // neighbour -> (live multiplicity, weight sum)
    Vertex() { std::memset(gi, -1, sizeof gi); }
    Group& grp(int k) {
      if (gi[k] < 0) {
        gi[k] = (int8_t)gl.size();
        gl.emplace_back();
      }
      return gl[gi[k]];
    }
    size_t gsize(int k) const { return gi[k] < 0 ? 0 : gl[gi[k]].slot.size(); }
    const Group* gptr(int k) const { return gi[k] < 0 ? nullptr : &gl[gi[k]]; }
  };

  uint32_t n = 0;
  std::vector<Vertex> vx;

  explicit ExactGraph(uint32_t n_) : n(n_), vx(n_) {}

  static inline uint32_t rank_of(uint32_t w, int k) { return __builtin_popcount(w & ((1u << k) - 1u)); }

  static void adj_add(Vertex& X, uint32_t v, uint32_t w) {
    auto& e = X.adj[v];
    ++e.first;
    e.second += w;
  }
  static void adj_sub(Vertex& X, uint32_t v, uint32_t w) {
    auto it = X.adj.find(v);
    if (it == X.adj.end() || !it->second.first) return;
    it->second.second -= w;
    if (--it->second.first == 0) X.adj.erase(it);
  }
  static bool adj_has(const Vertex& X, uint32_t v) {
    auto it = X.adj.find(v);
    return it != X.adj.end() && it->second.first > 0;
  }
  static uint64_t adj_weight(const Vertex& X, uint32_t v) {
    auto it = X.adj.find(v);
    return it != X.adj.end() && it->second.first > 0 ? it->second.second : 0;
  }

  // Append one edge to u (include/Bingo.cuh:182-198): slot = current slot count,
  // each set bit appends the slot to that group and records the back-pointer.
  uint32_t append(uint32_t u, uint32_t v, uint32_t w) {
    Vertex& X = vx[u];
    const uint32_t s = (uint32_t)X.ev.size();
    X.ev.push_back(v);
    X.ew.push_back(w);
    X.ebp.push_back((uint32_t)X.bp.size());
    for (uint32_t r = w; r; r &= r - 1) {
      Group& G = X.grp(__builtin_ctz(r));
      X.bp.push_back((uint32_t)G.slot.size());
      G.slot.push_back(s);
      G.v.push_back(v);
    }
    ++X.live;
    adj_add(X, v, w);
    return s;
  }

  // Swap-remove slot s of u from each of its groups (include/Bingo.cuh:199-218),
  // then tombstone it (include/operation.cuh:209-210). Returns false when the
  // slot is out of range or already a tombstone.
  bool remove(uint32_t u, uint32_t s) {
    Vertex& X = vx[u];
    if (s >= X.ev.size() || X.ew[s] == 0) return false;
    const uint32_t w = X.ew[s];
    for (uint32_t r = w; r; r &= r - 1) {
      const int k = __builtin_ctz(r);
      Group& G = X.grp(k);
      const uint32_t pos = X.bp[X.ebp[s] + rank_of(w, k)];
      const uint32_t last = (uint32_t)G.slot.size() - 1;
      const uint32_t ms = G.slot[last];
      G.slot[pos] = ms;
      G.v[pos] = G.v[last];
      X.bp[X.ebp[ms] + rank_of(X.ew[ms], k)] = pos;
      G.slot.pop_back();
      G.v.pop_back();
    }
    X.ew[s] = 0;
    --X.live;
    adj_sub(X, X.ev[s], w);
    return true;
  }

  void rebuild_alias(uint32_t u) {
    Vertex& X = vx[u];
    uint64_t mass[32];
    for (int k = 0; k < 32; ++k) mass[k] = (uint64_t)X.gsize(k) << k;
    X.m = build_exact_alias(mass, X.alias);
  }

  // Stable grouping by source (include/operation.cuh:82-90 / :147).
  static std::vector<uint64_t> stable_order(const uint32_t* key, uint64_t k) {
    std::vector<uint64_t> ord(k);
    for (uint64_t i = 0; i < k; ++i) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](uint64_t a, uint64_t b) { return key[a] < key[b]; });
    return ord;
  }

  void load(const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t m) {
    insert(src, dst, w, m, nullptr);
  }

  void insert(const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t k, uint32_t* out_slots) {
    std::vector<uint64_t> ord = stable_order(src, k);
    std::vector<uint64_t> starts;
    for (uint64_t i = 0; i < k; ++i)
      if (i == 0 || src[ord[i]] != src[ord[i - 1]]) starts.push_back(i);
    starts.push_back(k);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t sg = 0; sg < (int64_t)starts.size() - 1; ++sg) {
      const uint32_t u = src[ord[starts[sg]]];
      for (uint64_t i = starts[sg]; i < starts[sg + 1]; ++i) {
        const uint64_t e = ord[i];
        const uint32_t s = append(u, dst[e], w[e]);
        if (out_slots) out_slots[e] = s;
      }
      rebuild_alias(u);
    }
  }

  // Returns the number of rejected (out-of-range or tombstoned) deletes.
  uint64_t erase(const uint32_t* u, const uint32_t* slot, uint64_t k) {
    std::vector<uint64_t> ord = stable_order(u, k);
    std::vector<uint64_t> starts;
    for (uint64_t i = 0; i < k; ++i)
      if (i == 0 || u[ord[i]] != u[ord[i - 1]]) starts.push_back(i);
    starts.push_back(k);
    uint64_t bad = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : bad)
    for (int64_t sg = 0; sg < (int64_t)starts.size() - 1; ++sg) {
      const uint32_t x = u[ord[starts[sg]]];
      for (uint64_t i = starts[sg]; i < starts[sg + 1]; ++i)
        if (!remove(x, slot[ord[i]])) ++bad;
      rebuild_alias(x);
    }
    return bad;
  }

  // Delete by (u, v): the r-th occurrence of a pair in the batch takes the
  // r-th lowest live slot of u with neighbour v (~0 when there is none); the
  // slot list then goes through erase(). Returns erase()'s rejected count.
  uint64_t erase_pairs(const uint32_t* u, const uint32_t* v, uint64_t k, uint32_t* slots_out = nullptr) {
    std::vector<uint32_t> slot(k, 0xffffffffu);
    std::map<std::pair<uint32_t, uint32_t>, uint32_t> next;  // first slot not yet examined per pair
    for (uint64_t i = 0; i < k; ++i) {
      const Vertex& X = vx[u[i]];
      uint32_t& c = next[{u[i], v[i]}];
      while (c < X.ev.size() && !(X.ev[c] == v[i] && X.ew[c] != 0)) ++c;
      if (c < X.ev.size()) slot[i] = c++;
    }
    if (slots_out) std::copy(slot.begin(), slot.end(), slots_out);
    return erase(u, slot.data(), k);
  }

  // One weighted neighbour draw from the alias table, then a uniform member.
  inline int64_t sample(uint32_t cur, const U4& r) const {
    const Vertex& X = vx[cur];
    if (!X.m) return -1;
    const AliasSlot& A = X.alias[mulhi32(r.x, (uint32_t)X.m)];
    const uint64_t d = mulhi64(((uint64_t)r.y << 32) | r.z, A.T);
    const Group& G = *X.gptr(d < A.thr ? A.own : A.alias);
    return G.v[mulhi32(r.w, (uint32_t)G.v.size())];
  }

  // Walks: out is [n_starts][L] (sampling: [n_starts]). Counter = (walk, step, trial, job).
  void walk(int app, uint32_t L, const uint32_t* starts, uint64_t n_starts, uint64_t seed, uint32_t job,
            double p, double q, double stop, uint32_t flags, int32_t* out) const {
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    const WalkThresholds th = walk_thresholds(p, q, stop);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t ii = 0; ii < (int64_t)n_starts; ++ii) {
      const uint32_t i = (uint32_t)ii;
      if (app == APP_SAMPLING) {
        out[i] = (int32_t)sample(starts[i], philox4x32_10(U4{i, 1, 0, job}, k0, k1));
        continue;
      }
      int32_t* row = out + (uint64_t)i * L;
      if (L == 0) continue;
      int64_t cur = starts[i], prev = -1;
      row[0] = (int32_t)cur;
      uint32_t pos = 0;
      const bool tail = app == APP_PPR && (flags & WALK_PPR_TAIL);
      for (uint32_t j = 1;; ++j) {
        if (j >= L && !tail) break;
        if (tail && j >= kMaxPprSteps) break;
        pos = j < L ? j : L - 1;
        int64_t x;
        if (!vx[cur].m) {
          x = -1;
        } else if (app == APP_NODE2VEC && prev >= 0) {
          // Trial t: block (i, j, 2t+1) word y selects the return region,
          // block (i, j, 2t) proposes, word x of (i, j, 2t+1) accepts.
          const Vertex& C = vx[cur];
          const uint64_t region =
              region_threshold(th.ret_excess, adj_weight(C, (uint32_t)prev), C.alias[0].T);
          for (uint32_t t = 0;; ++t) {
            const U4 a = philox4x32_10(U4{i, j, 2 * t + 1, job}, k0, k1);
            if ((uint64_t)a.y < region) {
              x = prev;
              break;
            }
            x = sample((uint32_t)cur, philox4x32_10(U4{i, j, 2 * t, job}, k0, k1));
            const uint64_t thr = x == prev ? th.ret : (adj_has(vx[prev], (uint32_t)x) ? th.in : th.out);
            if ((uint64_t)a.x < thr || t + 1 == kMaxNode2vecTrials) break;
          }
        } else {
          x = sample((uint32_t)cur, philox4x32_10(U4{i, j, 0, job}, k0, k1));
        }
        row[pos] = (int32_t)x;
        if (x < 0) break;
        prev = cur;
        cur = x;
        if (app == APP_PPR && (uint64_t)philox4x32_10(U4{i, j, 1, job}, k0, k1).x < th.stop) break;
      }
      for (uint32_t j = pos + 1; j < L; ++j) row[j] = -1;
    }
  }

  // The same DeepWalk and PPR walks as walk() (PPR without the tail flag),
  // bit for bit, arranged for speed: each thread advances kLanes walks in
  // turn, one dependent read per visit (vertex record, alias slot, group,
  // member), and prefetches the next read of a walk before moving to the
  // next one, so a thread keeps kLanes cache misses in flight instead of
  // one. This is the timed CPU baseline; walk() stays the checker.
  void walk_interleaved(int app, uint32_t L, const uint32_t* starts, uint64_t n_starts, uint64_t seed, uint32_t job,
                        double stop, int32_t* out) const {
    constexpr int kLanes = 16;
    enum Stage { S_FREE, S_VERT, S_ALIAS, S_GROUP, S_MEMBER };
    struct Lane {
      int stage = S_FREE;
      uint32_t i = 0, j = 0, cur = 0, slot = 0, idx = 0;
      int32_t* row = nullptr;
      const Vertex* X = nullptr;
      const Group* G = nullptr;
      U4 r{};
    };
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    const uint64_t thr_stop = prob_threshold(stop);
    const bool ppr = app == APP_PPR;
    std::atomic<uint64_t> next{0};
#pragma omp parallel
    {
      Lane lane[kLanes];
      int busy = 0;
      bool drained = false;
      // Ends walk l after writing row[pos]: the rest of the row is -1.
      auto finish = [&](Lane& w, uint32_t pos) {
        for (uint32_t j = pos + 1; j < L; ++j) w.row[j] = -1;
        w.stage = S_FREE;
        --busy;
      };
      for (;;) {
        for (int l = 0; l < kLanes; ++l) {
          Lane& w = lane[l];
          switch (w.stage) {
            case S_FREE: {
              if (drained) break;
              const uint64_t i = next.fetch_add(1, std::memory_order_relaxed);
              if (i >= n_starts) {
                drained = true;
                break;
              }
              w.i = (uint32_t)i;
              w.row = out + i * L;
              if (L == 0) break;
              w.cur = starts[i];
              w.row[0] = (int32_t)w.cur;
              if (L == 1) break;
              w.j = 1;
              w.stage = S_VERT;
              ++busy;
              __builtin_prefetch(&vx[w.cur].m);
              break;
            }
            case S_VERT: {
              w.X = &vx[w.cur];
              if (!w.X->m) {
                w.row[w.j] = -1;
                finish(w, w.j);
                break;
              }
              w.r = philox4x32_10(U4{w.i, w.j, 0, job}, k0, k1);
              w.slot = mulhi32(w.r.x, (uint32_t)w.X->m);
              __builtin_prefetch(&w.X->alias[w.slot]);
              __builtin_prefetch(&w.X->gl);
              w.stage = S_ALIAS;
              break;
            }
            case S_ALIAS: {
              const AliasSlot& A = w.X->alias[w.slot];
              const uint64_t d = mulhi64(((uint64_t)w.r.y << 32) | w.r.z, A.T);
              w.G = w.X->gptr(d < A.thr ? A.own : A.alias);
              __builtin_prefetch(w.G);
              w.stage = S_GROUP;
              break;
            }
            case S_GROUP: {
              w.idx = mulhi32(w.r.w, (uint32_t)w.G->v.size());
              __builtin_prefetch(w.G->v.data() + w.idx);
              w.stage = S_MEMBER;
              break;
            }
            case S_MEMBER: {
              const uint32_t x = w.G->v[w.idx];
              w.row[w.j] = (int32_t)x;
              w.cur = x;
              if (ppr && (uint64_t)philox4x32_10(U4{w.i, w.j, 1, job}, k0, k1).x < thr_stop) {
                finish(w, w.j);
                break;
              }
              if (++w.j >= L) {
                w.stage = S_FREE;
                --busy;
                break;
              }
              __builtin_prefetch(&vx[x].m);
              w.stage = S_VERT;
              break;
            }
          }
        }
        if (drained && busy == 0) break;
      }
    }
  }
};

// ---------------------------------------------------------------------------
// RefGraph: the reference NodeData state machine (float masses, LOGT frozen at
// build, sparse/dense classification, float alias with EPS fudge).
struct RefGraph {
  static constexpr int MAXLOG = 16;   // include/api.h:11
  static constexpr int ORIGINAL = 16; // include/api.h:13
  static constexpr double EPS = 1e-3; // include/api.h:5
  struct AliasElement {
    float p;
    int8_t a, b;
  };
  struct Node {
    int LOGT = 0, BITS = 0, SZ = ORIGINAL;
    std::vector<int8_t> groupTP;                 // [LOGT]: sparse id or MAXLOG
    std::vector<float> num;                      // [LOGT]
    std::vector<uint32_t> ev;                    // slot -> neighbour
    std::vector<float> ew;                       // slot -> weight (0 = tombstone)
    std::vector<std::vector<uint32_t>> group;    // [BITS] member slot lists
    std::vector<std::vector<int32_t>> idx;       // [BITS][slot] position in group
    std::vector<AliasElement> alias;
  };
  uint32_t n;
  float RATE;
  std::vector<Node> nd;
  std::vector<int64_t> d;  // the caller-side slot counter (graph.cuh:41, :66)

  RefGraph(uint32_t n_, float rate) : n(n_), RATE(rate), nd(n_), d(n_, 0) {}

  static int bitlen(uint32_t x) { return x ? 32 - __builtin_clz(x) : 0; }

  // include/Bingo.cuh:111-158, single lane, float arithmetic as on the device.
  static void build_alias(Node& N) {
    N.alias.clear();
    struct TEMP {
      float p;
      int id;
    };
    std::vector<TEMP> l(1), s(1);
    int nonZ = 0;
    double sum = 0;
    for (int i = 0; i < N.LOGT; ++i)
      if (N.num[i] > EPS) ++nonZ, sum += N.num[i];
    if (sum < EPS) return;
    const float pFactor = (float)(1. * nonZ / sum);
    for (int i = 0; i < N.LOGT; ++i) {
      const float numi = N.num[i];
      if (numi < EPS) continue;
      TEMP t{numi * pFactor, i};
      if ((double)t.p + EPS >= 1)
        l.push_back(t);
      else
        s.push_back(t);
    }
    while (l.size() > 1) {
      TEMP a = l.back();
      l.pop_back();
      while ((double)a.p + EPS >= 1) {
        AliasElement e;
        if (s.size() > 1) {
          TEMP b = s.back();
          s.pop_back();
          e.p = b.p, e.a = (int8_t)b.id, e.b = (int8_t)a.id;
          a.p += b.p;
        } else {
          e.p = 1, e.a = (int8_t)a.id, e.b = -1;
        }
        N.alias.push_back(e);
        a.p -= 1;
      }
      if (a.p > 0) s.push_back(a);
    }
  }

  // include/operation.cuh:33-121 + include/Bingo.cuh:59-84, :159-181.
  void load(const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t m) {
    for (uint64_t i = 0; i < m; ++i) ++d[src[i]];
    std::vector<int> mxlog(n, 0);
    std::vector<std::array<int, MAXLOG>> groupNum(n);
    for (auto& a : groupNum) a.fill(0);
    for (uint64_t i = 0; i < m; ++i) {
      const unsigned wi = (unsigned)(float)w[i];
      mxlog[src[i]] = std::max(mxlog[src[i]], bitlen(wi));
      for (int j = 0; j < MAXLOG; ++j) groupNum[src[i]][j] += ((int)wi & (1 << j)) != 0;
    }
    for (uint32_t u = 0; u < n; ++u) {
      Node& N = nd[u];
      N.SZ = ORIGINAL;
      while (N.SZ < d[u]) N.SZ <<= 1;
      N.LOGT = mxlog[u];
      int bits = 0;
      int8_t tp[MAXLOG];
      for (int j = 0; j < MAXLOG; ++j)
        tp[j] = (int8_t)((groupNum[u][j] == 0 || (float)groupNum[u][j] >= (float)d[u] * RATE) ? MAXLOG : bits++);
      N.BITS = bits;
      N.groupTP.assign(tp, tp + std::min(N.LOGT, MAXLOG));
      N.groupTP.resize(N.LOGT, (int8_t)MAXLOG);
      N.num.assign(N.LOGT, 0.f);
      N.group.assign(bits, {});
      N.idx.assign(bits, {});
    }
    std::vector<uint64_t> ord = ExactGraph::stable_order(src, m);
    for (uint64_t i : ord) {
      Node& N = nd[src[i]];
      N.ev.push_back(dst[i]);
      N.ew.push_back((float)w[i]);
    }
    for (uint32_t u = 0; u < n; ++u) {
      Node& N = nd[u];
      for (auto& ix : N.idx) ix.assign(N.SZ, -1);
      for (uint32_t s = 0; s < N.ev.size(); ++s) {
        const unsigned wi = (unsigned)N.ew[s];
        for (int j = 0; j < N.LOGT; ++j)
          if (wi & (1ull << j)) {
            N.num[j] += (float)(1ull << j);
            if (N.groupTP[j] != MAXLOG) {
              const int g = N.groupTP[j];
              N.idx[g][s] = (int32_t)N.group[g].size();
              N.group[g].push_back(s);
            }
          }
      }
      if (!N.ev.empty()) build_alias(N);
    }
  }

  // include/operation.cuh:144-197 + include/Bingo.cuh:85-94, :182-198.
  void insert(const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t k) {
    for (uint64_t i = 0; i < k; ++i) ++d[src[i]];
    std::vector<uint64_t> ord = ExactGraph::stable_order(src, k);
    std::vector<uint32_t> touched;
    for (uint64_t t = 0; t < k; ++t) {
      const uint64_t i = ord[t];
      const uint32_t u = src[i];
      Node& N = nd[u];
      if (t == 0 || src[ord[t - 1]] != u) {
        touched.push_back(u);
        if (N.SZ < d[u]) {
          while (N.SZ < d[u]) N.SZ <<= 1;
          for (auto& ix : N.idx) ix.resize(N.SZ, -1);
        }
      }
      const unsigned wi = (unsigned)(float)w[i];
      const uint32_t s = (uint32_t)N.ev.size();
      for (int j = 0; j < N.LOGT; ++j)
        if (wi & (1ull << j)) {
          N.num[j] += (float)(1ull << j);
          if (N.groupTP[j] != MAXLOG) {
            const int g = N.groupTP[j];
            N.idx[g][s] = (int32_t)N.group[g].size();
            N.group[g].push_back(s);
          }
        }
      N.ev.push_back(dst[i]);
      N.ew.push_back((float)wi);
    }
    for (uint32_t u : touched) build_alias(nd[u]);
  }

  // include/operation.cuh:198-251 (stable order within a vertex) + Bingo.cuh:199-218.
  void erase(const uint32_t* u, const uint32_t* slot, uint64_t k) {
    std::vector<uint64_t> ord = ExactGraph::stable_order(u, k);
    uint64_t b = 0;
    while (b < k) {
      uint64_t e = b;
      const uint32_t x = u[ord[b]];
      while (e < k && u[ord[e]] == x) ++e;
      Node& N = nd[x];
      for (uint64_t t = b; t < e; ++t) {
        const uint32_t id = slot[ord[t]];
        const unsigned wi = (unsigned)N.ew[id];
        for (int j = 0; j < N.LOGT; ++j)
          if (wi & (1ull << j)) {
            N.num[j] -= (float)(1ull << j);
            if (N.groupTP[j] == MAXLOG) continue;
            const int g = N.groupTP[j];
            std::vector<uint32_t>& G = N.group[g];
            const uint32_t backid = G.back();
            const int32_t pos = N.idx[g][id];
            std::swap(G[pos], G.back());
            N.idx[g][backid] = pos;
            G.pop_back();
          }
      }
      for (uint64_t t = b; t < e; ++t) N.ew[slot[ord[t]]] = 0.f;
      build_alias(N);
      b = e;
    }
  }

  // Per-group probability implied by the float alias table
  // (include/Bingo.cuh:231-234: slot uniform, own with prob p, alias otherwise).
  static void implied_probs(const Node& N, double out[32]) {
    for (int i = 0; i < 32; ++i) out[i] = 0;
    const double sz = (double)N.alias.size();
    for (const AliasElement& e : N.alias) {
      const double p = std::min(1.0, std::max(0.0, (double)e.p));
      if (e.a >= 0) out[(int)e.a] += p / sz;
      if (e.b >= 0) out[(int)e.b] += (1.0 - p) / sz;
    }
  }
};

}  // namespace oracle
