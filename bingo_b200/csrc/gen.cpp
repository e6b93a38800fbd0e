// Seeded synthetic workloads: R-MAT graphs, weight distributions and update
// batches (see include/bingo_gen.h). Host code, OpenMP-parallel where the
// result does not depend on the thread count.
#include <parallel/algorithm>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/bingo_gen.h"
#include "philox.cuh"

namespace {

using bingo::philox;
using bingo::Rand4;

constexpr uint32_t kTagRmat = 0x524D4154u;  // stream tags keep the draws of each use apart
constexpr uint32_t kTagWeight = 0x57454947u;
constexpr uint32_t kTagUpdate = 0x55504454u;

inline Rand4 draw(uint64_t item, uint32_t sub, uint32_t tag, uint64_t seed) {
  return philox((uint32_t)item, (uint32_t)(item >> 32), sub, tag, (uint32_t)seed, (uint32_t)(seed >> 32));
}

inline double unit53(uint32_t hi, uint32_t lo) {
  return (double)((((uint64_t)hi << 32) | lo) >> 11) * (1.0 / 9007199254740992.0);
}

// Zipf(s) on [lo, hi] by rejection-inversion (Hoermann and Derflinger, "Rejection-
// inversion to generate variates from monotone discrete distributions", ACM TOMACS
// 6(3), 1996): invert the integral H of the hat x^-s, accept when the point lies
// under the histogram of the target.
struct Zipf {
  double s, lo, hi, hx1, hn, thr;
  double H(double x) const { return std::fabs(s - 1.0) < 1e-12 ? std::log(x) : (std::pow(x, 1.0 - s) - 1.0) / (1.0 - s); }
  double Hinv(double y) const {
    return std::fabs(s - 1.0) < 1e-12 ? std::exp(y) : std::pow(1.0 + y * (1.0 - s), 1.0 / (1.0 - s));
  }
  double h(double x) const { return std::pow(x, -s); }
  Zipf(double s_, double lo_, double hi_) : s(s_), lo(lo_), hi(hi_) {
    hx1 = H(lo + 0.5) - h(lo);
    hn = H(hi + 0.5);
    thr = (lo + 1) - Hinv(H(lo + 1.5) - h(lo + 1));
  }
  uint32_t sample(uint64_t item, uint64_t seed) const {
    for (uint32_t t = 0;; ++t) {
      const Rand4 r = draw(item, 1 + t, kTagWeight, seed);
      const double u = hn + unit53(r.x, r.y) * (hx1 - hn);
      const double x = Hinv(u);
      double k = std::floor(x + 0.5);
      k = std::min(std::max(k, lo), hi);
      if (k - x <= thr || u >= H(k + 0.5) - h(k) || t > 1000) return (uint32_t)k;
    }
  }
};

uint32_t weight_of(uint64_t i, int dist, double lo, double hi, double s, uint64_t seed, const Zipf* z) {
  if (dist == BINGO_W_ZIPF) return z->sample(i, seed);
  const Rand4 r = draw(i, 0, kTagWeight, seed);
  if (dist == BINGO_W_LOGUNIFORM) {
    const double x = lo * std::exp(unit53(r.x, r.y) * std::log(hi / lo));
    double f = std::floor(x);
    f = std::min(std::max(f, lo), hi - 1.0);
    return (uint32_t)f;
  }
  const uint64_t l = (uint64_t)lo, range = (uint64_t)hi - l + 1;
  return (uint32_t)(l + (((uint64_t)r.x * range) >> 32));
}

// Open-addressing set of 64-bit keys (linear probing, tombstones).
struct KeySet {
  static constexpr uint64_t kEmpty = ~0ull, kTomb = ~0ull - 1;
  std::vector<uint64_t> t;
  uint64_t mask = 0, used = 0;
  static uint64_t mix(uint64_t x) {  // SplitMix64 finaliser (Steele, Lea, Flood, OOPSLA 2014)
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    return x ^ (x >> 31);
  }
  void reserve(uint64_t n) {
    uint64_t c = 16;
    while (c < 2 * n + 16) c <<= 1;
    std::vector<uint64_t> old;
    old.swap(t);
    t.assign(c, kEmpty);
    mask = c - 1;
    used = 0;
    for (uint64_t k : old)
      if (k != kEmpty && k != kTomb) insert(k);
  }
  bool contains(uint64_t k) const {
    for (uint64_t h = mix(k) & mask;; h = (h + 1) & mask) {
      if (t[h] == k) return true;
      if (t[h] == kEmpty) return false;
    }
  }
  void insert(uint64_t k) {
    if (2 * (used + 1) > t.size()) reserve(t.size());
    uint64_t h = mix(k) & mask;
    while (t[h] != kEmpty && t[h] != kTomb) h = (h + 1) & mask;
    if (t[h] == kEmpty) ++used;
    t[h] = k;
  }
  void erase(uint64_t k) {
    for (uint64_t h = mix(k) & mask;; h = (h + 1) & mask) {
      if (t[h] == k) {
        t[h] = kTomb;
        return;
      }
      if (t[h] == kEmpty) return;
    }
  }
};

}  // namespace

struct bingo_updgen {
  uint32_t n;
  uint64_t seed, ctr = 0;
  std::vector<uint32_t> ecnt;
  struct Live {
    uint32_t u, v, slot;
  };
  std::vector<Live> live;
  KeySet keys;
};

extern "C" {

uint64_t bingo_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                        uint32_t* src, uint32_t* dst) {
  if (scale == 0 || scale > 31) return 0;
  const uint64_t draws = (uint64_t)edge_factor << scale;
  const uint64_t ta = (uint64_t)std::ldexp(a, 32), tab = (uint64_t)std::ldexp(a + b, 32),
                 tabc = (uint64_t)std::ldexp(a + b + c, 32);
  std::vector<uint64_t> key(draws);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)draws; ++i) {
    uint64_t u = 0, v = 0;
    Rand4 r{0, 0, 0, 0};
    for (uint32_t l = 0; l < scale; ++l) {
      if ((l & 3) == 0) r = draw((uint64_t)i, l >> 2, kTagRmat, seed);
      const uint32_t x = (l & 3) == 0 ? r.x : (l & 3) == 1 ? r.y : (l & 3) == 2 ? r.z : r.w;
      const uint32_t su = x >= tab, sv = (x >= ta && x < tab) || x >= tabc;
      u = (u << 1) | su;
      v = (v << 1) | sv;
    }
    key[i] = u == v ? ~0ull : (u << 32) | v;
  }
  __gnu_parallel::sort(key.begin(), key.end());
  uint64_t m = 0;
  for (uint64_t i = 0; i < draws; ++i) {
    if (key[i] == ~0ull) break;
    if (i && key[i] == key[i - 1]) continue;
    if (src) src[m] = (uint32_t)(key[i] >> 32), dst[m] = (uint32_t)key[i];
    ++m;
  }
  return m;
}

void bingo_gen_weights(uint64_t m, int dist, double lo, double hi, double s, uint64_t seed, uint32_t* w) {
  const Zipf z(s > 0 ? s : 1.0, lo, hi);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)m; ++i) w[i] = weight_of((uint64_t)i, dist, lo, hi, s, seed, &z);
}

bingo_updgen* bingo_updgen_create(uint32_t n, const uint32_t* src, const uint32_t* dst, uint64_t m, uint64_t seed) {
  bingo_updgen* g = new bingo_updgen;
  g->n = n;
  g->seed = seed;
  g->ecnt.assign(n, 0);
  g->live.resize(m);
  g->keys.reserve(m + 1024);
  for (uint64_t i = 0; i < m; ++i) {
    g->live[i] = bingo_updgen::Live{src[i], dst[i], g->ecnt[src[i]]++};
    g->keys.insert(((uint64_t)src[i] << 32) | dst[i]);
  }
  return g;
}

void bingo_updgen_destroy(bingo_updgen* g) { delete g; }

uint64_t bingo_updgen_live(const bingo_updgen* g) { return g->live.size(); }

uint64_t bingo_updgen_inserts(bingo_updgen* g, uint64_t k, int dist, double lo, double hi, double s, uint32_t* src,
                              uint32_t* dst, uint32_t* w) {
  const Zipf z(s > 0 ? s : 1.0, lo, hi);
  const uint64_t wseed = g->seed ^ 0x9E3779B97F4A7C15ull;
  for (uint64_t i = 0; i < k; ++i) {
    uint32_t u, v;
    for (;;) {
      const Rand4 r = draw(g->ctr++, 0, kTagUpdate, g->seed);
      u = (uint32_t)(((uint64_t)r.x * g->n) >> 32);
      v = (uint32_t)(((uint64_t)r.y * g->n) >> 32);
      if (u != v && !g->keys.contains(((uint64_t)u << 32) | v)) break;
    }
    g->keys.insert(((uint64_t)u << 32) | v);
    src[i] = u, dst[i] = v;
    w[i] = weight_of(g->ctr, dist, lo, hi, s, wseed, &z);
    g->live.push_back(bingo_updgen::Live{u, v, g->ecnt[u]++});
  }
  return k;
}

uint64_t bingo_updgen_deletes(bingo_updgen* g, uint64_t k, uint32_t* u, uint32_t* slot) {
  uint64_t made = 0;
  for (; made < k && !g->live.empty(); ++made) {
    const Rand4 r = draw(g->ctr++, 1, kTagUpdate, g->seed);
    const uint64_t pick = (((uint64_t)r.x << 32 | r.y) % g->live.size());
    const bingo_updgen::Live e = g->live[pick];
    g->live[pick] = g->live.back();
    g->live.pop_back();
    g->keys.erase(((uint64_t)e.u << 32) | e.v);
    u[made] = e.u, slot[made] = e.slot;
  }
  return made;
}

// ---- the reference's own inputs (include/graph.cuh:22-51) -------------------

int bingo_edge_list_read(const char* path, uint32_t* src, uint32_t* dst, uint64_t cap, uint64_t* m, uint32_t* n) {
  if (!path || !m || !n) return -1;
  FILE* f = std::fopen(path, "rb");
  if (!f) return -1;
  std::vector<char> buf(1 << 22);
  uint64_t count = 0, offset = 0, maxid = 0;
  uint64_t val = 0, pair[2] = {0, 0};
  int state = 0;       // 0 between tokens, 1 in a number, 2 in a comment line
  int half = 0;        // ids of the current pair read so far
  bool line_start = true;
  int rc = 0;
  auto emit = [&](uint64_t x) -> int {
    if (x > 0xFFFFFFFEull) return -4;
    pair[half++] = x;
    if (half == 2) {
      if (src) {
        if (count >= cap) return -3;
        src[count] = (uint32_t)pair[0], dst[count] = (uint32_t)pair[1];
      }
      maxid = std::max(maxid, std::max(pair[0], pair[1]));
      ++count;
      half = 0;
    }
    return 0;
  };
  size_t got;
  while (rc == 0 && (got = std::fread(buf.data(), 1, buf.size(), f)) > 0) {
    for (size_t i = 0; i < got && rc == 0; ++i, ++offset) {
      const char c = buf[i];
      if (state == 2) {
        if (c == '\n') state = 0, line_start = true;
        continue;
      }
      if (c >= '0' && c <= '9') {
        if (state == 0) val = 0, state = 1;
        val = val * 10 + (uint64_t)(c - '0');
        if (val > 0xFFFFFFFFull) val = 0x100000000ull;  // saturate; rejected as too large
        line_start = false;
      } else if (c == ' ' || c == '\t' || c == '\r' || c == '\n') {
        if (state == 1) rc = emit(val), state = 0;
        if (c == '\n') line_start = true;
      } else if ((c == '#' || c == '%') && line_start && state == 0) {
        state = 2;
      } else {
        *m = offset;
        rc = -2;
      }
    }
  }
  if (std::ferror(f) && rc == 0) rc = -1;
  std::fclose(f);
  if (rc == 0 && state == 1) rc = emit(val);
  if (rc == 0 && half) {  // a trailing lone id: the reference's scanf("%d%d") would not form an edge
    *m = offset;
    rc = -2;
  }
  if (rc) return rc;
  *m = count;
  *n = count ? (uint32_t)(maxid + 1) : 0;
  return 0;
}

int bingo_driver_weights(int kind, const uint32_t* src, const uint32_t* dst, uint64_t m, uint32_t n, uint32_t* w) {
  if (kind == BINGO_DRIVER_AUTO) kind = n > 1e7 ? BINGO_DRIVER_DEGREE_POW03 : BINGO_DRIVER_DEGREE;
  if (kind != BINGO_DRIVER_DEGREE && kind != BINGO_DRIVER_DEGREE_POW03) return -1;
  std::vector<uint32_t> d(n, 0);
  for (uint64_t i = 0; i < m; ++i) {
    if (src[i] >= n || dst[i] >= n) return -1;
    ++d[src[i]];
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)m; ++i) {
    const uint32_t dv = d[dst[i]];
    // The reference computes int w = bias(d) + 1 with bias returning float.
    const float b = kind == BINGO_DRIVER_DEGREE ? (float)dv : (float)std::pow((double)dv, 0.3);
    w[i] = (uint32_t)(b + 1.0f);
  }
  return 0;
}

}  // extern "C"
