// Walk-step sampler and the per-app walk loops. Replaces NodeData::sample
// (include/Bingo.cuh:220-267) and the loops of deepwalkKernel, node2vecKernel,
// pprKernel and samplingKernel (include/operation.cuh:252-368, :407-430).
//
// One step is three dependent loads: the 16 B VertexRec of the current
// vertex, the 32 B AliasRec of the drawn slot (which carries both candidate
// groups' member-list base and count), and the 4 B member id. All three go
// through the read-only path: the store does not change during a walk phase.
#pragma once
#include "common.cuh"
#include "store.cuh"

namespace bingo {

constexpr uint32_t kMaxNode2vecTrials = 1u << 16;
constexpr uint32_t kMaxPprSteps = 1u << 20;
constexpr uint32_t kWalkPprTail = 1u;

enum AppId : int { APP_DEEPWALK = 0, APP_NODE2VEC = 1, APP_PPR = 2, APP_SAMPLING = 3 };

// One walk job as the kernels see it (starts/out are device pointers).
struct WalkJobDev {
  int32_t app;
  uint32_t L;
  const uint32_t* starts;  // null: first + walk index
  unsigned long long n;
  uint32_t first;
  uint32_t job;
  uint32_t k0, k1;  // Philox key (seed)
  uint32_t flags;
  uint32_t pad;
  unsigned long long thr_ret, thr_in, thr_out, thr_stop;  // 33-bit acceptance thresholds
  int32_t* out;
};

struct WalkView {
  uint32_t n;
  const VertexRec* __restrict__ vrec;
  const AliasRec* __restrict__ alias;
  const uint32_t* __restrict__ gv;
  const HashEntry* __restrict__ hash;
  uint32_t* err;
  unsigned long long* steps;  // running count of produced steps (moves to a neighbour)
};

__device__ __forceinline__ VertexRec load_vrec(const WalkView& W, uint32_t u) {
  const uint4 r = __ldg(reinterpret_cast<const uint4*>(W.vrec) + u);
  return VertexRec{r.x, r.y, r.z, r.w};
}

// Weighted neighbour draw at a vertex with R.m > 0: slot = mulhi(x, m),
// r = mulhi64(y:z, T), group = r < thr ? own : alias, member = mulhi(w, cnt).
__device__ __forceinline__ uint32_t sample_at(const WalkView& W, const VertexRec& R, const Rand4& r) {
  const ulonglong2* a = reinterpret_cast<const ulonglong2*>(W.alias + R.aoff + mulhi32(r.x, R.m));
  const ulonglong2 tt = __ldg(a);                                   // thr, T
  const uint4 g = __ldg(reinterpret_cast<const uint4*>(a + 1));     // own base/cnt, alt base/cnt
  const unsigned long long d = mulhi64(((unsigned long long)r.y << 32) | r.z, tt.y);
  const bool own = d < tt.x;
  const uint32_t base = own ? g.x : g.z, cnt = own ? g.y : g.w;
  return __ldg(W.gv + (size_t)base * 4 + mulhi32(r.w, cnt));
}

__device__ __forceinline__ bool adjacent(const WalkView& W, const VertexRec& Rprev, uint32_t x) {
  return hash_has(W.hash + Rprev.hoff, Rprev.hmask, x);
}

// Runs walk `i` of job J to completion, writing its row. Returns the number
// of moves made (the produced steps).
template <int APP>
__device__ __forceinline__ uint32_t run_walk(const WalkView& W, const WalkJobDev& J, uint32_t i) {
  const uint32_t start = J.starts ? J.starts[i] : J.first + i;
  if (APP == APP_SAMPLING) {
    int32_t x = -1;
    if (start < W.n) {
      const VertexRec R = load_vrec(W, start);
      if (R.m) x = (int32_t)sample_at(W, R, philox(i, 1, 0, J.job, J.k0, J.k1));
    } else {
      set_err(W.err, E_RANGE);
    }
    J.out[i] = x;
    return x >= 0;
  }
  const uint32_t L = J.L;
  int32_t* row = J.out + (size_t)i * L;
  if (L == 0) return 0;
  if (start >= W.n) {
    set_err(W.err, E_RANGE);
    for (uint32_t j = 0; j < L; ++j) row[j] = -1;
    return 0;
  }
  row[0] = (int32_t)start;
  uint32_t cur = start, pos = 0, moves = 0;
  int64_t prev = -1;
  VertexRec Rprev{0, 0, 0, 0};
  const bool tail = APP == APP_PPR && (J.flags & kWalkPprTail);
  for (uint32_t j = 1;; ++j) {
    if (j >= L && !tail) break;
    if (tail && j >= kMaxPprSteps) break;
    pos = j < L ? j : L - 1;
    const VertexRec R = load_vrec(W, cur);
    if (!R.m) {
      row[pos] = -1;
      break;
    }
    uint32_t x;
    if (APP == APP_NODE2VEC && prev >= 0) {
      for (uint32_t t = 0;; ++t) {
        x = sample_at(W, R, philox(i, j, 2 * t, J.job, J.k0, J.k1));
        const unsigned long long thr =
            (int64_t)x == prev ? J.thr_ret : (adjacent(W, Rprev, x) ? J.thr_in : J.thr_out);
        const uint32_t a = philox(i, j, 2 * t + 1, J.job, J.k0, J.k1).x;
        if ((unsigned long long)a < thr || t + 1 == kMaxNode2vecTrials) break;
      }
    } else {
      x = sample_at(W, R, philox(i, j, 0, J.job, J.k0, J.k1));
    }
    row[pos] = (int32_t)x;
    ++moves;
    prev = cur;
    Rprev = R;
    cur = x;
    if (APP == APP_PPR && (unsigned long long)philox(i, j, 1, J.job, J.k0, J.k1).x < J.thr_stop) break;
  }
  for (uint32_t j = pos + 1; j < L; ++j) row[j] = -1;
  return moves;
}

__device__ __forceinline__ uint32_t run_walk_any(const WalkView& W, const WalkJobDev& J, uint32_t i) {
  switch (J.app) {
    case APP_DEEPWALK: return run_walk<APP_DEEPWALK>(W, J, i);
    case APP_NODE2VEC: return run_walk<APP_NODE2VEC>(W, J, i);
    case APP_PPR: return run_walk<APP_PPR>(W, J, i);
    default: return run_walk<APP_SAMPLING>(W, J, i);
  }
}

// One atomic per warp: adds the warp's produced steps to the running count.
__device__ __forceinline__ void add_steps(const WalkView& W, unsigned long long mine) {
#pragma unroll
  for (int o = 16; o; o >>= 1) mine += __shfl_xor_sync(kFull, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(W.steps, mine);
}

}  // namespace bingo
