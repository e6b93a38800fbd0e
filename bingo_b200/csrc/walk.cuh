// Walk-step sampler and the per-app walk loops. Replaces NodeData::sample
// (include/Bingo.cuh:220-267) and the loops of deepwalkKernel, node2vecKernel,
// pprKernel and samplingKernel (include/operation.cuh:252-368, :407-430).
//
// One step is at most three dependent loads: the 16 B VertexRec of the
// current vertex, the 32 B AliasRec of the drawn slot (which names both
// candidate groups: member-list base and count, or for a one-member group the
// member itself), and the 4 B member id (skipped for a one-member group). All
// go through the read-only path: the store does not change during a walk
// phase.
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
  uint32_t seq;  // serving ring: the job's sequence number (0 elsewhere)
  unsigned long long thr_ret, thr_in, thr_out, thr_stop;  // 33-bit acceptance thresholds
  double ret_excess;  // node2vec: (1/p) / max(1, 1/q) - 1 when positive, else 0
  int32_t* out;
};

// p in [0, 1] -> 33-bit threshold floor(p * 2^32) (2^32 = always); the same
// formula as the host side, with IEEE-rounded operations.
__device__ __forceinline__ unsigned long long prob_threshold_dev(double p) {
  if (!(p > 0.0)) return 0ull;
  if (p >= 1.0) return 1ull << 32;
  const double t = floor(__dmul_rn(p, 4294967296.0));
  return t >= 4294967296.0 ? (1ull << 32) : (unsigned long long)t;
}

struct WalkView {
  uint32_t n;
  const VertexRec* __restrict__ vrec;
  const AliasRec* __restrict__ alias;
  const uint32_t* __restrict__ gv;
  const HashEntry* __restrict__ hash;
  uint32_t* err;
  unsigned long long* steps;  // running count of produced steps (moves to a neighbour)
  unsigned long long* n2v;    // node2vec: [0] proposals drawn, [1] adjacency probes
};

__device__ __forceinline__ VertexRec load_vrec(const WalkView& W, uint32_t u) {
  const uint4 r = __ldg(reinterpret_cast<const uint4*>(W.vrec) + u);
  return VertexRec{r.x, r.y, r.z, r.w};
}

// Weighted neighbour draw at a vertex with R.m > 0: slot = mulhi(x, m),
// r = mulhi64(y:z, T), group = r < thr ? own : alias, member = mulhi(w, cnt)
// (a one-member group carries its member in the slot: mulhi(w, 1) = 0).
__device__ __forceinline__ uint32_t sample_at(const WalkView& W, const VertexRec& R, const Rand4& r) {
  // The whole 32-byte slot in one 256-bit read-only load (one L1 / L2
  // request instead of two 16-byte ones; slots are 32-byte aligned and no
  // kernel writes the store while walks run).
  const AliasRec* a = W.alias + R.aoff + mulhi32(r.x, R.m);
  unsigned long long thr, T, own_rc, alt_rc;
  asm("ld.global.nc.v4.u64 {%0, %1, %2, %3}, [%4];" : "=l"(thr), "=l"(T), "=l"(own_rc), "=l"(alt_rc) : "l"(a));
  const unsigned long long d = mulhi64(((unsigned long long)r.y << 32) | r.z, T);
  const unsigned long long rc = d < thr ? own_rc : alt_rc;  // ref | count word << 32
  const uint32_t ref = (uint32_t)rc, cw = (uint32_t)(rc >> 32);
  if (cw & kInlineGroup) return ref;  // one member, carried in the slot
  return __ldg(W.gv + (size_t)ref * 4 + mulhi32(r.w, cw));
}


// ---------------------------------------------------------------------------
// Step-at-a-time walks for the persistent kernels: a lane advances its walk
// one step per iteration and pulls a new walk as soon as its walk ends, so
// dead-ended and early-stopped walks do not idle their warp.
//
// Counters: step j of walk i in job `job` draws Philox block
// (i, j, trial, job) under key seed. DeepWalk uses trial 0; PPR samples with
// trial 0 and tests its stop with trial 1; node2vec proposes with trial 2t
// and accepts with trial 2t + 1 (t = 0, 1, ...; the first step is
// first-order and takes trial 0). Row position j holds the j-th move; a walk
// that reaches a vertex without out-edges writes -1 there and pads the rest.
//
// Row output goes through an 8-entry (one 32-byte sector) staging buffer per
// lane in shared memory: a lane writes its row a whole sector at a time with
// streaming (evict-first) stores, so the write-once walk output neither
// lands in L2 as partial sectors nor evicts graph data.
struct RowStage {
  uint32_t sec;   // index of the buffered 32-byte sector within the job output; kNoSec: empty
  uint32_t lohi;  // valid entries [lo, hi) of the sector: lo | hi << 8
};
constexpr uint32_t kNoSec = 0xffffffffu;

// This lane's 8 staging entries (16-byte aligned, blockDim.x rows of 8).
__device__ __forceinline__ int32_t* stage_buf(int32_t (*obuf)[8]) { return obuf[threadIdx.x]; }

__device__ __forceinline__ void stage_flush(RowStage& o, int32_t* out, int32_t (*obuf)[8]) {
  if (o.sec == kNoSec) return;
  const int32_t* buf = stage_buf(obuf);
  int32_t* sec = out + (size_t)o.sec * 8;
  const uint32_t lo = o.lohi & 0xff, hi = o.lohi >> 8;
  if (lo == 0 && hi == 8) {
    const int4* b = reinterpret_cast<const int4*>(buf);
    __stcs(reinterpret_cast<int4*>(sec), b[0]);
    __stcs(reinterpret_cast<int4*>(sec) + 1, b[1]);
  } else {
    for (uint32_t t = lo; t < hi; ++t) __stcs(sec + t, buf[t]);
  }
  o.sec = kNoSec;
}

// Writes v to out[g] through the stage; a row's positions arrive in
// non-decreasing order (PPR tail mode rewrites the last one). Job outputs are
// 32-byte aligned, so sectors are counted from out.
__device__ __forceinline__ void stage_put(RowStage& o, int32_t* out, int32_t (*obuf)[8], unsigned long long g,
                                          int32_t v) {
  const uint32_t sec = (uint32_t)(g >> 3), t = (uint32_t)(g & 7);
  if (sec != o.sec) {
    stage_flush(o, out, obuf);
    o.sec = sec;
    o.lohi = t | (t << 8);
  }
  stage_buf(obuf)[t] = v;
  if (t + 1 > (o.lohi >> 8)) o.lohi = (o.lohi & 0xff) | ((t + 1) << 8);
}

// Pads out[g, g_end) with -1: the open sector through the stage, then whole
// sectors with two 16-byte streaming stores each.
__device__ __forceinline__ void stage_pad(RowStage& o, int32_t* out, int32_t (*obuf)[8], unsigned long long g,
                                          unsigned long long g_end) {
  for (; g < g_end && (g & 7); ++g) stage_put(o, out, obuf, g, -1);
  stage_flush(o, out, obuf);
  const int4 m1 = make_int4(-1, -1, -1, -1);
  for (; g + 8 <= g_end; g += 8) {
    __stcs(reinterpret_cast<int4*>(out + g), m1);
    __stcs(reinterpret_cast<int4*>(out + g) + 1, m1);
  }
  for (; g < g_end; ++g) __stcs(out + g, -1);
}

// node2vec trials a lane runs before it yields the rest of the step to the
// next call (the rest of its warp moves on meanwhile).
constexpr uint32_t kNode2vecTrialsPerCall = 3;

struct LaneWalk {
  uint32_t i;      // walk index within its job
  uint32_t j;      // step being produced
  uint32_t cur;    // current vertex
  uint32_t pos;    // last row position written
  int32_t prev;    // previous vertex (node2vec), -1 before the first move
  uint32_t phoff;  // previous vertex's adjacency index (node2vec)
  uint32_t phmask;
  uint32_t trials;  // node2vec proposals drawn by this lane (kept across its walks)
  uint32_t probes;  // node2vec adjacency-index lookups by this lane
  uint32_t t;       // node2vec: trial of the step in progress (0 = a new step)
  unsigned long long region;  // node2vec: return-region threshold of the step in progress
};

// Starts walk i; returns true if it still has steps to produce. Sampling jobs
// complete here.
template <int APP>
__device__ __forceinline__ bool walk_begin(const WalkView& W, const WalkJobDev& J, uint32_t i, LaneWalk& s,
                                           RowStage& o, int32_t (*obuf)[8], uint32_t& moves) {
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
    moves += x >= 0;
    return false;
  }
  const uint32_t L = J.L;
  if (L == 0) return false;
  const unsigned long long g0 = (unsigned long long)i * L;
  if (start >= W.n) {
    set_err(W.err, E_RANGE);
    stage_pad(o, J.out, obuf, g0, g0 + L);
    return false;
  }
  stage_put(o, J.out, obuf, g0, (int32_t)start);
  s.i = i;
  s.j = 1;
  s.cur = start;
  s.pos = 0;
  s.prev = -1;
  s.t = 0;
  const bool tail = APP == APP_PPR && (J.flags & kWalkPprTail);
  if (L > 1 || tail) return true;
  stage_flush(o, J.out, obuf);
  return false;
}

// Produces one step; returns false when the walk has ended (row padded and
// flushed).
template <int APP>
__device__ __forceinline__ bool walk_advance(const WalkView& W, const WalkJobDev& J, LaneWalk& s, RowStage& o,
                                             int32_t (*obuf)[8], uint32_t& moves) {
  const uint32_t L = J.L;
  const bool tail = APP == APP_PPR && (J.flags & kWalkPprTail);
  s.pos = s.j < L ? s.j : L - 1;
  const unsigned long long g0 = (unsigned long long)s.i * L;
  const VertexRec R = load_vrec(W, s.cur);
  bool done = false;
  if (!R.m) {
    stage_put(o, J.out, obuf, g0 + s.pos, -1);
    done = true;
  } else {
    uint32_t x;
    if (APP == APP_NODE2VEC && s.prev >= 0) {
      // One trial per call: a rejected lane keeps its step and retries on the
      // next call while the other lanes of its warp go on, so the lanes of a
      // warp stay on the same instruction path (the trial count per step
      // varies from lane to lane). Trial t reads the same Philox blocks as in
      // a loop, so the walk is unchanged.
      if (s.t == 0) {
        // Return region: when 1/p exceeds the envelope max(1, 1/q), the
        // excess mass (ret_excess x w(cur -> prev)) returns to prev directly,
        // with probability D / (T + D) per trial (word y of the acceptance
        // block).
        s.region = 0;
        if (J.ret_excess > 0.0) {
          const unsigned long long wp = hash_weight(W.hash + R.hoff, R.hmask, (uint32_t)s.prev);
          ++s.probes;
          if (wp) {
            const double T = (double)__ldg(&W.alias[R.aoff].T);
            const double D = __dmul_rn(J.ret_excess, (double)wp);
            s.region = prob_threshold_dev(__ddiv_rn(D, __dadd_rn(T, D)));
          }
        }
      }
      // Otherwise accept a proposal x with probability weight(class(x)) /
      // envelope. The adjacency probe is skipped when the acceptance draw is
      // below both the in- and out-class thresholds (the outcome is then the
      // same for every class x can be in).
      bool ok = false;
      for (uint32_t k = 0; k < kNode2vecTrialsPerCall && !ok; ++k) {
        if (k) ++s.t;
        const Rand4 a = philox(s.i, s.j, 2 * s.t + 1, J.job, J.k0, J.k1);
        if ((unsigned long long)a.y < s.region) {
          x = (uint32_t)s.prev;
          ok = true;
        } else {
          x = sample_at(W, R, philox(s.i, s.j, 2 * s.t, J.job, J.k0, J.k1));
          ++s.trials;
          const unsigned long long io_min = J.thr_in < J.thr_out ? J.thr_in : J.thr_out;
          if ((int32_t)x == s.prev) {
            ok = a.x < J.thr_ret;
          } else if (a.x < io_min) {
            ok = true;
          } else {
            ok = a.x < (hash_has(W.hash + s.phoff, s.phmask, x) ? J.thr_in : J.thr_out);
            ++s.probes;
          }
          ok = ok || s.t + 1 == kMaxNode2vecTrials;
        }
      }
      if (!ok) {
        ++s.t;
        return true;  // the step continues on the next call
      }
      s.t = 0;
    } else {
      x = sample_at(W, R, philox(s.i, s.j, 0, J.job, J.k0, J.k1));
    }
    stage_put(o, J.out, obuf, g0 + s.pos, (int32_t)x);
    ++moves;
    if (APP == APP_NODE2VEC) {
      s.prev = (int32_t)s.cur;
      s.phoff = R.hoff;
      s.phmask = R.hmask;
    }
    s.cur = x;
    if (APP == APP_PPR && (unsigned long long)philox(s.i, s.j, 1, J.job, J.k0, J.k1).x < J.thr_stop) done = true;
    ++s.j;
    if ((s.j >= L && !tail) || (tail && s.j >= kMaxPprSteps)) done = true;
  }
  if (done) stage_pad(o, J.out, obuf, g0 + s.pos + 1, g0 + L);
  return !done;
}

__device__ __forceinline__ bool begin_any(const WalkView& W, const WalkJobDev& J, uint32_t i, LaneWalk& s,
                                          RowStage& o, int32_t (*obuf)[8], uint32_t& mv) {
  switch (J.app) {
    case APP_DEEPWALK: return walk_begin<APP_DEEPWALK>(W, J, i, s, o, obuf, mv);
    case APP_NODE2VEC: return walk_begin<APP_NODE2VEC>(W, J, i, s, o, obuf, mv);
    case APP_PPR: return walk_begin<APP_PPR>(W, J, i, s, o, obuf, mv);
    default: return walk_begin<APP_SAMPLING>(W, J, i, s, o, obuf, mv);
  }
}
__device__ __forceinline__ bool advance_any(const WalkView& W, const WalkJobDev& J, LaneWalk& s, RowStage& o,
                                            int32_t (*obuf)[8], uint32_t& mv) {
  switch (J.app) {
    case APP_DEEPWALK: return walk_advance<APP_DEEPWALK>(W, J, s, o, obuf, mv);
    case APP_NODE2VEC: return walk_advance<APP_NODE2VEC>(W, J, s, o, obuf, mv);
    default: return walk_advance<APP_PPR>(W, J, s, o, obuf, mv);
  }
}

// One atomic per warp: adds the warp's produced steps to the running count.
__device__ __forceinline__ void add_steps(const WalkView& W, unsigned long long mine) {
#pragma unroll
  for (int o = 16; o; o >>= 1) mine += __shfl_xor_sync(kFull, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(W.steps, mine);
}

// The same for the node2vec proposal and probe counts (zero, and folded
// away, in kernels without node2vec walks).
__device__ __forceinline__ void add_n2v(const WalkView& W, const LaneWalk& s) {
  unsigned long long t = s.trials, p = s.probes;
#pragma unroll
  for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(kFull, t, o), p += __shfl_xor_sync(kFull, p, o);
  if ((threadIdx.x & 31) == 0 && (t | p)) atomicAdd(W.n2v, t), atomicAdd(W.n2v + 1, p);
}

}  // namespace bingo
