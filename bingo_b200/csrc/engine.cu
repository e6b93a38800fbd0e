// Engine: kernels and host orchestration for load / insert / delete / walk.
//
// Update batches run as: group by vertex (batches up to kGroupMax edges: one
// cluster kernel that validates, sorts stably and lists the segments; larger
// ones: validate -> CUB radix sort -> gather + segment heads -> segment
// select) -> plan (per-vertex growth sizes, prefix inside each plan block) ->
// prefix of the plan-block sums and the batch's arena reservation (one
// block) -> apply (warp per vertex). Arena offsets come from these prefix
// sums in segment order, so the layout is a deterministic function of the
// inputs; arenas are index-addressed and grow by reallocation on the host
// (before a load, or when a batch did not fit).
#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "engine.cuh"
#include "group.cuh"
#include "serve.cuh"
#include "store.cuh"
#include "walk.cuh"

namespace bingo {

namespace {

constexpr int kBlock = 256;
constexpr unsigned long long kUnitBytes[kArenas] = {4, sizeof(EdgeRec), 4, sizeof(AliasRec), sizeof(HashEntry)};
// Index limits imposed by the 32-bit offsets in the walk-side records.
// (member lists are named by their offset in 4-entry units plus one, a 32-bit word)
constexpr unsigned long long kArenaLimit[kArenas] = {(1ull << 34) - 4, ~0ull, ~0ull, (1ull << 32), (1ull << 32)};
constexpr unsigned long long kArenaFloor[kArenas] = {1024, 1024, 1024, 256, 1024};
const char* const kArenaName[kArenas] = {"member", "edge", "back-pointer", "alias", "adjacency"};

int sm_count() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

size_t pow2_bytes(size_t b) {
  size_t p = 256;
  while (p < b) p <<= 1;
  return p;
}

unsigned grid_for(unsigned long long items, unsigned per_block, unsigned max_per_sm = 8) {
  const unsigned long long want = (items + per_block - 1) / per_block;
  const unsigned long long cap = (unsigned long long)sm_count() * max_per_sm;
  return (unsigned)std::max(1ull, std::min(want, cap));
}

// Launch with programmatic stream serialization (the kernel starts with
// pdl_wait()): its scheduling overlaps the end of the kernel before it.
template <typename... KArgs, typename... Args>
void launch_pdl(void (*kern)(KArgs...), unsigned grid, unsigned block, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(grid);
  lc.blockDim = dim3(block);
  lc.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  cuda_check(cudaLaunchKernelEx(&lc, kern, static_cast<KArgs>(args)...), "launch");
}

// ------------------------------------------------------------------ kernels
__global__ void k_iota(uint32_t* a, unsigned long long n) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    a[i] = (uint32_t)i;
}

// Range / weight checks of a batch. Any bit set in ctl aborts the batch.
__global__ void k_validate(const uint32_t* a, const uint32_t* b, const uint32_t* w, unsigned long long k, uint32_t n,
                           uint32_t* ctl, uint32_t* err) {
  uint32_t bits = 0;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < k;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    if ((a && a[i] >= n) || (b && b[i] >= n)) bits |= E_RANGE;
    if (w && w[i] == 0u) bits |= E_ZERO_WEIGHT;
  }
  bits = __reduce_or_sync(kFull, bits);
  if (bits && (threadIdx.x & 31) == 0) {
    atomicOr(ctl, bits);
    atomicOr(err, bits);
  }
}

// Sorted order -> payload columns in sorted order + segment heads.
__global__ void k_gather(const uint32_t* key, const uint32_t* perm, const uint32_t* a, const uint32_t* b,
                         uint32_t* sa, uint32_t* sb, uint8_t* head, unsigned long long k) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < k;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t p = perm[i];
    sa[i] = a[p];
    if (b) sb[i] = b[p];
    head[i] = (i == 0 || key[i] != key[i - 1]) ? 1 : 0;
  }
}

__device__ __forceinline__ void seg_bounds(const uint32_t* seg, uint32_t S, uint32_t s, unsigned long long k,
                                           uint32_t* b, uint32_t* e) {
  *b = seg[s];
  *e = s + 1 < S ? seg[s + 1] : (uint32_t)k;
}

// Arena sizes one segment needs (units of each arena).
struct ArenaNeed {
  unsigned long long v[kArenas];
};

// Plan blocks: one segment per warp, kPlanSegs consecutive segments per block.
constexpr int kPlanThreads = 1024;
constexpr int kPlanSegs = kPlanThreads / 32;
constexpr int kTotalsThreads = 1024;

// Plan blocks of a batch with ks segment slots.
__host__ __device__ inline uint32_t plan_blocks(uint32_t ks) { return (ks + kPlanSegs - 1) / kPlanSegs; }

// Per-segment arena sizes as an exclusive prefix inside the segment's plan
// block (excl[s], s < ks) and each block's sums, column-major per arena
// (bsum[a * nb + block]); segments past the last one need nothing. A
// segment's offset in arena a is then the prefix of bsum over blocks (which
// k_totals writes in place) plus excl[s].
__global__ void __launch_bounds__(kPlanThreads) k_plan(StoreView S, const uint32_t* skey, const uint32_t* sw,
                                                       const uint32_t* seg, const uint32_t* nseg,
                                                       unsigned long long k, uint32_t ks, const uint32_t* ctl,
                                                       ArenaNeed* excl, unsigned long long* bsum) {
  pdl_wait();
  pdl_trigger();
  __shared__ unsigned long long nd_s[kPlanSegs][kArenas];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t s = blockIdx.x * kPlanSegs + w;
  const uint32_t nS = *nseg;
  unsigned long long nd[kArenas] = {0, 0, 0, 0, 0};
  if (*ctl == 0 && s < nS) {
    uint32_t b, e;
    seg_bounds(seg, nS, s, k, &b, &e);
    const uint32_t u = skey[b];
    if (u < S.n) plan_append(S, u, sw + b, e - b, nd);
  }
  if (lane == 0) {
#pragma unroll
    for (int a = 0; a < kArenas; ++a) nd_s[w][a] = nd[a];
  }
  __syncthreads();
  if (w == 0) {  // lane v: the block's segment v
    const uint32_t nb = plan_blocks(ks), sv = blockIdx.x * kPlanSegs + lane;
#pragma unroll
    for (int a = 0; a < kArenas; ++a) {
      const unsigned long long y = nd_s[lane][a];
      unsigned long long yi = y;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long z = __shfl_up_sync(kFull, yi, o);
        if (lane >= o) yi += z;
      }
      if (sv < ks) excl[sv].v[a] = yi - y;
      if (lane == 31) bsum[(size_t)a * nb + blockIdx.x] = yi;
    }
  }
}

// Device reservation modes of k_totals and the outcome it publishes.
enum ReserveMode { kReserveNone = 0, kReservePublish = 1, kReserveSticky = 2 };
constexpr unsigned long long kReserveOk = 1, kReserveFull = 2, kReserveRejected = 3;
constexpr int kPlanStatusSlot = 2 * kArenas + 1;  // after totals, status word and tops in the published plan

// Exclusive prefix of the nb plan-block sums (column-major per arena), in
// place, and the batch totals per arena (one block; two tiles of
// kTotalsThreads block sums per barrier pass). With `out` (mapped host
// memory) it also publishes the insert plan: out[0..5) totals, out[5] the
// batch status word, out[6..11) the arena tops before this batch, and last
// (after a system fence) out[kPlanStatusSlot], nonzero once the rest is
// visible to the host.
// `reserve` != kReserveNone then reserves the batch's arena space, all or
// nothing: base = the tops, tops += totals. A full arena sets E_CAPACITY in
// the batch status word (the apply kernel then skips the batch); with
// kReservePublish the outcome goes to out[kPlanStatusSlot] and the host grows
// the arena and applies the batch again, with kReserveSticky (programs) the
// error also goes to the sticky error word.
__global__ void __launch_bounds__(kTotalsThreads) k_totals(StoreView S, unsigned long long* bsum, uint32_t nb,
                                                           unsigned long long* tot, uint32_t* ctl,
                                                           unsigned long long* base, int reserve,
                                                           volatile unsigned long long* out) {
  pdl_wait();
  pdl_trigger();
  constexpr int kTiles = 2;  // tiles of kTotalsThreads block sums scanned per barrier pass
  __shared__ unsigned long long wtot[kTiles][kTotalsThreads / 32][kArenas];
  __shared__ unsigned long long carry[kArenas];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  if (t < kArenas) carry[t] = 0;
  for (uint32_t base = 0; base < nb; base += kTiles * kTotalsThreads) {
    unsigned long long x[kTiles][kArenas], inc[kTiles][kArenas];
#pragma unroll
    for (int q = 0; q < kTiles; ++q) {
      const uint32_t r = base + (uint32_t)(q * kTotalsThreads + t);
#pragma unroll
      for (int a = 0; a < kArenas; ++a) x[q][a] = r < nb ? bsum[(size_t)a * nb + r] : 0ull;
    }
#pragma unroll
    for (int q = 0; q < kTiles; ++q)
#pragma unroll
      for (int a = 0; a < kArenas; ++a) {
        inc[q][a] = x[q][a];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const unsigned long long y = __shfl_up_sync(kFull, inc[q][a], o);
          if (lane >= o) inc[q][a] += y;
        }
        if (lane == 31) wtot[q][w][a] = inc[q][a];
        inc[q][a] -= x[q][a];  // exclusive within the warp
      }
    __syncthreads();
    if (w == 0) {  // lane v scans warp v's totals, tile by tile and arena by arena
#pragma unroll
      for (int a = 0; a < kArenas; ++a) {
        unsigned long long run = carry[a];
#pragma unroll
        for (int q = 0; q < kTiles; ++q) {
          const unsigned long long y = wtot[q][lane][a];
          unsigned long long yi = y;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long z = __shfl_up_sync(kFull, yi, o);
            if (lane >= o) yi += z;
          }
          wtot[q][lane][a] = run + yi - y;
          run += __shfl_sync(kFull, yi, 31);
        }
        __syncwarp();
        if (lane == 0) carry[a] = run;
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kTiles; ++q) {
      const uint32_t r = base + (uint32_t)(q * kTotalsThreads + t);
      if (r < nb) {
#pragma unroll
        for (int a = 0; a < kArenas; ++a) bsum[(size_t)a * nb + r] = wtot[q][w][a] + inc[q][a];
      }
    }
    __syncthreads();  // wtot and carry are reused by the next pass
  }
  __syncthreads();
  unsigned long long top0 = 0;
  uint32_t ctl0 = 0;
  if (t < kArenas) {
    tot[t] = carry[t];
    top0 = S.top[t];
  }
  if (t == kArenas) ctl0 = *ctl;
  __syncthreads();  // the tops and the status word are read before the reservation changes them
  __shared__ unsigned long long status;
  if (reserve != kReserveNone && t == 0) {
    unsigned long long st = kReserveOk;
    if (*ctl) {
      st = kReserveRejected;
    } else {
      bool ok = true;
      for (int a = 0; a < kArenas; ++a)
        if (S.top[a] + carry[a] > S.cap[a]) ok = false;
      if (ok) {
        for (int a = 0; a < kArenas; ++a) {
          base[a] = S.top[a];
          S.top[a] += carry[a];
        }
      } else {
        st = kReserveFull;
        atomicOr(ctl, E_CAPACITY);
        if (reserve == kReserveSticky) atomicOr(S.err, E_CAPACITY);
      }
    }
    status = st;
  }
  if (!out) return;
  if (t < kArenas) {
    out[t] = carry[t];
    out[kArenas + 1 + t] = top0;
  } else if (t == kArenas) {
    out[kArenas] = ctl0;
  }
  if (t <= kArenas) __threadfence_system();
  __syncthreads();
  // The status word goes last: a host that sees it nonzero sees the plan.
  if (t == 0) out[kPlanStatusSlot] = reserve != kReserveNone ? status : kReserveOk;
}

// Arena bases of a batch reserved by the host (plain inserts, after the plan
// was read back and the arenas grown): the apply kernel uses them and moves
// the device tops to `top`.
struct HostReserve {
  unsigned long long base[kArenas], top[kArenas];
};



__global__ void __launch_bounds__(kBlock, 4) k_apply_insert(StoreView S, const uint32_t* skey, const uint32_t* sv,
                                                         const uint32_t* sw, const uint32_t* sorig,
                                                         const uint32_t* seg, const uint32_t* nseg,
                                                         unsigned long long k, uint32_t ks, const uint32_t* ctl,
                                                         const ArenaNeed* excl, const unsigned long long* boff,
                                                         const unsigned long long* base, HostReserve hr,
                                                         uint32_t* out_slots) {
  pdl_wait();
  pdl_trigger();
  __shared__ AliasScratch asc[kBlock / 32];
  if (*ctl) return;
  if (!base && blockIdx.x == 0) {
#pragma unroll
    for (int a = 0; a < kArenas; ++a)
      if (threadIdx.x == a) S.top[a] = hr.top[a];  // constant indices keep hr in parameter space
  }
  const uint32_t warps = gridDim.x * blockDim.x / 32;
  const uint32_t nS = *nseg, nb = plan_blocks(ks);
  for (uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) / 32; s < nS; s += warps) {
    uint32_t b, e;
    seg_bounds(seg, nS, s, k, &b, &e);
    const uint32_t u = skey[b];
    if (u >= S.n) continue;
    const ArenaNeed off = excl[s];
    unsigned long long res[kArenas];
#pragma unroll
    for (int a = 0; a < kArenas; ++a)
      res[a] = (base ? base[a] : hr.base[a]) + boff[(size_t)a * nb + s / kPlanSegs] + off.v[a];
    apply_append(S, u, sv + b, sw + b, sorig + b, e - b, out_slots, res, &asc[threadIdx.x / 32]);
  }
}

__global__ void __launch_bounds__(kBlock, 3) k_apply_delete(StoreView S, const uint32_t* skey, const uint32_t* sslot,
                                                         const uint32_t* seg, const uint32_t* nseg,
                                                         unsigned long long k, const uint32_t* ctl) {
  pdl_wait();
  pdl_trigger();
  __shared__ AliasScratch asc[kBlock / 32];
  __shared__ uint32_t stage[kBlock / 32][64];
  if (*ctl) return;
  const uint32_t warps = gridDim.x * blockDim.x / 32;
  const uint32_t nS = *nseg;
  for (uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) / 32; s < nS; s += warps) {
    uint32_t b, e;
    seg_bounds(seg, nS, s, k, &b, &e);
    const uint32_t u = skey[b];
    if (u >= S.n) continue;
    apply_delete(S, u, sslot + b, e - b, stage[threadIdx.x / 32], &asc[threadIdx.x / 32]);
  }
}

// Float weights -> 16.16 fixed point, round half to even (the scaling by
// 2^16 is exact in float). bad |= 1 for w <= 0, NaN or a weight that rounds
// to 0; bad |= 2 for w >= 65536 (inf included).
__global__ void k_fixed16(const float* w, unsigned long long k, uint32_t* out, uint32_t* bad) {
  uint32_t bits = 0;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < k;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const float x = w[i];
    uint32_t q = 0;
    if (!(x > 0.0f))
      bits |= 1u;
    else if (!(x < 65536.0f))
      bits |= 2u;
    else if (!(q = __float2uint_rn(x * 65536.0f)))
      bits |= 1u;
    out[i] = q;
  }
  bits = __reduce_or_sync(kFull, bits);
  if (bits && (threadIdx.x & 31) == 0) atomicOr(bad, bits);
}

// Delete by pair, step 1: 64-bit sort keys (u << 32) | v.
__global__ void k_pair_keys(const uint32_t* u, const uint32_t* v, unsigned long long k, unsigned long long* key) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < k;
       i += (unsigned long long)gridDim.x * blockDim.x)
    key[i] = ((unsigned long long)u[i] << 32) | v[i];
}

// Step 2: run heads of equal pairs in the sorted keys.
__global__ void k_pair_heads(const unsigned long long* key, unsigned long long k, uint8_t* head) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < k;
       i += (unsigned long long)gridDim.x * blockDim.x)
    head[i] = i == 0 || key[i] != key[i - 1];
}

// Step 3: one warp per run of equal pairs (u, v), in batch order (the sort is
// stable): its r-th member takes the r-th lowest live slot of u whose
// neighbour is v, or ~0 (an absent slot, skipped and counted by the delete)
// when u has fewer such slots. Slots are scanned 32 at a time with one
// 16-byte load per lane.
__global__ void __launch_bounds__(kBlock) k_pair_slots(StoreView S, const unsigned long long* key,
                                                       const uint32_t* perm, const uint32_t* seg,
                                                       const uint32_t* nseg, unsigned long long k,
                                                       const uint32_t* ctl, uint32_t* slot_out) {
  if (*ctl) return;
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * blockDim.x / 32;
  const uint32_t nS = *nseg;
  for (uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) / 32; s < nS; s += warps) {
    uint32_t b, e;
    seg_bounds(seg, nS, s, k, &b, &e);
    const uint32_t u = (uint32_t)(key[b] >> 32), v = (uint32_t)key[b];
    const uint32_t want = e - b;
    const VertexMeta M = S.meta[u];
    uint32_t got = 0;
    for (uint32_t c = 0; c < M.ecnt && got < want; c += 32) {
      const uint32_t i = c + lane;
      EdgeRec r{0, 0, 0, 0};
      if (i < M.ecnt) r = S.edges[M.eoff + i];
      const uint32_t hit = __ballot_sync(kFull, i < M.ecnt && r.v == v && r.w != 0);
      const uint32_t rank = got + __popc(hit & lanemask_lt());
      if (((hit >> lane) & 1) && rank < want) slot_out[perm[b + rank]] = i;
      got += __popc(hit);
    }
    for (uint32_t r = got + lane; r < want; r += 32) slot_out[perm[b + r]] = 0xffffffffu;
  }
}

// Persistent walk kernel with per-lane refill. Each warp owns a range of
// walk items and hands them to idle lanes; when the range runs out it pulls
// the next `chunk` items from one device counter (reset by the host before
// launch). MULTI = false: every item is a walk of the single job J0.
// MULTI = true: items index the concatenated jobs of a device job table
// (prefix = running walk counts) and each lane follows its own job; APP >= 0
// when every job of the table has that app, APP < 0 for a mixed table.
// `chunk` (walks per warp refill) is a tuning knob (Tuning::walk_chunk).
static_assert(kBlock % 32 == 0, "whole warps");

// Resident 256-thread blocks per SM each walk variant is compiled for
// (register budget 65536 / (256 * blocks)): DeepWalk and sampling 32
// registers; PPR 40 (48 with a job table); node2vec 48 (64 with a job
// table); the mixed-app kernel 64.
constexpr int walk_min_blocks(int app, bool multi) {
  return app == APP_DEEPWALK || app == APP_SAMPLING ? 8
         : app == APP_PPR                           ? (multi ? 5 : 6)
         : app == APP_NODE2VEC                      ? (multi ? 4 : 5)
                                                    : 4;
}

template <int APP, bool MULTI>
__global__ void __launch_bounds__(kBlock, walk_min_blocks(APP, MULTI))
    k_walk(WalkView W, WalkJobDev J0, const WalkJobDev* __restrict__ jobs, const uint32_t* __restrict__ prefix,
           uint32_t n_jobs, uint32_t total, uint32_t* queue, uint32_t chunk) {
  __shared__ __align__(16) int32_t obuf[kBlock][8];
  const int lane = threadIdx.x & 31;
  LaneWalk s;
  RowStage o{kNoSec, 0};
  uint32_t jid = 0, moves = 0, wb = 0, we = 0;
  s.trials = 0, s.probes = 0;
  bool active = false, drained = false;
  for (;;) {
    uint32_t idle = __ballot_sync(kFull, !active);
    while (idle && !drained) {
      if (wb >= we) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(queue, chunk);
        base = __shfl_sync(kFull, base, 0);
        if (base >= total) {
          drained = true;
          break;
        }
        wb = base;
        we = base + min(chunk, total - base);
      }
      const uint32_t take = min((uint32_t)__popc(idle), we - wb);
      const uint32_t rank = __popc(idle & lanemask_lt());
      if (!active && rank < take) {
        const uint32_t item = wb + rank;
        if (!MULTI) {
          active = walk_begin<APP>(W, J0, item, s, o, obuf, moves);
        } else {
          uint32_t lo = 0, hi = n_jobs;
          while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (prefix[mid] <= item)
              lo = mid;
            else
              hi = mid;
          }
          jid = lo;
          if (APP >= 0)
            active = walk_begin<APP>(W, jobs[lo], item - prefix[lo], s, o, obuf, moves);
          else
            active = begin_any(W, jobs[lo], item - prefix[lo], s, o, obuf, moves);
        }
      }
      wb += take;
      idle = __ballot_sync(kFull, !active);
    }
    if (!__any_sync(kFull, active)) break;
    if (active) {
      constexpr int A = APP == APP_SAMPLING ? APP_DEEPWALK : APP;
      if (!MULTI)
        active = walk_advance<A>(W, J0, s, o, obuf, moves);
      else if (APP >= 0)
        active = walk_advance<A>(W, jobs[jid], s, o, obuf, moves);
      else
        active = advance_any(W, jobs[jid], s, o, obuf, moves);
    }
  }
  add_steps(W, moves);
  add_n2v(W, s);
}

__global__ void k_philox(const uint32_t* ctr, unsigned long long count, uint32_t k0, uint32_t k1, uint32_t* out) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < count;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const Rand4 r = philox(ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3], k0, k1);
    out[4 * i] = r.x;
    out[4 * i + 1] = r.y;
    out[4 * i + 2] = r.z;
    out[4 * i + 3] = r.w;
  }
}

// Resident 256-thread blocks per SM of walk kernel k_walk<APP, MULTI>
// (register-limited): the persistent grid is exactly one full wave.
template <int APP, bool MULTI>
unsigned walk_blocks_per_sm() {
  static int b = 0;
  if (!b) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_walk<APP, MULTI>, kBlock, 0) != cudaSuccess || b <= 0) {
      cudaGetLastError();
      b = 4;
    }
  }
  return (unsigned)b;
}

// Default launch shape of each walk kernel (the knobs' value 0), measured on
// B200 with fixed graphs, launches interleaved: resident 256-thread blocks
// per SM (0 = the occupancy limit) and walks a warp claims per refill.
// DeepWalk (R-MAT scale 20, 16 M edges, log-uniform weights): 26.3 G
// steps/s at 4 blocks and 8 walks against 21.7 G at its 8-block occupancy
// limit and 32 (more resident warps issue more concurrent random reads than
// DRAM turns into throughput; 2 blocks: 23.0 G). PPR: 11.3 G at 4 blocks and
// 32 against 11.0 G at 6. node2vec (R-MAT scale 22, Zipf weights) and the
// mixed-app table (R-MAT scale 22, 16 mixed jobs) run best at their
// occupancy limits (5 and 4 blocks) with 32. One-hop sampling (one step per
// item) keeps the occupancy limit and 32.
constexpr unsigned walk_default_bps(int app) { return app == APP_DEEPWALK || app == APP_PPR ? 4 : 0; }
constexpr uint32_t walk_default_chunk(int app) { return app == APP_DEEPWALK ? 8 : 32; }

// Blocks per SM for a walk launch of `app` (-1: mixed table): the tuned or
// default figure, capped by occupancy.
unsigned walk_bps(unsigned occ, const Tuning& t, int app) {
  const unsigned want = t.walk_blocks_per_sm ? t.walk_blocks_per_sm : walk_default_bps(app);
  return want ? std::max(1u, std::min(occ, want)) : occ;
}
uint32_t walk_chunk_of(const Tuning& t, int app) { return t.walk_chunk ? t.walk_chunk : walk_default_chunk(app); }

// Launches the persistent walk kernel for a device job table whose jobs all
// have app `app` (or any app when app < 0).
void launch_walk_table(cudaStream_t st, int app, const WalkView& W, const WalkJobDev& J0, const WalkJobDev* jobs,
                       const uint32_t* prefix, uint32_t n_jobs, uint32_t total, uint32_t* queue, const Tuning& t) {
  const uint32_t c = walk_chunk_of(t, app);
  switch (app) {
    case APP_DEEPWALK:
      k_walk<APP_DEEPWALK, true>
          <<<grid_for(total, kBlock, walk_bps(walk_blocks_per_sm<APP_DEEPWALK, true>(), t, APP_DEEPWALK)), kBlock, 0, st>>>(
              W, J0, jobs, prefix, n_jobs, total, queue, c);
      break;
    case APP_NODE2VEC:
      k_walk<APP_NODE2VEC, true>
          <<<grid_for(total, kBlock, walk_bps(walk_blocks_per_sm<APP_NODE2VEC, true>(), t, APP_NODE2VEC)), kBlock, 0, st>>>(
              W, J0, jobs, prefix, n_jobs, total, queue, c);
      break;
    case APP_PPR:
      k_walk<APP_PPR, true><<<grid_for(total, kBlock, walk_bps(walk_blocks_per_sm<APP_PPR, true>(), t, APP_PPR)), kBlock, 0, st>>>(
          W, J0, jobs, prefix, n_jobs, total, queue, c);
      break;
    case APP_SAMPLING:
      k_walk<APP_SAMPLING, true>
          <<<grid_for(total, kBlock, walk_bps(walk_blocks_per_sm<APP_SAMPLING, true>(), t, APP_SAMPLING)), kBlock, 0, st>>>(
              W, J0, jobs, prefix, n_jobs, total, queue, c);
      break;
    default:
      k_walk<-1, true><<<grid_for(total, kBlock, walk_bps(walk_blocks_per_sm<-1, true>(), t, -1)), kBlock, 0, st>>>(
          W, J0, jobs, prefix, n_jobs, total, queue, c);
      break;
  }
  cuda_check(cudaGetLastError(), "walk launch");
}

// A job table for one persistent launch: jobs of one app (or all apps).
struct WalkGroup {
  int app;            // app of every job, or -1 for a mixed table
  size_t job_off;     // first job in the concatenated table
  size_t pf_off;      // first prefix entry (n_jobs + 1 entries)
  uint32_t n_jobs;
  uint32_t total;     // walks
};

double walk_cost(const WalkJobDev& J);

// Appends the jobs `in` to (table, prefix) as one group per app present
// (or one mixed group), each ordered by expected walk cost, most expensive
// first, so the longest walks start earliest (longest_first = false keeps
// the given order). Outputs are per job, so the order does not change any
// result.
void build_walk_groups(const WalkJobDev* in, uint32_t n, bool split, bool longest_first,
                       std::vector<WalkJobDev>& table, std::vector<uint32_t>& prefix, std::vector<WalkGroup>& groups) {
  std::vector<uint32_t> idx;
  for (int app = split ? 0 : -1; app <= (split ? 3 : -1); ++app) {
    idx.clear();
    for (uint32_t j = 0; j < n; ++j)
      if ((app < 0 || in[j].app == app) && in[j].n) idx.push_back(j);
    if (idx.empty()) continue;
    if (longest_first)
      std::stable_sort(idx.begin(), idx.end(),
                       [&](uint32_t a, uint32_t b) { return walk_cost(in[a]) > walk_cost(in[b]); });
    WalkGroup g{app, table.size(), prefix.size(), (uint32_t)idx.size(), 0};
    uint64_t t = 0;
    prefix.push_back(0);
    for (uint32_t j : idx) {
      table.push_back(in[j]);
      t += in[j].n;
      prefix.push_back((uint32_t)t);
    }
    g.total = (uint32_t)t;
    groups.push_back(g);
  }
}

// Expected relative cost of one walk of a job, used to hand out the most
// expensive walks first (shorter tails in persistent launches).
double walk_cost(const WalkJobDev& J) {
  if (J.app == APP_SAMPLING) return 1.0;
  double L = J.L;
  if (J.app == APP_PPR) {
    const double stop = (double)J.thr_stop / 4294967296.0;
    const double geo = stop > 0 ? 1.0 / stop : 1e9;
    L = (J.flags & kWalkPprTail) ? geo : std::min(L, geo);
  }
  if (J.app == APP_NODE2VEC) L *= 3.0;
  return L;
}

uint64_t prob_threshold(double p);

// node2vec weights 1/p (return), 1 (neighbour of the previous vertex), 1/q
// (other); acceptance against the envelope max(1, 1/q); a larger 1/p is
// handled by the return region (ret_excess). PPR stop threshold.
void set_thresholds(WalkJobDev& D, const bingo_walk_job& J) {
  const bool n2v = J.app == BINGO_NODE2VEC;
  const double wr = n2v ? 1.0 / J.p : 1.0, wo = n2v ? 1.0 / J.q : 1.0;
  const double am = std::max(1.0, wo), rr = wr / am;
  D.thr_ret = prob_threshold(rr);
  D.ret_excess = rr > 1.0 ? rr - 1.0 : 0.0;
  D.thr_in = prob_threshold(1.0 / am);
  D.thr_out = prob_threshold(wo / am);
  D.thr_stop = prob_threshold(J.app == BINGO_PPR ? J.stop_prob : 0.0);
}

uint64_t prob_threshold(double p) {
  if (!(p > 0.0)) return 0;
  if (p >= 1.0) return 1ull << 32;
  const double t = std::floor(std::ldexp(p, 32));
  return t >= 4294967296.0 ? (1ull << 32) : (uint64_t)t;
}

int status_of(uint32_t bits) {
  if (bits & E_RANGE) return BINGO_ERR_OUT_OF_RANGE;
  if (bits & E_ZERO_WEIGHT) return BINGO_ERR_ZERO_WEIGHT;
  if (bits & E_CAPACITY) return BINGO_ERR_CAPACITY;
  if (bits & E_INVALID_SLOT) return BINGO_ERR_INVALID_SLOT;
  if (bits & E_TIMEOUT) return BINGO_ERR_TIMEOUT;
  return BINGO_OK;
}

}  // namespace

// ------------------------------------------------------------------ basics
void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(e == cudaErrorMemoryAllocation ? BINGO_ERR_CAPACITY : BINGO_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
  }
}

void DevBuf::ensure(size_t want, const char* what) {
  if (want <= bytes && p) return;
  release();
  const size_t b = std::max(want, (size_t)256);
  cuda_check(cudaMalloc(&p, b), what);
  bytes = b;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

Engine::Engine(const bingo_config& cfg) : cfg_(cfg) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
    cudaGetLastError();
    throw Error(BINGO_ERR_NO_DEVICE, "no CUDA device is available");
  }
  if (cfg.device < 0 || cfg.device >= count) throw Error(BINGO_ERR_INVALID_ARGUMENT, "device ordinal out of range");
  if (!(cfg.arena_factor >= 1.0)) throw Error(BINGO_ERR_INVALID_ARGUMENT, "arena_factor must be >= 1");
  cuda_check(cudaSetDevice(cfg.device), "cudaSetDevice");
  cuda_check(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  stream_ = own_stream_;
  cuda_check(cudaStreamCreateWithFlags(&xstream_, cudaStreamNonBlocking), "cudaStreamCreate");
  for (int k = 0; k < 2; ++k) {
    cuda_check(cudaEventCreateWithFlags(&walk_ev_[k], cudaEventDisableTiming), "cudaEventCreate");
    cuda_check(cudaEventCreateWithFlags(&copy_ev_[k], cudaEventDisableTiming), "cudaEventCreate");
  }
  cuda_check(cudaMalloc(&d_err_, 4 * sizeof(uint32_t)), "cudaMalloc(err)");
  cuda_check(cudaMemset(d_err_, 0, 4 * sizeof(uint32_t)), "memset(err)");
  cuda_check(cudaMalloc(&d_top_, kArenas * sizeof(unsigned long long)), "cudaMalloc(top)");
  cuda_check(cudaMalloc(&d_steps_, 3 * sizeof(unsigned long long)), "cudaMalloc(steps)");
  cuda_check(cudaMemset(d_steps_, 0, 3 * sizeof(unsigned long long)), "memset(steps)");
  cuda_check(cudaMemset(d_top_, 0, kArenas * sizeof(unsigned long long)), "memset(top)");
  cuda_check(cudaMallocHost(&h_err_, 4 * sizeof(uint32_t)), "cudaMallocHost(err)");
  cuda_check(cudaMallocHost(&h_top_, kArenas * sizeof(unsigned long long)), "cudaMallocHost(top)");
  std::memset(h_top_, 0, kArenas * sizeof(unsigned long long));
  cuda_check(cudaHostAlloc((void**)&h_plan_, 16 * sizeof(unsigned long long), cudaHostAllocMapped),
             "cudaHostAlloc(plan)");
  cuda_check(cudaHostGetDevicePointer((void**)&d_plan_, (void*)h_plan_, 0), "plan mapping");
  cuda_check(cudaEventCreateWithFlags(&slots_ev_, cudaEventDisableTiming), "cudaEventCreate");
}

Engine::~Engine() {
  cudaSetDevice(cfg_.device);
  server_.reset();
  if (stream_) cudaStreamSynchronize(stream_);
  if (xstream_) cudaStreamSynchronize(xstream_);
  drop_graph();
  prog_jobs_.release(), prog_prefix_.release(), prog_queue_.release();
  DevBuf* bufs[] = {&vrec_, &meta_, &gdesc_, &gs_, &in_a_, &in_b_, &in_c_, &key_s_, &perm_, &iota_, &sa_,
                    &sb_, &head_, &seg_, &nseg_, &need_, &scan_, &base_, &ctl_, &slots_, &cub_tmp_, &jobs_,
                    &prefix_, &queue_, &wstart_, &wout_[0], &wout_[1], &pair_key_, &pair_key_s_, &pair_slot_,
                    &fw_in_, &fw_fixed_, &check_buf_, &check_big_};
  for (DevBuf* b : bufs) b->release();
  for (int k = 0; k < 2; ++k) {
    if (walk_ev_[k]) cudaEventDestroy(walk_ev_[k]);
    if (copy_ev_[k]) cudaEventDestroy(copy_ev_[k]);
  }
  if (xstream_) cudaStreamDestroy(xstream_);
  if (slots_ev_) cudaEventDestroy(slots_ev_);
  if (h_plan_) cudaFreeHost((void*)h_plan_);
  for (auto& a : arena_) a.release();
  if (d_err_) cudaFree(d_err_);
  if (d_top_) cudaFree(d_top_);
  if (d_steps_) cudaFree(d_steps_);
  if (h_err_) cudaFreeHost(h_err_);
  if (h_top_) cudaFreeHost(h_top_);
  if (own_stream_) cudaStreamDestroy(own_stream_);
}

StoreView Engine::view() const {
  StoreView S;
  S.n = n_;
  S.vrec = vrec_.as<VertexRec>();
  S.meta = meta_.as<VertexMeta>();
  S.gdesc = gdesc_.as<GroupDesc>();
  S.gv = arena_[A_MEMBER].as<uint32_t>();
  S.gs = gs_.as<uint32_t>();
  S.edges = arena_[A_EDGE].as<EdgeRec>();
  S.bp = arena_[A_BP].as<uint32_t>();
  S.alias = arena_[A_ALIAS].as<AliasRec>();
  S.hash = arena_[A_HASH].as<HashEntry>();
  S.top = d_top_;
  for (int a = 0; a < kArenas; ++a) S.cap[a] = cap_[a];
  S.err = d_err_;
  S.node2vec = cfg_.node2vec;
  return S;
}

WalkView Engine::wview() const {
  WalkView W;
  W.n = n_;
  W.vrec = vrec_.as<VertexRec>();
  W.alias = arena_[A_ALIAS].as<AliasRec>();
  W.gv = arena_[A_MEMBER].as<uint32_t>();
  W.hash = arena_[A_HASH].as<HashEntry>();
  W.err = d_err_;
  W.steps = d_steps_;
  W.n2v = d_steps_ + 1;
  return W;
}

void Engine::require_loaded() const {
  if (!loaded_) throw Error(BINGO_ERR_NOT_LOADED, "no graph loaded");
}

void Engine::set_stream(void* s) { stream_ = s ? (cudaStream_t)s : own_stream_; }

int Engine::sync() {
  cuda_check(cudaStreamSynchronize(stream_), "stream synchronize");
  cuda_check(cudaStreamSynchronize(xstream_), "result copies");
  cuda_check(cudaMemcpy(h_err_, d_err_, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost), "read status");
  const uint32_t bits = h_err_[0], rejected = h_err_[1];
  if (!bits) return BINGO_OK;
  cuda_check(cudaMemset(d_err_, 0, 2 * sizeof(uint32_t)), "clear status");
  const int st = status_of(bits);
  last_error = "device reported error bits 0x" + std::to_string(bits);
  if (bits & E_INVALID_SLOT) last_error += " (" + std::to_string(rejected) + " deletes of absent slots skipped)";
  if (bits & E_RANGE) last_error += " (vertex id out of range)";
  if (bits & E_ZERO_WEIGHT) last_error += " (zero weight)";
  return st;
}

void Engine::finish_call() {
  if (!cfg_.synchronous || defer_sync_) return;
  const int st = sync();
  if (st) throw Error(st, last_error);
}

// ------------------------------------------------------------------ staging
void Engine::ensure_batch_scratch(uint64_t k) {
  const uint64_t kk = std::max<uint64_t>(k, 1);
  if (slots_busy_ && slots_.bytes < kk * 4) {  // slots_ is about to move: its copy-out must be over
    cuda_check(cudaEventSynchronize(slots_ev_), "slot copy");
    slots_busy_ = false;
  }
  const uint64_t ks = std::max<uint64_t>(std::min<uint64_t>(kk, n_ ? n_ : kk), 1);
  in_a_.ensure(kk * 4, "scratch");
  in_b_.ensure(kk * 4, "scratch");
  in_c_.ensure(kk * 4, "scratch");
  key_s_.ensure(kk * 4, "scratch");
  perm_.ensure(kk * 4, "scratch");
  sa_.ensure(kk * 4, "scratch");
  sb_.ensure(kk * 4, "scratch");
  head_.ensure(kk, "scratch");
  seg_.ensure(kk * 4, "scratch");
  slots_.ensure(kk * 4, "scratch");
  nseg_.ensure(16, "scratch");
  ctl_.ensure(16, "scratch");
  base_.ensure(kArenas * 8 * 2, "scratch");
  need_.ensure((size_t)plan_blocks((uint32_t)ks) * sizeof(ArenaNeed), "scratch");  // plan-block sums
  scan_.ensure((size_t)ks * sizeof(ArenaNeed), "scratch");                                   // in-block offsets
  if (iota_n_ < kk) {
    iota_.ensure(kk * 4, "scratch");
    k_iota<<<grid_for(kk, kBlock), kBlock, 0, stream_>>>(iota_.as<uint32_t>(), kk);
    cuda_check(cudaGetLastError(), "iota");
    ++launches_;
    iota_n_ = kk;
  }
  size_t t_sort = 0, t_sel = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, t_sort, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)kk, 0, 32, stream_);
  cub::DeviceSelect::Flagged(nullptr, t_sel, (const uint32_t*)nullptr, (const uint8_t*)nullptr, (uint32_t*)nullptr,
                             (uint32_t*)nullptr, (int)kk, stream_);
  cub_tmp_.ensure(std::max(t_sort, t_sel), "scratch");
  group_cluster_ok();  // probed here, outside any stream capture
}

const uint32_t* Engine::stage(const uint32_t* p, uint64_t k, DevBuf& buf, const char* what) {
  if (!p) return nullptr;
  if (is_device_ptr(p)) return p;
  cuda_check(cudaMemcpyAsync(buf.p, p, k * 4, cudaMemcpyHostToDevice, stream_), what);
  return buf.as<uint32_t>();
}

// Stable sort of the batch by vertex; leaves sorted keys in key_s_, the
// original index in perm_, payloads a/b in sorted order in sa_/sb_, and the
// segment start list in seg_ with its count in nseg_.
namespace {
void group_launch_config(cudaLaunchConfig_t& lc, cudaLaunchAttribute* at, int ctas, uint32_t ipt, cudaStream_t s) {
  lc = cudaLaunchConfig_t{};
  lc.gridDim = dim3(ctas);
  lc.blockDim = dim3(kGroupThreads);
  lc.dynamicSmemBytes = group_smem_bytes(ipt);
  lc.stream = s;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = ctas;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = 2;
}

// The grouping kernel for CTAS-CTA clusters can be resident on this device.
template <int CTAS, int IPT>
bool group_kernel_ready() {
  auto kern = k_group_small<CTAS, IPT>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)group_smem_bytes(IPT)) !=
      cudaSuccess)
    return false;
  if (CTAS > 8 && cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
    return false;
  cudaLaunchConfig_t lc;
  cudaLaunchAttribute at[2];
  group_launch_config(lc, at, CTAS, IPT, nullptr);
  int clusters = 0;
  return cudaOccupancyMaxActiveClusters(&clusters, kern, &lc) == cudaSuccess && clusters > 0;
}

template <int CTAS, int IPT>
cudaError_t launch_group(cudaStream_t s, const uint32_t* key, const uint32_t* a, const uint32_t* b, uint32_t k,
                         uint32_t n, int end_bit, bool insert, uint32_t* key_s, uint32_t* perm, uint32_t* sa,
                         uint32_t* sb, uint32_t* seg, uint32_t* nseg, uint32_t* ctl, uint32_t* err) {
  const uint32_t ipt = group_ipt(k, CTAS);
  cudaLaunchConfig_t lc;
  cudaLaunchAttribute at[2];
  group_launch_config(lc, at, CTAS, ipt, s);
  return cudaLaunchKernelEx(&lc, k_group_small<CTAS, IPT>, key, a, b, k, n, end_bit, ipt, insert ? 1 : 0, key_s,
                            perm, sa, sb, seg, nseg, ctl, err);
}
}  // namespace

// Bit 0: 8-CTA grouping clusters can run; bit 1: 16-CTA ones.
int Engine::group_cluster_ok() {
  if (group_cluster_ < 0) {
    group_cluster_ = (group_kernel_ready<8, kGroupIptSmall>() ? 1 : 0) |
                     (group_kernel_ready<16, kGroupIptLarge>() ? 2 : 0);
    cudaGetLastError();  // a refused query leaves the CUB path in place, not a sticky error
  }
  return group_cluster_;
}

void Engine::group_by_vertex(const uint32_t* key, const uint32_t* a, const uint32_t* b, uint64_t k, bool insert) {
  int end_bit = 1;
  while (end_bit < 32 && (1ull << end_bit) < n_) ++end_bit;
  const int gc = k >= 1 && k <= kGroupMax ? group_cluster_ok() : 0;
  const bool small = (gc & 1) && (k <= kGroupSmallMax || (!(gc & 2) && k <= 8ull * kGroupThreads * kGroupIptSmall));
  if (small || (gc & 2)) {
    auto* launch = small ? launch_group<8, kGroupIptSmall> : launch_group<16, kGroupIptLarge>;
    cuda_check(launch(stream_, key, a, b, (uint32_t)k, n_, end_bit, insert, key_s_.as<uint32_t>(),
                      perm_.as<uint32_t>(), sa_.as<uint32_t>(), sb_.as<uint32_t>(), seg_.as<uint32_t>(),
                      nseg_.as<uint32_t>(), ctl_.as<uint32_t>(), d_err_),
               "group batch");
    ++launches_;
    return;
  }
  cuda_check(cudaMemsetAsync(ctl_.p, 0, 16, stream_), "ctl");
  k_validate<<<grid_for(k, kBlock, 16), kBlock, 0, stream_>>>(key, insert ? a : nullptr, insert ? b : nullptr, k, n_,
                                                              ctl_.as<uint32_t>(), d_err_);
  cuda_check(cudaGetLastError(), "validate");
  ++launches_;
  size_t tb = cub_tmp_.bytes;
  cuda_check(cub::DeviceRadixSort::SortPairs(cub_tmp_.p, tb, key, key_s_.as<uint32_t>(), iota_.as<uint32_t>(),
                                             perm_.as<uint32_t>(), (int)k, 0, end_bit, stream_),
             "radix sort");
  k_gather<<<grid_for(k, kBlock, 16), kBlock, 0, stream_>>>(key_s_.as<uint32_t>(), perm_.as<uint32_t>(), a, b,
                                                             sa_.as<uint32_t>(), sb_.as<uint32_t>(),
                                                             head_.as<uint8_t>(), k);
  cuda_check(cudaGetLastError(), "gather");
  ++launches_;
  tb = cub_tmp_.bytes;
  cuda_check(cub::DeviceSelect::Flagged(cub_tmp_.p, tb, iota_.as<uint32_t>(), head_.as<uint8_t>(),
                                        seg_.as<uint32_t>(), nseg_.as<uint32_t>(), (int)k, stream_),
             "segment select");
}

void Engine::read_tops() {
  cuda_check(cudaMemcpyAsync(h_top_, d_top_, kArenas * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_),
             "read tops");
  cuda_check(cudaStreamSynchronize(stream_), "read tops");
}

void Engine::grow_arena(int a, unsigned long long min_cap) {
  unsigned long long nc = std::max<unsigned long long>(min_cap, cap_[a] + cap_[a] / 2);
  nc = std::min(nc, kArenaLimit[a]);
  if (nc < min_cap)
    throw Error(BINGO_ERR_CAPACITY, std::string(kArenaName[a]) + " arena would exceed its 32-bit index range");
  const unsigned long long used = h_top_[a];
  DevBuf fresh;
  fresh.ensure(nc * kUnitBytes[a], "grow arena");
  if (used) cuda_check(cudaMemcpyAsync(fresh.p, arena_[a].p, used * kUnitBytes[a], cudaMemcpyDeviceToDevice, stream_),
                       "grow arena copy");
  if (a == A_MEMBER) {
    DevBuf fgs;
    fgs.ensure(nc * 4, "grow arena");
    if (used) cuda_check(cudaMemcpyAsync(fgs.p, gs_.p, used * 4, cudaMemcpyDeviceToDevice, stream_), "grow copy");
    cuda_check(cudaStreamSynchronize(stream_), "grow arena");
    gs_.release();
    gs_ = fgs;
    fgs.p = nullptr;
  }
  cuda_check(cudaStreamSynchronize(stream_), "grow arena");
  arena_[a].release();
  arena_[a] = fresh;
  fresh.p = nullptr;
  cap_[a] = nc;
  ++arena_gen_;
}

void Engine::alloc_arenas(const unsigned long long need[kArenas]) {
  for (int a = 0; a < kArenas; ++a) {
    if (a == A_HASH && !cfg_.node2vec) {
      cap_[a] = 0;
      arena_[a].ensure(256, "arena");
      continue;
    }
    unsigned long long c = (unsigned long long)std::ceil((double)need[a] * cfg_.arena_factor);
    c = std::max(c, need[a] + kArenaFloor[a]);
    c = std::min(c, kArenaLimit[a]);
    if (c < need[a]) throw Error(BINGO_ERR_CAPACITY, std::string(kArenaName[a]) + " arena exceeds its index range");
    arena_[a].release();
    arena_[a].ensure(c * kUnitBytes[a], "allocate arena");
    if (a == A_MEMBER) {
      gs_.release();
      gs_.ensure(c * 4, "allocate arena");
    }
    cap_[a] = c;
  }
  if (cfg_.arena_bytes) {
    // Spread an explicit minimum over the arenas in proportion to their need.
    unsigned long long total = 0;
    for (int a = 0; a < kArenas; ++a) total += cap_[a] * kUnitBytes[a] + (a == A_MEMBER ? cap_[a] * 4 : 0);
    if (total < cfg_.arena_bytes) {
      const double scale = (double)cfg_.arena_bytes / (double)std::max<unsigned long long>(total, 1);
      for (int a = 0; a < kArenas; ++a)
        if (cap_[a]) grow_arena(a, (unsigned long long)std::ceil(cap_[a] * scale));
    }
  }
  cuda_check(cudaMemsetAsync(d_top_, 0, kArenas * sizeof(unsigned long long), stream_), "reset tops");
  std::memset(h_top_, 0, kArenas * sizeof(unsigned long long));
  ++arena_gen_;
}

// Per-segment arena offsets of the grouped insert batch relative to the
// batch's base (excl in scan_, block prefixes in need_) and the batch totals,
// which it returns (device memory); publish != null also writes the insert
// plan there.
unsigned long long* Engine::plan_needs(const StoreView& S, uint64_t k, uint32_t ks,
                                       volatile unsigned long long* publish, int reserve) {
  const uint32_t nb = plan_blocks(ks);
  launch_pdl(k_plan, nb, kPlanThreads, stream_, S, key_s_.as<uint32_t>(), sb_.as<uint32_t>(), seg_.as<uint32_t>(),
             nseg_.as<uint32_t>(), k, ks, ctl_.as<uint32_t>(), scan_.as<ArenaNeed>(), need_.as<unsigned long long>());
  cuda_check(cudaGetLastError(), "plan");
  ++launches_;
  unsigned long long* d_tot = base_.as<unsigned long long>() + kArenas;
  launch_pdl(k_totals, 1, kTotalsThreads, stream_, S, need_.as<unsigned long long>(), nb, d_tot, ctl_.as<uint32_t>(),
             base_.as<unsigned long long>(), reserve, publish);
  cuda_check(cudaGetLastError(), "totals");
  ++launches_;
  return d_tot;
}

// Waits until k_totals has published the insert plan (its status word turns
// nonzero), with the apply kernel already enqueued behind it so the stream
// is never drained here. Bounded: after kPlanWaitSeconds the stream is
// synchronised instead (which also surfaces a device fault).
void Engine::wait_plan() {
  constexpr double kPlanWaitSeconds = 5.0;
  const auto t0 = std::chrono::steady_clock::now();
  uint32_t spins = 0;
  while (h_plan_[kPlanStatusSlot] == 0) {
    if (++spins < 4096) continue;  // the plan is usually a few tens of microseconds away
    std::this_thread::yield();     // a long wait (work queued before the insert) leaves the core to others
    if ((spins & 255u) == 0 &&
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > kPlanWaitSeconds) {
      cuda_check(cudaStreamSynchronize(stream_), "plan sync");
      break;
    }
  }
  std::atomic_thread_fence(std::memory_order_acquire);
}

// Plan, size, reserve and apply an append batch whose grouped columns are in
// key_s_/sa_ (dst)/sb_ (w)/perm_ (original index) and segments in seg_/nseg_.
// A load sizes the arenas from the plan it reads back. An insert reserves on
// the device and launches the apply kernel at once; the host then waits only
// for the reservation (the apply kernel runs meanwhile) and, when an arena
// was full (the apply kernel skipped the batch), grows it and applies the
// batch again before returning, so later work always sees the batch applied.
void Engine::run_insert(uint64_t k, uint32_t* dev_out_slots, bool load_mode, uint64_t) {
  const uint32_t ks = (uint32_t)std::max<uint64_t>(std::min<uint64_t>(k, n_), 1);
  const StoreView S0 = view();
  h_plan_[kPlanStatusSlot] = 0;  // k_totals publishes the plan and then a nonzero status here
  plan_needs(S0, k, ks, d_plan_, load_mode ? kReserveNone : kReservePublish);
  auto apply = [&](const StoreView& S, const unsigned long long* dev_base, const HostReserve& hr) {
    launch_pdl(k_apply_insert, grid_for((unsigned long long)ks * 32, kBlock, tuning_.apply_blocks_per_sm), kBlock,
               stream_, S, key_s_.as<uint32_t>(), sa_.as<uint32_t>(), sb_.as<uint32_t>(), perm_.as<uint32_t>(),
               seg_.as<uint32_t>(), nseg_.as<uint32_t>(), k, ks, ctl_.as<uint32_t>(), scan_.as<ArenaNeed>(),
               need_.as<unsigned long long>(), dev_base, hr, dev_out_slots);
    cuda_check(cudaGetLastError(), "apply insert");
    ++launches_;
  };
  if (!load_mode) {
    apply(S0, base_.as<unsigned long long>(), HostReserve{});
    wait_plan();
  } else {
    cuda_check(cudaStreamSynchronize(stream_), "plan sync");
  }
  unsigned long long tot[kArenas];
  for (int a = 0; a < kArenas; ++a) tot[a] = h_plan_[a];
  const uint32_t ctl = (uint32_t)h_plan_[kArenas];
  if (!load_mode)
    for (int a = 0; a < kArenas; ++a) h_top_[a] = h_plan_[kArenas + 1 + a];
  if (ctl) {
    cuda_check(cudaStreamSynchronize(stream_), "rejected batch");
    cuda_check(cudaMemset(d_err_, 0, 2 * sizeof(uint32_t)), "clear status");
    const int st = status_of(ctl);
    throw Error(st, st == BINGO_ERR_ZERO_WEIGHT ? "batch holds a zero weight" : "batch holds a vertex id >= n");
  }
  if (load_mode) {
    alloc_arenas(tot);
    HostReserve hr;
    for (int a = 0; a < kArenas; ++a) hr.base[a] = h_top_[a], hr.top[a] = h_top_[a] + tot[a];
    apply(view(), nullptr, hr);
  } else if (h_plan_[kPlanStatusSlot] != kReserveOk) {
    // An arena was full: nothing was applied. Grow, clear the status word and
    // apply with bases from the host.
    for (int a = 0; a < kArenas; ++a)
      if (h_top_[a] + tot[a] > cap_[a]) grow_arena(a, h_top_[a] + tot[a]);
    cuda_check(cudaMemsetAsync(ctl_.p, 0, 4, stream_), "ctl");
    HostReserve hr;
    for (int a = 0; a < kArenas; ++a) hr.base[a] = h_top_[a], hr.top[a] = h_top_[a] + tot[a];
    apply(view(), nullptr, hr);
  }
  for (int a = 0; a < kArenas; ++a) h_top_[a] += tot[a];
}

// ------------------------------------------------------------------ API ops
namespace {
void host_check_ids(const uint32_t* a, uint64_t k, uint32_t n, const char* what) {
  for (uint64_t i = 0; i < k; ++i)
    if (a[i] >= n) throw Error(BINGO_ERR_OUT_OF_RANGE, std::string(what) + " id " + std::to_string(a[i]) + " >= n");
}
void host_check_weights(const uint32_t* w, uint64_t k) {
  for (uint64_t i = 0; i < k; ++i)
    if (w[i] == 0) throw Error(BINGO_ERR_ZERO_WEIGHT, "weight 0 at index " + std::to_string(i));
}
}  // namespace

void Engine::load(const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t m, uint32_t n) {
  const NvtxRange nvtx_("bingo load");
  if (n == 0) throw Error(BINGO_ERR_INVALID_ARGUMENT, "n must be > 0");
  if (m && (!src || !dst || !w)) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null edge array");
  if (m >= (1ull << 31)) throw Error(BINGO_ERR_UNSUPPORTED, "more than 2^31 edges in one load");
  if (m && !is_device_ptr(src)) host_check_ids(src, m, n, "source");
  if (m && !is_device_ptr(dst)) host_check_ids(dst, m, n, "destination");
  if (m && !is_device_ptr(w)) host_check_weights(w, m);
  cuda_check(cudaStreamSynchronize(stream_), "load");
  loaded_ = false;
  n_ = n;
  ++arena_gen_;
  vrec_.release(), meta_.release(), gdesc_.release();
  vrec_.ensure((size_t)n * sizeof(VertexRec), "vertex records");
  meta_.ensure((size_t)n * sizeof(VertexMeta), "vertex metadata");
  gdesc_.ensure((size_t)n * kBits * sizeof(GroupDesc), "group descriptors");
  cuda_check(cudaMemsetAsync(vrec_.p, 0, (size_t)n * sizeof(VertexRec), stream_), "memset");
  cuda_check(cudaMemsetAsync(meta_.p, 0, (size_t)n * sizeof(VertexMeta), stream_), "memset");
  cuda_check(cudaMemsetAsync(gdesc_.p, 0, (size_t)n * kBits * sizeof(GroupDesc), stream_), "memset");
  for (int a = 0; a < kArenas; ++a) arena_[a].release(), cap_[a] = 0;
  gs_.release();
  cuda_check(cudaMemsetAsync(d_top_, 0, kArenas * sizeof(unsigned long long), stream_), "reset tops");
  std::memset(h_top_, 0, kArenas * sizeof(unsigned long long));
  if (m == 0) {
    const unsigned long long zero[kArenas] = {0, 0, 0, 0, 0};
    alloc_arenas(zero);
    loaded_ = true;
    finish_call();
    return;
  }
  ensure_batch_scratch(m);
  const uint32_t* ds = stage(src, m, in_a_, "stage src");
  const uint32_t* dd = stage(dst, m, in_b_, "stage dst");
  const uint32_t* dw = stage(w, m, in_c_, "stage w");
  group_by_vertex(ds, dd, dw, m, true);
  run_insert(m, nullptr, true, m);
  loaded_ = true;
  // Release load-sized scratch; update batches re-grow what they need.
  DevBuf* big[] = {&in_a_, &in_b_, &in_c_, &key_s_, &perm_, &sa_, &sb_, &head_, &seg_, &slots_, &need_,
                   &scan_, &iota_, &cub_tmp_};
  cuda_check(cudaStreamSynchronize(stream_), "load");
  for (DevBuf* b : big) b->release();
  iota_n_ = 0;
  finish_call();
}

void Engine::insert(const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t k, uint32_t* out_slots) {
  const NvtxRange nvtx_("bingo insert");
  require_loaded();
  if (k == 0) return;
  if (!src || !dst || !w) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null edge array");
  if (k >= (1ull << 31)) throw Error(BINGO_ERR_UNSUPPORTED, "more than 2^31 edges in one batch");
  if (!is_device_ptr(src)) host_check_ids(src, k, n_, "source");
  if (!is_device_ptr(dst)) host_check_ids(dst, k, n_, "destination");
  if (!is_device_ptr(w)) host_check_weights(w, k);
  const uint64_t c = tuning_.update_chunk;
  if (c && k > c) {
    // Sub-batches in batch order append every source's edges in the same
    // order, so slots and state equal the whole batch's; the whole batch is
    // checked first, so a bad edge still rejects all of it.
    check_batch_on_device(src, dst, w, k);
    for (uint64_t o = 0; o < k; o += c)
      insert_one(src + o, dst + o, w + o, std::min(c, k - o), out_slots ? out_slots + o : nullptr);
  } else {
    insert_one(src, dst, w, k, out_slots);
  }
  finish_call();
}

// Float-weight mode (bingo_load_edges_f32 / bingo_insert_batch_f32): the
// weights become 16.16 fixed point on the device, then take the integer path.
const uint32_t* Engine::fixed_weights(const float* w, uint64_t k) {
  if (cfg_.weight_mode != BINGO_WEIGHTS_F32)
    throw Error(BINGO_ERR_INVALID_ARGUMENT, "float weights need a handle created with weight_mode = BINGO_WEIGHTS_F32");
  if (!w) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null weight array");
  const float* dw = w;
  if (!is_device_ptr(w)) {
    fw_in_.ensure(k * 4, "float weights");
    cuda_check(cudaMemcpyAsync(fw_in_.p, w, k * 4, cudaMemcpyHostToDevice, stream_), "stage float weights");
    dw = fw_in_.as<float>();
  }
  fw_fixed_.ensure(k * 4, "float weights");
  ctl_.ensure(16, "scratch");
  cuda_check(cudaMemsetAsync(ctl_.p, 0, 4, stream_), "ctl");
  k_fixed16<<<grid_for(k, kBlock, 16), kBlock, 0, stream_>>>(dw, k, fw_fixed_.as<uint32_t>(), ctl_.as<uint32_t>());
  cuda_check(cudaGetLastError(), "fixed-point weights");
  ++launches_;
  uint32_t bad = 0;
  cuda_check(cudaMemcpyAsync(&bad, ctl_.p, 4, cudaMemcpyDeviceToHost, stream_), "read ctl");
  cuda_check(cudaStreamSynchronize(stream_), "fixed-point weights");
  if (bad & 2u) throw Error(BINGO_ERR_OUT_OF_RANGE, "float weight >= 65536 (the fixed-point range)");
  if (bad & 1u) throw Error(BINGO_ERR_ZERO_WEIGHT, "float weight <= 0, NaN, or below 2^-17 (rounds to 0)");
  return fw_fixed_.as<uint32_t>();
}

void Engine::load_f32(const uint32_t* src, const uint32_t* dst, const float* w, uint64_t m, uint32_t n) {
  if (m >= (1ull << 31)) throw Error(BINGO_ERR_UNSUPPORTED, "more than 2^31 edges in one load");
  const uint32_t* q = m ? fixed_weights(w, m) : nullptr;
  load(src, dst, m ? q : nullptr, m, n);
  fw_in_.release(), fw_fixed_.release();
}

void Engine::insert_f32(const uint32_t* src, const uint32_t* dst, const float* w, uint64_t k, uint32_t* out_slots) {
  if (k == 0) return;
  if (k >= (1ull << 31)) throw Error(BINGO_ERR_UNSUPPORTED, "more than 2^31 edges in one batch");
  insert(src, dst, fixed_weights(w, k), k, out_slots);
}

// Rejects the batch (status, nothing applied) when a device-resident column
// holds an id >= n or a zero weight; host columns are checked on the host.
void Engine::check_batch_on_device(const uint32_t* a, const uint32_t* b, const uint32_t* w, uint64_t k) {
  const uint32_t* da = a && is_device_ptr(a) ? a : nullptr;
  const uint32_t* db = b && is_device_ptr(b) ? b : nullptr;
  const uint32_t* dw = w && is_device_ptr(w) ? w : nullptr;
  if (!da && !db && !dw) return;
  ctl_.ensure(16, "scratch");
  cuda_check(cudaMemsetAsync(ctl_.p, 0, 16, stream_), "ctl");
  k_validate<<<grid_for(k, kBlock, 16), kBlock, 0, stream_>>>(da, db, dw, k, n_, ctl_.as<uint32_t>(), d_err_);
  cuda_check(cudaGetLastError(), "validate");
  ++launches_;
  uint32_t ctl = 0;
  cuda_check(cudaMemcpyAsync(&ctl, ctl_.p, 4, cudaMemcpyDeviceToHost, stream_), "read ctl");
  cuda_check(cudaStreamSynchronize(stream_), "validate sync");
  if (ctl) {
    cuda_check(cudaMemset(d_err_, 0, 2 * sizeof(uint32_t)), "clear status");
    const int st = status_of(ctl);
    throw Error(st, st == BINGO_ERR_ZERO_WEIGHT ? "batch holds a zero weight" : "batch holds a vertex id >= n");
  }
}

void Engine::insert_one(const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint64_t k, uint32_t* out_slots) {
  if (slots_busy_) {  // the last host-bound slot copy reads slots_: finish it before slots_ changes
    if (slots_.bytes < std::max<uint64_t>(k, 1) * 4)
      cuda_check(cudaEventSynchronize(slots_ev_), "slot copy");
    else
      cuda_check(cudaStreamWaitEvent(stream_, slots_ev_, 0), "slot copy");
    slots_busy_ = false;
  }
  ensure_batch_scratch(k);
  const uint32_t* ds = stage(src, k, in_a_, "stage src");
  const uint32_t* dd = stage(dst, k, in_b_, "stage dst");
  const uint32_t* dw = stage(w, k, in_c_, "stage w");
  group_by_vertex(ds, dd, dw, k, true);
  const bool dev_out = out_slots && is_device_ptr(out_slots);
  uint32_t* dslots = out_slots ? (dev_out ? out_slots : slots_.as<uint32_t>()) : nullptr;
  run_insert(k, dslots, false, k);
  if (out_slots && !dev_out) {
    if (cfg_.synchronous) {
      cuda_check(cudaMemcpyAsync(out_slots, dslots, k * 4, cudaMemcpyDeviceToHost, stream_), "slots D2H");
    } else {
      // Copied out beside the walk results; bingo_sync waits for it.
      cuda_check(cudaEventRecord(slots_ev_, stream_), "slots ready");
      cuda_check(cudaStreamWaitEvent(xstream_, slots_ev_, 0), "slots ready");
      cuda_check(cudaMemcpyAsync(out_slots, dslots, k * 4, cudaMemcpyDeviceToHost, xstream_), "slots D2H");
      cuda_check(cudaEventRecord(slots_ev_, xstream_), "slots copied");
      slots_busy_ = true;
    }
  }
}

void Engine::erase(const uint32_t* u, const uint32_t* slot, uint64_t k) {
  const NvtxRange nvtx_("bingo delete");
  require_loaded();
  if (k == 0) return;
  if (!u || !slot) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null delete array");
  if (k >= (1ull << 31)) throw Error(BINGO_ERR_UNSUPPORTED, "more than 2^31 deletes in one batch");
  if (!is_device_ptr(u)) host_check_ids(u, k, n_, "vertex");
  const uint64_t c = tuning_.update_chunk;
  if (c && k > c) {
    // Sub-batches in batch order run the same swap-remove sequences; skipped
    // deletes add up in the status word until the one check at the end.
    check_batch_on_device(u, nullptr, nullptr, k);
    for (uint64_t o = 0; o < k; o += c) erase_one(u + o, slot + o, std::min(c, k - o));
  } else {
    erase_one(u, slot, k);
  }
  finish_call();
}

void Engine::erase_one(const uint32_t* u, const uint32_t* slot, uint64_t k) {
  ensure_batch_scratch(k);
  const uint32_t* du = stage(u, k, in_a_, "stage u");
  const uint32_t* dsl = stage(slot, k, in_b_, "stage slot");
  group_by_vertex(du, dsl, nullptr, k, false);
  const uint32_t ks = (uint32_t)std::max<uint64_t>(std::min<uint64_t>(k, n_), 1);
  launch_pdl(k_apply_delete, grid_for((unsigned long long)ks * 32, kBlock, tuning_.apply_blocks_per_sm), kBlock,
             stream_, view(), key_s_.as<uint32_t>(), sa_.as<uint32_t>(), seg_.as<uint32_t>(), nseg_.as<uint32_t>(), k,
             ctl_.as<uint32_t>());
  cuda_check(cudaGetLastError(), "apply delete");
  ++launches_;
}

// Delete by (u, v) pair. No reference counterpart (the reference deletes by
// (u, slot), include/operation.cuh:215): the r-th occurrence of a pair in
// the batch deletes the r-th lowest live slot of u whose neighbour is v;
// pairs without such a slot are skipped and reported like deletes of absent
// slots. The translated (u, slot) batch then takes the slot-delete path, so
// the swap-remove order is the batch order.
void Engine::erase_pairs(const uint32_t* u, const uint32_t* v, uint64_t k) {
  const NvtxRange nvtx_("bingo delete pairs");
  require_loaded();
  if (k == 0) return;
  if (!u || !v) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null delete array");
  if (k >= (1ull << 31)) throw Error(BINGO_ERR_UNSUPPORTED, "more than 2^31 deletes in one batch");
  if (!is_device_ptr(u)) host_check_ids(u, k, n_, "vertex");
  if (!is_device_ptr(v)) host_check_ids(v, k, n_, "vertex");
  ensure_batch_scratch(k);
  ensure_pair_scratch(k);
  const uint32_t* du = stage(u, k, in_a_, "stage u");
  const uint32_t* dv = stage(v, k, in_b_, "stage v");
  translate_pairs(du, dv, k);
  erase(du, pair_slot_.as<uint32_t>(), k);
}

// Scratch for translating k pairs (sized before a program is captured).
void Engine::ensure_pair_scratch(uint64_t k) {
  const uint64_t kk = std::max<uint64_t>(k, 1);
  pair_key_.ensure(kk * 8, "scratch");
  pair_key_s_.ensure(kk * 8, "scratch");
  pair_slot_.ensure(kk * 4, "scratch");
  size_t t_sort = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, t_sort, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                  (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)kk, 0, 64, stream_);
  cub_tmp_.ensure(t_sort, "scratch");
}

// Device arrays u, v -> pair_slot_ (stream-ordered, no host synchronisation):
// stable sort of (u << 32 | v), runs of equal pairs, one warp per run
// scanning u's slots. A batch that fails validation keeps every slot absent.
void Engine::translate_pairs(const uint32_t* du, const uint32_t* dv, uint64_t k) {
  int end_bit = 33;
  while (end_bit < 64 && (1ull << (end_bit - 32)) < n_) ++end_bit;
  cuda_check(cudaMemsetAsync(ctl_.p, 0, 16, stream_), "ctl");
  k_validate<<<grid_for(k, kBlock, 16), kBlock, 0, stream_>>>(du, dv, nullptr, k, n_, ctl_.as<uint32_t>(), d_err_);
  k_pair_keys<<<grid_for(k, kBlock, 16), kBlock, 0, stream_>>>(du, dv, k, pair_key_.as<unsigned long long>());
  cuda_check(cudaGetLastError(), "pair keys");
  launches_ += 2;
  size_t tb = cub_tmp_.bytes;
  cuda_check(cub::DeviceRadixSort::SortPairs(cub_tmp_.p, tb, pair_key_.as<unsigned long long>(),
                                             pair_key_s_.as<unsigned long long>(), iota_.as<uint32_t>(),
                                             perm_.as<uint32_t>(), (int)k, 0, end_bit, stream_),
             "pair sort");
  k_pair_heads<<<grid_for(k, kBlock, 16), kBlock, 0, stream_>>>(pair_key_s_.as<unsigned long long>(), k,
                                                                  head_.as<uint8_t>());
  cuda_check(cudaGetLastError(), "pair heads");
  ++launches_;
  tb = cub_tmp_.bytes;
  cuda_check(cub::DeviceSelect::Flagged(cub_tmp_.p, tb, iota_.as<uint32_t>(), head_.as<uint8_t>(),
                                        seg_.as<uint32_t>(), nseg_.as<uint32_t>(), (int)k, stream_),
             "pair runs");
  // Absent until matched: a batch rejected by validation deletes nothing.
  cuda_check(cudaMemsetAsync(pair_slot_.p, 0xff, k * 4, stream_), "pair slots");
  const uint32_t ks = (uint32_t)std::max<uint64_t>(std::min<uint64_t>(k, n_), 1);
  k_pair_slots<<<grid_for((unsigned long long)ks * 32, kBlock, 8), kBlock, 0, stream_>>>(
      view(), pair_key_s_.as<unsigned long long>(), perm_.as<uint32_t>(), seg_.as<uint32_t>(),
      nseg_.as<uint32_t>(), k, ctl_.as<uint32_t>(), pair_slot_.as<uint32_t>());
  cuda_check(cudaGetLastError(), "pair slots");
  ++launches_;
}

void Engine::walk(const bingo_walk_job* jobs, uint32_t n_jobs, uint32_t mode) {
  const NvtxRange nvtx_("bingo walk");
  require_loaded();
  if (n_jobs == 0) return;
  if (!jobs) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null job array");
  if (mode != BINGO_WALK_BATCHED && mode != BINGO_WALK_PLAIN) throw Error(BINGO_ERR_INVALID_ARGUMENT, "bad mode");
  std::vector<WalkJobDev> dj(n_jobs);
  std::vector<uint64_t> prefix(n_jobs + 1, 0);
  // staging layout for host starts / outputs
  std::vector<uint64_t> s_off(n_jobs, ~0ull), o_off(n_jobs, ~0ull);
  uint64_t s_total = 0, o_total = 0;
  for (uint32_t j = 0; j < n_jobs; ++j) {
    const bingo_walk_job& J = jobs[j];
    check_walk_job(J);
    if (J.n_starts && !J.out) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null output");
    if (J.n_starts >= (1ull << 32)) throw Error(BINGO_ERR_UNSUPPORTED, "more than 2^32 walks in one job");
    if (J.starts) {
      if (!is_device_ptr(J.starts)) {
        host_check_ids(J.starts, J.n_starts, n_, "start");
        s_off[j] = s_total;
        s_total += J.n_starts;
      }
    } else if ((uint64_t)J.first + J.n_starts > n_) {
      throw Error(BINGO_ERR_OUT_OF_RANGE, "start range exceeds n");
    }
    const uint64_t per = J.app == BINGO_SAMPLING ? 1 : J.length;
    if (J.n_starts && !is_device_ptr(J.out)) {
      o_off[j] = o_total;
      o_total += (J.n_starts * per + 7) & ~7ull;  // 32-byte aligned job outputs
    }
    prefix[j + 1] = prefix[j] + J.n_starts;
  }
  // Staging grows to the next power of two, so a stream of queries of
  // varying size reallocates (a device-wide synchronising cudaFree plus a
  // cudaMalloc) only a few times.
  if (s_total) wstart_.ensure(pow2_bytes(s_total * 4), "walk staging");
  // Host-bound outputs go through the next staging buffer; its previous
  // copy-out must finish before these kernels overwrite it (a device-side
  // wait, no host synchronisation).
  int32_t* wout = nullptr;
  const int ring = wout_next_;
  if (o_total) {
    wout_next_ ^= 1;
    if (wout_busy_[ring]) {
      if (wout_[ring].bytes < pow2_bytes(o_total * 4))  // about to reallocate: its copy-out must be over first
        cuda_check(cudaEventSynchronize(copy_ev_[ring]), "staging reuse");
      else
        cuda_check(cudaStreamWaitEvent(stream_, copy_ev_[ring], 0), "staging reuse");
    }
    wout_[ring].ensure(pow2_bytes(o_total * 4), "walk staging");
    wout = wout_[ring].as<int32_t>();
  }
  for (uint32_t j = 0; j < n_jobs; ++j) {
    const bingo_walk_job& J = jobs[j];
    WalkJobDev& D = dj[j];
    D = make_job(J);
    D.starts = J.starts;
    if (s_off[j] != ~0ull) {
      uint32_t* d = wstart_.as<uint32_t>() + s_off[j];
      cuda_check(cudaMemcpyAsync(d, J.starts, J.n_starts * 4, cudaMemcpyHostToDevice, stream_), "starts H2D");
      D.starts = d;
    }
    D.out = o_off[j] != ~0ull ? wout + o_off[j] : J.out;
  }
  if (mode == BINGO_WALK_BATCHED && prefix[n_jobs] >= (1ull << 32))
    throw Error(BINGO_ERR_UNSUPPORTED, "more than 2^32 walks in one batched call");
  for (uint32_t j = 0; j < n_jobs; ++j) {
    const uint64_t per = jobs[j].app == BINGO_SAMPLING ? 1 : jobs[j].length;
    if (jobs[j].n_starts * per >= (32ull << 32)) throw Error(BINGO_ERR_UNSUPPORTED, "job output exceeds 2^35 entries");
    if (jobs[j].n_starts && o_off[j] == ~0ull && jobs[j].app != BINGO_SAMPLING &&
        (reinterpret_cast<uintptr_t>(jobs[j].out) & 31))
      throw Error(BINGO_ERR_INVALID_ARGUMENT, "device output must be 32-byte aligned");
  }
  const WalkView W = wview();
  auto launch = [&](auto kern, unsigned occ, const WalkJobDev& J0, const WalkJobDev* jb, const uint32_t* pf,
                    uint32_t nj, uint32_t tot, uint32_t* qq) {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(grid_for(tot, kBlock, walk_bps(occ, tuning_, J0.app)));
    lc.blockDim = dim3(kBlock);
    lc.stream = stream_;
    cuda_check(cudaLaunchKernelEx(&lc, kern, W, J0, jb, pf, nj, tot, qq, walk_chunk_of(tuning_, J0.app)),
               "walk launch");
    ++launches_;
  };
  queue_.ensure(4 * std::max<uint32_t>(n_jobs, 4), "walk queue");
  uint32_t* q = queue_.as<uint32_t>();
  if (mode == BINGO_WALK_PLAIN) {
    // One launch per job, each with its own work counter.
    cuda_check(cudaMemsetAsync(q, 0, 4 * n_jobs, stream_), "queue reset");
    for (uint32_t j = 0; j < n_jobs; ++j) {
      if (!dj[j].n) continue;
      const uint32_t nw = (uint32_t)dj[j].n;
      switch (dj[j].app) {
        case APP_DEEPWALK:
          launch(k_walk<APP_DEEPWALK, false>, walk_blocks_per_sm<APP_DEEPWALK, false>(), dj[j], nullptr,
                 nullptr, 0, nw, q + j);
          break;
        case APP_NODE2VEC:
          launch(k_walk<APP_NODE2VEC, false>, walk_blocks_per_sm<APP_NODE2VEC, false>(), dj[j], nullptr,
                 nullptr, 0, nw, q + j);
          break;
        case APP_PPR:
          launch(k_walk<APP_PPR, false>, walk_blocks_per_sm<APP_PPR, false>(), dj[j], nullptr, nullptr, 0,
                 nw, q + j);
          break;
        default:
          launch(k_walk<APP_SAMPLING, false>, walk_blocks_per_sm<APP_SAMPLING, false>(), dj[j], nullptr,
                 nullptr, 0, nw, q + j);
          break;
      }
    }
  } else if (prefix[n_jobs]) {
    // One persistent launch per app present (or one mixed launch).
    std::vector<WalkJobDev> table;
    std::vector<uint32_t> pf;
    std::vector<WalkGroup> groups;
    build_walk_groups(dj.data(), n_jobs, tuning_.walk_split != 0, tuning_.walk_order != 0, table, pf, groups);
    jobs_.ensure(table.size() * sizeof(WalkJobDev), "walk jobs");
    prefix_.ensure(pf.size() * 4, "walk jobs");
    cuda_check(cudaMemcpyAsync(jobs_.p, table.data(), table.size() * sizeof(WalkJobDev), cudaMemcpyHostToDevice,
                               stream_),
               "jobs H2D");
    cuda_check(cudaMemcpyAsync(prefix_.p, pf.data(), pf.size() * 4, cudaMemcpyHostToDevice, stream_), "prefix H2D");
    cuda_check(cudaMemsetAsync(q, 0, 4 * groups.size(), stream_), "queue reset");
    for (size_t gi = 0; gi < groups.size(); ++gi) {
      const WalkGroup& G = groups[gi];
      launch_walk_table(stream_, G.app, W, table[G.job_off], jobs_.as<WalkJobDev>() + G.job_off,
                        prefix_.as<uint32_t>() + G.pf_off, G.n_jobs, G.total, q + gi, tuning_);
      ++launches_;
    }
  }
  if (o_total) {
    // Asynchronous handles copy out on xstream_, after this call's kernels;
    // the next call's kernels proceed meanwhile. bingo_sync waits for both.
    cudaStream_t cs = stream_;
    if (!cfg_.synchronous) {
      cs = xstream_;
      cuda_check(cudaEventRecord(walk_ev_[ring], stream_), "walk done");
      cuda_check(cudaStreamWaitEvent(xstream_, walk_ev_[ring], 0), "copy after walk");
    }
    for (uint32_t j = 0; j < n_jobs; ++j)
      if (o_off[j] != ~0ull) {
        const uint64_t per = jobs[j].app == BINGO_SAMPLING ? 1 : jobs[j].length;
        cuda_check(cudaMemcpyAsync(jobs[j].out, wout + o_off[j], jobs[j].n_starts * per * 4, cudaMemcpyDeviceToHost,
                                   cs),
                   "walk D2H");
      }
    cuda_check(cudaEventRecord(copy_ev_[ring], cs), "copy done");
    wout_busy_[ring] = true;
  }
  finish_call();
}

// ------------------------------------------------------------------ jobs, serving
void Engine::check_walk_job(const bingo_walk_job& J) const {
  if (J.app < 0 || J.app > 3) throw Error(BINGO_ERR_INVALID_ARGUMENT, "unknown app");
  if (J.app == BINGO_NODE2VEC && !cfg_.node2vec)
    throw Error(BINGO_ERR_UNSUPPORTED, "node2vec needs the adjacency index (config.node2vec)");
  if (J.app == BINGO_NODE2VEC && !(J.p > 0 && J.q > 0)) throw Error(BINGO_ERR_INVALID_ARGUMENT, "p, q must be > 0");
  if (J.app == BINGO_PPR && !(J.stop_prob >= 0 && J.stop_prob <= 1))
    throw Error(BINGO_ERR_INVALID_ARGUMENT, "stop_prob must be in [0, 1]");
  if (J.app != BINGO_SAMPLING && J.length == 0 && J.n_starts)
    throw Error(BINGO_ERR_INVALID_ARGUMENT, "length must be >= 1");
}

WalkJobDev Engine::make_job(const bingo_walk_job& J) const {
  WalkJobDev D;
  D.app = J.app;
  D.L = J.length;
  D.starts = J.starts;
  D.n = J.n_starts;
  D.first = J.first;
  D.job = J.job_id;
  D.k0 = (uint32_t)J.seed;
  D.k1 = (uint32_t)(J.seed >> 32);
  D.flags = J.flags;
  D.seq = 0;
  set_thresholds(D, J);
  D.out = J.out;
  return D;
}

void Engine::require_idle() const {
  if (server_) throw Error(BINGO_ERR_BUSY, "the handle is serving (bingo_serve_stop first)");
}

void Engine::serve_start(const bingo_serve_config& cfg) {
  require_loaded();
  require_idle();
  cuda_check(cudaStreamSynchronize(stream_), "serve start");
  server_.reset(new Server(*this, cfg));
}

void Engine::serve_stop() {
  if (!server_) throw Error(BINGO_ERR_INVALID_ARGUMENT, "not serving");
  server_.reset();
  finish_call();
}

// ------------------------------------------------------------------ programs
void Engine::drop_graph() {
  if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
  if (graph_) cudaGraphDestroy(graph_);
  graph_exec_ = nullptr;
  graph_ = nullptr;
  graph_sig_ = 0;
}

// Insert without host synchronisation: the batch's arena needs are reserved
// on the device (all or nothing); a batch that does not fit is not applied
// and raises E_CAPACITY. Inputs are device arrays.
void Engine::enqueue_insert(const uint32_t* a, const uint32_t* b, const uint32_t* c, uint64_t k,
                            uint32_t* out_slots) {
  const uint32_t ks = (uint32_t)std::max<uint64_t>(std::min<uint64_t>(k, n_), 1);
  group_by_vertex(a, b, c, k, true);
  const StoreView S = view();
  plan_needs(S, k, ks, nullptr, kReserveSticky);
  launch_pdl(k_apply_insert, grid_for((unsigned long long)ks * 32, kBlock, tuning_.apply_blocks_per_sm), kBlock,
             stream_, S, key_s_.as<uint32_t>(), sa_.as<uint32_t>(), sb_.as<uint32_t>(), perm_.as<uint32_t>(),
             seg_.as<uint32_t>(), nseg_.as<uint32_t>(), k, ks, ctl_.as<uint32_t>(), scan_.as<ArenaNeed>(),
             need_.as<unsigned long long>(), base_.as<unsigned long long>(), HostReserve{}, out_slots);
  cuda_check(cudaGetLastError(), "apply insert");
  ++launches_;
}

void Engine::enqueue_delete(const uint32_t* u, const uint32_t* slot, uint64_t k) {
  group_by_vertex(u, slot, nullptr, k, false);
  const uint32_t ks = (uint32_t)std::max<uint64_t>(std::min<uint64_t>(k, n_), 1);
  launch_pdl(k_apply_delete, grid_for((unsigned long long)ks * 32, kBlock, tuning_.apply_blocks_per_sm), kBlock,
             stream_, view(), key_s_.as<uint32_t>(), sa_.as<uint32_t>(), seg_.as<uint32_t>(), nseg_.as<uint32_t>(), k,
             ctl_.as<uint32_t>());
  cuda_check(cudaGetLastError(), "apply delete");
  ++launches_;
}

// Grows arenas so that a program inserting k edges in total is unlikely to
// run out on the device: free space >= a quarter of the used space plus a
// per-edge allowance (every set bit may double its group, every slot its
// vertex arrays).
void Engine::ensure_headroom(uint64_t k_ins) {
  static const unsigned long long per_edge[kArenas] = {64, 2, 64, 2, 4};
  read_tops();
  for (int a = 0; a < kArenas; ++a) {
    if (a == A_HASH && !cfg_.node2vec) continue;
    const unsigned long long want = h_top_[a] / 4 + per_edge[a] * k_ins + kArenaFloor[a];
    if (cap_[a] - h_top_[a] < want) grow_arena(a, h_top_[a] + 2 * want);
  }
}

void Engine::run(const bingo_op* ops, uint32_t n_ops, uint32_t flags) {
  const NvtxRange nvtx_("bingo run");
  require_loaded();
  if (n_ops == 0) return;
  if (!ops) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null op array");
  const bool use_graph = flags & BINGO_RUN_GRAPH;
  // ---- validate, size scratch, lay out the job tables
  uint64_t kmax = 0, k_ins = 0, n_jobs_total = 0, n_walk_ops = 0, kpairs = 0;
  uint64_t sig = 1469598103934665603ull;
  auto mix = [&](uint64_t x) { sig = (sig ^ x) * 1099511628211ull; };
  for (uint32_t i = 0; i < n_ops; ++i) {
    const bingo_op& o = ops[i];
    mix((uint64_t)o.kind);
    if (o.kind == BINGO_OP_INSERT || o.kind == BINGO_OP_DELETE || o.kind == BINGO_OP_DELETE_PAIRS) {
      const bool ins = o.kind == BINGO_OP_INSERT;
      if (o.kind == BINGO_OP_DELETE_PAIRS && o.k) kpairs = std::max<uint64_t>(kpairs, o.k);
      if (!o.k) continue;
      if (o.k >= (1ull << 31)) throw Error(BINGO_ERR_UNSUPPORTED, "batch larger than 2^31");
      if (!o.a || !o.b || (ins && !o.c)) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null batch array");
      if (!is_device_ptr(o.a) || !is_device_ptr(o.b) || (ins && !is_device_ptr(o.c)) ||
          (o.out_slots && !is_device_ptr(o.out_slots)))
        throw Error(BINGO_ERR_INVALID_ARGUMENT, "program batches must be device arrays");
      kmax = std::max<uint64_t>(kmax, o.k);
      if (ins) k_ins += o.k;
      mix(o.k), mix((uint64_t)(uintptr_t)o.a), mix((uint64_t)(uintptr_t)o.b), mix((uint64_t)(uintptr_t)o.c);
      mix((uint64_t)(uintptr_t)o.out_slots);
    } else if (o.kind == BINGO_OP_WALK) {
      if (o.n_jobs && !o.jobs) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null job array");
      n_jobs_total += o.n_jobs;
      ++n_walk_ops;
      mix(o.n_jobs);
      for (uint32_t j = 0; j < o.n_jobs; ++j) mix(o.jobs[j].n_starts);
    } else {
      throw Error(BINGO_ERR_INVALID_ARGUMENT, "unknown op kind");
    }
  }
  if (kmax) ensure_batch_scratch(kmax);
  if (kpairs) ensure_pair_scratch(kpairs);
  ensure_headroom(k_ins);
  mix(arena_gen_), mix(n_);
  std::vector<WalkJobDev> dj, table;
  std::vector<uint32_t> pf;
  std::vector<WalkGroup> groups;
  std::vector<size_t> grp_begin(n_ops, 0), grp_end(n_ops, 0);
  const bool split = tuning_.walk_split != 0;
  mix(tuning_.walk_chunk), mix(tuning_.walk_blocks_per_sm), mix(tuning_.walk_split), mix(tuning_.walk_order);
  mix(tuning_.apply_blocks_per_sm);
  dj.reserve(n_jobs_total);
  for (uint32_t i = 0; i < n_ops; ++i) {
    const bingo_op& o = ops[i];
    if (o.kind != BINGO_OP_WALK) continue;
    dj.clear();
    uint64_t t = 0;
    for (uint32_t j = 0; j < o.n_jobs; ++j) {
      const bingo_walk_job& J = o.jobs[j];
      if (J.app < 0 || J.app > 3) throw Error(BINGO_ERR_INVALID_ARGUMENT, "unknown app");
      if (J.app == BINGO_NODE2VEC && !cfg_.node2vec)
        throw Error(BINGO_ERR_UNSUPPORTED, "node2vec needs the adjacency index (config.node2vec)");
      if (J.app == BINGO_NODE2VEC && !(J.p > 0 && J.q > 0)) throw Error(BINGO_ERR_INVALID_ARGUMENT, "p, q must be > 0");
      if (J.app == BINGO_PPR && !(J.stop_prob >= 0 && J.stop_prob <= 1))
        throw Error(BINGO_ERR_INVALID_ARGUMENT, "stop_prob must be in [0, 1]");
      if (J.n_starts) {
        if (J.app != BINGO_SAMPLING && J.length == 0) throw Error(BINGO_ERR_INVALID_ARGUMENT, "length must be >= 1");
        if (!J.out || !is_device_ptr(J.out)) throw Error(BINGO_ERR_INVALID_ARGUMENT, "program outputs must be device arrays");
        if (J.starts && !is_device_ptr(J.starts))
          throw Error(BINGO_ERR_INVALID_ARGUMENT, "program start arrays must be device arrays");
        if (J.app != BINGO_SAMPLING && (reinterpret_cast<uintptr_t>(J.out) & 31))
          throw Error(BINGO_ERR_INVALID_ARGUMENT, "device output must be 32-byte aligned");
        if (!J.starts && (uint64_t)J.first + J.n_starts > n_) throw Error(BINGO_ERR_OUT_OF_RANGE, "start range exceeds n");
      }
      t += J.n_starts;
      if (t >= (1ull << 32)) throw Error(BINGO_ERR_UNSUPPORTED, "more than 2^32 walks in one op");
      if (split) mix((uint64_t)J.app);
      WalkJobDev D;
      D.app = J.app;
      D.L = J.length;
      D.starts = J.starts;
      D.n = J.n_starts;
      D.first = J.first;
      D.job = J.job_id;
      D.k0 = (uint32_t)J.seed;
      D.k1 = (uint32_t)(J.seed >> 32);
      D.flags = J.flags;
      D.seq = 0;
      set_thresholds(D, J);
      D.out = J.out;
      dj.push_back(D);
    }
    grp_begin[i] = groups.size();
    build_walk_groups(dj.data(), (uint32_t)dj.size(), split, tuning_.walk_order != 0, table, pf, groups);
    grp_end[i] = groups.size();
  }
  // Job tables are read by the walk kernels from device memory, so their
  // contents may change between replays of a captured program.
  if (!table.empty()) {
    const size_t jb = table.size() * sizeof(WalkJobDev), pb = pf.size() * 4, qb = groups.size() * 4;
    if (jb > prog_jobs_.bytes || pb > prog_prefix_.bytes || qb > prog_queue_.bytes) drop_graph();
    prog_jobs_.ensure(jb, "program jobs");
    prog_prefix_.ensure(pb, "program jobs");
    prog_queue_.ensure(std::max<size_t>(qb, 4), "program queue");
    cuda_check(cudaMemcpyAsync(prog_jobs_.p, table.data(), jb, cudaMemcpyHostToDevice, stream_), "program jobs H2D");
    cuda_check(cudaMemcpyAsync(prog_prefix_.p, pf.data(), pb, cudaMemcpyHostToDevice, stream_), "program jobs H2D");
  }
  (void)n_walk_ops;
  mix((uint64_t)(uintptr_t)prog_jobs_.p), mix((uint64_t)(uintptr_t)ctl_.p), mix((uint64_t)(uintptr_t)cub_tmp_.p);
  mix(cub_tmp_.bytes);

  const uint64_t launches0 = launches_;
  auto enqueue_all = [&]() {
    if (!groups.empty())
      cuda_check(cudaMemsetAsync(prog_queue_.p, 0, groups.size() * 4, stream_), "program queue reset");
    const WalkView W = wview();
    for (uint32_t i = 0; i < n_ops; ++i) {
      const bingo_op& o = ops[i];
      if (o.kind == BINGO_OP_INSERT && o.k) {
        enqueue_insert(o.a, o.b, o.c, o.k, o.out_slots);
      } else if (o.kind == BINGO_OP_DELETE && o.k) {
        enqueue_delete(o.a, o.b, o.k);
      } else if (o.kind == BINGO_OP_DELETE_PAIRS && o.k) {
        translate_pairs(o.a, o.b, o.k);
        enqueue_delete(o.a, pair_slot_.as<uint32_t>(), o.k);
      } else if (o.kind == BINGO_OP_WALK) {
        for (size_t gi = grp_begin[i]; gi < grp_end[i]; ++gi) {
          const WalkGroup& G = groups[gi];
          launch_walk_table(stream_, G.app, W, table[G.job_off], prog_jobs_.as<WalkJobDev>() + G.job_off,
                            prog_prefix_.as<uint32_t>() + G.pf_off, G.n_jobs, G.total,
                            prog_queue_.as<uint32_t>() + gi, tuning_);
          ++launches_;
        }
      }
    }
  };
  if (use_graph) {
    if (!graph_exec_ || graph_sig_ != sig) {
      drop_graph();
      cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
      try {
        enqueue_all();
      } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(stream_, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        throw;
      }
      cuda_check(cudaStreamEndCapture(stream_, &graph_), "end capture");
      cuda_check(cudaGraphInstantiate(&graph_exec_, graph_, 0), "instantiate graph");
      graph_sig_ = sig;
      graph_launches_ = launches_ - launches0;
      launches_ = launches0;
    }
    cuda_check(cudaGraphLaunch(graph_exec_, stream_), "graph launch");
    launches_ += graph_launches_;
  } else {
    enqueue_all();
  }
  if (cfg_.synchronous) {
    const int st = sync();
    read_tops();
    if (st) throw Error(st, last_error);
  }
}

// ------------------------------------------------------------------ no-alloc walks
// Scratch of bingo_walk_noalloc: job table, walk prefix and work counter in a
// file-scope device array (every GPU that loads the library holds it until
// exit). Host code reaches it only through the address cudaGetSymbolAddress
// returns for the current device.
constexpr uint32_t kNoAllocMaxJobs = 64;
struct NoAllocScratch {
  WalkJobDev jobs[kNoAllocMaxJobs];
  uint32_t prefix[kNoAllocMaxJobs + 1];
  uint32_t queue;
};
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// The call's job table and walk offsets travel as one kernel parameter
// (values, not a pointer to host memory; 6,404 bytes, under the 32,764-byte
// parameter limit), and this kernel writes them into the scratch and zeroes
// the work counter, ahead of the walk launch on the same stream.
struct NoAllocJobs {
  WalkJobDev jobs[kNoAllocMaxJobs];
  uint32_t prefix[kNoAllocMaxJobs + 1];
  uint32_t n_jobs;
};
static_assert(sizeof(NoAllocJobs) <= 32764, "kernel parameter limit");

__global__ void k_noalloc_stage(const __grid_constant__ NoAllocJobs in, NoAllocScratch* dst) {
  const uint32_t words = (uint32_t)(in.n_jobs * sizeof(WalkJobDev) / 4);
  const uint32_t* src = reinterpret_cast<const uint32_t*>(in.jobs);
  uint32_t* out = reinterpret_cast<uint32_t*>(dst->jobs);
  for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) out[i] = src[i];
  for (uint32_t i = threadIdx.x; i <= in.n_jobs; i += blockDim.x) dst->prefix[i] = in.prefix[i];
  if (threadIdx.x == 0) dst->queue = 0;
}
static_assert(sizeof(WalkJobDev) % 4 == 0, "word copy");

namespace {
constexpr int kNoAllocMaxDevices = 128;
std::mutex g_noalloc_mu;
NoAllocScratch* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch for `device` (must be current); looked up
// once per device. The ordinal is checked before it indexes the table.
NoAllocScratch* noalloc_scratch(int device) {
  if (device < 0 || device >= kNoAllocMaxDevices)
    throw Error(BINGO_ERR_INVALID_ARGUMENT, "bingo_walk_noalloc supports device ordinals 0.." +
                                                std::to_string(kNoAllocMaxDevices - 1));
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(no-alloc scratch)");
    g_noalloc_ptr[device] = static_cast<NoAllocScratch*>(p);
  }
  return g_noalloc_ptr[device];
}
}  // namespace

void Engine::walk_noalloc(const bingo_walk_job* jobs, uint32_t n_jobs) {
  const NvtxRange nvtx_("bingo walk noalloc");
  require_loaded();
  if (n_jobs == 0) return;
  if (!jobs) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null job array");
  if (n_jobs > kNoAllocMaxJobs)
    throw Error(BINGO_ERR_INVALID_ARGUMENT, "bingo_walk_noalloc takes at most " + std::to_string(kNoAllocMaxJobs) +
                                                " jobs per call (got " + std::to_string(n_jobs) + ")");
  NoAllocScratch* scratch = noalloc_scratch(cfg_.device);
  NoAllocJobs in;
  WalkJobDev* dj = in.jobs;
  uint32_t* prefix = in.prefix;
  in.n_jobs = n_jobs;
  prefix[0] = 0;
  uint64_t total = 0;
  for (uint32_t j = 0; j < n_jobs; ++j) {
    const bingo_walk_job& J = jobs[j];
    if (J.app < 0 || J.app > 3) throw Error(BINGO_ERR_INVALID_ARGUMENT, "unknown app");
    if (J.app == BINGO_NODE2VEC && !cfg_.node2vec)
      throw Error(BINGO_ERR_UNSUPPORTED, "node2vec needs the adjacency index (config.node2vec)");
    if (J.app == BINGO_NODE2VEC && !(J.p > 0 && J.q > 0)) throw Error(BINGO_ERR_INVALID_ARGUMENT, "p, q must be > 0");
    if (J.app == BINGO_PPR && !(J.stop_prob >= 0 && J.stop_prob <= 1))
      throw Error(BINGO_ERR_INVALID_ARGUMENT, "stop_prob must be in [0, 1]");
    if (J.app != BINGO_SAMPLING && J.length == 0 && J.n_starts)
      throw Error(BINGO_ERR_INVALID_ARGUMENT, "length must be >= 1");
    if (J.n_starts) {
      if (!J.out || !is_device_ptr(J.out))
        throw Error(BINGO_ERR_INVALID_ARGUMENT, "bingo_walk_noalloc needs device output buffers");
      if (J.starts && !is_device_ptr(J.starts))
        throw Error(BINGO_ERR_INVALID_ARGUMENT, "bingo_walk_noalloc needs device start arrays (or NULL)");
      if (J.app != BINGO_SAMPLING && (reinterpret_cast<uintptr_t>(J.out) & 31))
        throw Error(BINGO_ERR_INVALID_ARGUMENT, "device output must be 32-byte aligned");
      if (!J.starts && (uint64_t)J.first + J.n_starts > n_) throw Error(BINGO_ERR_OUT_OF_RANGE, "start range exceeds n");
    }
    total += J.n_starts;
    if (total >= (1ull << 32)) throw Error(BINGO_ERR_UNSUPPORTED, "more than 2^32 walks in one call");
    prefix[j + 1] = (uint32_t)total;
    WalkJobDev& D = dj[j];
    D.app = J.app;
    D.L = J.length;
    D.starts = J.starts;
    D.n = J.n_starts;
    D.first = J.first;
    D.job = J.job_id;
    D.k0 = (uint32_t)J.seed;
    D.k1 = (uint32_t)(J.seed >> 32);
    D.flags = J.flags;
    D.seq = 0;
    set_thresholds(D, J);
    D.out = J.out;
  }
  if (!total) return;
  // Job table, prefix and a zeroed work counter reach the scratch through a
  // kernel parameter: nothing is read from host memory after this call returns.
  k_noalloc_stage<<<1, 256, 0, stream_>>>(in, scratch);
  cuda_check(cudaGetLastError(), "no-alloc job staging");
  ++launches_;
  const WalkView W = wview();
  k_walk<-1, true><<<grid_for(total, kBlock, walk_bps(walk_blocks_per_sm<-1, true>(), tuning_, -1)), kBlock, 0, stream_>>>(
      W, dj[0], scratch->jobs, scratch->prefix, n_jobs, (uint32_t)total, &scratch->queue, walk_chunk_of(tuning_, -1));
  cuda_check(cudaGetLastError(), "no-alloc walk launch");
  ++launches_;
  finish_call();
}

void Engine::philox_batch(const uint32_t* ctr4, uint64_t count, uint64_t key, uint32_t* out4) {
  if (!count) return;
  if (!ctr4 || !out4) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null array");
  DevBuf c, o;
  c.ensure(count * 16, "philox");
  o.ensure(count * 16, "philox");
  cuda_check(cudaMemcpyAsync(c.p, ctr4, count * 16, cudaMemcpyDefault, stream_), "philox H2D");
  k_philox<<<grid_for(count, kBlock), kBlock, 0, stream_>>>(c.as<uint32_t>(), count, (uint32_t)key,
                                                           (uint32_t)(key >> 32), o.as<uint32_t>());
  cuda_check(cudaGetLastError(), "philox");
  ++launches_;
  cuda_check(cudaMemcpyAsync(out4, o.p, count * 16, cudaMemcpyDefault, stream_), "philox D2H");
  cuda_check(cudaStreamSynchronize(stream_), "philox");
  c.release();
  o.release();
}

// ------------------------------------------------------------------ state access
void Engine::stats(bingo_stats* out) {
  std::memset(out, 0, sizeof *out);
  out->n = n_;
  out->weight_mode = cfg_.weight_mode;
  if (server_) {  // the scheduler owns the stream and the host mirrors
    unsigned long long c[3];
    cuda_check(cudaMemcpy(c, d_steps_, sizeof c, cudaMemcpyDeviceToHost), "stats");
    out->walk_steps = c[0], out->walk_trials = c[1], out->walk_probes = c[2];
    out->kernel_launches = launches_;
    return;
  }
  cuda_check(cudaStreamSynchronize(stream_), "stats");
  {
    unsigned long long c[3];
    cuda_check(cudaMemcpy(c, d_steps_, sizeof c, cudaMemcpyDeviceToHost), "stats");
    out->walk_steps = c[0], out->walk_trials = c[1], out->walk_probes = c[2];
  }
  out->kernel_launches = launches_;
  if (!loaded_) return;
  read_tops();
  std::vector<VertexMeta> meta(n_);
  cuda_check(cudaMemcpy(meta.data(), meta_.p, (size_t)n_ * sizeof(VertexMeta), cudaMemcpyDeviceToHost), "stats");
  for (const auto& M : meta) out->slots += M.ecnt, out->live_edges += M.live;
  for (int a = 0; a < kArenas; ++a) {
    out->arena_bytes += cap_[a] * kUnitBytes[a] + (a == A_MEMBER ? cap_[a] * 4 : 0);
    out->arena_used += h_top_[a] * kUnitBytes[a] + (a == A_MEMBER ? h_top_[a] * 4 : 0);
  }
  const DevBuf* sc[] = {&in_a_, &in_b_, &in_c_, &key_s_, &perm_, &iota_, &sa_, &sb_, &head_, &seg_, &nseg_,
                        &need_, &scan_, &base_, &ctl_, &slots_, &cub_tmp_, &jobs_, &prefix_, &queue_, &wstart_,
                        &wout_[0], &wout_[1], &pair_key_, &pair_key_s_, &pair_slot_, &fw_in_, &fw_fixed_,
                        &prog_jobs_, &prog_prefix_, &prog_queue_};
  for (const DevBuf* b : sc) out->scratch_bytes += b->bytes;
}

namespace {
struct HostState {
  std::vector<VertexMeta> meta;
  std::vector<GroupDesc> gd;
  std::vector<VertexRec> vr;
  std::vector<uint32_t> gv, gs, bp;
  std::vector<EdgeRec> edges;
  std::vector<AliasRec> alias;
};
}  // namespace

static void fetch(HostState& H, uint32_t n, const DevBuf& meta, const DevBuf& gd, const DevBuf& vr,
                  const DevBuf* arena, const DevBuf& gs, const unsigned long long* top) {
  H.meta.resize(n);
  H.gd.resize((size_t)n * kBits);
  H.vr.resize(n);
  cuda_check(cudaMemcpy(H.meta.data(), meta.p, (size_t)n * sizeof(VertexMeta), cudaMemcpyDeviceToHost), "dump");
  cuda_check(cudaMemcpy(H.gd.data(), gd.p, H.gd.size() * sizeof(GroupDesc), cudaMemcpyDeviceToHost), "dump");
  cuda_check(cudaMemcpy(H.vr.data(), vr.p, (size_t)n * sizeof(VertexRec), cudaMemcpyDeviceToHost), "dump");
  H.gv.resize(top[A_MEMBER]);
  H.gs.resize(top[A_MEMBER]);
  H.edges.resize(top[A_EDGE]);
  H.bp.resize(top[A_BP]);
  H.alias.resize(top[A_ALIAS]);
  if (top[A_MEMBER]) {
    cuda_check(cudaMemcpy(H.gv.data(), arena[A_MEMBER].p, top[A_MEMBER] * 4, cudaMemcpyDeviceToHost), "dump");
    cuda_check(cudaMemcpy(H.gs.data(), gs.p, top[A_MEMBER] * 4, cudaMemcpyDeviceToHost), "dump");
  }
  if (top[A_EDGE])
    cuda_check(cudaMemcpy(H.edges.data(), arena[A_EDGE].p, top[A_EDGE] * sizeof(EdgeRec), cudaMemcpyDeviceToHost),
               "dump");
  if (top[A_BP]) cuda_check(cudaMemcpy(H.bp.data(), arena[A_BP].p, top[A_BP] * 4, cudaMemcpyDeviceToHost), "dump");
  if (top[A_ALIAS])
    cuda_check(
        cudaMemcpy(H.alias.data(), arena[A_ALIAS].p, top[A_ALIAS] * sizeof(AliasRec), cudaMemcpyDeviceToHost),
        "dump");
}

void Engine::dump_sizes(uint64_t sizes[3]) {
  require_loaded();
  cuda_check(cudaStreamSynchronize(stream_), "dump");
  std::vector<VertexMeta> meta(n_);
  std::vector<GroupDesc> gd((size_t)n_ * kBits);
  std::vector<VertexRec> vr(n_);
  cuda_check(cudaMemcpy(meta.data(), meta_.p, (size_t)n_ * sizeof(VertexMeta), cudaMemcpyDeviceToHost), "dump");
  cuda_check(cudaMemcpy(gd.data(), gdesc_.p, gd.size() * sizeof(GroupDesc), cudaMemcpyDeviceToHost), "dump");
  cuda_check(cudaMemcpy(vr.data(), vrec_.p, (size_t)n_ * sizeof(VertexRec), cudaMemcpyDeviceToHost), "dump");
  uint64_t s = 0, mem = 0, a = 0;
  for (uint32_t u = 0; u < n_; ++u) {
    s += meta[u].ecnt;
    for (int k = 0; k < kBits; ++k) mem += gd[(size_t)u * kBits + k].cnt;
    a += vr[u].m;
  }
  sizes[0] = s, sizes[1] = mem, sizes[2] = a;
}

void Engine::dump(uint32_t* ecnt, uint32_t* live, uint32_t* ev, uint32_t* ew, uint32_t* gcnt, uint32_t* mslot,
                  uint32_t* mv, uint32_t* mbp, uint32_t* am, uint64_t* athr, uint64_t* aT, uint8_t* aown,
                  uint8_t* aalias) {
  require_loaded();
  read_tops();
  HostState H;
  fetch(H, n_, meta_, gdesc_, vrec_, arena_, gs_, h_top_);
  uint64_t s = 0, mem = 0, a = 0;
  std::vector<uint32_t> ebp;
  for (uint32_t u = 0; u < n_; ++u) {
    const VertexMeta& M = H.meta[u];
    ecnt[u] = M.ecnt;
    live[u] = M.live;
    ebp.resize(M.ecnt);
    for (uint32_t i = 0; i < M.ecnt; ++i, ++s) {
      const EdgeRec& e = H.edges[M.eoff + i];
      ev[s] = e.v;
      ew[s] = e.w;
      ebp[i] = e.ebp;
    }
    for (int k = 0; k < kBits; ++k) {
      const GroupDesc& G = H.gd[(size_t)u * kBits + k];
      gcnt[(size_t)u * kBits + k] = G.cnt;
      for (uint32_t p = 0; p < G.cnt; ++p, ++mem) {
        // A member holds its slot's back-pointer index for the group; the
        // slot is the last one whose back-pointer range starts at or below it.
        const size_t idx = (size_t)group_base(G) * 4 + p;
        const uint32_t bi = H.gs[idx];
        const uint32_t sl = (uint32_t)(std::upper_bound(ebp.begin(), ebp.end(), bi) - ebp.begin()) - 1;
        mslot[mem] = sl;
        mv[mem] = H.gv[idx];
        mbp[mem] = H.bp[M.bpoff + bi];
      }
    }
    const VertexRec& R = H.vr[u];
    am[u] = R.m;
    int nzbits[kBits], nnz = 0;
    for (int k = 0; k < kBits; ++k)
      if (H.gd[(size_t)u * kBits + k].cnt) nzbits[nnz++] = k;
    for (uint32_t j = 0; j < R.m; ++j, ++a) {
      const AliasRec& A = H.alias[R.aoff + j];
      athr[a] = A.thr;
      aT[a] = A.T;
      aown[a] = j < (uint32_t)nnz ? (uint8_t)nzbits[j] : 255;
      uint8_t alt = 255;
      if (A.alt_cw & kInlineGroup) {
        alt = (uint8_t)(A.alt_cw & (kBits - 1));  // a one-member group names its bit
      } else {
        for (int k = 0; k < kBits; ++k) {
          const GroupDesc& G = H.gd[(size_t)u * kBits + k];
          if (G.cnt > 1 && group_base(G) == A.alt_ref && G.cnt == A.alt_cw) alt = (uint8_t)k;
        }
      }
      aalias[a] = alt;
    }
  }
}

// ------------------------------------------------------------------ tuning / state copy
void StateCopy::release() {
  vrec.release(), meta.release(), gdesc.release(), gs.release();
  for (auto& a : arena) a.release();
}

void Engine::set_tuning(const Tuning& t) {
  if (t.walk_chunk > 1024) throw Error(BINGO_ERR_INVALID_ARGUMENT, "walk_chunk must be in [0, 1024] (0: the kernel's default)");
  if (t.walk_blocks_per_sm > 32) throw Error(BINGO_ERR_INVALID_ARGUMENT, "walk_blocks_per_sm must be <= 32");
  if (t.walk_split > 1 || t.walk_order > 1) throw Error(BINGO_ERR_INVALID_ARGUMENT, "walk_split / walk_order are 0 or 1");
  if (t.apply_blocks_per_sm < 1 || t.apply_blocks_per_sm > 32)
    throw Error(BINGO_ERR_INVALID_ARGUMENT, "apply_blocks_per_sm must be in [1, 32]");
  tuning_ = t;
}

// Device copy of the store (used part of each arena); false when the device
// has no room for it.
bool Engine::save_state(StateCopy& c) {
  cuda_check(cudaStreamSynchronize(stream_), "state copy");
  read_tops();
  try {
    c.vrec.ensure((size_t)n_ * sizeof(VertexRec), "state copy");
    c.meta.ensure((size_t)n_ * sizeof(VertexMeta), "state copy");
    c.gdesc.ensure((size_t)n_ * kBits * sizeof(GroupDesc), "state copy");
    for (int a = 0; a < kArenas; ++a) c.arena[a].ensure(std::max(1ull, h_top_[a]) * kUnitBytes[a], "state copy");
    c.gs.ensure(std::max(1ull, h_top_[A_MEMBER]) * 4, "state copy");
  } catch (const Error&) {
    cudaGetLastError();
    c.release();
    return false;
  }
  cuda_check(cudaMemcpyAsync(c.vrec.p, vrec_.p, (size_t)n_ * sizeof(VertexRec), cudaMemcpyDeviceToDevice, stream_),
             "state copy");
  cuda_check(cudaMemcpyAsync(c.meta.p, meta_.p, (size_t)n_ * sizeof(VertexMeta), cudaMemcpyDeviceToDevice, stream_),
             "state copy");
  cuda_check(cudaMemcpyAsync(c.gdesc.p, gdesc_.p, (size_t)n_ * kBits * sizeof(GroupDesc), cudaMemcpyDeviceToDevice,
                             stream_),
             "state copy");
  for (int a = 0; a < kArenas; ++a) {
    c.top[a] = h_top_[a];
    if (h_top_[a])
      cuda_check(cudaMemcpyAsync(c.arena[a].p, arena_[a].p, h_top_[a] * kUnitBytes[a], cudaMemcpyDeviceToDevice,
                                 stream_),
                 "state copy");
  }
  if (h_top_[A_MEMBER])
    cuda_check(cudaMemcpyAsync(c.gs.p, gs_.p, h_top_[A_MEMBER] * 4, cudaMemcpyDeviceToDevice, stream_), "state copy");
  cuda_check(cudaStreamSynchronize(stream_), "state copy");
  return true;
}

// Puts a copy back. Arenas only grow, so each still holds the copy's used
// part at the same offsets.
void Engine::restore_state(const StateCopy& c) {
  cuda_check(cudaStreamSynchronize(stream_), "state restore");
  cuda_check(cudaMemcpyAsync(vrec_.p, c.vrec.p, (size_t)n_ * sizeof(VertexRec), cudaMemcpyDeviceToDevice, stream_),
             "state restore");
  cuda_check(cudaMemcpyAsync(meta_.p, c.meta.p, (size_t)n_ * sizeof(VertexMeta), cudaMemcpyDeviceToDevice, stream_),
             "state restore");
  cuda_check(cudaMemcpyAsync(gdesc_.p, c.gdesc.p, (size_t)n_ * kBits * sizeof(GroupDesc), cudaMemcpyDeviceToDevice,
                             stream_),
             "state restore");
  for (int a = 0; a < kArenas; ++a) {
    if (c.top[a] > cap_[a]) throw Error(BINGO_ERR_CUDA, "state copy larger than its arena");
    if (c.top[a])
      cuda_check(cudaMemcpyAsync(arena_[a].p, c.arena[a].p, c.top[a] * kUnitBytes[a], cudaMemcpyDeviceToDevice,
                                 stream_),
                 "state restore");
    h_top_[a] = c.top[a];
  }
  if (c.top[A_MEMBER])
    cuda_check(cudaMemcpyAsync(gs_.p, c.gs.p, c.top[A_MEMBER] * 4, cudaMemcpyDeviceToDevice, stream_), "state restore");
  cuda_check(cudaMemcpyAsync(d_top_, h_top_, kArenas * sizeof(unsigned long long), cudaMemcpyHostToDevice, stream_),
             "state restore");
  cuda_check(cudaMemsetAsync(d_err_, 0, 2 * sizeof(uint32_t), stream_), "state restore");
  cuda_check(cudaStreamSynchronize(stream_), "state restore");
}

// ------------------------------------------------------------------ snapshot files
// Layout: SnapHeader, then the vertex arrays (VertexRec, VertexMeta,
// GroupDesc x 32 per vertex), each arena's used part in arena order and the
// member slot ids, all as the device holds them (offsets stay valid because
// the arenas are restored at the same positions). The checksum covers the
// payload; record sizes and the format version guard against a file from an
// incompatible build.
namespace {

struct SnapHeader {
  char magic[8];
  uint32_t version, node2vec, n, bits;
  uint32_t rec_bytes[4];  // VertexRec, VertexMeta, GroupDesc, AliasRec
  uint64_t top[kArenas];
  uint64_t payload_bytes;
  uint64_t checksum;
};
constexpr char kSnapMagic[8] = {'B', 'I', 'N', 'G', 'O', 'S', 'N', 'P'};
// 2: 8-byte group descriptors, one-member groups named inline in the alias
// table; 3: members hold back-pointer indices instead of slot ids.
constexpr uint32_t kSnapVersion = 3;
constexpr size_t kSnapChunk = 64u << 20;

// Word-wise multiply-xor hash (64-bit lanes, tail bytes folded in one by one).
struct SnapSum {
  uint64_t h = 0x9E3779B97F4A7C15ull;
  void add(const char* p, size_t b) {
    size_t i = 0;
    for (; i + 8 <= b; i += 8) {
      uint64_t x;
      std::memcpy(&x, p + i, 8);
      h = (h ^ x) * 0x100000001B3ull;
      h ^= h >> 29;
    }
    for (; i < b; ++i) h = (h ^ (uint8_t)p[i]) * 0x100000001B3ull;
  }
};

struct Pinned {
  char* p = nullptr;
  explicit Pinned(size_t b) { cuda_check(cudaMallocHost((void**)&p, b), "snapshot staging"); }
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
};

struct File {
  FILE* f = nullptr;
  File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

}  // namespace

void Engine::save(const char* path) {
  const NvtxRange nvtx_("bingo save");
  require_loaded();
  require_idle();
  if (!path) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null path");
  cuda_check(cudaStreamSynchronize(stream_), "snapshot");
  read_tops();
  struct Part {
    const void* dev;
    uint64_t bytes;
  };
  std::vector<Part> parts = {{vrec_.p, (uint64_t)n_ * sizeof(VertexRec)},
                             {meta_.p, (uint64_t)n_ * sizeof(VertexMeta)},
                             {gdesc_.p, (uint64_t)n_ * kBits * sizeof(GroupDesc)}};
  for (int a = 0; a < kArenas; ++a) parts.push_back({arena_[a].p, h_top_[a] * kUnitBytes[a]});
  parts.push_back({gs_.p, h_top_[A_MEMBER] * 4});
  SnapHeader H{};
  std::memcpy(H.magic, kSnapMagic, 8);
  H.version = kSnapVersion;
  H.node2vec = cfg_.node2vec ? 1 : 0;
  H.n = n_;
  H.bits = kBits;
  H.rec_bytes[0] = sizeof(VertexRec), H.rec_bytes[1] = sizeof(VertexMeta);
  H.rec_bytes[2] = sizeof(GroupDesc), H.rec_bytes[3] = sizeof(AliasRec);
  for (int a = 0; a < kArenas; ++a) H.top[a] = h_top_[a];
  for (const Part& q : parts) H.payload_bytes += q.bytes;
  File F(path, "wb");
  if (!F.f) throw Error(BINGO_ERR_INVALID_ARGUMENT, std::string("cannot create ") + path);
  if (std::fwrite(&H, sizeof H, 1, F.f) != 1) throw Error(BINGO_ERR_INVALID_ARGUMENT, "snapshot write failed");
  // Double-buffered: the copy of the next chunk overlaps the write of this one.
  Pinned stage(2 * kSnapChunk);
  cudaEvent_t ev[2];
  cuda_check(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming), "event");
  cuda_check(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming), "event");
  SnapSum sum;
  struct Pending {
    size_t bytes = 0;
    int buf = 0;
  } pend;
  bool have = false;
  int next = 0;
  auto drain = [&]() {
    cuda_check(cudaEventSynchronize(ev[pend.buf]), "snapshot copy");
    const char* p = stage.p + (size_t)pend.buf * kSnapChunk;
    sum.add(p, pend.bytes);
    if (std::fwrite(p, 1, pend.bytes, F.f) != pend.bytes) throw Error(BINGO_ERR_INVALID_ARGUMENT, "snapshot write failed");
    have = false;
  };
  try {
    for (const Part& q : parts)
      for (uint64_t o = 0; o < q.bytes; o += kSnapChunk) {
        const size_t b = (size_t)std::min<uint64_t>(kSnapChunk, q.bytes - o);
        cuda_check(cudaMemcpyAsync(stage.p + (size_t)next * kSnapChunk, (const char*)q.dev + o, b,
                                   cudaMemcpyDeviceToHost, stream_),
                   "snapshot copy");
        cuda_check(cudaEventRecord(ev[next], stream_), "event");
        if (have) drain();
        pend = Pending{b, next};
        have = true;
        next ^= 1;
      }
    if (have) drain();
  } catch (...) {
    cudaStreamSynchronize(stream_);
    cudaEventDestroy(ev[0]), cudaEventDestroy(ev[1]);
    throw;
  }
  cudaEventDestroy(ev[0]), cudaEventDestroy(ev[1]);
  H.checksum = sum.h;
  if (std::fseek(F.f, 0, SEEK_SET) || std::fwrite(&H, sizeof H, 1, F.f) != 1 || std::fflush(F.f))
    throw Error(BINGO_ERR_INVALID_ARGUMENT, "snapshot write failed");
}

void Engine::restore(const char* path) {
  const NvtxRange nvtx_("bingo restore");
  require_idle();
  if (!path) throw Error(BINGO_ERR_INVALID_ARGUMENT, "null path");
  File F(path, "rb");
  if (!F.f) throw Error(BINGO_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
  SnapHeader H{};
  if (std::fread(&H, sizeof H, 1, F.f) != 1 || std::memcmp(H.magic, kSnapMagic, 8))
    throw Error(BINGO_ERR_INVALID_ARGUMENT, "not a graph snapshot");
  if (H.version != kSnapVersion || H.bits != (uint32_t)kBits || H.rec_bytes[0] != sizeof(VertexRec) ||
      H.rec_bytes[1] != sizeof(VertexMeta) || H.rec_bytes[2] != sizeof(GroupDesc) || H.rec_bytes[3] != sizeof(AliasRec))
    throw Error(BINGO_ERR_UNSUPPORTED, "snapshot from an incompatible build");
  if (H.node2vec != (cfg_.node2vec ? 1u : 0u))
    throw Error(BINGO_ERR_UNSUPPORTED, H.node2vec ? "snapshot carries the node2vec adjacency index; create the handle "
                                                    "with config.node2vec = 1"
                                                  : "snapshot has no node2vec adjacency index; create the handle with "
                                                    "config.node2vec = 0");
  if (!H.n) throw Error(BINGO_ERR_INVALID_ARGUMENT, "snapshot with n = 0");
  if (!H.node2vec && H.top[A_HASH]) throw Error(BINGO_ERR_INVALID_ARGUMENT, "corrupt snapshot header");
  uint64_t expect = (uint64_t)H.n * (sizeof(VertexRec) + sizeof(VertexMeta) + kBits * sizeof(GroupDesc));
  for (int a = 0; a < kArenas; ++a) {
    if (H.top[a] > kArenaLimit[a]) throw Error(BINGO_ERR_INVALID_ARGUMENT, "corrupt snapshot header");
    expect += H.top[a] * kUnitBytes[a];
  }
  expect += H.top[A_MEMBER] * 4;
  if (expect != H.payload_bytes) throw Error(BINGO_ERR_INVALID_ARGUMENT, "corrupt snapshot header");
  cuda_check(cudaStreamSynchronize(stream_), "restore");
  // From here the handle's old graph is gone; on failure it holds none.
  loaded_ = false;
  drop_graph();
  ++arena_gen_;
  n_ = H.n;
  vrec_.release(), meta_.release(), gdesc_.release();
  vrec_.ensure((size_t)n_ * sizeof(VertexRec), "vertex records");
  meta_.ensure((size_t)n_ * sizeof(VertexMeta), "vertex metadata");
  gdesc_.ensure((size_t)n_ * kBits * sizeof(GroupDesc), "group descriptors");
  const unsigned long long need[kArenas] = {H.top[0], H.top[1], H.top[2], H.top[3], H.top[4]};
  alloc_arenas(need);
  struct Part {
    void* dev;
    uint64_t bytes;
  };
  std::vector<Part> parts = {{vrec_.p, (uint64_t)n_ * sizeof(VertexRec)},
                             {meta_.p, (uint64_t)n_ * sizeof(VertexMeta)},
                             {gdesc_.p, (uint64_t)n_ * kBits * sizeof(GroupDesc)}};
  for (int a = 0; a < kArenas; ++a) parts.push_back({arena_[a].p, H.top[a] * kUnitBytes[a]});
  parts.push_back({gs_.p, H.top[A_MEMBER] * 4});
  // Double-buffered: reading the next chunk overlaps the copy of this one;
  // a half is refilled only after the copy issued from it has finished.
  Pinned stage(2 * kSnapChunk);
  cudaEvent_t ev[2];
  cuda_check(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming), "event");
  cuda_check(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming), "event");
  bool used[2] = {false, false};
  SnapSum sum;
  int next = 0;
  try {
    for (const Part& q : parts)
      for (uint64_t o = 0; o < q.bytes; o += kSnapChunk) {
        const size_t b = (size_t)std::min<uint64_t>(kSnapChunk, q.bytes - o);
        char* p = stage.p + (size_t)next * kSnapChunk;
        if (used[next]) cuda_check(cudaEventSynchronize(ev[next]), "restore copy");
        if (std::fread(p, 1, b, F.f) != b) throw Error(BINGO_ERR_INVALID_ARGUMENT, "snapshot file is truncated");
        sum.add(p, b);
        cuda_check(cudaMemcpyAsync((char*)q.dev + o, p, b, cudaMemcpyHostToDevice, stream_), "restore copy");
        cuda_check(cudaEventRecord(ev[next], stream_), "event");
        used[next] = true;
        next ^= 1;
      }
    cuda_check(cudaStreamSynchronize(stream_), "restore copy");
  } catch (...) {
    cudaStreamSynchronize(stream_);
    cudaEventDestroy(ev[0]), cudaEventDestroy(ev[1]);
    throw;
  }
  cudaEventDestroy(ev[0]), cudaEventDestroy(ev[1]);
  if (sum.h != H.checksum) throw Error(BINGO_ERR_INVALID_ARGUMENT, "snapshot checksum mismatch");
  for (int a = 0; a < kArenas; ++a) h_top_[a] = H.top[a];
  cuda_check(cudaMemcpyAsync(d_top_, h_top_, kArenas * sizeof(unsigned long long), cudaMemcpyHostToDevice, stream_),
             "restore");
  cuda_check(cudaMemsetAsync(d_err_, 0, 2 * sizeof(uint32_t), stream_), "restore");
  // The checksum only shows the file is the one written; the store check
  // shows its content is a store the kernels can index safely.
  bingo_check_report rep{};
  check_store(&rep);
  if (rep.bad_vertices)
    throw Error(BINGO_ERR_CORRUPT, "snapshot content fails the store check: " + std::to_string(rep.bad_vertices) +
                                       " vertices, first " + std::to_string(rep.first_bad) + ", kinds " +
                                       std::to_string(rep.kinds));
  loaded_ = true;
}

}  // namespace bingo
