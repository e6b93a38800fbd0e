// Store check (bingo_check): verifies every structural invariant the walk and
// update kernels rely on. A record is read only after the offsets that lead
// to it were checked against the used part of its arena, and every loop is
// bounded by a checked count, so a corrupt store yields a report, never an
// out-of-bounds access or an endless loop.
//
// k_check takes one warp per vertex. A vertex's group members are checked
// in one flattened range over all its groups (a lane finds its group by
// binary search over the 32 group offsets), so the three dependent reads per
// member are paid once per 32 x kMemberUnroll members, not once per group.
// Vertices with more than kBigMembers members are handed to k_check_big,
// where a whole CTA splits the member range, so a hub vertex does not keep
// one warp busy long after the rest of the grid has finished.
//
// The reference keeps no such checker; its structures (NodeData,
// include/Bingo.cuh:15-94) are trusted as built.
#include "engine.cuh"
#include "store.cuh"

namespace bingo {
namespace {

constexpr int kCheckBlock = 256;
constexpr int kWarpsPerBlock = kCheckBlock / 32;
constexpr int kBigBlock = 512;
constexpr int kMemberUnroll = 4;
constexpr uint32_t kBigMembers = 4096;

struct CheckTotals {
  unsigned long long live, wsum, members, slots, bad;
  uint32_t kinds, first_bad;
  uint32_t n_big;  // vertices handed to k_check_big (may exceed the list capacity)
  uint32_t pad;
};

// A vertex handed to k_check_big with the result of every other check.
struct BigVertex {
  uint32_t u, bad;
};

// Group offsets of one vertex: off[k] = members of groups below k (zero
// counts included), off[32] = all members; base[k] in 4-entry units.
struct GroupIndex {
  unsigned long long off[kBits + 1];
  uint32_t base[kBits];
};

// [off, off + len) inside [0, top).
__device__ __forceinline__ bool within(unsigned long long off, unsigned long long len, unsigned long long top) {
  return off <= top && len <= top - off;
}

__device__ __forceinline__ int nth_set_bit(uint32_t x, uint32_t j) {
  for (uint32_t t = 0; t < j && x; ++t) x &= x - 1;
  return x ? __ffs(x) - 1 : 0;
}

__device__ __forceinline__ bool group_extent_ok(const GroupDesc& G, unsigned long long top_member) {
  if (!G.base1) return G.cnt == 0;
  return G.cnt <= (1u << 31) && within((unsigned long long)group_base(G) * 4, group_cap(G), top_member);
}

// Lane k of the calling warp holds group k; fills X.
__device__ __forceinline__ void build_index(GroupIndex& X, const GroupDesc& G, int lane) {
  unsigned long long incl = G.cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  X.off[lane] = incl - G.cnt;
  X.base[lane] = group_base(G);
  if (lane == 31) X.off[kBits] = incl;
}

// The group holding flattened member f < off[32]: off[k] <= f < off[k + 1].
__device__ __forceinline__ int group_of(const GroupIndex& X, unsigned long long f) {
  int lo = 0, hi = kBits;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (X.off[mid] <= f)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// The slot whose back-pointer range holds back-pointer index bi: the last
// slot s < ecnt with ebp(s) <= bi (ebp grows with the slot id), or ecnt if
// there is none.
__device__ uint32_t slot_of_bp(const StoreView& S, const VertexMeta& M, uint32_t bi) {
  uint32_t lo = 0, hi = M.ecnt;  // answer in [lo, hi) or none
  if (hi == 0 || S.edges[M.eoff].ebp > bi) return M.ecnt;
  while (hi - lo > 1) {
    const uint32_t mid = lo + ((hi - lo) >> 1);
    if (S.edges[M.eoff + mid].ebp <= bi)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// Flattened members f0, f0 + stride, ... below end: each holds the
// back-pointer index of a live slot with the group's bit and the same
// neighbour (that slot's back-pointer for the group), and that back-pointer
// is the member's position. Returns BINGO_CHECK_MEMBER or 0.
__device__ uint32_t check_members(const StoreView& S, const VertexMeta& M, const GroupIndex& X,
                                  unsigned long long f0, unsigned long long stride, unsigned long long end) {
  uint32_t bad = 0;
  for (; f0 < end; f0 += stride * kMemberUnroll) {
    int k[kMemberUnroll];
    unsigned long long pos[kMemberUnroll];
    uint32_t b[kMemberUnroll], s[kMemberUnroll], v[kMemberUnroll];
    EdgeRec e[kMemberUnroll];
#pragma unroll
    for (int q = 0; q < kMemberUnroll; ++q) {
      const unsigned long long f = f0 + stride * q;
      k[q] = 0, pos[q] = 0, b[q] = 0xffffffffu, v[q] = 0;
      if (f < end) {
        k[q] = group_of(X, f);
        pos[q] = f - X.off[k[q]];
        const size_t at = (size_t)X.base[k[q]] * 4 + pos[q];
        b[q] = S.gs[at];
        v[q] = S.gv[at];
      }
    }
#pragma unroll
    for (int q = 0; q < kMemberUnroll; ++q) {
      e[q] = EdgeRec{0, 0, 0, 0};
      s[q] = M.ecnt;
      if (f0 + stride * q >= end) continue;
      if (b[q] < M.bpcnt) s[q] = slot_of_bp(S, M, b[q]);
      if (s[q] < M.ecnt)
        e[q] = S.edges[M.eoff + s[q]];
      else
        bad = BINGO_CHECK_MEMBER;
    }
#pragma unroll
    for (int q = 0; q < kMemberUnroll; ++q) {
      if (f0 + stride * q >= end || s[q] >= M.ecnt) continue;
      const unsigned long long bi = (unsigned long long)e[q].ebp + __popc(e[q].w & ((1u << k[q]) - 1u));
      if (!((e[q].w >> k[q]) & 1u) || e[q].v != v[q] || bi != b[q]) {
        bad = BINGO_CHECK_MEMBER;
        continue;
      }
      if (S.bp[M.bpoff + bi] != pos[q]) bad = BINGO_CHECK_MEMBER;
    }
  }
  return bad;
}

__device__ __forceinline__ void count_bad(CheckTotals* out, uint32_t u, uint32_t bad) {
  atomicAdd(&out->bad, 1ull);
  atomicOr(&out->kinds, bad);
  atomicMin(&out->first_bad, u);
}

__global__ void __launch_bounds__(kCheckBlock) k_check(StoreView S, CheckTotals* out, BigVertex* big,
                                                       uint32_t big_cap) {
  __shared__ GroupIndex gidx[kWarpsPerBlock];
  const int lane = threadIdx.x & 31;
  GroupIndex& X = gidx[threadIdx.x / 32];
  const unsigned long long warps = (unsigned long long)gridDim.x * kWarpsPerBlock;
  unsigned long long top[kArenas];
#pragma unroll
  for (int a = 0; a < kArenas; ++a) top[a] = S.top[a];
  unsigned long long t_live = 0, t_wsum = 0, t_members = 0, t_slots = 0;

  for (unsigned long long u = (unsigned long long)blockIdx.x * kWarpsPerBlock + threadIdx.x / 32; u < S.n;
       u += warps) {
    const VertexMeta M = S.meta[u];
    const VertexRec R = S.vrec[u];
    const GroupDesc G = S.gdesc[(size_t)u * kBits + lane];
    const unsigned long long hcap = R.hmask ? (unsigned long long)R.hmask + 1 : 0;
    uint32_t bad = 0;

    // --- extents: every offset against the used part of its arena ---
    if (M.ecnt > M.ecap || !within(M.eoff, M.ecap, top[A_EDGE])) bad |= BINGO_CHECK_EXTENT;
    if (M.bpcnt > M.bpcap || !within(M.bpoff, M.bpcap, top[A_BP])) bad |= BINGO_CHECK_EXTENT;
    if (!group_extent_ok(G, top[A_MEMBER])) bad |= BINGO_CHECK_EXTENT;
    if (R.m > M.acap || (M.acap && !within(R.aoff, M.acap, top[A_ALIAS]))) bad |= BINGO_CHECK_EXTENT;
    if (S.node2vec) {
      if (hcap != M.hcap || (hcap & (hcap - 1)) || (hcap && !within(R.hoff, hcap, top[A_HASH])))
        bad |= BINGO_CHECK_EXTENT;
    } else if (hcap || M.hcap) {
      bad |= BINGO_CHECK_EXTENT;
    }
    if (M.live > M.ecnt) bad |= BINGO_CHECK_COUNT;
    bad = __reduce_or_sync(kFull, bad);

    uint32_t live = 0;
    unsigned long long ws = 0;
    const unsigned long long members = warp_sum_u64(G.cnt);
    const uint32_t nz = __ballot_sync(kFull, G.cnt != 0);
    bool handed_off = false;
    if (!(bad & BINGO_CHECK_EXTENT)) {
      // --- live slots: range, back-pointer runs, per-bit counts, adjacency ---
      uint32_t bitcnt = 0;  // lane k: live slots whose weight has bit k
      for (unsigned long long c = 0; c < M.ecnt; c += 32) {
        const unsigned long long i = c + lane;
        EdgeRec e{0, 0, 0, 0};
        if (i < M.ecnt) e = S.edges[M.eoff + i];
        if (e.w) {
          ++live;
          ws += e.w;
          if (e.v >= S.n) bad |= BINGO_CHECK_RANGE;
          if ((unsigned long long)e.ebp + __popc(e.w) > M.bpcnt) bad |= BINGO_CHECK_MEMBER;
          if (S.node2vec && hcap && !hash_has(S.hash + R.hoff, R.hmask, e.v)) bad |= BINGO_CHECK_HASH;
        }
        uint32_t present = __reduce_or_sync(kFull, e.w);
        while (present) {
          const int k = __ffs(present) - 1;
          present &= present - 1;
          const uint32_t b = __ballot_sync(kFull, (e.w >> k) & 1u);
          if (lane == k) bitcnt += __popc(b);
        }
      }
      live = warp_sum_u32(live);
      ws = warp_sum_u64(ws);
      if (live != M.live || bitcnt != G.cnt) bad |= BINGO_CHECK_COUNT;

      // --- alias table: slot j is the j-th nonzero group; the slots carry
      //     exactly the scaled mass (cnt_k << k) * m of every group ---
      const uint32_t m = __popc(nz);
      if (R.m != m) {
        bad |= BINGO_CHECK_ALIAS;
      } else if (m) {
        const unsigned long long T = warp_sum_u64((unsigned long long)G.cnt << lane);
        AliasRec a{};
        const bool mine = (uint32_t)lane < m;
        if (mine) a = S.alias[R.aoff + lane];
        const int own = mine ? nth_set_bit(nz, lane) : 0;
        // lane k: the (ref, count word) its group is named by in the table
        // (a one-member group by its member; extents were checked above).
        const uint32_t gref = G.cnt == 1 ? S.gv[(size_t)group_base(G) * 4] : group_base(G);
        const uint32_t gcw = G.cnt == 1 ? (kInlineGroup | (uint32_t)lane) : (uint32_t)G.cnt;
        const uint32_t own_ref = __shfl_sync(kFull, gref, own), own_cw = __shfl_sync(kFull, gcw, own);
        int alt = -1;
        for (int l = 0; l < 32; ++l) {
          const uint32_t rl = __shfl_sync(kFull, gref, l), cl = __shfl_sync(kFull, gcw, l);
          if (mine && alt < 0 && ((nz >> l) & 1u) && rl == a.alt_ref && cl == a.alt_cw) alt = l;
        }
        if (mine && (a.T != T || a.thr > T || a.own_ref != own_ref || a.own_cw != own_cw || alt < 0))
          bad |= BINGO_CHECK_ALIAS;
        unsigned __int128 acc = 0;
        for (uint32_t j = 0; j < m; ++j) {
          const unsigned long long thr = __shfl_sync(kFull, a.thr, j);
          const int oj = __shfl_sync(kFull, own, j), aj = __shfl_sync(kFull, alt, j);
          if (lane == oj) acc += thr;
          if (lane == aj && thr <= T) acc += T - thr;
        }
        const unsigned __int128 want = (unsigned __int128)((unsigned long long)G.cnt << lane) * m;
        if (acc != want) bad |= BINGO_CHECK_ALIAS;
      }

      // --- adjacency index totals (node2vec handles) ---
      if (S.node2vec) {
        if (live && !hcap) bad |= BINGO_CHECK_HASH;
        uint32_t keys = 0, cnts = 0;
        unsigned long long hw = 0;
        for (unsigned long long h = lane; h < hcap; h += 32) {
          const HashEntry E = S.hash[R.hoff + h];
          if (E.key == kEmptyKey) continue;
          ++keys;
          cnts += (uint32_t)E.cnt;
          hw += E.wsum;
          if (E.cnt < 0 || (E.cnt > 0 && (uint32_t)E.key >= S.n)) bad |= BINGO_CHECK_HASH;
        }
        keys = warp_sum_u32(keys);
        cnts = warp_sum_u32(cnts);
        hw = warp_sum_u64(hw);
        if (hcap && (keys != M.hkeys || cnts != live || hw != ws)) bad |= BINGO_CHECK_HASH;
      }

      // --- group members: here, or by a whole CTA for a large vertex ---
      bad = __reduce_or_sync(kFull, bad);
      if (members > kBigMembers) {
        uint32_t slot = 0;
        if (lane == 0) slot = atomicAdd(&out->n_big, 1u);
        slot = __shfl_sync(kFull, slot, 0);
        if (slot < big_cap) {
          if (lane == 0) big[slot] = BigVertex{(uint32_t)u, bad};
          handed_off = true;
        }
      }
      if (!handed_off) {
        build_index(X, G, lane);
        __syncwarp();
        bad |= check_members(S, M, X, lane, 32, members);
        __syncwarp();
      }
    }
    bad = __reduce_or_sync(kFull, bad);
    if (lane == 0) {
      t_live += live;
      t_wsum += ws;
      t_members += members;
      t_slots += __popc(nz);
      if (bad && !handed_off) count_bad(out, (uint32_t)u, bad);
    }
  }
  if (lane == 0) {
    atomicAdd(&out->live, t_live);
    atomicAdd(&out->wsum, t_wsum);
    atomicAdd(&out->members, t_members);
    atomicAdd(&out->slots, t_slots);
  }
}

// One CTA per large vertex (block-stride over the list k_check wrote); the
// vertex's other checks already passed their extents there.
__global__ void __launch_bounds__(kBigBlock) k_check_big(StoreView S, CheckTotals* out, const BigVertex* big,
                                                         uint32_t big_cap) {
  __shared__ GroupIndex X;
  __shared__ uint32_t s_bad;
  const uint32_t nb = min(*(volatile uint32_t*)&out->n_big, big_cap);
  const unsigned long long top_member = S.top[A_MEMBER];
  for (uint32_t b = blockIdx.x; b < nb; b += gridDim.x) {
    const BigVertex V = big[b];
    const bool ok_u = V.u < S.n;
    if (threadIdx.x == 0) s_bad = ok_u ? 0u : (uint32_t)BINGO_CHECK_EXTENT;
    __syncthreads();
    if (threadIdx.x < 32 && ok_u) {
      const GroupDesc G = S.gdesc[(size_t)V.u * kBits + threadIdx.x];
      if (__any_sync(kFull, !group_extent_ok(G, top_member))) {
        if (threadIdx.x == 0) s_bad = BINGO_CHECK_EXTENT;
      } else {
        build_index(X, G, threadIdx.x);
      }
    }
    __syncthreads();
    const bool run = s_bad == 0;
    __syncthreads();  // every thread has read s_bad before any sets it
    if (run) {
      const VertexMeta M = S.meta[V.u];
      const uint32_t bad = check_members(S, M, X, threadIdx.x, kBigBlock, X.off[kBits]);
      if (bad) atomicOr(&s_bad, bad);
    }
    __syncthreads();
    if (threadIdx.x == 0 && (V.bad | s_bad)) count_bad(out, ok_u ? V.u : 0xffffffffu, V.bad | s_bad);
    __syncthreads();
  }
}

}  // namespace

void Engine::check_store(bingo_check_report* out) {
  read_tops();
  CheckTotals zero{};
  zero.first_bad = 0xffffffffu;
  check_buf_.ensure(sizeof(CheckTotals), "store check");
  // A sound store's vertices with more than kBigMembers members each own
  // that many entries of the used member arena, so this many list entries
  // suffice; a corrupt store that needs more is checked in place.
  const uint32_t big_cap = (uint32_t)std::min<unsigned long long>(n_, h_top_[A_MEMBER] / kBigMembers + 1);
  check_big_.ensure((size_t)big_cap * sizeof(BigVertex), "store check");
  cuda_check(cudaMemcpyAsync(check_buf_.p, &zero, sizeof zero, cudaMemcpyHostToDevice, stream_), "store check");
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_check, kCheckBlock, 0) != cudaSuccess || per_sm <= 0) {
    cudaGetLastError();
    per_sm = 4;
  }
  int sms = 0;
  cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cfg_.device), "device query");
  const uint64_t want = ((uint64_t)n_ + kWarpsPerBlock - 1) / kWarpsPerBlock;
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sms * per_sm));
  const StoreView S = view();
  k_check<<<grid, kCheckBlock, 0, stream_>>>(S, check_buf_.as<CheckTotals>(), check_big_.as<BigVertex>(), big_cap);
  cuda_check(cudaGetLastError(), "store check");
  k_check_big<<<2 * sms, kBigBlock, 0, stream_>>>(S, check_buf_.as<CheckTotals>(), check_big_.as<BigVertex>(),
                                                  big_cap);
  cuda_check(cudaGetLastError(), "store check");
  launches_ += 2;
  CheckTotals t{};
  cuda_check(cudaMemcpyAsync(&t, check_buf_.p, sizeof t, cudaMemcpyDeviceToHost, stream_), "store check");
  cuda_check(cudaStreamSynchronize(stream_), "store check");
  out->vertices = n_;
  out->live_edges = t.live;
  out->weight_sum = t.wsum;
  out->members = t.members;
  out->alias_slots = t.slots;
  out->bad_vertices = t.bad;
  out->kinds = t.kinds;
  out->first_bad = t.first_bad;
}

void Engine::check(bingo_check_report* out) {
  const NvtxRange nvtx_("bingo check");
  require_loaded();
  require_idle();
  check_store(out);
  if (out->bad_vertices)
    throw Error(BINGO_ERR_CORRUPT, "graph store check failed: " + std::to_string(out->bad_vertices) +
                                       " vertices, first " + std::to_string(out->first_bad) + ", kinds " +
                                       std::to_string(out->kinds));
}

}  // namespace bingo
