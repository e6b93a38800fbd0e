// Warp-cooperative operations on the graph store. One warp owns one vertex;
// lane k owns weight bit k (group k) for the whole operation.
#pragma once
#include "common.cuh"

namespace bingo {

// ---------------------------------------------------------------------------
// Integer Vose alias table over the vertex's nonzero groups (lane k = group k).
//
// Slot j belongs to the j-th nonzero group in ascending bit order. Scaled
// mass s_k = (cnt_k << k) * m, each slot holds exactly T scaled units. The
// pairing always takes the lowest small (s < T) and lowest large (s >= T)
// group, so the table is a pure function of the counts. Masks, ranks and
// the total come from ballots and shuffles; the pairing loop runs at most
// m - 1 times. Replaces the single-lane float construction of
// include/Bingo.cuh:111-158.
//
// single: the member of this lane's group when cnt == 1 (the table names a
// one-member group by its member, AliasRec). sc: this warp's shared-memory
// scratch for the pairing loop.
struct AliasScratch {
  unsigned long long s[kBits];    // scaled masses
  unsigned long long thr[kBits];  // thresholds out
  uint8_t al[kBits];              // alias groups out
};

__device__ __forceinline__ uint32_t warp_build_alias(int lane, uint32_t cnt, uint32_t base, uint32_t single,
                                                     AliasRec* out, AliasScratch* sc) {
  const unsigned long long mass = (unsigned long long)cnt << lane;
  const uint32_t nz = __ballot_sync(kFull, cnt != 0);
  const uint32_t m = __popc(nz);
  if (m == 0) return 0;
  const unsigned long long T = warp_sum_u64(mass);
  unsigned long long thr = T;
  int alias_lane = lane;
  if (T < (1ull << 58)) {
    // Every scaled mass is below 32 * 2^58: the pairing in 64 bits, run by
    // lane 0 over shared memory (about half the instructions of a
    // shuffle-per-step loop). The lowest large group stays the partner until
    // it turns small (larges are never added), so its residual lives in a
    // register meanwhile.
    const unsigned long long s = mass * m;
    uint32_t small = __ballot_sync(kFull, cnt != 0 && s < T);
    uint32_t large = nz & ~small;
    if (small && large) {
      sc->s[lane] = s;
      sc->thr[lane] = T;
      sc->al[lane] = (uint8_t)lane;
      __syncwarp();
      if (lane == 0) {
        int b = -1;
        unsigned long long sb = 0;
        while (small && large) {
          const int a = __ffs(small) - 1;
          if (b < 0) b = __ffs(large) - 1, sb = sc->s[b];
          const unsigned long long sa = sc->s[a];
          sc->thr[a] = sa;
          sc->al[a] = (uint8_t)b;
          sb -= T - sa;
          small &= ~(1u << a);
          if (sb < T) {
            sc->s[b] = sb;
            large &= ~(1u << b);
            small |= 1u << b;
            b = -1;
          }
        }
      }
      __syncwarp();
      thr = sc->thr[lane];
      alias_lane = sc->al[lane];
      __syncwarp();  // the scratch is reused by this warp's next vertex
    }
  } else {
    unsigned __int128 s = (unsigned __int128)mass * m;
    uint32_t small = __ballot_sync(kFull, cnt != 0 && s < T);
    uint32_t large = nz & ~small;
    while (small && large) {
      const int a = __ffs(small) - 1, b = __ffs(large) - 1;
      const unsigned long long sa = __shfl_sync(kFull, (unsigned long long)s, a);  // s_a < T fits 64 bits
      if (lane == a) {
        thr = sa;
        alias_lane = b;
      }
      if (lane == b) s -= (unsigned __int128)(T - sa);
      small &= ~(1u << a);
      const bool b_small = __shfl_sync(kFull, (int)(s < T), b);
      if (b_small) {
        large &= ~(1u << b);
        small |= 1u << b;
      }
    }
  }
  // Remaining groups hold exactly T: thr = T, alias = self (already set).
  // A one-member group is named by its member (AliasRec).
  const uint32_t ref = cnt == 1 ? single : base;
  const uint32_t cw = cnt == 1 ? (kInlineGroup | (uint32_t)lane) : cnt;
  const uint32_t alt_ref = __shfl_sync(kFull, ref, alias_lane);
  const uint32_t alt_cw = __shfl_sync(kFull, cw, alias_lane);
  if (cnt) {
    const uint32_t j = __popc(nz & lanemask_lt());
    AliasRec r;
    r.thr = thr;
    r.T = T;
    r.own_ref = ref;
    r.own_cw = cw;
    r.alt_ref = alt_ref;
    r.alt_cw = alt_cw;
    out[j] = r;
  }
  return m;
}

// ---------------------------------------------------------------------------
// Adjacency index (node2vec), linear probing on mix32: per neighbour the
// live edge count and live weight sum.
__device__ __forceinline__ void hash_add(HashEntry* tab, uint32_t hmask, uint32_t v, uint32_t w, uint32_t* claimed) {
  uint32_t h = mix32(v) & hmask;
  for (uint32_t probe = 0; probe <= hmask; ++probe) {
    const int prev = atomicCAS(&tab[h].key, kEmptyKey, (int)v);
    if (prev == kEmptyKey || prev == (int)v) {
      atomicAdd(&tab[h].cnt, 1);
      atomicAdd(&tab[h].wsum, (unsigned long long)w);
      if (prev == kEmptyKey) ++*claimed;
      return;
    }
    h = (h + 1) & hmask;
  }
}

__device__ __forceinline__ void hash_sub(HashEntry* tab, uint32_t hmask, uint32_t v, uint32_t w) {
  uint32_t h = mix32(v) & hmask;
  for (uint32_t probe = 0; probe <= hmask; ++probe) {
    const int k = tab[h].key;
    if (k == (int)v) {
      atomicSub(&tab[h].cnt, 1);
      atomicAdd(&tab[h].wsum, 0ull - (unsigned long long)w);
      return;
    }
    if (k == kEmptyKey) return;
    h = (h + 1) & hmask;
  }
}

// Index of v's entry, or -1.
__device__ __forceinline__ int hash_find(const HashEntry* tab, uint32_t hmask, uint32_t v) {
  uint32_t h = mix32(v) & hmask;
  for (uint32_t probe = 0; probe <= hmask; ++probe) {
    const int k = __ldg(&tab[h].key);
    if (k == (int)v) return (int)h;
    if (k == kEmptyKey) return -1;
    h = (h + 1) & hmask;
  }
  return -1;
}

__device__ __forceinline__ bool hash_has(const HashEntry* tab, uint32_t hmask, uint32_t v) {
  const int h = hash_find(tab, hmask, v);
  return h >= 0 && __ldg(&tab[h].cnt) > 0;
}

// Live weight sum of the edges to v (0 when there are none).
__device__ __forceinline__ unsigned long long hash_weight(const HashEntry* tab, uint32_t hmask, uint32_t v) {
  const int h = hash_find(tab, hmask, v);
  return h >= 0 && __ldg(&tab[h].cnt) > 0 ? __ldg(&tab[h].wsum) : 0ull;
}

// ---------------------------------------------------------------------------
// Growth plan for appending `len` edges to a vertex. All lanes compute the
// same values; lane k also knows whether group k grows and to what capacity.
struct GrowPlan {
  uint32_t new_ecap;   // 0 = no edge relocation
  uint32_t new_bpcap;  // 0 = no back-pointer relocation
  uint32_t new_acap;   // 0 = alias table fits
  uint32_t new_hcap;   // 0 = adjacency index fits
  uint32_t gcap_lane;  // this lane's new group capacity, 0 = fits
  uint32_t gsum;       // sum over lanes of gcap_lane
  uint32_t gpre;       // exclusive prefix of gcap_lane over lanes
};

// add_lane: how many of the appended edges carry bit `lane`; pc_total: sum of
// their popcounts. Called with the whole warp.
__device__ __forceinline__ GrowPlan plan_growth(int lane, const VertexMeta& M, const GroupDesc& G, uint32_t len,
                                                uint32_t add_lane, uint32_t pc_total, uint32_t node2vec) {
  GrowPlan p;
  const uint32_t ecnt = M.ecnt + len;
  p.new_ecap = ecnt > M.ecap ? pow2_at_least(ecnt, kMinEdgeCap) : 0;
  const uint32_t bpn = M.bpcnt + pc_total;
  p.new_bpcap = bpn > M.bpcap ? pow2_at_least(bpn, kMinEdgeCap) : 0;
  const uint32_t cnt = G.cnt + add_lane;
  p.gcap_lane = cnt > group_cap(G) ? pow2_at_least(cnt, kMinGroupCap) : 0;
  const uint32_t incl = warp_incl_scan(p.gcap_lane, lane);
  p.gsum = __shfl_sync(kFull, incl, 31);
  p.gpre = incl - p.gcap_lane;
  const uint32_t m = __popc(__ballot_sync(kFull, cnt != 0));
  p.new_acap = m > M.acap ? pow2_at_least(m, 1) : 0;
  p.new_hcap = 0;
  if (node2vec && (M.hkeys + len > M.hcap / 2)) p.new_hcap = pow2_at_least(2 * (M.live + len), kMinHashCap);
  return p;
}

// Per-lane count of segment edges carrying bit `lane`, and the segment's
// total popcount, from one ballot per bit per 32 edges.
__device__ __forceinline__ void count_bits(int lane, const uint32_t* seg_w, uint32_t len, uint32_t* add_lane,
                                           uint32_t* pc_total) {
  if (len == 1) {  // one edge (the common case): lane k counts bit k of its weight
    const uint32_t w = seg_w[0];
    *add_lane = (w >> lane) & 1u;
    *pc_total = __popc(w);
    return;
  }
  uint32_t add = 0, pc = 0;
  for (uint32_t c = 0; c < len; c += 32) {
    const uint32_t i = c + lane;
    const uint32_t w = i < len ? seg_w[i] : 0u;
    pc += __popc(w);
    uint32_t present = __reduce_or_sync(kFull, w);
    while (present) {
      const int k = __ffs(present) - 1;
      present &= present - 1;
      const uint32_t b = __ballot_sync(kFull, (w >> k) & 1u);
      if (lane == k) add += __popc(b);
    }
  }
  *add_lane = add;
  *pc_total = warp_sum_u32(pc);
}

// Warp copy of n 16-byte units between non-overlapping ranges, two 16-byte
// loads per lane in flight (a relocation of thousands of entries costs tens
// of round trips, not one per 32 entries; four in flight pushed the insert
// kernel past 64 registers).
__device__ __forceinline__ void warp_copy_v4(uint4* __restrict__ dst, const uint4* __restrict__ src, uint32_t n,
                                             int lane) {
  uint32_t i = lane;
  for (; i + 32 < n; i += 64) {
    const uint4 a = src[i], b = src[i + 32];
    dst[i] = a;
    dst[i + 32] = b;
  }
  for (; i < n; i += 32) dst[i] = src[i];
}

// Warp copy of the first n 32-bit entries of a list or pool that starts on a
// 16-byte boundary into another such range, rounded up to whole 16-byte
// units (both ranges hold at least that many entries: capacities are powers
// of two >= 4).
__device__ __forceinline__ void warp_copy_u32(uint32_t* dst, const uint32_t* src, uint32_t n, int lane) {
  warp_copy_v4(reinterpret_cast<uint4*>(dst), reinterpret_cast<const uint4*>(src), (n + 3) / 4, lane);
}

// ---------------------------------------------------------------------------
// Apply a growth plan (relocations drawn from per-arena bases reserved for
// this segment), append the segment's edges in order, refresh the adjacency
// index and rebuild the alias table. Replaces NodeData::copy / insert /
// buildAliasTable (include/Bingo.cuh:95-110, :182-198, :111-158) and the host
// reMalloc round trip (include/operation.cuh:163-174).
//
// seg_v / seg_w / seg_orig: the segment's edges in batch order; out_slots is
// indexed by seg_orig (may be null). res[a]: the arena offsets reserved for
// this segment (units of each arena).
static __device__ void apply_append(const StoreView& S, uint32_t u, const uint32_t* seg_v, const uint32_t* seg_w,
                             const uint32_t* seg_orig, uint32_t len, uint32_t* out_slots,
                             const unsigned long long res[kArenas], AliasScratch* sc) {
  const int lane = threadIdx.x & 31;
  VertexMeta M = S.meta[u];
  GroupDesc G = S.gdesc[(size_t)u * kBits + lane];
  const uint32_t cap0 = group_cap(G);
  uint32_t add_lane, pc_total;
  count_bits(lane, seg_w, len, &add_lane, &pc_total);
  const GrowPlan P = plan_growth(lane, M, G, len, add_lane, pc_total, S.node2vec);
  // Loaded here, before any store of this warp: the vertex record, and the
  // member of a one-member group the batch leaves alone (the alias table
  // names such a group by its member).
  VertexRec R = S.vrec[u];
  uint32_t single = G.cnt == 1 && add_lane == 0 ? S.gv[(size_t)group_base(G) * 4] : 0u;

  // --- relocations (old contents keep their order) ---
  if (P.new_ecap) {
    warp_copy_v4(reinterpret_cast<uint4*>(S.edges + res[A_EDGE]), reinterpret_cast<const uint4*>(S.edges + M.eoff),
                 M.ecnt, lane);
    M.eoff = res[A_EDGE];
    M.ecap = P.new_ecap;
  }
  if (P.new_bpcap) {
    warp_copy_u32(S.bp + res[A_BP], S.bp + M.bpoff, M.bpcnt, lane);
    M.bpoff = res[A_BP];
    M.bpcap = P.new_bpcap;
  }
  {
    // Lists that move: the whole warp copies the members of each non-empty
    // one in turn; every moving lane then takes its new base (a list that
    // held no members needs no copy, the common case for a new group).
    const uint32_t old_base = group_base(G);
    uint32_t copy = __ballot_sync(kFull, P.gcap_lane != 0 && G.cnt != 0);
    if (P.gcap_lane) {
      G.base1 = (uint32_t)((res[A_MEMBER] + P.gpre) >> 2) + 1u;  // reserved offsets are 4-entry aligned
      G.roomy = 0;
    }
    while (copy) {
      const int k = __ffs(copy) - 1;
      copy &= copy - 1;
      const uint32_t ob = __shfl_sync(kFull, old_base, k), oc = __shfl_sync(kFull, G.cnt, k);
      const size_t nb = (size_t)__shfl_sync(kFull, group_base(G), k) * 4;
      warp_copy_u32(S.gv + nb, S.gv + (size_t)ob * 4, oc, lane);
      warp_copy_u32(S.gs + nb, S.gs + (size_t)ob * 4, oc, lane);
    }
  }
  if (P.new_acap) {
    R.aoff = (uint32_t)res[A_ALIAS];
    M.acap = P.new_acap;
  }
  __syncwarp();

  // --- append in batch order ---
  uint32_t bpbase = M.bpcnt;
  if (len == 1) {
    // One edge: lane k appends it to group k at position cnt_k when its
    // weight has bit k (the same positions the general loop gives).
    const uint32_t v = seg_v[0], w = seg_w[0], slot = M.ecnt;
    if (lane == 0) {
      S.edges[M.eoff + slot] = EdgeRec{v, w, bpbase, 0u};
      if (out_slots) out_slots[seg_orig[0]] = slot;
    }
    if ((w >> lane) & 1u) {
      const uint32_t pos = G.cnt, bi = bpbase + __popc(w & ((1u << lane) - 1u));
      const size_t e = (size_t)group_base(G) * 4 + pos;
      S.gv[e] = v;
      S.gs[e] = bi;
      S.bp[M.bpoff + bi] = pos;
      if (pos == 0) single = v;
      ++G.cnt;
    }
    bpbase += __popc(w);
  }
  for (uint32_t c = 0; len > 1 && c < len; c += 32) {
    const uint32_t i = c + lane;
    const bool valid = i < len;
    const uint32_t v = valid ? seg_v[i] : 0u, w = valid ? seg_w[i] : 0u;
    const uint32_t pc = __popc(w);
    const uint32_t incl = warp_incl_scan(pc, lane);
    const uint32_t ebp = bpbase + incl - pc;
    bpbase += __shfl_sync(kFull, incl, 31);
    const uint32_t slot = M.ecnt + i;
    if (valid) {
      S.edges[M.eoff + slot] = EdgeRec{v, w, ebp, 0u};
      if (out_slots) out_slots[seg_orig[i]] = slot;
    }
    uint32_t present = __reduce_or_sync(kFull, w);
    while (present) {
      const int k = __ffs(present) - 1;
      present &= present - 1;
      const bool has = (w >> k) & 1u;
      const uint32_t b = __ballot_sync(kFull, has);
      const uint32_t kcnt = __shfl_sync(kFull, G.cnt, k), kbase = __shfl_sync(kFull, group_base(G), k);
      if (has) {
        const uint32_t pos = kcnt + __popc(b & lanemask_lt()), bi = ebp + __popc(w & ((1u << k) - 1u));
        const size_t e = (size_t)kbase * 4 + pos;
        S.gv[e] = v;
        S.gs[e] = bi;
        S.bp[M.bpoff + bi] = pos;
      }
      const uint32_t first_v = __shfl_sync(kFull, v, __ffs(b) - 1);  // b != 0: bit k is present
      if (lane == k) {
        if (kcnt == 0) single = first_v;
        G.cnt += __popc(b);
      }
    }
  }
  M.ecnt += len;
  M.bpcnt = bpbase;
  M.live += len;
  __syncwarp();

  // --- adjacency index ---
  if (S.node2vec) {
    uint32_t claimed = 0;
    if (P.new_hcap) {
      // Rebuild from every live slot into a fresh table.
      HashEntry* tab = S.hash + res[A_HASH];
      for (uint32_t i = lane; i < P.new_hcap; i += 32) tab[i] = HashEntry{kEmptyKey, 0, 0ull};
      __syncwarp();
      for (uint32_t i = lane; i < M.ecnt; i += 32) {
        const EdgeRec e = S.edges[M.eoff + i];
        if (e.w) hash_add(tab, P.new_hcap - 1, e.v, e.w, &claimed);
      }
      R.hoff = (uint32_t)res[A_HASH];
      R.hmask = P.new_hcap - 1;
      M.hcap = P.new_hcap;
      M.hkeys = warp_sum_u32(claimed);
    } else {
      for (uint32_t i = lane; i < len; i += 32) hash_add(S.hash + R.hoff, R.hmask, seg_v[i], seg_w[i], &claimed);
      M.hkeys += warp_sum_u32(claimed);
    }
  }
  __syncwarp();

  // --- alias table over the new counts ---
  R.m = warp_build_alias(lane, G.cnt, group_base(G), single, S.alias + R.aoff, sc);
  if (add_lane && !P.gcap_lane) G.roomy = group_roomy(G.cnt, cap0);
  if (add_lane || P.gcap_lane) S.gdesc[(size_t)u * kBits + lane] = G;  // only the descriptors that changed
  if (lane == 0) {
    S.meta[u] = M;
    S.vrec[u] = R;
  }
}

// Per-arena sizes the append of a segment needs (same decisions as
// apply_append). Lane 0 returns them.
__device__ __forceinline__ void plan_append(const StoreView& S, uint32_t u, const uint32_t* seg_w, uint32_t len,
                                            unsigned long long need[kArenas]) {
  const int lane = threadIdx.x & 31;
  const VertexMeta M = S.meta[u];
  const GroupDesc G = S.gdesc[(size_t)u * kBits + lane];
  uint32_t add_lane, pc_total;
  count_bits(lane, seg_w, len, &add_lane, &pc_total);
  const GrowPlan P = plan_growth(lane, M, G, len, add_lane, pc_total, S.node2vec);
  need[A_MEMBER] = P.gsum;
  need[A_EDGE] = P.new_ecap;
  need[A_BP] = P.new_bpcap;
  need[A_ALIAS] = P.new_acap;
  need[A_HASH] = P.new_hcap;
}

// Removals of one group a lane resolves per round of loads (apply_delete).
constexpr int kDeleteRound = 4;

// ---------------------------------------------------------------------------
// Delete a run of slots of one vertex in batch order. Each delete swap-removes
// the slot from every group its weight has a bit in (lane k = group k) and
// then tombstones the slot. Groups are independent, so each lane walks its
// own sequence of removals with no warp synchronisation per delete; the
// slot records of 32 deletes are fetched at once and the tombstones of a
// chunk are written after its removals (the reference also tombstones after
// its removal loop, include/operation.cuh:206-210). A delete is skipped and
// counted when its slot is out of range, already a tombstone, or repeats an
// earlier delete of the batch. Replaces NodeData::deleteE
// (include/Bingo.cuh:199-218) and deleteKernel (include/operation.cuh:198-214).
// stage: 64 words of shared memory owned by this warp.
static __device__ void apply_delete(const StoreView& S, uint32_t u, const uint32_t* seg_slot, uint32_t len,
                                    uint32_t* stage, AliasScratch* sc) {
  const int lane = threadIdx.x & 31;
  const uint32_t below = lanemask_lt();
  VertexMeta M = S.meta[u];
  GroupDesc G = S.gdesc[(size_t)u * kBits + lane];
  VertexRec R = S.vrec[u];
  const size_t gb = (size_t)group_base(G) * 4;
  const uint32_t cnt0 = G.cnt, cap0 = group_cap(G);
  uint32_t rejected = 0;
  bool front_known = false;  // this lane moved a member into position 0
  uint32_t front = 0;
  for (uint32_t c = 0; c < len; c += 32) {
    const uint32_t i = c + lane;
    const uint32_t slot = i < len ? seg_slot[i] : 0xffffffffu;
    EdgeRec e{0, 0, 0, 0};
    if (i < len && slot < M.ecnt) e = S.edges[M.eoff + slot];
    const bool dup = (__match_any_sync(kFull, slot) & below) != 0;
    const bool valid = i < len && e.w != 0 && !dup;
    const uint32_t vmask = __ballot_sync(kFull, valid);
    rejected += __popc(__ballot_sync(kFull, i < len && !valid));
    stage[lane] = valid ? e.w : 0u;
    stage[32 + lane] = e.ebp;
    __syncwarp();
    // This lane's removals, in batch order: the chunk's deletes with bit `lane`.
    uint32_t mine = 0;
    for (uint32_t r = vmask; r; r &= r - 1) {
      const int d = __ffs(r) - 1;
      if ((stage[d] >> lane) & 1u) mine |= 1u << d;
    }
    // Up to kDeleteRound removals at a time: their members' positions and
    // the list's last entries (neighbour and back-pointer index) are loaded
    // together, then the swap-removes run in registers, in batch order, and
    // are stored. A removal whose member was moved by an earlier one, or a
    // last entry that an earlier removal overwrote, is followed in registers
    // (entries are told apart by their back-pointer index, unique per
    // (slot, bit)). Removing the list's last entry itself moves nothing.
    uint32_t* const bpv = S.bp + M.bpoff;
    while (mine) {
      uint32_t bpi[kDeleteRound], pos[kDeleteRound], tv[kDeleteRound], tbi[kDeleteRound];
      int r = 0;
#pragma unroll
      for (int q = 0; q < kDeleteRound; ++q) {
        bpi[q] = 0;
        if (mine) {
          const int d = __ffs(mine) - 1;
          mine &= mine - 1;
          bpi[q] = stage[32 + d] + __popc(stage[d] & below);
          r = q + 1;
        }
      }
      const uint32_t c0 = G.cnt;  // >= r: every removal's member is in the list
#pragma unroll
      for (int q = 0; q < kDeleteRound; ++q) {
        pos[q] = tv[q] = tbi[q] = 0;
        if (q < r) {
          pos[q] = bpv[bpi[q]];
          tbi[q] = S.gs[gb + c0 - 1 - q];
          tv[q] = S.gv[gb + c0 - 1 - q];
        }
      }
#pragma unroll
      for (int i = 0; i < kDeleteRound; ++i) {
        if (i < r) {
          // Removal i: the entry at the current last position (c0 - 1 - i)
          // moves into the removed member's position p.
          const uint32_t p = pos[i], mv = tv[i], mbi = tbi[i];
          if (p != c0 - 1 - i) {
            S.gv[gb + p] = mv;
            S.gs[gb + p] = mbi;
            bpv[mbi] = p;
            if (p == 0) front_known = true, front = mv;
          }
#pragma unroll
          for (int t = i + 1; t < kDeleteRound; ++t) {
            if (t < r && p == c0 - 1 - t) tv[t] = mv, tbi[t] = mbi;  // a later last entry
            if (t < r && bpi[t] == mbi) pos[t] = p;                  // a later removal moved
          }
        }
      }
      G.cnt = c0 - r;
    }
    __syncwarp();
    if (valid) {
      S.edges[M.eoff + slot].w = 0u;
      if (S.node2vec && R.hmask) hash_sub(S.hash + R.hoff, R.hmask, e.v, e.w);
    }
    M.live -= __popc(vmask);
    __syncwarp();
  }
  if (rejected && lane == 0) {
    atomicAdd(&S.err[1], rejected);
    set_err(S.err, E_INVALID_SLOT);
  }
  // A group left with one member is named by it in the alias table.
  const uint32_t single = G.cnt == 1 ? (front_known ? front : S.gv[gb]) : 0u;
  R.m = warp_build_alias(lane, G.cnt, group_base(G), single, S.alias + R.aoff, sc);
  if (G.cnt != cnt0) {  // only the descriptors that changed
    G.roomy = group_roomy(G.cnt, cap0);
    S.gdesc[(size_t)u * kBits + lane] = G;
  }
  if (lane == 0) {
    S.meta[u] = M;
    S.vrec[u] = R;
  }
}

}  // namespace bingo
