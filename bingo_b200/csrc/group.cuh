// Stable grouping of an update batch by vertex in one thread-block cluster.
//
// A batch of up to kGroupMax edges is sorted by source vertex (stable: the
// edges of one vertex keep their batch order, the order the reference's
// per-edge loop applies them in, include/operation.cuh:122-251) entirely in
// the distributed shared memory of one cluster: least-significant-digit
// radix passes of 10 bits (two passes for up to 2^20 vertices), each CTA
// ranking its chunk with warp ballots and scattering every item straight
// into the shared memory of the CTA that owns its new position. The same
// launch zeroes the batch status word, validates the batch, writes the
// sorted columns (key, batch index, payload gathered by batch index) and the
// list of segment starts. It replaces the validate / radix sort / gather /
// segment-select launch sequence for the small batches that dominate
// streaming updates. Fixed costs (cluster barriers, remote shared-memory
// latency) favour 8 CTAs up to kGroupSmallMax edges and 16 CTAs above.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"

namespace bingo {

constexpr int kGroupThreads = 1024;
constexpr int kGroupWarps = kGroupThreads / 32;
constexpr int kGroupDigitBits = 10;
constexpr int kGroupBins = 1 << kGroupDigitBits;
// Per cluster size: items per thread and pass at most (shared memory bound).
constexpr int kGroupIptSmall = 8;  // 8 CTAs
constexpr int kGroupIptLarge = 6;  // 16 CTAs (non-portable cluster size)
constexpr uint32_t kGroupSmallMax = 12288;
constexpr uint32_t kGroupMax = 16u * kGroupThreads * kGroupIptLarge;  // 98,304 edges

// Items per thread for a batch of k edges on `ctas` CTAs (k >= 1).
inline uint32_t group_ipt(uint64_t k, int ctas) {
  const uint64_t per = (uint64_t)ctas * kGroupThreads;
  return (uint32_t)((k + per - 1) / per);
}
// Dynamic shared memory of one CTA: two buffers of (key, batch index) pairs
// and the per-warp digit counters.
inline size_t group_smem_bytes(uint32_t ipt) {
  return (size_t)2 * ipt * kGroupThreads * sizeof(uint2) + (size_t)kGroupWarps * kGroupBins * sizeof(uint16_t);
}

// key: source vertex of each edge; a: second column (destination for an
// insert, slot for a delete); b: weights or null. check_payload: a must be
// < n and b nonzero (inserts). Outputs, for positions g < k in sorted order:
// key_s[g], perm[g] (batch index), sa[g] = a[perm[g]], sb[g] = b[perm[g]];
// seg[0..*nseg) the positions where a new vertex starts. ctl[0..4) is zeroed
// and then gets the batch's validation bits (also OR-ed into err).
// Launch: a cluster of CTAS CTAs x kGroupThreads, group_smem_bytes(ipt)
// dynamic shared memory, ipt = group_ipt(k, CTAS) <= IPT_MAX.
template <int CTAS, int IPT_MAX>
__global__ void __launch_bounds__(kGroupThreads, 1)
    k_group_small(const uint32_t* __restrict__ key, const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                  uint32_t k, uint32_t n, int end_bit, uint32_t ipt, int check_payload, uint32_t* __restrict__ key_s,
                  uint32_t* __restrict__ perm, uint32_t* __restrict__ sa, uint32_t* __restrict__ sb,
                  uint32_t* __restrict__ seg, uint32_t* __restrict__ nseg, uint32_t* ctl, uint32_t* err) {
  namespace cg = cooperative_groups;
  constexpr int BINS = kGroupBins, BITS = kGroupDigitBits;
  static_assert(BINS == kGroupThreads, "one thread per digit in the digit scans");
  extern __shared__ uint2 g_items[];
  __shared__ uint32_t hist[BINS];   // this CTA's digit counts (read by the whole cluster)
  __shared__ uint32_t gbase[BINS];  // first global position of this CTA's items per digit
  __shared__ uint32_t wsum[kGroupWarps];
  __shared__ uint32_t wc[IPT_MAX * 32];
  __shared__ uint32_t heads, cta_heads[CTAS];
  cg::cluster_group cluster = cg::this_cluster();
  const uint32_t c = cluster.block_rank();
  const uint32_t t = threadIdx.x, w = t >> 5, l = t & 31;
  const uint32_t chunk = ipt * kGroupThreads;  // this CTA owns global positions [c * chunk, (c + 1) * chunk)
  // __umulhi(pos, cmagic) == pos / chunk for every pos < CTAS * chunk: with
  // cmagic = ceil(2^32 / chunk) the error is below pos / 2^32 < 2^-15 and
  // pos % chunk <= chunk - 1 < chunk * (1 - 2^-15) (chunk < 2^15).
  const uint32_t cmagic = (uint32_t)((0x100000000ull + chunk - 1) / chunk);
  uint2* in = g_items;                         // in[j] holds global position c * chunk + j
  uint2* out = g_items + chunk;
  uint16_t (*cnt)[BINS] = reinterpret_cast<uint16_t (*)[BINS]>(g_items + 2 * chunk);  // per warp and digit

  pdl_wait();  // launched with programmatic serialization: the batch and ctl are ready after this
  pdl_trigger();
  if (c == 0 && t < 4) {
    ctl[t] = 0;
    __threadfence();
  }
  // Positions past the batch hold all-ones keys: they take the last digit in
  // every pass and, placed after every edge, stay at positions >= k.
  {
    uint32_t kv[IPT_MAX];
#pragma unroll
    for (int i = 0; i < IPT_MAX; ++i) {
      const uint32_t g = c * chunk + i * kGroupThreads + t;
      kv[i] = (i < (int)ipt && g < k) ? key[g] : 0xFFFFFFFFu;
      // The payload is gathered by batch index after the sort: bring the
      // 128-byte lines this warp's positions cover into L2 now.
      if (i < (int)ipt && g < k && (l == 0 || l == 31)) {
        asm volatile("prefetch.global.L2 [%0];" ::"l"(a + g));
        if (b) asm volatile("prefetch.global.L2 [%0];" ::"l"(b + g));
      }
    }
#pragma unroll
    for (int i = 0; i < IPT_MAX; ++i)
      if (i < (int)ipt) in[i * kGroupThreads + t] = make_uint2(kv[i], c * chunk + i * kGroupThreads + t);
  }
  __syncthreads();

  // Ranking order inside the CTA: item (warp w, i, lane l) is local position
  // w * 32 * ipt + i * 32 + l; a warp ranks its items in (i, l) order.
  const uint32_t wbase = w * 32 * ipt;
  for (int shift = 0; shift < end_bit; shift += BITS) {
    const uint32_t mask = end_bit - shift >= BITS ? (uint32_t)BINS - 1 : (1u << (end_bit - shift)) - 1;
    for (uint32_t x = t; x < kGroupWarps * BINS / 8; x += kGroupThreads)
      reinterpret_cast<uint4*>(&cnt[0][0])[x] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    uint32_t rk[IPT_MAX];
#pragma unroll
    for (int i = 0; i < IPT_MAX; ++i) {
      rk[i] = 0;
      if (i < (int)ipt) {
        const uint32_t d = (in[wbase + i * 32 + l].x >> shift) & mask;
        uint32_t peers = kFull;  // lanes holding the same digit
#pragma unroll
        for (int bit = 0; bit < BITS; ++bit) {
          const uint32_t bal = __ballot_sync(kFull, (d >> bit) & 1u);
          peers &= ((d >> bit) & 1u) ? bal : ~bal;
        }
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t old = 0;
        if (l == leader) {
          old = cnt[w][d];
          cnt[w][d] = (uint16_t)(old + __popc(peers));
        }
        old = __shfl_sync(kFull, old, leader);
        rk[i] = old + __popc(peers & ((1u << l) - 1u));
        __syncwarp();
      }
    }
    __syncthreads();
    if (t < BINS / 2) {  // digits 2t and 2t + 1 as one word: exclusive prefix over warps, CTA counts
      // (a CTA holds at most 8,192 items, so the low half never carries into the high one)
      uint32_t* cw = reinterpret_cast<uint32_t*>(&cnt[0][0]);
      uint32_t run = 0;
#pragma unroll
      for (int v = 0; v < kGroupWarps; ++v) {
        const uint32_t x = cw[v * (BINS / 2) + t];
        cw[v * (BINS / 2) + t] = run;
        run += x;
      }
      hist[2 * t] = run & 0xFFFFu;
      hist[2 * t + 1] = run >> 16;
    }
    cluster.sync();  // every CTA's digit counts are complete
    uint32_t tot = 0, before = 0;
#pragma unroll
    for (int r = 0; r < CTAS; ++r) {
      const uint32_t x = cluster.map_shared_rank(hist, r)[t];
      tot += x;
      if ((uint32_t)r < c) before += x;
    }
    uint32_t inc = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, inc, o);
      if (l >= (uint32_t)o) inc += y;
    }
    if (l == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {  // exclusive prefix of the warp totals
      const uint32_t x = wsum[l];
      uint32_t y = x;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t z = __shfl_up_sync(kFull, y, o);
        if (l >= (uint32_t)o) y += z;
      }
      wsum[l] = y - x;
    }
    __syncthreads();
    gbase[t] = wsum[w] + inc - tot + before;  // all smaller digits + this digit in lower-ranked CTAs
    __syncthreads();
#pragma unroll
    for (int i = 0; i < IPT_MAX; ++i) {
      if (i < (int)ipt) {
        const uint2 v = in[wbase + i * 32 + l];
        const uint32_t d = (v.x >> shift) & mask;
        const uint32_t pos = gbase[d] + cnt[w][d] + rk[i];
        const uint32_t r = __umulhi(pos, cmagic);  // pos / chunk
        cluster.map_shared_rank(out, r)[pos - r * chunk] = v;
      }
    }
    cluster.sync();  // the pass's scatter has landed everywhere
    uint2* tmp = in;
    in = out;
    out = tmp;
  }

  // Sorted. Thread t covers local positions j = i * kGroupThreads + t.
  uint2 v[IPT_MAX];
  uint32_t av[IPT_MAX], bv[IPT_MAX], hmask = 0;
  const uint32_t prev_remote = (t == 0 && c > 0) ? cluster.map_shared_rank(in, c - 1)[chunk - 1].x : 0u;
#pragma unroll
  for (int i = 0; i < IPT_MAX; ++i) {
    v[i] = make_uint2(0xFFFFFFFFu, 0u);
    av[i] = bv[i] = 0;
    if (i < (int)ipt) {
      const uint32_t j = i * kGroupThreads + t, g = c * chunk + j;
      v[i] = in[j];
      const uint32_t pk = j > 0 ? in[j - 1].x : prev_remote;
      if (g < k) {
        if (g == 0 || v[i].x != pk) hmask |= 1u << i;
        av[i] = a[v[i].y];
        if (b) bv[i] = b[v[i].y];
      }
    }
  }
  // Segment starts are numbered in position order, (i, warp, lane).
#pragma unroll
  for (int i = 0; i < IPT_MAX; ++i)
    if (i < (int)ipt) {
      const uint32_t bal = __ballot_sync(kFull, (hmask >> i) & 1u);
      if (l == 0) wc[i * 32 + w] = __popc(bal);
    }
  __syncthreads();
  {
    const uint32_t nwc = ipt * 32;
    const bool act = t < 32 * IPT_MAX;
    uint32_t x = 0, incw = 0;
    if (act) {
      x = t < nwc ? wc[t] : 0u;
      incw = x;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, incw, o);
        if (l >= (uint32_t)o) incw += y;
      }
      if (l == 31) wsum[w] = incw;
    }
    __syncthreads();
    if (act) {
      uint32_t p = 0;
      for (uint32_t u = 0; u < w; ++u) p += wsum[u];
      if (t < nwc) wc[t] = p + incw - x;
      if (t == 32 * IPT_MAX - 1) heads = p + incw;
    }
  }
  cluster.sync();  // every CTA's head count is complete
  if (t < (uint32_t)CTAS) cta_heads[t] = *cluster.map_shared_rank(&heads, t);
  __syncthreads();
  uint32_t cb = 0, all = 0;
#pragma unroll
  for (int r = 0; r < CTAS; ++r) {
    all += cta_heads[r];
    if ((uint32_t)r < c) cb += cta_heads[r];
  }
  if (c == 0 && t == 0) *nseg = all;
  uint32_t bits = 0;
  const uint32_t below = (1u << l) - 1u;
#pragma unroll
  for (int i = 0; i < IPT_MAX; ++i) {
    if (i < (int)ipt) {
      const uint32_t g = c * chunk + i * kGroupThreads + t;
      const bool h = (hmask >> i) & 1u;
      const uint32_t bal = __ballot_sync(kFull, h);
      if (g < k) {
        key_s[g] = v[i].x;
        perm[g] = v[i].y;
        sa[g] = av[i];
        if (b) {
          sb[g] = bv[i];
          if (check_payload && bv[i] == 0u) bits |= E_ZERO_WEIGHT;
        }
        if (v[i].x >= n || (check_payload && av[i] >= n)) bits |= E_RANGE;
        if (h) seg[cb + wc[i * 32 + w] + __popc(bal & below)] = g;
      }
    }
  }
  bits = __reduce_or_sync(kFull, bits);
  if (bits && l == 0) {
    atomicOr(ctl, bits);
    atomicOr(err, bits);
  }
  cluster.sync();  // no CTA exits while another may still read its shared memory
}

}  // namespace bingo
