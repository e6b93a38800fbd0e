// Stable grouping of an update batch by vertex in one thread-block cluster.
//
// A batch of up to kGroupMax edges is sorted by source vertex (stable: the
// edges of one vertex keep their batch order, the order the reference's
// per-edge loop applies them in, include/operation.cuh:122-251) entirely in
// the distributed shared memory of an 8-CTA cluster: least-significant-digit
// radix passes of 8 bits, each CTA ranking its chunk with warp match masks
// and scattering every item straight into the shared memory of the CTA that
// owns its new position. The same launch zeroes the batch status word,
// validates the batch, writes the sorted columns (key, batch index, payload
// gathered by batch index) and the list of segment starts. It replaces the
// validate / radix sort / gather / segment-select launch sequence for the
// small batches that dominate streaming updates.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"

namespace bingo {

constexpr int kGroupCtas = 8;  // one portable-size cluster
constexpr int kGroupThreads = 1024;
constexpr int kGroupWarps = kGroupThreads / 32;
constexpr int kGroupIpt = 12;  // items per thread and pass, at most
constexpr uint32_t kGroupMax = (uint32_t)kGroupCtas * kGroupThreads * kGroupIpt;  // 98,304 edges
constexpr int kGroupDigitBits = 8;
constexpr int kGroupBins = 1 << kGroupDigitBits;

// Items per thread for a batch of k edges (1 <= k <= kGroupMax).
inline uint32_t group_ipt(uint64_t k) {
  const uint64_t per = (uint64_t)kGroupCtas * kGroupThreads;
  return (uint32_t)((k + per - 1) / per);
}
// Dynamic shared memory of one CTA: two buffers of (key, batch index) pairs.
inline size_t group_smem_bytes(uint32_t ipt) { return (size_t)2 * ipt * kGroupThreads * sizeof(uint2); }

// key: source vertex of each edge; a: second column (destination for an
// insert, slot for a delete); b: weights or null. check_payload: a must be
// < n and b nonzero (inserts). Outputs, for positions g < k in sorted order:
// key_s[g], perm[g] (batch index), sa[g] = a[perm[g]], sb[g] = b[perm[g]];
// seg[0..*nseg) the positions where a new vertex starts. ctl[0..4) is zeroed
// and then gets the batch's validation bits (also OR-ed into err).
// Launch: grid kGroupCtas x kGroupThreads, group_smem_bytes(ipt) dynamic
// shared memory, ipt = group_ipt(k).
__global__ void __cluster_dims__(kGroupCtas, 1, 1) __launch_bounds__(kGroupThreads, 1)
    k_group_small(const uint32_t* __restrict__ key, const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                  uint32_t k, uint32_t n, int end_bit, uint32_t ipt, int check_payload, uint32_t* __restrict__ key_s,
                  uint32_t* __restrict__ perm, uint32_t* __restrict__ sa, uint32_t* __restrict__ sb,
                  uint32_t* __restrict__ seg, uint32_t* __restrict__ nseg, uint32_t* ctl, uint32_t* err) {
  namespace cg = cooperative_groups;
  extern __shared__ uint2 g_items[];
  __shared__ uint16_t cnt[kGroupWarps][kGroupBins];  // per warp and digit: count, then exclusive prefix
  __shared__ uint32_t hist[kGroupBins];              // this CTA's digit counts (read by the whole cluster)
  __shared__ uint32_t gbase[kGroupBins];             // first global position of this CTA's items per digit
  __shared__ uint32_t wsum[kGroupWarps];
  __shared__ uint32_t heads, cta_heads[kGroupCtas];
  cg::cluster_group cluster = cg::this_cluster();
  const uint32_t c = cluster.block_rank();
  const uint32_t t = threadIdx.x, w = t >> 5, l = t & 31;
  const uint32_t chunk = ipt * kGroupThreads;  // this CTA owns global positions [c * chunk, (c + 1) * chunk)
  uint2* in = g_items;
  uint2* out = g_items + chunk;

  if (c == 0 && t < 4) ctl[t] = 0;
  if (c == 0 && t == 0) __threadfence();
  // Positions past the batch hold all-ones keys: they take the last digit in
  // every pass and, placed after every edge, stay at positions >= k.
  for (uint32_t j = t; j < chunk; j += kGroupThreads) {
    const uint32_t g = c * chunk + j;
    in[j] = make_uint2(g < k ? key[g] : 0xFFFFFFFFu, g);
  }
  __syncthreads();

  // Item (warp w, lane l, i) sits at local position w * 32 * ipt + i * 32 + l,
  // the order in which the match ranking below counts equal digits.
  const uint32_t wbase = w * 32 * ipt;
  for (int shift = 0; shift < end_bit; shift += kGroupDigitBits) {
    const uint32_t mask = end_bit - shift >= kGroupDigitBits ? (uint32_t)kGroupBins - 1 : (1u << (end_bit - shift)) - 1;
    for (uint32_t x = t; x < kGroupWarps * kGroupBins / 2; x += kGroupThreads)
      reinterpret_cast<uint32_t*>(&cnt[0][0])[x] = 0;
    __syncthreads();
    uint32_t rk[kGroupIpt];
#pragma unroll
    for (int i = 0; i < kGroupIpt; ++i) {
      rk[i] = 0;
      if (i < (int)ipt) {
        const uint32_t d = (in[wbase + i * 32 + l].x >> shift) & mask;
        const uint32_t peers = __match_any_sync(kFull, d);
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
    uint32_t tot = 0, before = 0, inc = 0;
    if (t < kGroupBins) {
      uint32_t s = 0;
      for (int v = 0; v < kGroupWarps; ++v) {
        const uint32_t x = cnt[v][t];
        cnt[v][t] = (uint16_t)s;
        s += x;
      }
      hist[t] = s;
    }
    cluster.sync();  // every CTA's digit counts are complete
    if (t < kGroupBins) {
      for (uint32_t r = 0; r < kGroupCtas; ++r) {
        const uint32_t x = cluster.map_shared_rank(hist, r)[t];
        tot += x;
        if (r < c) before += x;
      }
      inc = tot;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, inc, o);
        if (l >= (uint32_t)o) inc += y;
      }
      if (l == 31) wsum[w] = inc;
    }
    __syncthreads();
    if (t < kGroupBins) {
      uint32_t p = 0;
      for (uint32_t v = 0; v < w; ++v) p += wsum[v];
      gbase[t] = p + inc - tot + before;  // all smaller digits + this digit in lower-ranked CTAs
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kGroupIpt; ++i) {
      if (i < (int)ipt) {
        const uint2 v = in[wbase + i * 32 + l];
        const uint32_t d = (v.x >> shift) & mask;
        const uint32_t pos = gbase[d] + cnt[w][d] + rk[i];
        cluster.map_shared_rank(out, pos / chunk)[pos % chunk] = v;
      }
    }
    cluster.sync();  // the pass's scatter has landed everywhere
    uint2* tmp = in;
    in = out;
    out = tmp;
  }

  // Sorted. Thread t covers local positions [t * ipt, (t + 1) * ipt).
  const uint32_t j0 = t * ipt;
  const uint32_t g0 = c * chunk + j0;
  uint32_t prev = 0;  // key before this thread's first position (position 0 is a head regardless)
  if (j0 > 0)
    prev = in[j0 - 1].x;
  else if (c > 0)
    prev = cluster.map_shared_rank(in, c - 1)[chunk - 1].x;
  uint32_t nh = 0;
  {
    uint32_t pk = prev;
    for (uint32_t i = 0; i < ipt; ++i) {
      const uint32_t kk = in[j0 + i].x;
      if (g0 + i < k && (g0 + i == 0 || kk != pk)) ++nh;
      pk = kk;
    }
  }
  uint32_t inc = nh;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, inc, o);
    if (l >= (uint32_t)o) inc += y;
  }
  if (l == 31) wsum[w] = inc;
  __syncthreads();
  if (t == 0) {
    uint32_t s = 0;
    for (int v = 0; v < kGroupWarps; ++v) {
      const uint32_t x = wsum[v];
      wsum[v] = s;
      s += x;
    }
    heads = s;
  }
  cluster.sync();  // every CTA's head count is complete
  if (t < kGroupCtas) cta_heads[t] = *cluster.map_shared_rank(&heads, t);
  __syncthreads();
  uint32_t hb = wsum[w] + inc - nh, all = 0;
  for (uint32_t r = 0; r < kGroupCtas; ++r) {
    all += cta_heads[r];
    if (r < c) hb += cta_heads[r];
  }
  if (c == 0 && t == 0) *nseg = all;
  uint32_t bits = 0, pk = prev;
  for (uint32_t i = 0; i < ipt; ++i) {
    const uint32_t g = g0 + i;
    const uint2 v = in[j0 + i];
    if (g < k) {
      key_s[g] = v.x;
      perm[g] = v.y;
      const uint32_t av = a[v.y];
      sa[g] = av;
      if (b) {
        const uint32_t bv = b[v.y];
        sb[g] = bv;
        if (check_payload && bv == 0u) bits |= E_ZERO_WEIGHT;
      }
      if (v.x >= n || (check_payload && av >= n)) bits |= E_RANGE;
      if (g == 0 || v.x != pk) seg[hb++] = g;
    }
    pk = v.x;
  }
  bits = __reduce_or_sync(kFull, bits);
  if (bits && l == 0) {
    atomicOr(ctl, bits);
    atomicOr(err, bits);
  }
  cluster.sync();  // no CTA exits while another may still read its shared memory
}

}  // namespace bingo
