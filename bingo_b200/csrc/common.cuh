// Shared device definitions: HBM layout of the graph store, Philox4x32-10,
// multiply-shift range reduction and warp helpers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "philox.cuh"

namespace bingo {

constexpr unsigned kFull = 0xffffffffu;

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may be scheduled while the kernel before it still runs;
// pdl_wait() (first statement of such a kernel) returns once that kernel has
// completed and its memory is visible, and is a no-op for a plain launch.
// pdl_trigger() lets the next kernel be scheduled early (its CTAs then wait
// in pdl_wait()).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
constexpr int kBits = 32;            // weight bits = possible groups per vertex
constexpr uint32_t kMinEdgeCap = 16; // reference ORIGINAL (include/api.h:13)
constexpr uint32_t kMinGroupCap = 4; // member lists are allocated in 16-byte units
constexpr uint32_t kMinHashCap = 8;
constexpr int32_t kEmptyKey = -1;

// ---------------------------------------------------------------------------
// Walk-side records (read by every walk step; 3 dependent loads per step:
// VertexRec -> AliasRec -> member id).

// 16 B, one vector load. m == 0 marks a vertex with no live out-edge.
struct __align__(16) VertexRec {
  uint32_t aoff;   // first AliasRec of this vertex
  uint32_t m;      // alias slots = nonzero bit groups
  uint32_t hoff;   // first HashEntry of the adjacency index
  uint32_t hmask;  // adjacency index capacity - 1 (0 when absent)
};

// 32 B = one sector. Slot j of a vertex: draw r in [0, T); r < thr picks the
// slot's own group, otherwise its alias group. Each group is named by a
// (ref, count word) pair: for a list of two or more members, its base (in
// 4-entry units of the member arena) and its count; for a group of one
// member, that member's neighbour id and kInlineGroup | k (k = the group's
// bit), so a draw that lands there needs no member load.
constexpr uint32_t kInlineGroup = 0x80000000u;
struct __align__(32) AliasRec {
  unsigned long long thr;
  unsigned long long T;
  uint32_t own_ref, own_cw;
  uint32_t alt_ref, alt_cw;
};

struct __align__(16) HashEntry {
  int32_t key;                // neighbour id or kEmptyKey
  int32_t cnt;                // live multiplicity
  unsigned long long wsum;    // live weight sum of the edges to key
};

// ---------------------------------------------------------------------------
// Update-side records.

// One edge slot: neighbour, weight (0 = tombstone, include/operation.cuh:209-210)
// and the start of its back-pointer run (one entry per set weight bit, in
// ascending bit order).
struct __align__(16) EdgeRec {
  uint32_t v, w, ebp, pad;
};

// 8 B (a vertex's 32 descriptors fill two 128-byte lines). The capacity is
// not stored exactly: a list holds at least group_cap() entries, the power of
// two >= max(cnt, kMinGroupCap), doubled when `roomy` is set (the list holds
// at least twice that, as after deletes from a larger count). An append that
// would pass group_cap() moves the list; the bit keeps a list whose count
// dips below a power of two and comes back from moving each time. A list
// emptied by deletes keeps its storage (base1 != 0, cnt 0).
struct __align__(8) GroupDesc {
  uint32_t base1;      // member arena offset in 4-entry units, plus 1; 0 = no list
  uint32_t cnt : 31;   // members
  uint32_t roomy : 1;  // the list holds at least 2 x pow2(max(cnt, kMinGroupCap)) entries
};

struct __align__(16) VertexMeta {
  unsigned long long eoff;   // EdgeRec index of slot 0
  unsigned long long bpoff;  // back-pointer arena index of the vertex pool
  uint32_t ecnt, ecap;       // slots used (tombstones included) / capacity
  uint32_t bpcnt, bpcap;     // back-pointer entries used / capacity
  uint32_t live;             // non-tombstone slots
  uint32_t acap;             // AliasRec capacity at VertexRec::aoff
  uint32_t hkeys;            // occupied adjacency keys (zero-count keys included)
  uint32_t hcap;             // adjacency capacity (power of two) or 0
};

// Arenas (one device allocation each).
enum Arena : int { A_MEMBER = 0, A_EDGE = 1, A_BP = 2, A_ALIAS = 3, A_HASH = 4, kArenas = 5 };

// Device status words.
enum ErrBit : uint32_t {
  E_RANGE = 1u,
  E_ZERO_WEIGHT = 2u,
  E_INVALID_SLOT = 4u,
  E_CAPACITY = 8u,
  E_TIMEOUT = 16u,
};

// Everything a kernel needs to read or modify the store.
struct StoreView {
  uint32_t n;
  VertexRec* vrec;
  VertexMeta* meta;
  GroupDesc* gdesc;  // [n][32]
  uint32_t* gv;      // member arena: neighbour ids
  uint32_t* gs;      // member arena: each member's back-pointer index (its slot's entry for the group; same indexing as gv)
  EdgeRec* edges;
  uint32_t* bp;
  AliasRec* alias;
  HashEntry* hash;
  unsigned long long* top;  // [kArenas] bump pointers (arena units)
  unsigned long long cap[kArenas];
  uint32_t* err;            // [0] ErrBit mask, [1] rejected-delete count
  uint32_t node2vec;
};

// floor(a * b / 2^32): uniform pick in [0, b) from a 32-bit draw.
__device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) { return __umulhi(a, b); }
// floor(a * b / 2^64).
__device__ __forceinline__ unsigned long long mulhi64(unsigned long long a, unsigned long long b) {
  return __umul64hi(a, b);
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long x) {
#pragma unroll
  for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}
__device__ __forceinline__ uint32_t warp_sum_u32(uint32_t x) {
#pragma unroll
  for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}
// Inclusive prefix sum across the warp.
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// The smallest power of two >= max(x, lo) (lo a power of two); 0 when x
// exceeds 2^31.
__host__ __device__ __forceinline__ uint32_t pow2_at_least(uint32_t x, uint32_t lo) {
  if (x <= lo) return lo;
  if (x > 0x80000000u) return 0u;
#ifdef __CUDA_ARCH__
  return 1u << (32 - __clz(x - 1));
#else
  return 1u << (32 - __builtin_clz(x - 1));
#endif
}

// Entries the group's list holds at least (0 when it has no list).
__host__ __device__ __forceinline__ uint32_t group_cap(const GroupDesc& G) {
  return G.base1 ? pow2_at_least(G.cnt, kMinGroupCap) << G.roomy : 0u;
}
// The roomy bit after the count changed in place (no move) from a list
// whose group_cap() was cap0.
__host__ __device__ __forceinline__ uint32_t group_roomy(uint32_t cnt, uint32_t cap0) {
  return 2ull * pow2_at_least(cnt, kMinGroupCap) <= (unsigned long long)cap0 ? 1u : 0u;
}
// Member arena offset of the list in 4-entry units (0 when it has no list).
__host__ __device__ __forceinline__ uint32_t group_base(const GroupDesc& G) { return G.base1 ? G.base1 - 1u : 0u; }

// Adjacency index hash: MurmurHash3 32-bit finaliser (Appleby, public domain).
__host__ __device__ __forceinline__ uint32_t mix32(uint32_t h) {
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

__device__ __forceinline__ void set_err(uint32_t* err, uint32_t bit) { atomicOr(err, bit); }

}  // namespace bingo
