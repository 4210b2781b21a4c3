// common.cuh -- shared device types and helpers of the B200 delta-repair engine.
//
// Adjacency layout (one arena per direction, pinned + mapped host memory):
//   dst[slot]  uint32 neighbour id; bit 31 set = deleted occurrence (tombstone)
//   w[slot]    uint32 weight (only when weights are stored)
// Each vertex owns a block [off, off+cap) of slots; [0,len) is in use, of which
// [0,srt) is sorted by neighbour id (tombstones keep their id bits, so binary
// search still works) and [srt,len) holds appended occurrences in insertion
// order; live = occurrences in use minus tombstones.
//
// The arena is split into pages of 2^page_shift slots. page_slot[page] names
// the HBM cache slot holding a copy of the page, or PAGE_NONE. Every write goes
// to the host arena and, when the page is resident, to its cached copy, so the
// host copy is always authoritative and eviction never writes back.
//
// Vertex state for SSSP/BFS/CC is one 64-bit key per vertex:
//   key = (value << 32) | (parent + 1), parent field 0 = no parent.
// One 64-bit atomic keeps value and parent consistent. With weights >= 1
// (BFS, the (u+v)%128+1 rule) atomicMin is used and equal values break toward
// the smaller parent id; where zero weights can occur (CC, stored weights) the
// parent only moves on a strict value decrease (see repair.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/dycg_operators.h"

namespace dycg {

typedef unsigned long long u64;

constexpr uint32_t PAGE_NONE = 0xFFFFFFFFu;
constexpr uint32_t TOMB = 0x80000000u;
constexpr uint32_t VMASK = 0x7FFFFFFFu;
constexpr uint32_t INF32 = 0xFFFFFFFFu;
constexpr u64 KEY_INF = ~0ull;

constexpr uint32_t ALGO_SSSP = 0, ALGO_BFS = 1, ALGO_CC = 2, ALGO_PR = 3;
constexpr uint32_t WEIGHT_HASH128 = 0, WEIGHT_STORED = 1;

// Rows longer than HEAVY are split into TILE-slot tiles processed by whole CTAs.
constexpr uint32_t HEAVY = 1024;
constexpr uint32_t TILE = 4096;
constexpr int BLOCK = 256;

// Error codes written to Ctl::err by device code (never trap).
constexpr uint32_t ERR_BARRIER = 1;   // a grid barrier waited past its time limit
constexpr uint32_t ERR_WAVES = 2;     // a closure exceeded its wave cap
constexpr uint32_t ERR_TILES = 3;     // tile queue full
constexpr uint32_t ERR_ARENA = 4;     // adjacency arena exhausted
constexpr uint32_t ERR_QUEUE = 5;     // a vertex queue overflowed
constexpr uint32_t ERR_NONFINITE = 6; // PR produced a non-finite value

__host__ __device__ inline u64 pack_key(uint32_t value, uint32_t parent_plus1) {
  return ((u64)value << 32) | parent_plus1;
}
__host__ __device__ inline uint32_t key_value(u64 k) { return (uint32_t)(k >> 32); }
__host__ __device__ inline uint32_t key_parent1(u64 k) { return (uint32_t)k; }

// SplitMix64 finalizer (Steele, Lea, Flood 2014): counter-based randomness for
// the workload generators, identical on host and device.
__host__ __device__ inline u64 mix64(u64 z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__host__ __device__ inline uint32_t hash_weight(u64 seed, uint32_t u, uint32_t v,
                                                uint32_t wlo, uint32_t whi) {
  u64 r = mix64(seed ^ mix64(((u64)u << 32) | v));
  return wlo + (uint32_t)(r % (u64)(whi - wlo + 1));
}

// R-MAT draw number idx: quadrant a=(0,0) b=(0,1) c=(1,0) d=(1,1) per level,
// three levels per 64-bit hash (21-bit uniform fields).
__host__ __device__ inline void rmat_draw(u64 seed, u64 idx, uint32_t scale, uint32_t ta,
                                          uint32_t tab, uint32_t tabc, uint32_t &u,
                                          uint32_t &v) {
  uint32_t uu = 0, vv = 0;
  for (uint32_t level = 0; level < scale; level += 3) {
    u64 r = mix64(seed ^ mix64(idx * 0x9E3779B97F4A7C15ull + level + 1));
    for (uint32_t j = 0; j < 3 && level + j < scale; j++) {
      uint32_t x = (uint32_t)(r >> (21 * j)) & ((1u << 21) - 1);
      uint32_t bu = x >= tab;
      uint32_t bv = (x >= ta && x < tab) || x >= tabc;
      uu = (uu << 1) | bu;
      vv = (vv << 1) | bv;
    }
  }
  u = uu;
  v = vv;
}

// Device view of one adjacency direction. Slot p occupies `stride` 32-bit
// words at word index p*stride: the neighbour id, then (stride 2) its weight,
// so one 8-byte access moves both.
struct Adj {
  uint32_t *hdst;        // host arena words (device-mapped pointer)
  uint32_t *cdst;        // HBM page cache words, slot-major (shared by both directions)
  const uint32_t *page_slot;
  uint32_t *page_hits;   // per-page slot-access counters (hotness)
  uint32_t page_base;    // global id of this arena's first page
  uint32_t page_shift;
  uint32_t stride;       // 1: id only, 2: (id, weight)
  uint32_t fence_shift;  // one fence per 128 bytes of slots: 5 (stride 1) or 4 (stride 2)
  u64 *off;
  uint32_t *len;
  uint32_t *cap;
  uint32_t *srt;
  uint32_t *live;
  u64 *top;              // arena bump pointer (slots)
  u64 arena;             // arena size (slots)
  uint32_t *fence;       // HBM fence index: id bits of slot (f << fence_shift)
  uint32_t *tbits;       // HBM deletion bitmap, one bit per arena slot
};

constexpr uint32_t BAR_GROUPS = 16;

// Per-launch control block in device memory: barrier, queues, counters.
struct Ctl {
  uint32_t bar_count;
  uint32_t bar_gen;
  uint32_t err;
  uint32_t err_info;
  uint32_t n_aff;        // affected list length
  uint32_t q_count[3];   // wave queue lengths (q0/q1 alternate; q2: the ordered bucket)
  uint32_t tile_count;
  uint32_t vmin;         // ordered closure: minimum frontier value of the wave
  // snapshots taken by the last block to arrive at a barrier
  uint32_t snap_aff;
  uint32_t snap_q[3];
  uint32_t snap_tiles;
  uint32_t snap_vmin;
  uint32_t wave_tag;     // running wave tag (never reused)
  uint32_t waves;        // waves run in this launch
  uint32_t pad[2];       // PageRank: carried frontier (queue parity, length)
  uint32_t grab;         // claimed-item counter of a phase (reset by its barriers)
  uint32_t pad2;
  // range-ordered wave queues (batched form): entries per vertex range, per
  // queue parity (reset with the parity's queue count)
  uint32_t qrange[2][64];
  // asynchronous worklist (batched form): ring claim / append positions, items
  // pushed and not yet finished, mask records and tile items handed out
  u64 a_head, a_tail;
  uint32_t a_pend, a_pool, a_tiles, a_pad;
  u64 stat[20];
  u64 tphase[8];         // batched repair: global timer at phase boundaries (ns)
  // grid-barrier arrival groups, one 128-byte line each (frontier.cuh)
  uint32_t bar_sub[BAR_GROUPS * 32];
};
// read back to the host once per snapshot (dycgraph_b200/engine.py CTL_BYTES)
static_assert(sizeof(Ctl) == 2904, "Ctl layout changed: update CTL_BYTES in engine.py");

enum StatIdx {
  ST_LINK_BYTES = 0,
  ST_HBM_ADJ_BYTES,
  ST_STATE_BYTES,
  ST_EXPANDED,
  ST_SCANNED,
  ST_IMPROVED,
  ST_AFFECTED,
  ST_MISSING,
  ST_RELOCATED,
  ST_INVALID,
  ST_TOUCHED,
  ST_PAGES_LOADED,
  ST_PAGES_EVICTED,
  ST_MUT_LINK_BYTES,   // mutation kernels' adjacency bytes over the host link
  ST_MUT_HBM_BYTES,    // mutation kernels' adjacency bytes in the HBM cache
  ST_T_START,          // batched repair: global timer at launch start (ns)
  ST_T_END,            // batched repair: latest block exit (ns)
  ST_COUNT
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

__device__ __forceinline__ u64 globaltimer_ns() {
  u64 t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Warp-aggregated append of `val` by the lanes with want=true. The calling
// code keeps the warp converged (loops are warp-uniform).
__device__ __forceinline__ bool warp_append(uint32_t *q, uint32_t *count, uint32_t cap,
                                            bool want, uint32_t val, uint32_t *err) {
  unsigned mask = __activemask();
  unsigned m = __ballot_sync(mask, want);
  if (!m) return true;
  int leader = __ffs(m) - 1;
  uint32_t base = 0;
  if ((int)lane_id() == leader) base = atomicAdd(count, (uint32_t)__popc(m));
  base = __shfl_sync(mask, base, leader);
  uint32_t rank = __popc(m & ((1u << lane_id()) - 1));
  if (base + __popc(m) > cap) {
    if ((int)lane_id() == leader) atomicExch(err, ERR_QUEUE);
    return false;
  }
  if (want) q[base + rank] = val;
  return true;
}

__device__ __forceinline__ u64 warp_sum(u64 x) {
  for (int o = 16; o; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  return x;
}

// Minimum of a 64-bit key over the warp, in every lane: the high words'
// minimum, then the minimum low word among the lanes that hold it (the same
// order as the 64-bit comparison), each one warp reduction instruction.
__device__ __forceinline__ u64 warp_min_all(u64 x) {
  const uint32_t hi = __reduce_min_sync(0xffffffffu, (uint32_t)(x >> 32));
  const uint32_t lo =
      __reduce_min_sync(0xffffffffu, (uint32_t)(x >> 32) == hi ? (uint32_t)x : 0xFFFFFFFFu);
  return ((u64)hi << 32) | lo;
}

// Slot address through the page table.
__device__ __forceinline__ uint32_t page_of(const Adj &a, u64 p) {
  return a.page_base + (uint32_t)(p >> a.page_shift);
}

__device__ __forceinline__ u64 cache_index(const Adj &a, uint32_t cslot, u64 p) {
  return ((u64)cslot << a.page_shift) | (p & ((1ull << a.page_shift) - 1));
}

// Word address of slot p (HBM copy when its page is resident) for readers.
__device__ __forceinline__ const uint32_t *slot_ptr(const Adj &a, u64 p, bool &cached) {
  const uint32_t cs = __ldg(a.page_slot + page_of(a, p));
  cached = cs != PAGE_NONE;
  return cached ? a.cdst + cache_index(a, cs, p) * a.stride : a.hdst + p * a.stride;
}

// Same, for kernels that also write the arena (no read-only cache path).
__device__ __forceinline__ const uint32_t *slot_ptr_rw(const Adj &a, u64 p) {
  const uint32_t cs = a.page_slot[page_of(a, p)];
  return cs != PAGE_NONE ? a.cdst + cache_index(a, cs, p) * a.stride : a.hdst + p * a.stride;
}

__device__ __forceinline__ uint32_t read_dst(const Adj &a, u64 p, bool &cached) {
  return __ldg(slot_ptr(a, p, cached));
}

// (id, weight) of slot p in one access; weight 0 without stored weights.
__device__ __forceinline__ uint2 read_pair(const Adj &a, u64 p, bool &cached) {
  const uint32_t *q = slot_ptr(a, p, cached);
  if (a.stride == 2) return __ldg(reinterpret_cast<const uint2 *>(q));
  return make_uint2(__ldg(q), 0u);
}

__device__ __forceinline__ uint32_t read_dst_rw(const Adj &a, u64 p) { return *slot_ptr_rw(a, p); }

__device__ __forceinline__ uint2 read_pair_rw(const Adj &a, u64 p) {
  const uint32_t *q = slot_ptr_rw(a, p);
  if (a.stride == 2) return *reinterpret_cast<const uint2 *>(q);
  return make_uint2(*q, 0u);
}

// Deleted: tombstone bit in the slot (materialised by a row relocation) or the
// slot's bit in the HBM deletion bitmap (set by the deletion kernels).
__device__ __forceinline__ bool slot_deleted(const Adj &a, u64 p, uint32_t d) {
  return (d & TOMB) || ((__ldg(a.tbits + (p >> 5)) >> (p & 31)) & 1u);
}

__device__ __forceinline__ bool slot_deleted_rw(const Adj &a, u64 p, uint32_t d) {
  return (d & TOMB) || ((*(volatile uint32_t *)(a.tbits + (p >> 5)) >> (p & 31)) & 1u);
}

// Write-through store of one slot: host arena (one 8-byte store with
// weights), the resident cached copy, and the fence entry when the slot opens
// a 128-byte group. Returns whether the page is resident.
__device__ __forceinline__ bool write_slot(const Adj &a, u64 p, uint32_t d, uint32_t w) {
  const uint32_t cs = a.page_slot[page_of(a, p)];
  if (a.stride == 2) {
    *reinterpret_cast<uint2 *>(a.hdst + p * 2) = make_uint2(d, w);
    if (cs != PAGE_NONE) *reinterpret_cast<uint2 *>(a.cdst + cache_index(a, cs, p) * 2) = make_uint2(d, w);
  } else {
    a.hdst[p] = d;
    if (cs != PAGE_NONE) a.cdst[cache_index(a, cs, p)] = d;
  }
  if ((p & ((1ull << a.fence_shift) - 1)) == 0) a.fence[p >> a.fence_shift] = d & VMASK;
  return cs != PAGE_NONE;
}

// Edge weight by algorithm (BFS 1, CC 0, SSSP (u+v)%128+1 unless weights are
// stored): the operator's TraversalEdgeWeight (the reference's,
// include/framework/variants/api.cuh:26-28).
template <uint32_t ALGO>
__device__ __forceinline__ uint32_t rule_weight(uint32_t u, uint32_t v) {
  return dycg_ops::ForAlgo<ALGO>::type::TraversalEdgeWeight(u, v);
}

}  // namespace dycg
