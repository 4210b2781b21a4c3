// frontier.cuh -- bounded grid barrier and the row-expansion engine shared by
// the persistent repair kernels (SSSP/BFS/CC closures and PageRank pushes).
//
// Work distribution (the B200 form of the reference's degree-aware CTA/warp
// scheduler, include/groute/device/cta_scheduler_hybrid.cuh:60-240): one warp
// per frontier vertex walks its row 32 slots at a time (coalesced 128-byte
// reads, from the HBM page cache or zero-copy from the host arena); rows
// longer than HEAVY are cut into TILE-slot tiles that whole CTAs process after
// a grid barrier, so a million-edge hub row spreads over the whole GPU.
#pragma once
#include <type_traits>

#include "common.cuh"

namespace dycg {

// Ops that declare `static constexpr int kBatch` take a lane's UNROLL slots in
// one call (edges()), so they can issue independent atomics back to back
// instead of waiting on each before the next.
template <class T, class = void>
struct batch_edges : std::false_type {};
template <class T>
struct batch_edges<T, std::void_t<decltype(T::kBatch)>> : std::true_type {};

constexpr uint32_t SYNC_RESET_TILES = 1;
constexpr uint32_t SYNC_RESET_Q0 = 2;
constexpr uint32_t SYNC_RESET_Q1 = 4;
constexpr uint32_t SYNC_RESET_Q2 = 8;
constexpr uint32_t SYNC_RESET_VMIN = 16;
constexpr uint32_t SYNC_RESET_GRAB = 32;
constexpr uint32_t SYNC_RESET_ASYNC = 64;

// Back-off of a block waiting at the grid barrier between polls (ns).
#ifndef DYCG_SPIN_NS
#define DYCG_SPIN_NS 100
#endif

// Grid-wide barrier for cooperative launches. Arrival is two-level: a block
// arrives at one of BAR_GROUPS group counters (separate 128-byte lines) and
// only the last arriver of each group arrives at the top counter, so the
// serialised atomics per barrier drop from one per block to about
// blocks / BAR_GROUPS + BAR_GROUPS. Every wait is bounded: past timeout_ns
// the waiting block records ERR_BARRIER and all blocks leave at their next
// barrier. The last block to arrive snapshots the queue counters and applies
// the requested resets while every other block is waiting.
__device__ __forceinline__ bool grid_sync(Ctl *c, uint32_t flags, u64 timeout_ns) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile uint32_t *vgen = &c->bar_gen;
    volatile uint32_t *verr = &c->err;
    uint32_t g = *vgen;
    __threadfence();
    const uint32_t groups = min(gridDim.x, BAR_GROUPS);
    const uint32_t grp = blockIdx.x % groups;
    const uint32_t members = (gridDim.x - grp + groups - 1) / groups;
    bool last = false;
    if (atomicAdd(&c->bar_sub[grp * 32], 1u) + 1 == members) {
      atomicExch(&c->bar_sub[grp * 32], 0u);  // every member has arrived
      last = atomicAdd(&c->bar_count, 1u) + 1 == groups;
    }
    int ok = 1;
    if (last) {
      if (flags & SYNC_RESET_TILES) c->tile_count = 0;
      if (flags & SYNC_RESET_Q0) {
        c->q_count[0] = 0;
        for (int b = 0; b < 64; b++) c->qrange[0][b] = 0;
      }
      if (flags & SYNC_RESET_Q1) {
        c->q_count[1] = 0;
        for (int b = 0; b < 64; b++) c->qrange[1][b] = 0;
      }
      if (flags & SYNC_RESET_Q2) c->q_count[2] = 0;
      if (flags & SYNC_RESET_GRAB) c->grab = 0;
      if (flags & SYNC_RESET_ASYNC) {
        c->a_head = 0;
        c->a_tail = 0;
        c->a_pend = 0;
        c->a_pool = 0;
        c->a_tiles = 0;
      }
      c->snap_aff = *(volatile uint32_t *)&c->n_aff;
      c->snap_q[0] = *(volatile uint32_t *)&c->q_count[0];
      c->snap_q[1] = *(volatile uint32_t *)&c->q_count[1];
      c->snap_q[2] = *(volatile uint32_t *)&c->q_count[2];
      c->snap_tiles = *(volatile uint32_t *)&c->tile_count;
      c->snap_vmin = *(volatile uint32_t *)&c->vmin;
      if (flags & SYNC_RESET_VMIN) c->vmin = 0xFFFFFFFFu;
      atomicExch(&c->bar_count, 0u);
      __threadfence();
      atomicAdd(&c->bar_gen, 1u);
    } else {
      u64 t0 = globaltimer_ns();
      while (*vgen == g) {
        if (*verr) {
          ok = 0;
          break;
        }
        if (globaltimer_ns() - t0 > timeout_ns) {
          atomicCAS(&c->err, 0u, ERR_BARRIER);
          ok = 0;
          break;
        }
        if (DYCG_SPIN_NS) __nanosleep(DYCG_SPIN_NS);
      }
    }
    __threadfence();
    s_ok = ok && (*verr == 0);
  }
  __syncthreads();
  return s_ok != 0;
}

// Per-thread traffic counters, flushed once per kernel.
struct Acc {
  u64 link;
  u64 hbm;
  u64 scanned;
  u64 expanded;
  u64 improved;
  u64 state;  // vertex-state bytes counted by the kernel itself (batched form)
  __device__ void flush(Ctl *c) {
    u64 a = warp_sum(link), b = warp_sum(hbm), s = warp_sum(scanned), e = warp_sum(expanded),
        i = warp_sum(improved), k = warp_sum(state);
    if (lane_id() == 0) {
      if (k) atomicAdd(&c->stat[ST_STATE_BYTES], k);
      if (a) atomicAdd(&c->stat[ST_LINK_BYTES], a);
      if (b) atomicAdd(&c->stat[ST_HBM_ADJ_BYTES], b);
      if (s) atomicAdd(&c->stat[ST_SCANNED], s);
      if (e) atomicAdd(&c->stat[ST_EXPANDED], e);
      if (i) atomicAdd(&c->stat[ST_IMPROVED], i);
    }
  }
};

// Walk slots [b, e) of row v; this lane handles s0 + lane for s0 = b, b+stride...
// Loads are issued UNROLL iterations ahead of their use so that each lane keeps
// several zero-copy reads in flight (a host-link read costs ~1-2 us).
// Op interface (all lanes call every member, keeping the warp converged):
//   bool begin(uint32_t v, Row&)                  -- false: skip the row
//   void edge(uint32_t v, uint32_t nb, uint32_t w, bool valid, Row&, Acc&)
//     or, with kBatch, edges(v, nb[UNROLL], valid[UNROLL], Row&, Acc&)
//   void end(uint32_t v, Row&)
template <bool WITH_W, class Op>
__device__ __forceinline__ void warp_slots(const Adj &A, uint32_t v, u64 off, uint32_t b,
                                           uint32_t e, uint32_t stride, Op &op, Acc &acc) {
  constexpr int UNROLL = 4;
  typename Op::Row r;
  if (!op.begin(v, r)) return;
  const uint32_t lane = lane_id();
  if (lane == 0 && b == 0) acc.expanded++;
  uint32_t hit_pg = PAGE_NONE, hit_n = 0;  // lane 0: pending hotness count
  const uint32_t bytes = WITH_W ? 8u : 4u;
  for (uint32_t s0 = b; s0 < e; s0 += stride * UNROLL) {
    uint32_t d[UNROLL], w[UNROLL], pg[UNROLL];
    bool in[UNROLL], cached[UNROLL];
#pragma unroll
    for (int u = 0; u < UNROLL; u++) {
      const uint32_t s = s0 + u * stride + lane;
      in[u] = s < e;
      d[u] = TOMB;
      w[u] = 0;
      pg[u] = PAGE_NONE;
      cached[u] = false;
      if (in[u]) {
        const u64 p = off + s;
        pg[u] = page_of(A, p);
        if (WITH_W) {
          const uint2 pr = read_pair(A, p, cached[u]);
          d[u] = pr.x;
          w[u] = pr.y;
        } else {
          d[u] = read_dst(A, p, cached[u]);
        }
        if (slot_deleted(A, p, d[u])) d[u] |= TOMB;
      }
    }
    bool ok[UNROLL];  // valid slot (every entry set before the loop may break)
#pragma unroll
    for (int u = 0; u < UNROLL; u++) ok[u] = false;
#pragma unroll
    for (int u = 0; u < UNROLL; u++) {
      if (s0 + u * stride >= e) break;  // warp-uniform
      const bool valid = in[u] && !(d[u] & TOMB);
      ok[u] = valid;
      if (in[u]) {
        if (cached[u]) acc.hbm += valid ? bytes : 4u;
        else acc.link += valid ? bytes : 4u;
        acc.scanned++;
      }
      // hotness: lane 0 accumulates the warp's slots that share its page
      const uint32_t pg0 = __shfl_sync(0xffffffffu, pg[u], 0);
      const unsigned same = __ballot_sync(0xffffffffu, in[u] && pg[u] == pg0);
      if (lane == 0) {
        if (pg0 != hit_pg) {
          if (hit_n) atomicAdd(A.page_hits + hit_pg, hit_n);
          hit_pg = pg0;
          hit_n = 0;
        }
        hit_n += __popc(same);
      }
      if (in[u] && pg[u] != pg0) atomicAdd(A.page_hits + pg[u], 1u);
      if constexpr (!batch_edges<Op>::value) op.edge(v, d[u] & VMASK, w[u], valid, r, acc);
    }
    if constexpr (batch_edges<Op>::value) {
      uint32_t nb[UNROLL];
#pragma unroll
      for (int u = 0; u < UNROLL; u++) nb[u] = d[u] & VMASK;
      op.edges(v, nb, ok, r, acc);
    }
  }
  if (lane == 0 && hit_n) atomicAdd(A.page_hits + hit_pg, hit_n);
  op.end(v, r);
}

struct Tiles {
  uint4 *tiles;
  uint32_t cap;
};

// Expand the rows of items[0..cnt) over adjacency A. Ends with a grid barrier
// that also applies `reset_flags` (with the tile reset). Returns false when
// the launch has failed (error flag set).
// Items are taken statically (warp w: items w, w + warps, ...) or, with
// `claimed`, one at a time from the control block's claim counter (reset by
// the barriers that end the phase), so a warp that drew long rows does not
// hold the wave's barrier while the others idle.
template <bool WITH_W, class Op>
__device__ bool expand_rows(const Adj &A, const uint32_t *items, uint32_t cnt, Op &op,
                            Acc &acc, Tiles T, Ctl *ctl, uint32_t reset_flags,
                            u64 timeout_ns, bool claimed = false) {
  const uint32_t lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  uint32_t i = gw;
  if (claimed) {
    if (lane == 0) i = atomicAdd(&ctl->grab, 1u);
    i = __shfl_sync(0xffffffffu, i, 0);
  }
  while (i < cnt) {
    const uint32_t v = items[i];
    if (claimed) {
      if (lane == 0) i = atomicAdd(&ctl->grab, 1u);
      i = __shfl_sync(0xffffffffu, i, 0);
    } else {
      i += nw;
    }
    const uint32_t len = A.len[v];
    if (len > HEAVY) {
      if (lane == 0) {
        const uint32_t nt = (len + TILE - 1) / TILE;
        const uint32_t base = atomicAdd(&ctl->tile_count, nt);
        if (base + nt > T.cap) {
          atomicCAS(&ctl->err, 0u, ERR_TILES);
        } else {
          for (uint32_t t = 0; t < nt; t++)
            T.tiles[base + t] = make_uint4(v, t * TILE, min(len, (t + 1) * TILE), 0);
        }
      }
      continue;
    }
    warp_slots<WITH_W>(A, v, A.off[v], 0, len, 32, op, acc);
  }
  // The items have been consumed: the queue resets can apply here. When no row
  // was heavy this barrier's snapshot already holds every append of the
  // expansion and the tile phase (and its barrier) is skipped.
  if (!grid_sync(ctl, reset_flags | SYNC_RESET_GRAB, timeout_ns)) return false;
  const uint32_t nt = min(*(volatile uint32_t *)&ctl->snap_tiles, T.cap);
  if (nt == 0) return true;
  const uint32_t wib = threadIdx.x >> 5;
  __shared__ uint32_t s_tile;
  uint32_t t = blockIdx.x;
  if (claimed) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&ctl->grab, 1u);
    __syncthreads();
    t = s_tile;
  }
  while (t < nt) {
    const uint4 tl = T.tiles[t];
    if (claimed) {
      __syncthreads();  // every warp has read s_tile
      if (threadIdx.x == 0) s_tile = atomicAdd(&ctl->grab, 1u);
      __syncthreads();
      t = s_tile;
    } else {
      t += gridDim.x;
    }
    warp_slots<WITH_W>(A, tl.x, A.off[tl.x], tl.y + wib * 32, tl.z, blockDim.x, op, acc);
  }
  return grid_sync(ctl, SYNC_RESET_TILES | SYNC_RESET_GRAB, timeout_ns);
}

__device__ __forceinline__ u64 ld_key(const u64 *p) {
  return *(const volatile u64 *)p;
}

// Lower key[v] to cand only when the value strictly decreases. With
// zero-weight edges (CC labels; stored weights may be 0) an equal value must
// not move the parent: a switch to a smaller-id parent of equal value can
// close a cycle in the parent forest, and deletion repair follows parents.
// Returns true when this call lowered the value.
__device__ __forceinline__ bool strict_lower(u64 *addr, u64 cand) {
  u64 old = ld_key(addr);
  while (key_value(cand) < key_value(old)) {
    const u64 prev = atomicCAS(addr, old, cand);
    if (prev == old) return true;
    old = prev;
  }
  return false;
}

// Zero-weight edges possible: strict value decrease only.
template <uint32_t ALGO, bool STORED>
struct Strict {
  static constexpr bool value = ALGO == ALGO_CC || STORED;
};

}  // namespace dycg
