// multi.cu -- batched repair of many SSSP/BFS queries (sources) over one
// shared graph: one persistent cooperative launch repairs every query after a
// snapshot, so each adjacency row crosses the host link once per wave for all
// the queries that need it instead of once per query.
//
// Layout: key[v*Q + q] (Q = 32*NB, NB <= 8 blocks of 32 queries), so the keys
// of one vertex for one block of queries are one 256-byte line. Frontier items
// are vertices; per vertex and block a 32-bit mask names the queries for
// which it is active (affm: affected this snapshot; inew: newly affected, one
// buffer per invalidation-wave parity; nmask: improved, one buffer per
// closure-wave parity; cmask: the masks of a heavy row, read by its tiles).
//
// Two warp mappings, chosen per row by a cost model (qratio, tuned):
//   edge lanes  -- lane i takes slot i of each 32-slot chunk and works through
//                  the row's active queries four at a time (their key loads
//                  issued together); per-query state (the row's own value, or
//                  the best pull candidate) sits in the warp's shared memory.
//                  Every lane does useful work whatever the query count.
//   query lanes -- the warp visits the row's edges one by one and lane i works
//                  on query 32*b + i of every active block b (one coalesced
//                  key line per edge and block, all blocks' loads issued
//                  together); for rows active in many queries.
// Rows whose work (slot chunks x active queries, or edges) exceeds `heavy`
// are cut into tiles processed by whole CTAs after a grid barrier: an
// edge-lane tile is staged once in shared memory and the CTA's warps split
// its (chunk, query group) pairs; a query-lane tile's warps split its chunks.
// Per query the phases are the single-query repair's (repair.cu): deletion
// seeds (parent == u), invalidation waves over out-rows, reset, pull over
// in-rows, frontier + insertion seeds, push closure. The batched form has no
// counterpart in the reference engine, which repairs one source per engine
// (include/framework/framework.cuh:1803 InitGraph(src)).
#include "frontier.cuh"
#include "internal.h"

namespace dycg {

constexpr uint32_t WARPS = BLOCK / 32;
constexpr uint32_t QRANGES = 64;  // vertex ranges of a range-ordered wave queue

struct MultiParams {
  Adj out, in;
  u64 *key;
  uint32_t *affm;
  uint32_t *inew[2];
  uint32_t *nmask[2];
  uint32_t *cmask;
  uint32_t *mark;
  uint32_t *wtag;
  uint32_t *aff;
  uint32_t *q[2];
  Tiles tiles;
  Ctl *ctl;
  uint32_t *seq;
  const uint2 *del_uv;
  const uint32_t *del_found;
  const uint32_t *n_del_ptr;
  const uint3 *add_uvw;
  uint32_t n_add;
  uint32_t n, phases, max_waves, qratio, pull_qratio, heavy, tile;
  uint32_t sched;   // item distribution: 0 static, 1 claimed (dycg_query_mapping.queue bit 0)
  bool ranges;      // wave queues ordered by vertex range (dycg_query_mapping.queue bit 1)
  bool async;       // invalidation and closure on the asynchronous worklist (bit 2)
  uint32_t rsize;   // vertices per range: ceil(n / QRANGES)
  u64 *ring;        // asynchronous worklist: ring_cap items, A_EMPTY when free
  uint32_t ring_cap;
  uint32_t *inq;    // per vertex: an item of it is in the ring and not yet taken
  uint32_t *pool;   // mask records of split heavy rows, NB words each
  uint32_t pool_cap;
  u64 timeout_ns;
};

// Asynchronous worklist items: vertex v in the low 32 bits; a tile of a
// split heavy row carries its mask record + 1 (bits 32-47) and its tile index
// (bits 48-63).
constexpr u64 A_EMPTY = ~0ull;
constexpr uint32_t A_TILE_CAP = 1u << 20;   // tile items outstanding at once
constexpr uint32_t A_MAX_TILES = 1u << 16;  // tiles of one split row
constexpr uint32_t QPAR_ASYNC = 2;          // Ph queue parity that means "the worklist"

template <uint32_t ALGO, bool STORED>
__device__ __forceinline__ uint32_t mweight(uint32_t u, uint32_t v, uint32_t w) {
  return STORED ? w : rule_weight<ALGO>(u, v);
}

// Key reads inside a phase go to L2 (no L1 copy): within a phase values only
// decrease, so a read that misses a concurrent update only costs an atomic
// that turns out to be a no-op; across phases the grid barrier orders them.
__device__ __forceinline__ u64 ldk(const u64 *p) { return __ldcg(p); }

// Lower *addr to cand given a recent read `seen`; true when the value
// decreased (strict CAS form where zero weights are possible, atomicMin with
// parent tie-break otherwise).
template <bool STRICT>
__device__ __forceinline__ bool lower_from(u64 *addr, u64 cand, u64 seen) {
  if (cand >= seen) return false;
  if (STRICT) {
    u64 old = seen;
    while (key_value(cand) < key_value(old)) {
      const u64 prev = atomicCAS(addr, old, cand);
      if (prev == old) return true;
      old = prev;
    }
    return false;
  }
  return key_value(atomicMin(addr, cand)) > key_value(cand);
}

template <bool STRICT>
__device__ __forceinline__ bool lower_key(u64 *addr, u64 cand) {
  return lower_from<STRICT>(addr, cand, ldk(addr));
}

// lower_from split in two so that a lane can issue several independent
// first attempts before it looks at any result: first_lower issues the first
// atomic (false: cand cannot lower `seen`, nothing issued) and leaves its
// result in got; lowered finishes the attempt (the strict form retries from
// the value it lost to, exactly as lower_from's loop does).
template <bool STRICT>
__device__ __forceinline__ bool first_lower(u64 *addr, u64 cand, u64 seen, u64 &got) {
  if (cand >= seen) return false;
  if (STRICT) {
    if (key_value(cand) >= key_value(seen)) return false;
    got = atomicCAS(addr, seen, cand);
  } else {
    got = atomicMin(addr, cand);
  }
  return true;
}
template <bool STRICT>
__device__ __forceinline__ bool lowered(u64 *addr, u64 cand, u64 seen, u64 got) {
  if (!STRICT) return key_value(got) > key_value(cand);
  if (got == seen) return true;
  return lower_from<true>(addr, cand, got);
}

// Append y to the wave queue of parity par once per wave (tag). With range
// ordering the queue is cut into QRANGES regions of P.rsize slots, region b
// holding the vertices of [b * rsize, (b + 1) * rsize); a vertex enters a
// wave's queue at most once, so no region overflows. The queue count is kept
// either way (it ends the waves).
__device__ bool async_push(const MultiParams &P, u64 item);

__device__ __forceinline__ void enqueue_once(const MultiParams &P, uint32_t par, uint32_t y,
                                             uint32_t tag) {
  if (par == QPAR_ASYNC) {
    // asynchronous worklist: y's new mask bits are set; one item per vertex
    // until a consumer takes it (the fence orders the mask update before the
    // flag, the consumer clears the flag before it takes the masks)
    __threadfence();
    if (atomicExch(P.inq + y, 1u) == 0u) async_push(P, y);
    return;
  }
  if (atomicExch(P.wtag + y, tag) != tag) {
    Ctl *c = P.ctl;
    const uint32_t s = atomicAdd(&c->q_count[par], 1u);
    if (P.ranges) {
      const uint32_t b = y / P.rsize;
      const uint32_t k = atomicAdd(&c->qrange[par][b], 1u);
      if (b < QRANGES && k < P.rsize) P.q[par][b * P.rsize + k] = y;
      else atomicCAS(&c->err, 0u, ERR_QUEUE);
    } else if (s < P.n) {
      P.q[par][s] = y;
    } else {
      atomicCAS(&c->err, 0u, ERR_QUEUE);
    }
  }
}

__device__ __forceinline__ void note_affected(const MultiParams &P, uint32_t y, uint32_t epoch) {
  if (atomicExch(P.mark + y, epoch) != epoch) {
    const uint32_t s = atomicAdd(&P.ctl->n_aff, 1u);
    if (s < P.n) P.aff[s] = y;
    else atomicCAS(&P.ctl->err, 0u, ERR_QUEUE);
  }
}

// Slots [b, e) of the row at `off`, `stride` apart per lane: each lane loads
// its slot UNROLL chunks ahead of use, then the converged warp calls
// visit(id, weight, valid). Charges traffic and per-page hotness like
// warp_slots (frontier.cuh).
template <bool WITH_W, class Visit>
__device__ __forceinline__ void walk(const Adj &A, u64 off, uint32_t b, uint32_t e,
                                     uint32_t stride, Visit &visit, Acc &acc) {
  constexpr int UNROLL = 2;
  const uint32_t lane = lane_id();
  const uint32_t bytes = WITH_W ? 8u : 4u;
  uint32_t hit_pg = PAGE_NONE, hit_n = 0;
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
#pragma unroll
    for (int u = 0; u < UNROLL; u++) {
      if (s0 + u * stride >= e) break;  // warp-uniform
      const bool valid = in[u] && !(d[u] & TOMB);
      if (in[u]) {
        if (cached[u]) acc.hbm += valid ? bytes : 4u;
        else acc.link += valid ? bytes : 4u;
        acc.scanned++;
      }
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
      visit(d[u] & VMASK, w[u], valid);
    }
  }
  if (lane == 0 && hit_n) atomicAdd(A.page_hits + hit_pg, hit_n);
}

// Mapping of a row of `len` slots active in `act` queries: query lanes when
// 4*act >= qratio * min(len, 32) (qratio 0: always query lanes).
__device__ __forceinline__ bool use_query_lanes(uint32_t act, uint32_t len, uint32_t qratio) {
  return 4ull * act >= (u64)qratio * min(len, 32u);
}

// Expand slots [b, e) of v's row, `stride` apart per lane, for the queries
// in masks m (warp-uniform); s is the warp's shared per-query state (Q
// entries) for the edge-lane mapping.
// Ask L2 for the key lines of neighbour y that the active queries (masks m,
// warp-uniform) will read: one 256-byte bulk prefetch per block of 32 queries
// with any bit set (no registers held, no completion to wait for). A lane's
// loads for its later query groups, or for the warp's later edges, then find
// their sectors in L2 instead of waiting on HBM one group after another. The
// kernel is latency-bound with DRAM bandwidth mostly idle, so fetching whole
// lines costs nothing it is short of. Each line is 256-byte aligned inside the
// key array, and y is a live slot's vertex id (< n).
template <int NB>
__device__ __forceinline__ void prefetch_keys(const u64 *key, uint32_t y,
                                              const uint32_t (&m)[NB]) {
#pragma unroll
  for (int k = 0; k < NB; k++) {
    if (!m[k]) continue;  // warp-uniform
    const u64 *p = key + ((u64)y * NB + k) * 32;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], 256;" ::"l"(p) : "memory");
  }
}

template <int NB, bool WITH_W, class Ph>
__device__ __forceinline__ void expand_vertex(const Adj &A, uint32_t v, const uint32_t (&m)[NB],
                                              uint32_t b, uint32_t e, uint32_t stride, bool qlanes,
                                              Ph &ph, u64 *s, Acc &acc) {
  if (lane_id() == 0 && b == 0) acc.expanded++;
  const u64 off = A.off[v];
  uint32_t act = 0;
#pragma unroll
  for (int k = 0; k < NB; k++) act += __popc(m[k]);
  if (qlanes) {
    u64 st[NB];
#pragma unroll
    for (int k = 0; k < NB; k++) ph.beginQ(v, k, m[k], st[k]);
    auto visit = [&](uint32_t y, uint32_t w, bool valid) {
      // the warp takes these edges one at a time: their key lines are asked
      // for together first
      if (valid) prefetch_keys<NB>(ph.P->key, y, m);
      unsigned vb = __ballot_sync(0xffffffffu, valid);
      while (vb) {
        const int src = __ffs(vb) - 1;
        vb &= vb - 1;
        ph.edgeQ(v, __shfl_sync(0xffffffffu, y, src), __shfl_sync(0xffffffffu, w, src), m, st,
                 acc);
      }
    };
    walk<WITH_W>(A, off, b, e, stride, visit, acc);
#pragma unroll
    for (int k = 0; k < NB; k++)
      if (m[k]) ph.endQ(v, k, m[k], st[k]);
    return;
  }
#pragma unroll
  for (int k = 0; k < NB; k++)
    if (m[k]) ph.beginE(v, k, m[k], s);
  __syncwarp();
  auto visit = [&](uint32_t y, uint32_t w, bool valid) {
    // more than one group of four queries: the later groups' keys are
    // asked for before the first group's loads
    if (act > 4 && valid) prefetch_keys<NB>(ph.P->key, y, m);
    uint32_t qpk = 0, cnt = 0;
#pragma unroll
    for (int k = 0; k < NB; k++) {
      uint32_t mm = m[k];
      while (mm) {
        const uint32_t bit = __ffs(mm) - 1;
        mm &= mm - 1;
        qpk |= (k * 32 + bit) << (8 * cnt);
        if (++cnt == 4) {
          ph.edgesE(v, y, w, valid, qpk, 4, s, acc);
          qpk = 0;
          cnt = 0;
        }
      }
    }
    if (cnt) ph.edgesE(v, y, w, valid, qpk, cnt, s, acc);
  };
  walk<WITH_W>(A, off, b, e, stride, visit, acc);
  __syncwarp();
#pragma unroll
  for (int k = 0; k < NB; k++)
    if (m[k]) ph.endE(v, k, m[k], s);
  __syncwarp();
}

// Stage slots [b, e) (e - b <= MULTI_MIN_TILE) of v's row into shared
// memory, once per CTA: (id | TOMB when deleted, weight).
template <bool WITH_W>
__device__ __forceinline__ void stage_slots(const Adj &A, uint32_t v, uint32_t b, uint32_t e,
                                            uint2 *st, Acc &acc) {
  const uint32_t lane = lane_id();
  const u64 off = A.off[v] + b;
  const uint32_t len = e - b;
  const uint32_t bytes = WITH_W ? 8u : 4u;
  for (uint32_t i0 = threadIdx.x - lane; i0 < len; i0 += blockDim.x) {  // warp-uniform
    const uint32_t i = i0 + lane;
    const bool in = i < len;
    uint32_t d = TOMB, w = 0, pg = PAGE_NONE;
    bool cached = false;
    if (in) {
      const u64 p = off + i;
      pg = page_of(A, p);
      if (WITH_W) {
        const uint2 pr = read_pair(A, p, cached);
        d = pr.x;
        w = pr.y;
      } else {
        d = read_dst(A, p, cached);
      }
      if (slot_deleted(A, p, d)) d |= TOMB;
      const bool valid = !(d & TOMB);
      if (cached) acc.hbm += valid ? bytes : 4u;
      else acc.link += valid ? bytes : 4u;
      acc.scanned++;
      st[i] = make_uint2(d, w);
    }
    const uint32_t pg0 = __shfl_sync(0xffffffffu, pg, 0);
    const unsigned same = __ballot_sync(0xffffffffu, in && pg == pg0);
    if (lane == 0 && same) atomicAdd(A.page_hits + pg0, __popc(same));
    if (in && pg != pg0) atomicAdd(A.page_hits + pg, 1u);
  }
}

// Edge-lane expansion of a staged tile of len slots: the CTA's warps split
// the (32-slot chunk, group of four active queries) pairs.
template <int NB, class Ph>
__device__ __forceinline__ void staged_pairs(uint32_t v, const uint32_t (&m)[NB], uint32_t len,
                                             const uint2 *st, Ph &ph, u64 *s, Acc &acc) {
  const uint32_t lane = lane_id();
  const uint32_t wib = threadIdx.x >> 5;
  uint32_t act = 0;
#pragma unroll
  for (int k = 0; k < NB; k++) act += __popc(m[k]);
  const uint32_t C = (len + 31) / 32, G = (act + 3) / 4;
#pragma unroll
  for (int k = 0; k < NB; k++)
    if (m[k]) ph.beginE(v, k, m[k], s);
  __syncwarp();
  for (uint32_t p = wib; p < C * G; p += WARPS) {
    const uint32_t c = p % C, lo = (p / C) * 4;
    uint32_t j = 0, qpk = 0, cnt = 0;
#pragma unroll
    for (int k = 0; k < NB; k++) {
      const uint32_t pc = __popc(m[k]);
      if (j < lo + 4 && j + pc > lo) {
        uint32_t mm = m[k];
        while (mm) {
          const uint32_t bit = __ffs(mm) - 1;
          mm &= mm - 1;
          if (j >= lo && j < lo + 4) qpk |= (k * 32 + bit) << (8 * cnt++);
          j++;
        }
      } else {
        j += pc;
      }
    }
    const uint32_t slot = c * 32 + lane;
    const uint2 sl = slot < len ? st[slot] : make_uint2(TOMB, 0u);
    ph.edgesE(v, sl.x & VMASK, sl.y, !(sl.x & TOMB), qpk, cnt, s, acc);
  }
  __syncwarp();
#pragma unroll
  for (int k = 0; k < NB; k++)
    if (m[k]) ph.endE(v, k, m[k], s);
  __syncwarp();
}

// Expand items[0..cnt): prep(v, m) fills v's masks (false: skip). Rows whose
// work exceeds P.heavy are cut into P.tile-slot tiles (x = row, y/z = slot
// range, w = mapping) that whole CTAs process after a grid barrier; their
// masks travel through cmask. Ends with a barrier that applies reset_flags.
// Returns false when the launch has failed.
constexpr uint32_t NO_QUEUE = 0xFFFFFFFFu;

template <int NB, bool WITH_W, class Prep, class Ph>
__device__ bool multi_expand(const MultiParams &P, const Adj &A, const uint32_t *items,
                             uint32_t cnt, Prep &prep, Ph &ph, u64 *s, uint2 *stage, Acc &acc,
                             uint32_t qpar, uint32_t reset_flags, uint32_t qratio) {
  Ctl *ctl = P.ctl;
  const uint32_t lane = lane_id();
  // a range-ordered wave queue (qpar: its parity) is read range by range:
  // item i is entry i - pre[b] of region b, pre = prefix of the range counts
  __shared__ uint32_t s_pre[QRANGES + 1];
  const bool ranged = P.ranges && qpar != NO_QUEUE;
  if (ranged) {
    if (threadIdx.x < 32) {
      uint32_t x = ctl->qrange[qpar][lane], y = ctl->qrange[qpar][lane + 32];
      for (int o = 1; o < 32; o <<= 1) {  // inclusive warp scans of both halves
        const uint32_t xa = __shfl_up_sync(0xffffffffu, x, o);
        const uint32_t ya = __shfl_up_sync(0xffffffffu, y, o);
        if ((int)lane >= o) {
          x += xa;
          y += ya;
        }
      }
      const uint32_t tot_a = __shfl_sync(0xffffffffu, x, 31);
      s_pre[lane + 1] = x;
      s_pre[lane + 33] = tot_a + y;
      if (lane == 0) s_pre[0] = 0;
    }
    __syncthreads();
  }
  auto item = [&](uint32_t i) -> uint32_t {
    if (!ranged) return items[i];
    uint32_t lo = 0, hi = QRANGES;  // last b with s_pre[b] <= i
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) / 2;
      if (s_pre[mid] <= i) lo = mid; else hi = mid;
    }
    return items[lo * P.rsize + (i - s_pre[lo])];
  };
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  // Item distribution: static (warp w takes items w, w + nw, ...) or claimed
  // one at a time from a per-phase counter, so that a warp that drew long rows
  // does not hold the wave's barrier while the others idle (the counter is
  // reset by the barriers that end the phase).
  uint32_t i = gw;
  if (P.sched) {
    if (lane == 0) i = atomicAdd(&ctl->grab, 1u);
    i = __shfl_sync(0xffffffffu, i, 0);
  }
  for (; i < cnt;) {
    const uint32_t v = item(i);
    if (P.sched) {
      if (lane == 0) i = atomicAdd(&ctl->grab, 1u);
      i = __shfl_sync(0xffffffffu, i, 0);
    } else {
      i += nw;
    }
    uint32_t m[NB];
    if (!prep(v, m)) continue;
    const uint32_t len = A.len[v];
    if (len == 0) continue;
    uint32_t act = 0;
#pragma unroll
    for (int k = 0; k < NB; k++) act += __popc(m[k]);
    const bool ql = use_query_lanes(act, len, qratio);
    const u64 work = ql ? len : (u64)((len + 31) / 32) * act;
    if (work > P.heavy) {
#pragma unroll
      for (int k = 0; k < NB; k++)
        if (lane == (uint32_t)k) P.cmask[(u64)v * NB + k] = m[k];
      if (lane == 0) {
        // query-lane tiles: P.tile slots; edge-lane tiles: one staging buffer
        const uint32_t ts = ql ? P.tile : MULTI_MIN_TILE;
        const uint32_t nt = (len + ts - 1) / ts;
        const uint32_t base = atomicAdd(&ctl->tile_count, nt);
        if (base + nt > P.tiles.cap) {
          atomicCAS(&ctl->err, 0u, ERR_TILES);
        } else {
          for (uint32_t t = 0; t < nt; t++)
            P.tiles.tiles[base + t] = make_uint4(v, t * ts, min(len, (t + 1) * ts), ql ? 1u : 0u);
        }
      }
      continue;
    }
    expand_vertex<NB, WITH_W>(A, v, m, 0, len, 32, ql, ph, s, acc);
  }
  if (!grid_sync(ctl, reset_flags | SYNC_RESET_GRAB, P.timeout_ns)) return false;
  const uint32_t nt = min(*(volatile uint32_t *)&ctl->snap_tiles, P.tiles.cap);
  if (nt == 0) return true;
  const uint32_t wib = threadIdx.x >> 5;
  __shared__ uint32_t s_tile;
  uint32_t t = blockIdx.x;
  if (P.sched) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&ctl->grab, 1u);
    __syncthreads();
    t = s_tile;
  }
  while (t < nt) {
    const uint4 tl = P.tiles.tiles[t];
    if (P.sched) {
      __syncthreads();  // every warp has read s_tile
      if (threadIdx.x == 0) s_tile = atomicAdd(&ctl->grab, 1u);
      __syncthreads();
      t = s_tile;
    } else {
      t += gridDim.x;
    }
    uint32_t m[NB];
#pragma unroll
    for (int k = 0; k < NB; k++) m[k] = P.cmask[(u64)tl.x * NB + k];
    if (tl.w) {  // query lanes: the CTA's warps split the slot chunks
      expand_vertex<NB, WITH_W>(A, tl.x, m, tl.y + wib * 32, tl.z, blockDim.x, true, ph, s, acc);
    } else {     // edge lanes: slots staged once, warps split (chunk, query group) pairs
      __syncthreads();
      stage_slots<WITH_W>(A, tl.x, tl.y, tl.z, stage, acc);
      __syncthreads();
      if (threadIdx.x == 0 && tl.y == 0) acc.expanded++;
      staged_pairs<NB>(tl.x, m, tl.z - tl.y, stage, ph, s, acc);
    }
  }
  return grid_sync(ctl, SYNC_RESET_TILES | SYNC_RESET_GRAB, P.timeout_ns);
}

// Children y of a newly affected (x, q) with parent_q(y) == x become affected.
template <int NB>
struct InvalidatePh {
  const MultiParams *P;
  uint32_t *inew_next;
  uint32_t qpar;  // parity of the next wave's queue
  uint32_t tag, epoch;
  __device__ void mark(uint32_t y, uint32_t k, uint32_t bits) {
    const uint32_t old = atomicOr(P->affm + (u64)y * NB + k, bits);
    const uint32_t fresh = bits & ~old;
    if (fresh) {
      atomicOr(inew_next + (u64)y * NB + k, fresh);
      note_affected(*P, y, epoch);
      enqueue_once(*P, qpar, y, tag);
    }
  }
  __device__ void beginQ(uint32_t, int, uint32_t, u64 &) {}
  __device__ void edgeQ(uint32_t x, uint32_t y, uint32_t, const uint32_t (&m)[NB],
                        u64 (&)[NB], Acc &acc) {
    const uint32_t lane = lane_id();
    u64 cur[NB];
#pragma unroll
    for (int k = 0; k < NB; k++) {
      cur[k] = 0;
      if ((m[k] >> lane) & 1u) {
        cur[k] = ldk(P->key + ((u64)y * NB + k) * 32 + lane);
        acc.state += 8;
      }
    }
    // lane 0 takes every block's children; their affected-mask atomics are
    // independent and issued together, the fresh bits handled after
    uint32_t bits[NB], old[NB];
#pragma unroll
    for (int k = 0; k < NB; k++) {
      bits[k] = 0;
      if (!m[k]) continue;
      const bool child = ((m[k] >> lane) & 1u) && key_parent1(cur[k]) == x + 1u;
      bits[k] = __ballot_sync(0xffffffffu, child);
    }
    if (lane == 0) {
#pragma unroll
      for (int k = 0; k < NB; k++)
        old[k] = bits[k] ? atomicOr(P->affm + (u64)y * NB + k, bits[k]) : ~0u;
      bool fresh_any = false;
#pragma unroll
      for (int k = 0; k < NB; k++) {
        const uint32_t fresh = bits[k] & ~old[k];
        if (fresh) {
          atomicOr(inew_next + (u64)y * NB + k, fresh);
          fresh_any = true;
        }
      }
      if (fresh_any) {
        note_affected(*P, y, epoch);
        enqueue_once(*P, qpar, y, tag);
      }
    }
  }
  __device__ void endQ(uint32_t, int, uint32_t, u64 &) {}
  __device__ void beginE(uint32_t, int, uint32_t, u64 *) {}
  __device__ void edgesE(uint32_t x, uint32_t y, uint32_t, bool valid, uint32_t qpk,
                         uint32_t cnt, u64 *, Acc &acc) {
    u64 cur[4];
#pragma unroll
    for (uint32_t u = 0; u < 4; u++) {
      cur[u] = 0;
      if (u < cnt && valid) {
        cur[u] = ldk(P->key + (u64)y * NB * 32 + ((qpk >> (8 * u)) & 255));
        acc.state += 8;
      }
    }
    // the lane's children (one edge, up to four queries in ascending order),
    // merged per mask word: one affected-mask atomic per word
    uint32_t word = ~0u, bits = 0;
#pragma unroll
    for (uint32_t u = 0; u < 4; u++) {
      const uint32_t q = (qpk >> (8 * u)) & 255;
      if (u < cnt && valid && key_parent1(cur[u]) == x + 1u) {
        if ((q >> 5) != word) {
          if (bits) mark(y, word, bits);
          word = q >> 5;
          bits = 0;
        }
        bits |= 1u << (q & 31);
      }
    }
    if (bits) mark(y, word, bits);
  }
  __device__ void endE(uint32_t, int, uint32_t, u64 *) {}
};

// Affected (v, q) takes the best (value(x) + w, parent x) over live in-edges.
template <uint32_t ALGO, bool STORED, int NB>
struct PullPh {
  const MultiParams *P;
  static constexpr bool STRICT = Strict<ALGO, STORED>::value;
  __device__ u64 cand(uint32_t v, uint32_t x, uint32_t w, u64 kx) const {
    const uint32_t vx = key_value(kx);
    if (vx == INF32) return KEY_INF;
    const u64 c = (u64)vx + mweight<ALGO, STORED>(x, v, w);
    return c >= INF32 ? KEY_INF : pack_key((uint32_t)c, x + 1u);
  }
  __device__ void beginQ(uint32_t, int, uint32_t, u64 &best) { best = KEY_INF; }
  __device__ void edgeQ(uint32_t v, uint32_t x, uint32_t w, const uint32_t (&m)[NB],
                        u64 (&best)[NB], Acc &acc) {
    const uint32_t lane = lane_id();
    u64 cur[NB];
#pragma unroll
    for (int k = 0; k < NB; k++) {
      cur[k] = KEY_INF;
      if ((m[k] >> lane) & 1u) {
        cur[k] = ldk(P->key + ((u64)x * NB + k) * 32 + lane);
        acc.state += 8;
      }
    }
#pragma unroll
    for (int k = 0; k < NB; k++) {
      const u64 c = cand(v, x, w, cur[k]);
      best[k] = c < best[k] ? c : best[k];
    }
  }
  __device__ void endQ(uint32_t v, int k, uint32_t mk, u64 &best) {
    const uint32_t lane = lane_id();
    if (((mk >> lane) & 1u) && best != KEY_INF)
      lower_key<STRICT>(P->key + ((u64)v * NB + k) * 32 + lane, best);
  }
  __device__ void beginE(uint32_t, int k, uint32_t mk, u64 *s) {
    const uint32_t lane = lane_id();
    if ((mk >> lane) & 1u) s[k * 32 + lane] = KEY_INF;
  }
  __device__ void edgesE(uint32_t v, uint32_t x, uint32_t w, bool valid, uint32_t qpk,
                         uint32_t cnt, u64 *s, Acc &acc) {
    u64 cur[4];
#pragma unroll
    for (uint32_t u = 0; u < 4; u++) {
      cur[u] = KEY_INF;
      if (u < cnt && valid) {
        cur[u] = ldk(P->key + (u64)x * NB * 32 + ((qpk >> (8 * u)) & 255));
        acc.state += 8;
      }
    }
    // the four minima over the warp's slots are independent: their
    // reductions (two single-instruction 32-bit reductions each) overlap
    u64 mn[4];
#pragma unroll
    for (uint32_t u = 0; u < 4; u++)
      mn[u] = u < cnt ? warp_min_all(cand(v, x, w, cur[u])) : KEY_INF;  // cnt warp-uniform
    if (lane_id() == 0) {
#pragma unroll
      for (uint32_t u = 0; u < 4; u++) {
        const uint32_t q = (qpk >> (8 * u)) & 255;
        if (u < cnt && mn[u] < s[q]) s[q] = mn[u];
      }
    }
  }
  __device__ void endE(uint32_t v, int k, uint32_t mk, u64 *s) {
    const uint32_t lane = lane_id();
    if ((mk >> lane) & 1u) {
      const u64 best = s[k * 32 + lane];
      if (best != KEY_INF) lower_key<STRICT>(P->key + ((u64)v * NB + k) * 32 + lane, best);
    }
  }
};

// Push relaxation of an improved (x, q) over x's out-edges.
template <uint32_t ALGO, bool STORED, int NB>
struct RelaxPh {
  const MultiParams *P;
  uint32_t *nmask_next;
  uint32_t qpar;  // parity of the next wave's queue
  uint32_t tag;
  static constexpr bool STRICT = Strict<ALGO, STORED>::value;
  __device__ void beginQ(uint32_t x, int k, uint32_t mk, u64 &dx) {
    const uint32_t lane = lane_id();
    dx = INF32;
    if ((mk >> lane) & 1u) dx = key_value(ldk(P->key + ((u64)x * NB + k) * 32 + lane));
  }
  __device__ void edgeQ(uint32_t x, uint32_t y, uint32_t w, const uint32_t (&m)[NB],
                        u64 (&dx)[NB], Acc &acc) {
    const uint32_t lane = lane_id();
    const uint32_t wt = mweight<ALGO, STORED>(x, y, w);
    u64 cur[NB];
#pragma unroll
    for (int k = 0; k < NB; k++) {
      cur[k] = 0;
      if (dx[k] != INF32 && dx[k] + wt < INF32) {
        cur[k] = ldk(P->key + ((u64)y * NB + k) * 32 + lane);
        acc.state += 8;
      }
    }
    bool any = false;
#pragma unroll
    for (int k = 0; k < NB; k++) {
      if (!m[k]) continue;
      bool low = false;
      if (dx[k] != INF32 && dx[k] + wt < INF32)
        low = lower_from<STRICT>(P->key + ((u64)y * NB + k) * 32 + lane,
                                 pack_key((uint32_t)(dx[k] + wt), x + 1u), cur[k]);
      const unsigned bits = __ballot_sync(0xffffffffu, low);
      if (bits && lane == 0) {
        atomicOr(nmask_next + (u64)y * NB + k, bits);
        acc.improved += __popc(bits);
        any = true;
      }
    }
    if (lane == 0 && any) enqueue_once(*P, qpar, y, tag);
  }
  __device__ void endQ(uint32_t, int, uint32_t, u64 &) {}
  __device__ void beginE(uint32_t x, int k, uint32_t mk, u64 *s) {
    const uint32_t lane = lane_id();
    if ((mk >> lane) & 1u)
      s[k * 32 + lane] = key_value(ldk(P->key + ((u64)x * NB + k) * 32 + lane));
  }
  __device__ void edgesE(uint32_t x, uint32_t y, uint32_t w, bool valid, uint32_t qpk,
                         uint32_t cnt, u64 *s, Acc &acc) {
    const uint32_t wt = mweight<ALGO, STORED>(x, y, w);
    u64 cur[4], c[4];
#pragma unroll
    for (uint32_t u = 0; u < 4; u++) {
      cur[u] = 0;
      c[u] = INF32;
      if (u < cnt && valid) {
        const uint32_t q = (qpk >> (8 * u)) & 255;
        const uint32_t dx = (uint32_t)s[q];
        if (dx != INF32 && (u64)dx + wt < INF32) {
          c[u] = (u64)dx + wt;
          cur[u] = ldk(P->key + (u64)y * NB * 32 + q);
          acc.state += 8;
        }
      }
    }
    // first lowering attempts, independent and issued together
    u64 cand[4], got[4];
    bool tried[4];
#pragma unroll
    for (uint32_t u = 0; u < 4; u++) {
      tried[u] = false;
      cand[u] = KEY_INF;
      got[u] = 0;
      if (c[u] == INF32) continue;
      const uint32_t q = (qpk >> (8 * u)) & 255;
      cand[u] = pack_key((uint32_t)c[u], x + 1u);
      tried[u] = first_lower<STRICT>(P->key + (u64)y * NB * 32 + q, cand[u], cur[u], got[u]);
    }
    // improvements of this edge's queries (ascending), merged per mask word;
    // y enters the next wave's queue once
    uint32_t word = ~0u, bits = 0;
    bool any = false;
#pragma unroll
    for (uint32_t u = 0; u < 4; u++) {
      if (!tried[u]) continue;
      const uint32_t q = (qpk >> (8 * u)) & 255;
      if (!lowered<STRICT>(P->key + (u64)y * NB * 32 + q, cand[u], cur[u], got[u])) continue;
      if ((q >> 5) != word) {
        if (bits) atomicOr(nmask_next + (u64)y * NB + word, bits);
        word = q >> 5;
        bits = 0;
      }
      bits |= 1u << (q & 31);
      acc.improved++;
      any = true;
    }
    if (bits) atomicOr(nmask_next + (u64)y * NB + word, bits);
    if (any) enqueue_once(*P, qpar, y, tag);
  }
  __device__ void endE(uint32_t, int, uint32_t, u64 *) {}
};

// Masks of v taken from src[v] (cleared when `consume`; nobody else writes
// the buffer during the wave, so plain loads and stores suffice).
template <int NB>
__device__ __forceinline__ bool take_masks(uint32_t *src, uint32_t v, bool consume,
                                           uint32_t (&m)[NB]) {
  const uint32_t lane = lane_id();
  uint32_t x = 0;
  if (lane < (uint32_t)NB) {
    x = src[(u64)v * NB + lane];
    if (consume && x) src[(u64)v * NB + lane] = 0;
  }
  bool any = false;
#pragma unroll
  for (int k = 0; k < NB; k++) {
    m[k] = __shfl_sync(0xffffffffu, x, k);
    any |= m[k] != 0;
  }
  return any;
}

// ---- asynchronous worklist ----------------------------------------------------
// Invalidation and closure without wave barriers: producers set a vertex's
// mask bits and, unless an item of the vertex is already waiting, append the
// vertex to a ring; every warp claims ring positions in order and processes
// what arrives there. a_pend counts items appended and not yet finished (an
// item's own appends come before its completion), so once it reaches zero no
// item can appear any more and the waiting warps leave. Every wait is bounded
// by the launch's time limit (ERR_BARRIER).

__device__ bool async_push(const MultiParams &P, u64 item) {
  Ctl *c = P.ctl;
  atomicAdd(&c->a_pend, 1u);
  const u64 t = atomicAdd(&c->a_tail, 1ull);
  u64 *slot = P.ring + (t % P.ring_cap);
  // the position is free unless the item of the previous lap is still being
  // read by the warp that claimed it
  const u64 t0 = globaltimer_ns();
  while (atomicCAS(slot, A_EMPTY, item) != A_EMPTY) {
    if (*(volatile uint32_t *)&c->err) return false;
    if (globaltimer_ns() - t0 > P.timeout_ns) {
      atomicCAS(&c->err, 0u, ERR_BARRIER);
      return false;
    }
    __nanosleep(64);
  }
  return true;
}

// Lane 0 claims the next ring position and waits for its item; A_EMPTY when
// the worklist has drained (or the launch failed). Warp-uniform result.
__device__ __forceinline__ u64 async_pop(const MultiParams &P) {
  // (the caller's lanes read the item's mask record after this returns: the
  // fence below orders those reads after the item's arrival)
  Ctl *c = P.ctl;
  u64 item = A_EMPTY;
  if (lane_id() == 0) {
    const u64 h = atomicAdd(&c->a_head, 1ull);
    u64 *slot = P.ring + (h % P.ring_cap);
    const u64 t0 = globaltimer_ns();
    for (;;) {
      const u64 x = *(volatile u64 *)slot;
      if (x != A_EMPTY) {
        atomicExch(slot, A_EMPTY);
        item = x;
        break;
      }
      if (*(volatile uint32_t *)&c->a_pend == 0u || *(volatile uint32_t *)&c->err) break;
      if (globaltimer_ns() - t0 > P.timeout_ns) {
        atomicCAS(&c->err, 0u, ERR_BARRIER);
        break;
      }
      __nanosleep(32);
    }
  }
  item = __shfl_sync(0xffffffffu, item, 0);
  __threadfence();
  return item;
}

// Masks of v taken atomically from pend (producers may set bits meanwhile).
template <int NB>
__device__ __forceinline__ bool take_masks_atomic(uint32_t *pend, uint32_t v, uint32_t (&m)[NB]) {
  const uint32_t lane = lane_id();
  uint32_t x = 0;
  if (lane < (uint32_t)NB) x = atomicExch(pend + (u64)v * NB + lane, 0u);
  bool any = false;
#pragma unroll
  for (int k = 0; k < NB; k++) {
    m[k] = __shfl_sync(0xffffffffu, x, k);
    any |= m[k] != 0;
  }
  return any;
}

// One asynchronous phase over adjacency A: the vertices items[0..cnt) (their
// masks already in pend) are appended, a barrier, then every warp drains the
// worklist; rows whose work exceeds P.heavy are split into tile items with
// their masks in a pool record (or expanded by the warp itself when the pool
// or the tile budget is exhausted). Ends with a barrier that resets the ring.
template <int NB, bool WITH_W, class Ph>
__device__ bool async_phase(const MultiParams &P, const Adj &A, const uint32_t *items,
                            uint32_t cnt, uint32_t *pend, Ph &ph, u64 *s, Acc &acc,
                            uint32_t qratio) {
  Ctl *c = P.ctl;
  const uint32_t lane = lane_id();
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  for (uint32_t i = gtid; i < cnt; i += gridDim.x * blockDim.x) {
    const uint32_t v = items[i];
    if (atomicExch(P.inq + v, 1u) == 0u) async_push(P, v);
  }
  if (!grid_sync(c, SYNC_RESET_Q0 | SYNC_RESET_Q1, P.timeout_ns)) return false;
  for (;;) {
    const u64 item = async_pop(P);
    if (item == A_EMPTY) break;
    const uint32_t v = (uint32_t)item;
    const uint32_t rec1 = (uint32_t)(item >> 32) & 0xFFFFu;
    uint32_t m[NB];
    const uint32_t len = A.len[v];
    if (rec1) {  // one tile of a split row
      const uint32_t t = (uint32_t)(item >> 48);
      uint32_t x = 0;
      if (lane < (uint32_t)NB) x = P.pool[(u64)(rec1 - 1) * NB + lane];
      uint32_t act = 0;
#pragma unroll
      for (int k = 0; k < NB; k++) {
        m[k] = __shfl_sync(0xffffffffu, x, k);
        act += __popc(m[k]);
      }
      const bool ql = use_query_lanes(act, len, qratio);
      const uint32_t ts = ql ? P.tile : MULTI_MIN_TILE;
      expand_vertex<NB, WITH_W>(A, v, m, t * ts, min(len, (t + 1) * ts), 32, ql, ph, s, acc);
      if (lane == 0) atomicSub(&c->a_tiles, 1u);
    } else {
      if (lane == 0) atomicExch(P.inq + v, 0u);
      __threadfence();
      __syncwarp();
      if (take_masks_atomic<NB>(pend, v, m) && len) {
        uint32_t act = 0;
#pragma unroll
        for (int k = 0; k < NB; k++) act += __popc(m[k]);
        const bool ql = use_query_lanes(act, len, qratio);
        const u64 work = ql ? len : (u64)((len + 31) / 32) * act;
        const uint32_t ts = ql ? P.tile : MULTI_MIN_TILE;
        const uint32_t nt = (len + ts - 1) / ts;
        bool split = false;
        if (work > P.heavy && nt > 1 && nt <= A_MAX_TILES) {
          uint32_t rec = 0;
          if (lane == 0) {
            rec = atomicAdd(&c->a_pool, 1u);
            if (rec < P.pool_cap && atomicAdd(&c->a_tiles, nt) + nt <= A_TILE_CAP) {
              split = true;
            } else if (rec < P.pool_cap) {
              atomicSub(&c->a_tiles, nt);
            }
          }
          split = __shfl_sync(0xffffffffu, split, 0);
          rec = __shfl_sync(0xffffffffu, rec, 0);
          if (split) {
#pragma unroll
            for (int k = 0; k < NB; k++)
              if (lane == (uint32_t)k) P.pool[(u64)rec * NB + k] = m[k];
            __threadfence();
            __syncwarp();
            for (uint32_t t = lane; t < nt; t += 32)
              async_push(P, (u64)v | ((u64)(rec + 1) << 32) | ((u64)t << 48));
          }
        }
        if (!split) expand_vertex<NB, WITH_W>(A, v, m, 0, len, 32, ql, ph, s, acc);
      }
    }
    __syncwarp();
    __threadfence();
    if (lane == 0) atomicSub(&c->a_pend, 1u);
  }
  return grid_sync(c, SYNC_RESET_ASYNC | SYNC_RESET_Q0 | SYNC_RESET_Q1, P.timeout_ns);
}

// CTAs per SM the register allocation is sized for at 8 blocks of queries:
// 3 (85 registers, ~140 bytes of spills per thread) measured ~3% faster on
// the R-MAT 24 / 256-query workload than 2 (104 registers, no spills)
#ifndef DYCG_MULTI_MIN_BLOCKS
#define DYCG_MULTI_MIN_BLOCKS 3
#endif

template <uint32_t ALGO, bool STORED, int NB>
__global__ void __launch_bounds__(BLOCK, NB >= 8 ? DYCG_MULTI_MIN_BLOCKS : 3)
    multi_repair_kernel(MultiParams P) {
  Ctl *ctl = P.ctl;
  Acc acc = {0, 0, 0, 0, 0, 0};
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t lane = lane_id();
  const uint32_t gw = gtid >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  constexpr uint32_t Q = NB * 32;
  // every block reads the sequence counters before its first barrier
  const uint32_t epoch = *(volatile uint32_t *)&P.seq[0];
  const uint32_t tag0 = *(volatile uint32_t *)&P.seq[1];
  uint32_t tag = tag0 + 1;  // next unused wave tag (uniform over the grid)
  uint32_t waves = 0;
  if (gtid == 0) ctl->stat[ST_T_START] = globaltimer_ns();
  __shared__ u64 s_state[WARPS][Q];  // edge-lane per-query state of each warp
  __shared__ uint2 s_stage[MULTI_MIN_TILE];  // staged slots of an edge-lane tile
  u64 *s = s_state[threadIdx.x >> 5];

  if (P.phases & PH_DELETE) {
    // 1. seeds: (v, q) with parent_q(v) == u for a deleted (u, v); one warp per record
    const uint32_t n_del = *P.n_del_ptr;
    for (uint32_t i = gw; i < n_del; i += nw) {
      if (!P.del_found[i]) continue;
      const uint2 e = P.del_uv[i];
      bool any = false;
#pragma unroll
      for (int k = 0; k < NB; k++) {
        const u64 kv = ld_key(P.key + (u64)e.y * Q + k * 32 + lane);
        const unsigned bits = __ballot_sync(0xffffffffu, key_parent1(kv) == e.x + 1u);
        if (bits && lane == 0) {
          const uint32_t old = atomicOr(P.affm + (u64)e.y * NB + k, bits);
          if (bits & ~old) {
            atomicOr(P.inew[0] + (u64)e.y * NB + k, bits & ~old);
            any = true;
          }
        }
      }
      if (lane == 0 && any) {
        note_affected(P, e.y, epoch);
        enqueue_once(P, 0, e.y, tag0);
      }
    }
    if (!grid_sync(ctl, 0, P.timeout_ns)) goto done;
    // 2. invalidation waves (or one asynchronous phase)
    if (P.async) {
      const uint32_t cnt = *(volatile uint32_t *)&ctl->snap_q[0];
      InvalidatePh<NB> ph{&P, P.inew[0], QPAR_ASYNC, tag++, epoch};
      if (!async_phase<NB, false>(P, P.out, P.q[0], cnt, P.inew[0], ph, s, acc, P.qratio))
        goto done;
      waves++;
    } else {
      uint32_t cur = 0;
      for (uint32_t wave = 0;; wave++) {
        const uint32_t cnt = *(volatile uint32_t *)&ctl->snap_q[cur];
        if (cnt == 0) break;
        if (wave >= P.max_waves) {
          if (gtid == 0) atomicCAS(&ctl->err, 0u, ERR_WAVES);
          break;
        }
        const uint32_t par = wave & 1;
        InvalidatePh<NB> ph{&P, P.inew[par ^ 1], cur ^ 1, tag++, epoch};
        uint32_t *src = P.inew[par];
        auto prep = [&](uint32_t v, uint32_t (&m)[NB]) { return take_masks<NB>(src, v, true, m); };
        if (!multi_expand<NB, false>(P, P.out, P.q[cur], cnt, prep, ph, s, s_stage, acc, cur,
                                     cur ? SYNC_RESET_Q1 : SYNC_RESET_Q0, P.qratio))
          goto done;
        waves++;
        cur ^= 1;
      }
    }
    if (gtid == 0) ctl->tphase[0] = globaltimer_ns();  // seeds + invalidation done
    // 3. reset the affected (v, q)
    {
      const uint32_t na = *(volatile uint32_t *)&ctl->snap_aff;
      for (uint32_t i = gw; i < na; i += nw) {
        const uint32_t v = P.aff[i];
#pragma unroll
        for (int k = 0; k < NB; k++) {
          const uint32_t mk = P.affm[(u64)v * NB + k];
          if ((mk >> lane) & 1u) P.key[(u64)v * Q + k * 32 + lane] = KEY_INF;
        }
      }
      if (!grid_sync(ctl, 0, P.timeout_ns)) goto done;
      // 4. pull over in-rows
      PullPh<ALGO, STORED, NB> ph{&P};
      auto prep = [&](uint32_t v, uint32_t (&m)[NB]) { return take_masks<NB>(P.affm, v, false, m); };
      if (!multi_expand<NB, STORED>(P, P.in, P.aff, na, prep, ph, s, s_stage, acc, NO_QUEUE, 0,
                                    P.pull_qratio))
        goto done;
      if (gtid == 0) ctl->tphase[1] = globaltimer_ns();  // reset + pull done
    }
  }
  {
    // 5. frontier: affected (v, q) with a finite value, then insertion seeds
    const uint32_t ftag = tag++;
    if (P.phases & PH_DELETE) {
      const uint32_t na = *(volatile uint32_t *)&ctl->snap_aff;
      for (uint32_t i = gw; i < na; i += nw) {
        const uint32_t v = P.aff[i];
        bool any = false;
#pragma unroll
        for (int k = 0; k < NB; k++) {
          const uint32_t mk = P.affm[(u64)v * NB + k];
          const bool fin = ((mk >> lane) & 1u) &&
                           key_value(ld_key(P.key + (u64)v * Q + k * 32 + lane)) != INF32;
          const unsigned bits = __ballot_sync(0xffffffffu, fin);
          if (bits && lane == 0) {
            atomicOr(P.nmask[0] + (u64)v * NB + k, bits);
            any = true;
          }
        }
        if (lane == 0 && any) enqueue_once(P, 0, v, ftag);
      }
    }
    if (P.phases & PH_INSERT) {
      for (uint32_t i = gw; i < P.n_add; i += nw) {
        const uint3 e = P.add_uvw[i];
        if (e.x >= P.n || e.y >= P.n) continue;
        bool any = false;
#pragma unroll
        for (int k = 0; k < NB; k++) {
          bool low = false;
          const uint32_t du = key_value(ld_key(P.key + (u64)e.x * Q + k * 32 + lane));
          if (du != INF32) {
            const u64 c = (u64)du + mweight<ALGO, STORED>(e.x, e.y, e.z);
            if (c < INF32)
              low = lower_key<Strict<ALGO, STORED>::value>(P.key + (u64)e.y * Q + k * 32 + lane,
                                                           pack_key((uint32_t)c, e.x + 1u));
          }
          const unsigned bits = __ballot_sync(0xffffffffu, low);
          if (bits && lane == 0) {
            atomicOr(P.nmask[0] + (u64)e.y * NB + k, bits);
            any = true;
          }
        }
        if (lane == 0 && any) enqueue_once(P, 0, e.y, ftag);
      }
    }
  }
  if (!grid_sync(ctl, 0, P.timeout_ns)) goto done;
  if (gtid == 0) ctl->tphase[2] = globaltimer_ns();  // frontier + insertion seeds done
  // 6. closure waves (or one asynchronous phase)
  if ((P.phases & PH_CLOSE) && P.async) {
    const uint32_t cnt = *(volatile uint32_t *)&ctl->snap_q[0];
    RelaxPh<ALGO, STORED, NB> ph{&P, P.nmask[0], QPAR_ASYNC, tag++};
    if (!async_phase<NB, STORED>(P, P.out, P.q[0], cnt, P.nmask[0], ph, s, acc, P.qratio))
      goto done;
    waves++;
  } else if (P.phases & PH_CLOSE) {
    uint32_t cur = 0;
    for (uint32_t wave = 0;; wave++) {
      const uint32_t cnt = *(volatile uint32_t *)&ctl->snap_q[cur];
      if (cnt == 0) break;
      if (wave >= P.max_waves) {
        if (gtid == 0) atomicCAS(&ctl->err, 0u, ERR_WAVES);
        break;
      }
      const uint32_t par = wave & 1;
      RelaxPh<ALGO, STORED, NB> ph{&P, P.nmask[par ^ 1], cur ^ 1, tag++};
      uint32_t *src = P.nmask[par];
      auto prep = [&](uint32_t v, uint32_t (&m)[NB]) { return take_masks<NB>(src, v, true, m); };
      if (!multi_expand<NB, STORED>(P, P.out, P.q[cur], cnt, prep, ph, s, s_stage, acc, cur,
                                    cur ? SYNC_RESET_Q1 : SYNC_RESET_Q0, P.qratio))
        goto done;
      waves++;
      cur ^= 1;
    }
  }
  if (gtid == 0) ctl->tphase[3] = globaltimer_ns();  // closure done
  // 7. clear the snapshot's affected masks
  if (P.phases & PH_DELETE) {
    const uint32_t na = *(volatile uint32_t *)&ctl->snap_aff;
    for (uint32_t i = gw; i < na; i += nw)
      if (lane < (uint32_t)NB) P.affm[(u64)P.aff[i] * NB + lane] = 0;
  }
done:
  acc.flush(ctl);
  __syncthreads();
  if (threadIdx.x == 0) atomicMax(&ctl->stat[ST_T_END], globaltimer_ns());
  if (gtid == 0) {
    atomicAdd(&ctl->stat[ST_AFFECTED], (u64)ctl->snap_aff);
    ctl->waves = waves;
    ctl->wave_tag = tag;
    P.seq[0] = epoch + 1;
    P.seq[1] = tag + 1;
  }
}

// Static solve set-up: every (v, q) unreachable, then (source_q, q) = 0 in
// the first closure frontier.
__global__ void multi_init_kernel(u64 *key, u64 total) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < total;
       i += (u64)gridDim.x * blockDim.x)
    key[i] = KEY_INF;
}

__global__ void multi_seed_kernel(u64 *key, uint32_t n, uint32_t nb, const uint32_t *sources,
                                  uint32_t *nmask0, uint32_t *q0, uint32_t *wtag,
                                  const uint32_t *seq, Ctl *ctl, bool ranges) {
  const uint32_t Q = nb * 32;
  const uint32_t tag = seq[1];
  const uint32_t rsize = (n + QRANGES - 1) / QRANGES;
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < Q; q += gridDim.x * blockDim.x) {
    const uint32_t s = sources[q];
    if (s >= n) continue;
    key[(u64)s * Q + q] = pack_key(0, 0);
    atomicOr(nmask0 + (u64)s * nb + q / 32, 1u << (q % 32));
    if (atomicExch(wtag + s, tag) != tag) {
      const uint32_t k = atomicAdd(&ctl->q_count[0], 1u);  // ranges: seeds into their regions
      if (ranges) {
        const uint32_t b = s / rsize;
        q0[b * rsize + atomicAdd(&ctl->qrange[0][b], 1u)] = s;
      } else {
        q0[k] = s;
      }
    }
  }
}

__global__ void multi_gather_kernel(const u64 *key, uint32_t n, uint32_t Q, uint32_t q,
                                    uint32_t *values, uint32_t *parents) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const u64 k = Q ? key[(u64)v * Q + q] : key[v];
    const uint32_t val = key_value(k), p1 = key_parent1(k);
    values[v] = val;
    parents[v] = (val == INF32 || p1 == 0) ? INF32 : p1 - 1;
  }
}

template <uint32_t ALGO, bool STORED, int NB>
static cudaError_t launch_multi_t(const MultiLaunch &L, cudaStream_t s) {
  MultiParams P;
  P.out = L.out;
  P.in = L.in;
  P.key = L.key;
  P.affm = L.affm;
  P.inew[0] = L.inew0;
  P.inew[1] = L.inew1;
  P.nmask[0] = L.nmask0;
  P.nmask[1] = L.nmask1;
  P.cmask = L.cmask;
  P.mark = L.mark;
  P.wtag = L.wtag;
  P.aff = L.aff;
  P.q[0] = L.q0;
  P.q[1] = L.q1;
  P.tiles = Tiles{L.tiles, L.tile_cap};
  P.ctl = L.ctl;
  P.seq = L.seq;
  P.del_uv = L.del_uv;
  P.del_found = L.del_found;
  P.n_del_ptr = L.n_del_ptr;
  P.add_uvw = L.add_uvw;
  P.n_add = L.n_add;
  P.n = L.n;
  P.phases = L.phases;
  P.max_waves = L.max_waves;
  P.qratio = L.qratio;
  P.pull_qratio = L.pull_qratio;
  P.heavy = std::max(L.heavy, 1u);
  P.tile = std::max(L.tile, MULTI_MIN_TILE);
  P.sched = L.sched & 1u;
  P.async = (L.sched & 4u) != 0;
  P.ranges = (L.sched & 2u) != 0 && !P.async;  // the worklist reads the plain queue
  P.ring = L.ring;
  P.ring_cap = L.ring_cap;
  P.inq = L.inq;
  P.pool = L.pool;
  P.pool_cap = L.pool_cap;
  P.rsize = (L.n + QRANGES - 1) / QRANGES;
  P.timeout_ns = L.timeout_ns;
  static int blocks_per_sm = -1;
  if (blocks_per_sm < 0) {
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &blocks_per_sm, multi_repair_kernel<ALGO, STORED, NB>, BLOCK, 0);
    if (e != cudaSuccess) return e;
    if (blocks_per_sm < 1) return cudaErrorLaunchOutOfResources;
  }
  // cooperative (co-resident blocks for the grid barrier); this launch form
  // can also be recorded into a CUDA graph
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks_per_sm * L.num_sms);
  cfg.blockDim = dim3(BLOCK);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, multi_repair_kernel<ALGO, STORED, NB>, P);
}

template <uint32_t ALGO, bool STORED>
static cudaError_t launch_multi_nb(const MultiLaunch &L, cudaStream_t s) {
  switch (L.nb) {
    case 1: return launch_multi_t<ALGO, STORED, 1>(L, s);
    case 2: return launch_multi_t<ALGO, STORED, 2>(L, s);
    case 4: return launch_multi_t<ALGO, STORED, 4>(L, s);
    case 8: return launch_multi_t<ALGO, STORED, 8>(L, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_multi(const MultiLaunch &L, cudaStream_t s) {
  if (L.algo == ALGO_SSSP)
    return L.stored ? launch_multi_nb<ALGO_SSSP, true>(L, s)
                    : launch_multi_nb<ALGO_SSSP, false>(L, s);
  if (L.algo == ALGO_BFS) return launch_multi_nb<ALGO_BFS, false>(L, s);
  return cudaErrorInvalidValue;
}

cudaError_t launch_multi_init(u64 *key, uint32_t n, uint32_t nb, const uint32_t *sources,
                              uint32_t *nmask0, uint32_t *q0, uint32_t *wtag, const uint32_t *seq,
                              Ctl *ctl, uint32_t sched, cudaStream_t s) {
  multi_init_kernel<<<148 * 16, BLOCK, 0, s>>>(key, (u64)n * nb * 32);
  multi_seed_kernel<<<1, BLOCK, 0, s>>>(key, n, nb, sources, nmask0, q0, wtag, seq, ctl,
                                        (sched & 2u) != 0 && (sched & 4u) == 0);
  return cudaGetLastError();
}

cudaError_t launch_multi_gather(const u64 *key, uint32_t n, uint32_t Q, uint32_t q,
                                uint32_t *values, uint32_t *parents, cudaStream_t s) {
  multi_gather_kernel<<<148 * 8, BLOCK, 0, s>>>(key, n, Q, q, values, parents);
  return cudaGetLastError();
}

}  // namespace dycg
