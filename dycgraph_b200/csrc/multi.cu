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
// Two warp mappings, chosen per vertex by the number of active queries
// (edge_lanes, the tuned threshold):
//   query lanes -- the warp loads 32 slots, then visits them one by one; for
//                  each edge lane i works on query 32*b + i of every active
//                  block b (one coalesced key line per edge and block);
//   edge lanes  -- lane i works on slot i for each active query in turn (the
//                  single-query mapping), for vertices active in few queries.
// Per query the phases are the single-query repair's (repair.cu): deletion
// seeds (parent == u), invalidation waves over out-rows, reset, pull over
// in-rows, frontier + insertion seeds, push closure. The batched form has no
// counterpart in the reference engine, which repairs one source per engine
// (include/framework/framework.cuh:1803 InitGraph(src)).
#include "frontier.cuh"
#include "internal.h"

namespace dycg {

constexpr int ST = 8;  // per-vertex state slots: max(blocks, edge-lane queries)
static_assert(MULTI_MAX_BLOCKS <= ST && MULTI_EDGE_LANES_MAX <= ST, "state slots");

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
  uint32_t n, phases, max_waves, edge_lanes, heavy, tile;
  u64 timeout_ns;
};

template <uint32_t ALGO, bool STORED>
__device__ __forceinline__ uint32_t mweight(uint32_t u, uint32_t v, uint32_t w) {
  return STORED ? w : rule_weight<ALGO>(u, v);
}

// Lower *addr to cand; true when the value decreased (strict CAS form where
// zero weights are possible, atomicMin with parent tie-break otherwise).
template <bool STRICT>
__device__ __forceinline__ bool lower_key(u64 *addr, u64 cand) {
  if (STRICT) return strict_lower(addr, cand);
  if (cand < ld_key(addr)) return key_value(atomicMin(addr, cand)) > key_value(cand);
  return false;
}

__device__ __forceinline__ void enqueue_once(const MultiParams &P, uint32_t *q, uint32_t *count,
                                             uint32_t y, uint32_t tag) {
  if (atomicExch(P.wtag + y, tag) != tag) {
    const uint32_t s = atomicAdd(count, 1u);
    if (s < P.n) q[s] = y;
    else atomicCAS(&P.ctl->err, 0u, ERR_QUEUE);
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

// Expand slots [b, e) of v's row for the queries in masks m (warp-uniform).
// Ph supplies, for the query-lane mapping, beginQ/visitQ/endQ over blocks and,
// for the edge-lane mapping, beginE/visitE/endE over single queries.
template <int NB, bool WITH_W, class Ph>
__device__ __forceinline__ void expand_vertex(const MultiParams &P, const Adj &A, uint32_t v,
                                              const uint32_t (&m)[NB], uint32_t b, uint32_t e,
                                              uint32_t stride, Ph &ph, Acc &acc) {
  const uint32_t lane = lane_id();
  uint32_t tot = 0;
#pragma unroll
  for (int k = 0; k < NB; k++) tot += __popc(m[k]);
  if (tot == 0) return;
  if (lane == 0 && b == 0) acc.expanded++;
  const u64 off = A.off[v];
  u64 st[ST];
  if (tot <= P.edge_lanes) {
    // lane j < tot finds the j-th active query; broadcast into registers
    uint32_t mine = INF32, seen = 0;
#pragma unroll
    for (int k = 0; k < NB; k++) {
      const uint32_t c = __popc(m[k]);
      if (mine == INF32 && lane >= seen && lane < seen + c) {
        uint32_t mm = m[k];
        for (uint32_t r = lane - seen; r; r--) mm &= mm - 1;
        mine = k * 32 + __ffs(mm) - 1;
      }
      seen += c;
    }
    uint32_t qj[MULTI_EDGE_LANES_MAX];
#pragma unroll
    for (int j = 0; j < (int)MULTI_EDGE_LANES_MAX; j++) {
      qj[j] = __shfl_sync(0xffffffffu, mine, j);
      if (j < (int)tot) ph.beginE(v, qj[j], st[j]);
    }
    auto visit = [&](uint32_t y, uint32_t w, bool valid) {
#pragma unroll
      for (int j = 0; j < (int)MULTI_EDGE_LANES_MAX; j++)
        if (j < (int)tot) ph.visitE(v, y, w, valid, qj[j], st[j], acc);
    };
    walk<WITH_W>(A, off, b, e, stride, visit, acc);
#pragma unroll
    for (int j = 0; j < (int)MULTI_EDGE_LANES_MAX; j++)
      if (j < (int)tot) ph.endE(v, qj[j], st[j]);
  } else {
#pragma unroll
    for (int k = 0; k < NB; k++) ph.beginQ(v, k, m[k], st[k]);
    auto visit = [&](uint32_t y, uint32_t w, bool valid) {
      unsigned vb = __ballot_sync(0xffffffffu, valid);
      while (vb) {
        const int src = __ffs(vb) - 1;
        vb &= vb - 1;
        const uint32_t yy = __shfl_sync(0xffffffffu, y, src);
        const uint32_t ww = __shfl_sync(0xffffffffu, w, src);
#pragma unroll
        for (int k = 0; k < NB; k++)
          if (m[k]) ph.visitQ(v, yy, ww, k, m[k], st[k], acc);
      }
    };
    walk<WITH_W>(A, off, b, e, stride, visit, acc);
#pragma unroll
    for (int k = 0; k < NB; k++)
      if (m[k]) ph.endQ(v, k, m[k], st[k]);
  }
}

// Expand items[0..cnt): prep(v, m) fills v's masks (false: skip). Rows longer
// than P.heavy are cut into P.tile-slot tiles that whole CTAs process after a
// grid barrier; their masks travel through cmask. Ends with a barrier that
// applies reset_flags. Returns false when the launch has failed.
template <int NB, bool WITH_W, class Prep, class Ph>
__device__ bool multi_expand(const MultiParams &P, const Adj &A, const uint32_t *items,
                             uint32_t cnt, Prep &prep, Ph &ph, Acc &acc, uint32_t reset_flags) {
  Ctl *ctl = P.ctl;
  const uint32_t lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = gw; i < cnt; i += nw) {
    const uint32_t v = items[i];
    uint32_t m[NB];
    if (!prep(v, m)) continue;
    const uint32_t len = A.len[v];
    if (len > P.heavy) {
#pragma unroll
      for (int k = 0; k < NB; k++)
        if (lane == (uint32_t)k) P.cmask[(u64)v * NB + k] = m[k];
      if (lane == 0) {
        const uint32_t nt = (len + P.tile - 1) / P.tile;
        const uint32_t base = atomicAdd(&ctl->tile_count, nt);
        if (base + nt > P.tiles.cap) {
          atomicCAS(&ctl->err, 0u, ERR_TILES);
        } else {
          for (uint32_t t = 0; t < nt; t++)
            P.tiles.tiles[base + t] = make_uint4(v, t * P.tile, min(len, (t + 1) * P.tile), 0);
        }
      }
      continue;
    }
    expand_vertex<NB, WITH_W>(P, A, v, m, 0, len, 32, ph, acc);
  }
  if (!grid_sync(ctl, reset_flags, P.timeout_ns)) return false;
  const uint32_t nt = min(*(volatile uint32_t *)&ctl->snap_tiles, P.tiles.cap);
  if (nt == 0) return true;
  const uint32_t wib = threadIdx.x >> 5;
  for (uint32_t t = blockIdx.x; t < nt; t += gridDim.x) {
    const uint4 tl = P.tiles.tiles[t];
    uint32_t m[NB];
#pragma unroll
    for (int k = 0; k < NB; k++) m[k] = P.cmask[(u64)tl.x * NB + k];
    expand_vertex<NB, WITH_W>(P, A, tl.x, m, tl.y + wib * 32, tl.z, blockDim.x, ph, acc);
  }
  return grid_sync(ctl, SYNC_RESET_TILES, P.timeout_ns);
}

// Children y of a newly affected (x, q) with parent_q(y) == x become affected.
template <int NB>
struct InvalidatePh {
  const MultiParams *P;
  uint32_t *inew_next, *nq, *nc;
  uint32_t tag, epoch;
  __device__ void mark(uint32_t y, uint32_t k, uint32_t bits) {
    const uint32_t old = atomicOr(P->affm + (u64)y * NB + k, bits);
    const uint32_t fresh = bits & ~old;
    if (fresh) {
      atomicOr(inew_next + (u64)y * NB + k, fresh);
      note_affected(*P, y, epoch);
      enqueue_once(*P, nq, nc, y, tag);
    }
  }
  __device__ void beginQ(uint32_t, int, uint32_t, u64 &) {}
  __device__ void visitQ(uint32_t x, uint32_t y, uint32_t, int k, uint32_t mk, u64 &, Acc &acc) {
    const uint32_t lane = lane_id();
    bool child = false;
    if ((mk >> lane) & 1u) {
      child = key_parent1(ld_key(P->key + ((u64)y * NB + k) * 32 + lane)) == x + 1u;
      acc.state += 8;
    }
    const unsigned bits = __ballot_sync(0xffffffffu, child);
    if (bits && lane == 0) mark(y, k, bits);
  }
  __device__ void endQ(uint32_t, int, uint32_t, u64 &) {}
  __device__ void beginE(uint32_t, uint32_t, u64 &) {}
  __device__ void visitE(uint32_t x, uint32_t y, uint32_t, bool valid, uint32_t q, u64 &,
                         Acc &acc) {
    if (!valid) return;
    acc.state += 8;
    if (key_parent1(ld_key(P->key + (u64)y * NB * 32 + q)) == x + 1u)
      mark(y, q >> 5, 1u << (q & 31));
  }
  __device__ void endE(uint32_t, uint32_t, u64 &) {}
};

// Affected (v, q) takes the best (value(x) + w, parent x) over live in-edges.
template <uint32_t ALGO, bool STORED, int NB>
struct PullPh {
  const MultiParams *P;
  static constexpr bool STRICT = Strict<ALGO, STORED>::value;
  __device__ void beginQ(uint32_t, int, uint32_t, u64 &best) { best = KEY_INF; }
  __device__ void visitQ(uint32_t v, uint32_t x, uint32_t w, int k, uint32_t mk, u64 &best,
                         Acc &acc) {
    const uint32_t lane = lane_id();
    if (!((mk >> lane) & 1u)) return;
    acc.state += 8;
    const uint32_t vx = key_value(ld_key(P->key + ((u64)x * NB + k) * 32 + lane));
    if (vx == INF32) return;
    const u64 c = (u64)vx + mweight<ALGO, STORED>(x, v, w);
    if (c >= INF32) return;
    const u64 cand = pack_key((uint32_t)c, x + 1u);
    best = cand < best ? cand : best;
  }
  __device__ void endQ(uint32_t v, int k, uint32_t mk, u64 &best) {
    const uint32_t lane = lane_id();
    if (((mk >> lane) & 1u) && best != KEY_INF)
      lower_key<STRICT>(P->key + ((u64)v * NB + k) * 32 + lane, best);
  }
  __device__ void beginE(uint32_t, uint32_t, u64 &best) { best = KEY_INF; }
  __device__ void visitE(uint32_t v, uint32_t x, uint32_t w, bool valid, uint32_t q, u64 &best,
                         Acc &acc) {
    if (!valid) return;
    acc.state += 8;
    const uint32_t vx = key_value(ld_key(P->key + (u64)x * NB * 32 + q));
    if (vx == INF32) return;
    const u64 c = (u64)vx + mweight<ALGO, STORED>(x, v, w);
    if (c >= INF32) return;
    const u64 cand = pack_key((uint32_t)c, x + 1u);
    best = cand < best ? cand : best;
  }
  __device__ void endE(uint32_t v, uint32_t q, u64 &best) {
    const u64 mn = warp_min(best);
    if (lane_id() == 0 && mn != KEY_INF) lower_key<STRICT>(P->key + (u64)v * NB * 32 + q, mn);
  }
};

// Push relaxation of an improved (x, q) over x's out-edges.
template <uint32_t ALGO, bool STORED, int NB>
struct RelaxPh {
  const MultiParams *P;
  uint32_t *nmask_next, *nq, *nc;
  uint32_t tag;
  static constexpr bool STRICT = Strict<ALGO, STORED>::value;
  __device__ void beginQ(uint32_t x, int k, uint32_t mk, u64 &dx) {
    const uint32_t lane = lane_id();
    dx = INF32;
    if ((mk >> lane) & 1u) dx = key_value(ld_key(P->key + ((u64)x * NB + k) * 32 + lane));
  }
  __device__ void visitQ(uint32_t x, uint32_t y, uint32_t w, int k, uint32_t, u64 &dx, Acc &acc) {
    const uint32_t lane = lane_id();
    bool low = false;
    if (dx != INF32) {
      acc.state += 8;
      const u64 c = dx + mweight<ALGO, STORED>(x, y, w);
      if (c < INF32)
        low = lower_key<STRICT>(P->key + ((u64)y * NB + k) * 32 + lane,
                                pack_key((uint32_t)c, x + 1u));
    }
    const unsigned bits = __ballot_sync(0xffffffffu, low);
    if (bits && lane == 0) {
      atomicOr(nmask_next + (u64)y * NB + k, bits);
      enqueue_once(*P, nq, nc, y, tag);
      acc.improved += __popc(bits);
    }
  }
  __device__ void endQ(uint32_t, int, uint32_t, u64 &) {}
  __device__ void beginE(uint32_t x, uint32_t q, u64 &dx) {
    dx = key_value(ld_key(P->key + (u64)x * NB * 32 + q));
  }
  __device__ void visitE(uint32_t x, uint32_t y, uint32_t w, bool valid, uint32_t q, u64 &dx,
                         Acc &acc) {
    if (!valid || dx == INF32) return;
    acc.state += 8;
    const u64 c = dx + mweight<ALGO, STORED>(x, y, w);
    if (c >= INF32) return;
    if (lower_key<STRICT>(P->key + (u64)y * NB * 32 + q, pack_key((uint32_t)c, x + 1u))) {
      atomicOr(nmask_next + (u64)y * NB + (q >> 5), 1u << (q & 31));
      enqueue_once(*P, nq, nc, y, tag);
      acc.improved++;
    }
  }
  __device__ void endE(uint32_t, uint32_t, u64 &) {}
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

template <uint32_t ALGO, bool STORED, int NB>
__global__ void __launch_bounds__(BLOCK) multi_repair_kernel(MultiParams P) {
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
        enqueue_once(P, P.q[0], &ctl->q_count[0], e.y, tag0);
      }
    }
    if (!grid_sync(ctl, 0, P.timeout_ns)) goto done;
    // 2. invalidation waves
    {
      uint32_t cur = 0;
      for (uint32_t wave = 0;; wave++) {
        const uint32_t cnt = *(volatile uint32_t *)&ctl->snap_q[cur];
        if (cnt == 0) break;
        if (wave >= P.max_waves) {
          if (gtid == 0) atomicCAS(&ctl->err, 0u, ERR_WAVES);
          break;
        }
        const uint32_t par = wave & 1;
        InvalidatePh<NB> ph{&P, P.inew[par ^ 1], P.q[cur ^ 1], &ctl->q_count[cur ^ 1], tag++, epoch};
        uint32_t *src = P.inew[par];
        auto prep = [&](uint32_t v, uint32_t (&m)[NB]) { return take_masks<NB>(src, v, true, m); };
        if (!multi_expand<NB, false>(P, P.out, P.q[cur], cnt, prep, ph, acc,
                                     cur ? SYNC_RESET_Q1 : SYNC_RESET_Q0))
          goto done;
        waves++;
        cur ^= 1;
      }
    }
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
      if (!multi_expand<NB, STORED>(P, P.in, P.aff, na, prep, ph, acc, 0)) goto done;
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
        if (lane == 0 && any) enqueue_once(P, P.q[0], &ctl->q_count[0], v, ftag);
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
        if (lane == 0 && any) enqueue_once(P, P.q[0], &ctl->q_count[0], e.y, ftag);
      }
    }
  }
  if (!grid_sync(ctl, 0, P.timeout_ns)) goto done;
  // 6. closure waves
  if (P.phases & PH_CLOSE) {
    uint32_t cur = 0;
    for (uint32_t wave = 0;; wave++) {
      const uint32_t cnt = *(volatile uint32_t *)&ctl->snap_q[cur];
      if (cnt == 0) break;
      if (wave >= P.max_waves) {
        if (gtid == 0) atomicCAS(&ctl->err, 0u, ERR_WAVES);
        break;
      }
      const uint32_t par = wave & 1;
      RelaxPh<ALGO, STORED, NB> ph{&P, P.nmask[par ^ 1], P.q[cur ^ 1], &ctl->q_count[cur ^ 1], tag++};
      uint32_t *src = P.nmask[par];
      auto prep = [&](uint32_t v, uint32_t (&m)[NB]) { return take_masks<NB>(src, v, true, m); };
      if (!multi_expand<NB, STORED>(P, P.out, P.q[cur], cnt, prep, ph, acc,
                                    cur ? SYNC_RESET_Q1 : SYNC_RESET_Q0))
        goto done;
      waves++;
      cur ^= 1;
    }
  }
  // 7. clear the snapshot's affected masks
  if (P.phases & PH_DELETE) {
    const uint32_t na = *(volatile uint32_t *)&ctl->snap_aff;
    for (uint32_t i = gw; i < na; i += nw)
      if (lane < (uint32_t)NB) P.affm[(u64)P.aff[i] * NB + lane] = 0;
  }
done:
  acc.flush(ctl);
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
                                  const uint32_t *seq, Ctl *ctl) {
  const uint32_t Q = nb * 32;
  const uint32_t tag = seq[1];
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < Q; q += gridDim.x * blockDim.x) {
    const uint32_t s = sources[q];
    if (s >= n) continue;
    key[(u64)s * Q + q] = pack_key(0, 0);
    atomicOr(nmask0 + (u64)s * nb + q / 32, 1u << (q % 32));
    if (atomicExch(wtag + s, tag) != tag) q0[atomicAdd(&ctl->q_count[0], 1u)] = s;
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
  P.edge_lanes = std::min(L.edge_lanes, MULTI_EDGE_LANES_MAX);
  P.heavy = std::max(L.heavy, MULTI_MIN_TILE);
  P.tile = std::max(L.tile, MULTI_MIN_TILE);
  P.timeout_ns = L.timeout_ns;
  static int blocks_per_sm = -1;
  if (blocks_per_sm < 0) {
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &blocks_per_sm, multi_repair_kernel<ALGO, STORED, NB>, BLOCK, 0);
    if (e != cudaSuccess) return e;
    if (blocks_per_sm < 1) return cudaErrorLaunchOutOfResources;
  }
  void *args[] = {&P};
  return cudaLaunchCooperativeKernel((const void *)multi_repair_kernel<ALGO, STORED, NB>,
                                     blocks_per_sm * L.num_sms, BLOCK, args, 0, s);
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
                              Ctl *ctl, cudaStream_t s) {
  multi_init_kernel<<<148 * 16, BLOCK, 0, s>>>(key, (u64)n * nb * 32);
  multi_seed_kernel<<<1, BLOCK, 0, s>>>(key, n, nb, sources, nmask0, q0, wtag, seq, ctl);
  return cudaGetLastError();
}

cudaError_t launch_multi_gather(const u64 *key, uint32_t n, uint32_t Q, uint32_t q,
                                uint32_t *values, uint32_t *parents, cudaStream_t s) {
  multi_gather_kernel<<<148 * 8, BLOCK, 0, s>>>(key, n, Q, q, values, parents);
  return cudaGetLastError();
}

}  // namespace dycg
