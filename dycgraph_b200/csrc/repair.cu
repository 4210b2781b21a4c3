// repair.cu -- one persistent cooperative kernel repairs SSSP / BFS / CC after
// a snapshot, after the topology mutation kernels have run.
//
// Phases (each ends at a bounded grid barrier):
//   1. deletion seeds: for every deleted (u,v) that removed an occurrence and
//      where u is v's parent, v is affected (reset_del_edges,
//      include/framework/variants/driver.cuh:401-441, IsDeletionDependency
//      api.cuh:42-49; with parents always tight the rule reduces to parent==u).
//   2. invalidation waves: children y of affected x (parent(y)==x) become
//      affected (PushFunctorDB_Del, push_functor.h:1180-1213), over out-rows.
//   3. reset affected state (reset_affected_values, driver.cuh:448-463).
//   4. pull: each affected v takes min over live in-edges of
//      (value(x)+w, parent x) (GpuAffectedPullRelax, framework.cuh:189-263;
//      equal values break toward the smaller parent).
//   5. frontier: affected vertices with a finite value, plus insertion seeds
//      (SeedAddedEdgeFrontier, framework.cuh:297-370).
//   6. closure waves: push relaxation until the frontier is empty
//      (RunExactGpuClosure, framework.cuh:504-616, AccumulateBuffer
//      samples/hybrid_sssp/hybrid_sssp.cu:125-145).
// The reference drives phases 2 and 4 from the host with one synchronisation
// per level/iteration; here the whole repair is a single launch.
#include "frontier.cuh"
#include "internal.h"

namespace dycg {

struct RepairParams {
  Adj out, in;
  u64 *key;
  uint32_t *mark;
  uint32_t *wtag;
  uint32_t *aff;
  uint32_t *q[2];
  Tiles tiles;
  Ctl *ctl;
  const uint2 *del_uv;      // unique deleted (u,v)
  const uint32_t *del_found; // occurrences removed per unique record
  const uint32_t *n_del_ptr; // device count of unique records
  const uint3 *add_uvw;     // valid insertions (u,v,w)
  uint32_t n_add;
  uint32_t n;
  uint32_t source;
  uint32_t epoch;
  uint32_t tag_base;
  uint32_t phases;
  uint32_t max_waves;
  uint32_t delta;           // ordered closure: expand values < wave min + delta (0: unordered)
  uint32_t *q2;             // ordered closure: the wave's bucket
  uint32_t *tag_dev;        // non-null: wave tags start at *tag_dev, which the
                            // launch advances past the tags it used
  u64 timeout_ns;
  bool claimed;             // waves' items claimed one at a time (else static)
};

template <uint32_t ALGO>
__device__ __forceinline__ u64 reset_key(uint32_t v) {
  return ALGO == ALGO_CC ? pack_key(v, 0) : KEY_INF;
}

// Children of an affected vertex become affected.
template <uint32_t ALGO>
struct InvalidateOp {
  const RepairParams *P;
  struct Row {};
  __device__ bool begin(uint32_t, Row &) { return true; }
  __device__ void edge(uint32_t x, uint32_t y, uint32_t, bool valid, Row &, Acc &) {
    bool want = false;
    if (valid && !(ALGO != ALGO_CC && y == P->source)) {
      if (key_parent1(ld_key(P->key + y)) == x + 1u)
        want = atomicExch(P->mark + y, P->epoch) != P->epoch;
    }
    warp_append(P->aff, &P->ctl->n_aff, P->n, want, y, &P->ctl->err);
  }
  __device__ void end(uint32_t, Row &) {}
};

// Affected v pulls the best candidate over its live in-edges.
template <uint32_t ALGO, bool STORED>
struct PullOp {
  const RepairParams *P;
  struct Row {
    u64 best;
  };
  __device__ bool begin(uint32_t, Row &r) {
    r.best = KEY_INF;
    return true;
  }
  __device__ void edge(uint32_t v, uint32_t x, uint32_t w, bool valid, Row &r, Acc &) {
    if (!valid) return;
    const u64 kx = ld_key(P->key + x);
    const uint32_t vx = key_value(kx);
    if (vx == INF32) return;
    const u64 c = (u64)vx + (STORED ? w : rule_weight<ALGO>(x, v));
    if (c >= INF32) return;
    const u64 cand = pack_key((uint32_t)c, x + 1u);
    r.best = cand < r.best ? cand : r.best;
  }
  __device__ void end(uint32_t v, Row &r) {
    const u64 m = warp_min_all(r.best);
    if (lane_id() == 0 && m != KEY_INF) {
      if (Strict<ALGO, STORED>::value) strict_lower(P->key + v, m);
      else atomicMin(P->key + v, m);
    }
  }
};

// Push relaxation of the out-edges of a frontier vertex. In the ordered
// closure (vmin set) every improvement also lowers *vmin, the next wave's
// running minimum.
template <uint32_t ALGO, bool STORED>
struct RelaxOp {
  const RepairParams *P;
  uint32_t *outq;
  uint32_t *outc;
  uint32_t tag;
  uint32_t *vmin;  // ordered closure: running minimum of the next wave (or null)
  struct Row {
    uint32_t dv;
  };
  __device__ bool begin(uint32_t x, Row &r) {
    // one read, broadcast: the key may change under concurrent relaxations
    r.dv = __shfl_sync(0xffffffffu, key_value(ld_key(P->key + x)), 0);
    return r.dv != INF32;
  }
  __device__ void edge(uint32_t x, uint32_t y, uint32_t w, bool valid, Row &r, Acc &acc) {
    bool want = false;
    uint32_t imp = INF32;  // value this lane lowered y to
    if (valid) {
      const u64 c = (u64)r.dv + (STORED ? w : rule_weight<ALGO>(x, y));
      if (c < INF32) {
        const u64 cand = pack_key((uint32_t)c, x + 1u);
        bool lowered = false;
        if (Strict<ALGO, STORED>::value) {
          lowered = strict_lower(P->key + y, cand);
        } else if (cand < ld_key(P->key + y)) {
          lowered = key_value(atomicMin(P->key + y, cand)) > (uint32_t)c;
        }
        if (lowered) {
          acc.improved++;
          want = atomicExch(P->wtag + y, tag) != tag;
          imp = (uint32_t)c;
        }
      }
    }
    warp_append(outq, outc, P->n, want, y, &P->ctl->err);
    if (vmin) {
      imp = __reduce_min_sync(0xffffffffu, imp);
      if (lane_id() == 0 && imp != INF32) atomicMin(vmin, imp);
    }
  }
  __device__ void end(uint32_t, Row &) {}
};

// One wave of the ordered closure in a single pass: a warp takes 32
// consecutive queue items, its lanes split them by value (below thr: expand
// now; at or above: carry to the next queue, with the carried values' minimum
// lowering the next wave's running minimum, one atomic per warp), then the
// warp expands the items kept for now one by one (rows longer than HEAVY as
// CTA tiles after the barrier, as expand_rows does).
template <bool WITH_W, class Op>
__device__ bool expand_ordered(const RepairParams &P, const uint32_t *items, uint32_t cnt,
                               uint32_t thr, Op &op, Acc &acc, Ctl *ctl, uint32_t reset_flags) {
  const Adj &A = P.out;
  const uint32_t lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i0 = gw * 32; i0 < cnt; i0 += nw * 32) {
    const uint32_t i = i0 + lane;
    uint32_t v = 0, dv = INF32;
    if (i < cnt) {
      v = items[i];
      dv = key_value(ld_key(P.key + v));
    }
    const bool now = dv < thr;
    const bool carry = dv != INF32 && !now && atomicExch(P.wtag + v, op.tag) != op.tag;
    warp_append(op.outq, op.outc, P.n, carry, v, &ctl->err);
    const uint32_t cm = __reduce_min_sync(0xffffffffu, carry ? dv : INF32);
    if (lane == 0 && cm != INF32) atomicMin(op.vmin, cm);
    unsigned todo = __ballot_sync(0xffffffffu, now);
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1;
      const uint32_t x = __shfl_sync(0xffffffffu, v, src);
      const uint32_t len = A.len[x];
      if (len > HEAVY) {
        if (lane == 0) {
          const uint32_t nt = (len + TILE - 1) / TILE;
          const uint32_t base = atomicAdd(&ctl->tile_count, nt);
          if (base + nt > P.tiles.cap) {
            atomicCAS(&ctl->err, 0u, ERR_TILES);
          } else {
            for (uint32_t t = 0; t < nt; t++)
              P.tiles.tiles[base + t] = make_uint4(x, t * TILE, min(len, (t + 1) * TILE), 0);
          }
        }
        continue;
      }
      warp_slots<WITH_W>(A, x, A.off[x], 0, len, 32, op, acc);
    }
  }
  if (!grid_sync(ctl, reset_flags, P.timeout_ns)) return false;
  const uint32_t nt = min(*(volatile uint32_t *)&ctl->snap_tiles, P.tiles.cap);
  if (nt == 0) return true;
  const uint32_t wib = threadIdx.x >> 5;
  for (uint32_t t = blockIdx.x; t < nt; t += gridDim.x) {
    const uint4 tl = P.tiles.tiles[t];
    warp_slots<WITH_W>(A, tl.x, A.off[tl.x], tl.y + wib * 32, tl.z, blockDim.x, op, acc);
  }
  return grid_sync(ctl, SYNC_RESET_TILES, P.timeout_ns);
}

template <uint32_t ALGO, bool STORED>
__global__ void __launch_bounds__(BLOCK) repair_kernel(RepairParams P) {
  Ctl *ctl = P.ctl;
  Acc acc = {0, 0, 0, 0, 0};
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t gstride = gridDim.x * blockDim.x;
  const uint32_t lane = lane_id();
  const uint32_t tag_base = P.tag_dev ? *(volatile uint32_t *)P.tag_dev : P.tag_base;
  if (gtid == 0) ctl->stat[ST_T_START] = globaltimer_ns();

  if (P.phases & PH_DELETE) {
    // 1. deletion seeds (warp-uniform loop so appends can aggregate)
    const uint32_t n_del = *P.n_del_ptr;
    for (uint32_t i0 = gtid - lane; i0 < n_del; i0 += gstride) {
      const uint32_t i = i0 + lane;
      bool want = false;
      uint32_t v = 0;
      if (i < n_del && P.del_found[i] != 0) {
        const uint2 e = P.del_uv[i];
        v = e.y;
        if (!(ALGO != ALGO_CC && v == P.source) &&
            key_parent1(ld_key(P.key + v)) == e.x + 1u)
          want = atomicExch(P.mark + v, P.epoch) != P.epoch;
      }
      warp_append(P.aff, &ctl->n_aff, P.n, want, v, &ctl->err);
    }
    if (!grid_sync(ctl, 0, P.timeout_ns)) goto done;
    // 2. invalidation waves over the growing affected list
    {
      uint32_t lo = 0;
      for (;;) {
        const uint32_t hi = *(volatile uint32_t *)&ctl->snap_aff;
        if (hi == lo) break;
        InvalidateOp<ALGO> op{&P};
        if (!expand_rows<false>(P.out, P.aff + lo, hi - lo, op, acc, P.tiles, ctl, 0,
                                P.timeout_ns, P.claimed))
          goto done;
        lo = hi;
      }
    }
    if (gtid == 0) ctl->tphase[0] = globaltimer_ns();  // seeds + invalidation done
    // 3. reset
    {
      const uint32_t na = *(volatile uint32_t *)&ctl->snap_aff;
      for (uint32_t i = gtid; i < na; i += gstride) {
        const uint32_t v = P.aff[i];
        P.key[v] = reset_key<ALGO>(v);
      }
      if (!grid_sync(ctl, 0, P.timeout_ns)) goto done;
      // 4. pull over incoming rows
      PullOp<ALGO, STORED> op{&P};
      if (!expand_rows<STORED>(P.in, P.aff, na, op, acc, P.tiles, ctl, 0, P.timeout_ns, P.claimed))
        goto done;
      if (gtid == 0) ctl->tphase[1] = globaltimer_ns();  // reset + pull done
      // 5a. frontier from affected vertices with a finite value
      for (uint32_t i0 = gtid - lane; i0 < na; i0 += gstride) {
        const uint32_t i = i0 + lane;
        bool want = false;
        uint32_t v = 0;
        if (i < na) {
          v = P.aff[i];
          if (key_value(ld_key(P.key + v)) != INF32)
            want = atomicExch(P.wtag + v, tag_base) != tag_base;
        }
        warp_append(P.q[0], &ctl->q_count[0], P.n, want, v, &ctl->err);
      }
    }
  }
  if (P.phases & PH_INSERT) {
    // 5b. insertion seeds
    for (uint32_t i0 = gtid - lane; i0 < P.n_add; i0 += gstride) {
      const uint32_t i = i0 + lane;
      bool want = false;
      uint32_t v = 0;
      const uint3 e = i < P.n_add ? P.add_uvw[i] : make_uint3(INF32, INF32, 0);
      if (e.x < P.n) {
        v = e.y;
        const uint32_t du = key_value(ld_key(P.key + e.x));
        if (du != INF32) {
          const u64 c = (u64)du + (STORED ? e.z : rule_weight<ALGO>(e.x, e.y));
          if (c < INF32) {
            const u64 cand = pack_key((uint32_t)c, e.x + 1u);
            bool lowered = false;
            if (Strict<ALGO, STORED>::value) {
              lowered = strict_lower(P.key + v, cand);
            } else if (cand < ld_key(P.key + v)) {
              lowered = key_value(atomicMin(P.key + v, cand)) > (uint32_t)c;
            }
            if (lowered) want = atomicExch(P.wtag + v, tag_base) != tag_base;
          }
        }
      }
      warp_append(P.q[0], &ctl->q_count[0], P.n, want, v, &ctl->err);
    }
  }
  if (!grid_sync(ctl, SYNC_RESET_VMIN, P.timeout_ns)) goto done;
  if (gtid == 0) ctl->tphase[2] = globaltimer_ns();  // frontier + insertion seeds done
  // 6. closure waves
  if ((P.phases & PH_CLOSE) && P.delta) {
    // Ordered (bucketed) closure for high-diameter graphs, the B200 form of
    // the reference's ordered insertion schedule (framework.cuh:537-556):
    // each wave expands only the frontier vertices whose value is below the
    // wave's minimum + delta and carries the rest to the next wave, so a
    // vertex is expanded about once instead of once per improvement. The
    // next wave's minimum is kept on the fly (carried values and every
    // improvement lower ctl->vmin, which the wave's closing barrier snapshots
    // and resets), so only the first wave needs a reduction pass. SSSP and
    // BFS split each wave's queue into a compact bucket first (a barrier),
    // which spreads the bucket's rows over all warps (their buckets hold
    // runs of consecutive queue entries); CC splits and expands in one pass
    // (its waves are mostly carried entries, for which the split barrier is
    // the larger cost).
    uint32_t cur = 0;
    {
      const uint32_t cnt = *(volatile uint32_t *)&ctl->snap_q[0];
      uint32_t m = INF32;
      for (uint32_t i = gtid; i < cnt; i += gstride)
        m = min(m, key_value(ld_key(P.key + P.q[0][i])));
      for (int o = 16; o; o >>= 1) m = min(m, __shfl_down_sync(0xffffffffu, m, o));
      if (lane == 0 && m != INF32) atomicMin(&ctl->vmin, m);
      if (!grid_sync(ctl, SYNC_RESET_VMIN, P.timeout_ns)) goto done;
    }
    for (uint32_t wave = 0;; wave++) {
      const uint32_t cnt = *(volatile uint32_t *)&ctl->snap_q[cur];
      if (cnt == 0) break;
      if (wave >= P.max_waves) {
        if (gtid == 0) atomicCAS(&ctl->err, 0u, ERR_WAVES);
        break;
      }
      const uint32_t tag = tag_base + 1 + wave;
      const uint32_t vm = *(volatile uint32_t *)&ctl->snap_vmin;
      const uint32_t thr = vm > INF32 - P.delta ? INF32 : vm + P.delta;
      RelaxOp<ALGO, STORED> op{&P, P.q[cur ^ 1], &ctl->q_count[cur ^ 1], tag, &ctl->vmin};
      const uint32_t close = (cur ? SYNC_RESET_Q1 : SYNC_RESET_Q0) | SYNC_RESET_VMIN;
      if (ALGO == ALGO_CC) {
        if (!expand_ordered<STORED>(P, P.q[cur], cnt, thr, op, acc, ctl, close)) goto done;
      } else {
        // split: values below thr form this wave's bucket, the rest carry over
        for (uint32_t i0 = gtid - lane; i0 < cnt; i0 += gstride) {
          const uint32_t i = i0 + lane;
          uint32_t v = 0, d = INF32;
          if (i < cnt) {
            v = P.q[cur][i];
            d = key_value(ld_key(P.key + v));
          }
          const bool now = d < thr;
          const bool carry = !now && d != INF32 && atomicExch(P.wtag + v, tag) != tag;
          warp_append(P.q2, &ctl->q_count[2], P.n, now, v, &ctl->err);
          warp_append(P.q[cur ^ 1], &ctl->q_count[cur ^ 1], P.n, carry, v, &ctl->err);
          const uint32_t cm = __reduce_min_sync(0xffffffffu, carry ? d : INF32);
          if (lane == 0 && cm != INF32) atomicMin(&ctl->vmin, cm);
        }
        if (!grid_sync(ctl, cur ? SYNC_RESET_Q1 : SYNC_RESET_Q0, P.timeout_ns)) goto done;
        const uint32_t nb = *(volatile uint32_t *)&ctl->snap_q[2];
        if (!expand_rows<STORED>(P.out, P.q2, nb, op, acc, P.tiles, ctl,
                                 SYNC_RESET_Q2 | SYNC_RESET_VMIN, P.timeout_ns, P.claimed))
          goto done;
      }
      if (gtid == 0) ctl->waves = wave + 1;
      cur ^= 1;
    }
  } else if (P.phases & PH_CLOSE) {
    uint32_t cur = 0;
    for (uint32_t wave = 0;; wave++) {
      const uint32_t cnt = *(volatile uint32_t *)&ctl->snap_q[cur];
      if (cnt == 0) break;
      if (wave >= P.max_waves) {
        if (gtid == 0) atomicCAS(&ctl->err, 0u, ERR_WAVES);
        break;
      }
      RelaxOp<ALGO, STORED> op{&P, P.q[cur ^ 1], &ctl->q_count[cur ^ 1], tag_base + 1 + wave,
                               nullptr};
      if (!expand_rows<STORED>(P.out, P.q[cur], cnt, op, acc, P.tiles, ctl,
                               cur ? SYNC_RESET_Q1 : SYNC_RESET_Q0, P.timeout_ns, P.claimed))
        goto done;
      if (gtid == 0) ctl->waves = wave + 1;
      cur ^= 1;
    }
  }
  if (gtid == 0) ctl->tphase[3] = globaltimer_ns();  // closure done
done:
  acc.flush(ctl);
  if (gtid == 0) {
    atomicAdd(&ctl->stat[ST_AFFECTED], (u64)ctl->snap_aff);
    // every block read *tag_dev before the first barrier
    if (P.tag_dev) *P.tag_dev = tag_base + ctl->waves + 2;
  }
}

// Static solve set-up: every key reset, the initial frontier in q[0].
template <uint32_t ALGO>
__global__ void init_state_kernel(u64 *key, uint32_t n, uint32_t source, uint32_t *q0,
                                  Ctl *ctl) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += gridDim.x * blockDim.x) {
    if (ALGO == ALGO_CC) {
      key[v] = pack_key(v, 0);
      q0[v] = v;
    } else {
      key[v] = v == source ? pack_key(0, 0) : KEY_INF;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (ALGO == ALGO_CC) {
      ctl->q_count[0] = n;
    } else if (source < n) {
      q0[0] = source;
      ctl->q_count[0] = 1;
    }
  }
}

template <uint32_t ALGO, bool STORED>
static cudaError_t launch_one(const RepairLaunch &L, cudaStream_t s) {
  RepairParams P;
  P.out = L.out;
  P.in = L.in;
  P.key = L.key;
  P.mark = L.mark;
  P.wtag = L.wtag;
  P.aff = L.aff;
  P.q[0] = L.q0;
  P.q[1] = L.q1;
  P.tiles = Tiles{L.tiles, L.tile_cap};
  P.ctl = L.ctl;
  P.del_uv = L.del_uv;
  P.del_found = L.del_found;
  P.n_del_ptr = L.n_del_ptr;
  P.add_uvw = L.add_uvw;
  P.n_add = L.n_add;
  P.n = L.n;
  P.source = L.source;
  P.epoch = L.epoch;
  P.tag_base = L.tag_base;
  P.phases = L.phases;
  P.max_waves = L.max_waves;
  P.delta = L.delta;
  P.q2 = L.q2;
  P.tag_dev = L.tag_dev;
  P.timeout_ns = L.timeout_ns;
  P.claimed = L.sched != 0;
  static int blocks_per_sm = -1;
  if (blocks_per_sm < 0) {
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &blocks_per_sm, repair_kernel<ALGO, STORED>, BLOCK, 0);
    if (e != cudaSuccess) return e;
  }
  const int grid = blocks_per_sm * L.num_sms;
  void *args[] = {&P};
  return cudaLaunchCooperativeKernel((const void *)repair_kernel<ALGO, STORED>, grid, BLOCK,
                                     args, 0, s);
}

cudaError_t launch_repair(const RepairLaunch &L, cudaStream_t s) {
  switch (L.algo) {
    case ALGO_SSSP:
      return L.stored ? launch_one<ALGO_SSSP, true>(L, s) : launch_one<ALGO_SSSP, false>(L, s);
    case ALGO_BFS:
      return launch_one<ALGO_BFS, false>(L, s);
    case ALGO_CC:
      return launch_one<ALGO_CC, false>(L, s);
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t launch_init_state(uint32_t algo, u64 *key, uint32_t n, uint32_t source,
                              uint32_t *q0, Ctl *ctl, cudaStream_t s) {
  const int grid = (int)std::min<u64>((n + BLOCK - 1) / BLOCK + 1, 148ull * 16);
  if (algo == ALGO_CC)
    init_state_kernel<ALGO_CC><<<grid, BLOCK, 0, s>>>(key, n, source, q0, ctl);
  else
    init_state_kernel<ALGO_SSSP><<<grid, BLOCK, 0, s>>>(key, n, source, q0, ctl);
  return cudaGetLastError();
}

}  // namespace dycg
