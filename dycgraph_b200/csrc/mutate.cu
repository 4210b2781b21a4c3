// mutate.cu -- GPU ingest of an update batch and in-place mutation of the
// pinned host adjacency (with write-through to resident HBM pages).
//
// Ingest replaces the reference's CPU GroupedUpdateBatch
// (include/framework/effective_update_batch.h:36-207): records are keyed
// (row << 32 | neighbour), radix-sorted on the GPU, run-length de-duplicated
// (identical deletions become one record with a multiplicity) and grouped by
// row. Mutation keeps the chunk store's occurrence semantics
// (include/groute/graphs/source_local_chunk_store.h:220-406,
// BuildDeletionPlan :685-739): a deletion requested r times removes r live
// occurrences (fewer if fewer exist: the rest are counted missing), additions
// append occurrences, and a row that outgrows its block moves to a new
// power-of-two block at the arena tail. Rows stay sorted in their prefix, so
// a deletion finds its target with a 32-ary warp search instead of the
// reference's linear row scan, and deleted occurrences become tombstones.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "frontier.cuh"
#include "internal.h"

namespace dycg {

__global__ void prep_keys_kernel(const dycg_edge_dev *e, uint32_t cnt, uint32_t n, u64 *kout,
                                 u64 *kin, uint32_t *w, u64 *invalid) {
  uint32_t bad = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += gridDim.x * blockDim.x) {
    const dycg_edge_dev r = e[i];
    const bool ok = r.u < n && r.v < n;
    bad += !ok;
    kout[i] = ok ? (((u64)r.u << 32) | r.v) : KEY_INF;
    if (kin) kin[i] = ok ? (((u64)r.v << 32) | r.u) : KEY_INF;
    if (w) w[i] = r.w;
  }
  const u64 b = warp_sum(bad);
  if (lane_id() == 0 && b) atomicAdd(invalid, b);
}

// Runs of a sorted key array, found without any serial walk (a hub row or a
// heavily repeated edge can span tens of thousands of keys): head flags, an
// exclusive sum for the output slots, one start index per run, and the run
// lengths as differences of consecutive starts. ROWS: runs of equal row
// (key >> 32); otherwise runs of equal key. Sentinel keys (KEY_INF, the
// invalid records, sorted last) belong to no run. Runs come out in ascending
// key order, so the records of one row are contiguous.
template <bool ROWS>
__device__ __forceinline__ bool same_run(u64 a, u64 b) {
  return ROWS ? (a >> 32) == (b >> 32) : a == b;
}

template <bool ROWS>
__global__ void run_heads_kernel(const u64 *k, uint32_t cnt, uint32_t *flags, uint32_t *valid) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const u64 key = k[i];
    flags[i] = key != KEY_INF && (i == 0 || !same_run<ROWS>(k[i - 1], key));
    // end of the non-sentinel keys
    if (key != KEY_INF && (i + 1 == cnt || k[i + 1] == KEY_INF)) *valid = i + 1;
  }
}

__global__ void run_starts_kernel(uint32_t cnt, const uint32_t *flags, const uint32_t *pos,
                                  uint32_t *start, uint32_t *n_out, uint32_t cap, uint32_t *err) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    if (i == cnt - 1) *n_out = min(pos[i] + flags[i], cap);
    if (!flags[i]) continue;
    if (pos[i] < cap) start[pos[i]] = i;
    else atomicCAS(err, 0u, ERR_QUEUE);
  }
}

// unique (u, v) records with their multiplicity
__global__ void runs_emit_kernel(const u64 *k, const uint32_t *start, const uint32_t *n_ptr,
                                 const uint32_t *valid, uint2 *uv, uint32_t *mult) {
  const uint32_t n = *n_ptr;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const uint32_t b = start[r], e = r + 1 < n ? start[r + 1] : *valid;
    const u64 key = k[b];
    uv[r] = make_uint2((uint32_t)(key >> 32), (uint32_t)key);
    mult[r] = e - b;
  }
}

// row segments (row, first index, count)
__global__ void segs_emit_kernel(const u64 *k, const uint32_t *start, const uint32_t *n_ptr,
                                 const uint32_t *valid, uint3 *seg) {
  const uint32_t n = *n_ptr;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const uint32_t b = start[r], e = r + 1 < n ? start[r + 1] : *valid;
    seg[r] = make_uint3((uint32_t)(k[b] >> 32), b, e - b);
  }
}

// First index (row-relative) in the sorted prefix [0, srt) of the row at
// arena offset off whose id is >= target; all lanes return the same index.
// The HBM fence index holds the id of the first slot of every 128-byte group
// of slots (G = 32 slots without weights, 16 with), so a 32-ary warp search
// over the row's fences (HBM reads) narrows the answer to one group, read
// from the row with a single coalesced 128-byte request.
__device__ uint32_t warp_lower_bound(const Adj &A, u64 off, uint32_t srt, uint32_t target,
                                     uint32_t &reads) {
  const uint32_t lane = lane_id();
  const uint32_t fs = A.fence_shift;
  const u64 G = 1ull << fs;
  // fences inside the prefix: groups f with off <= f*G < off + srt
  const u64 flo = (off + G - 1) >> fs;
  u64 fhi = srt ? ((off + srt - 1) >> fs) + 1 : flo;  // exclusive
  if (fhi < flo) fhi = flo;
  // first fence index f in [flo, fhi) with fence[f] >= target (fhi if none)
  u64 lo = flo, hi = fhi;
  while (hi - lo > 32) {
    const u64 step = (hi - lo + 31) / 32;
    u64 f = lo + (lane + 1) * step - 1;
    if (f >= hi) f = hi - 1;
    const unsigned ge = __ballot_sync(0xffffffffu, A.fence[f] >= target);
    if (!ge) {
      lo = hi;
      break;
    }
    const uint32_t k = __ffs(ge) - 1;
    const u64 nlo = lo + k * step;
    hi = min(lo + (k + 1) * step, hi);
    lo = nlo;
  }
  if (hi > lo) {
    const u64 f = lo + lane;
    const unsigned ge = __ballot_sync(0xffffffffu, f < hi && A.fence[f] >= target);
    lo = ge ? lo + __ffs(ge) - 1 : hi;
  }
  // the answer lies in ((lo-1)*G, lo*G] clipped to the prefix
  const u64 pend = off + srt;
  u64 wbeg = lo > flo ? ((lo - 1) << fs) + 1 : off;
  u64 wend = lo < fhi ? (lo << fs) + 1 : pend;
  if (wbeg < off) wbeg = off;
  if (wend > pend) wend = pend;
  uint32_t ans = (uint32_t)(wend - off);
  for (u64 b = wbeg; b < wend; b += 32) {
    const u64 p = b + lane;
    const bool in = p < wend;
    const uint32_t val = in ? (read_dst_rw(A, p) & VMASK) : 0xFFFFFFFFu;
    reads += in;
    const unsigned ge = __ballot_sync(0xffffffffu, in && val >= target);
    if (ge) {
      ans = (uint32_t)(b + __ffs(ge) - 1 - off);
      break;
    }
  }
  return ans;
}

// Warp per unique deletion record: find up to mult live occurrences (reads
// only) and record their slots; tombstone_kernel then sets their bits in the
// HBM deletion bitmap, so a deletion costs no host-link write.
__global__ void delete_rows_kernel(Adj A, const uint2 *uv, const uint32_t *mult,
                                   const uint32_t *n_ptr, uint32_t *found_out, Ctl *ctl,
                                   int count_missing, Tombs T, DeferDel D) {
  const uint32_t lane = lane_id();
  const uint32_t nrec = *n_ptr;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  u64 link = 0, hbm = 0, missing = 0;
  for (uint32_t i = gw; i < nrec; i += nw) {
    const uint2 e = uv[i];
    const uint32_t row = e.x, target = e.y;
    uint32_t remaining = mult[i], found = 0, reads = 0;
    const u64 off = A.off[row];
    const uint32_t len = A.len[row], srt = A.srt[row];
    const uint32_t pos = warp_lower_bound(A, off, srt, target, reads);
    const bool defer = D.on && len - srt > DEFER_SUFFIX;
    for (uint32_t pass = 0; pass < (defer ? 1u : 2u); pass++) {
      // pass 0: the run of target in the sorted prefix; pass 1: the unsorted suffix
      const uint32_t b = pass ? srt : pos, e2 = pass ? len : srt;
      for (uint32_t s0 = b; s0 < e2 && remaining; s0 += 32) {
        const uint32_t s = s0 + lane;
        const bool in = s < e2;
        const uint32_t d = in ? read_dst_rw(A, off + s) : 0xFFFFFFFFu;
        reads += in;
        const bool live = in && (d & VMASK) == target && !slot_deleted_rw(A, off + s, d);
        const unsigned lm = __ballot_sync(0xffffffffu, live);
        const uint32_t rank = __popc(lm & ((1u << lane) - 1));
        const uint32_t take = min((uint32_t)__popc(lm), remaining);
        uint32_t base = 0;
        if (lane == 0 && take) base = atomicAdd(T.count, take);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (live && rank < remaining && base + rank < T.cap) T.pos[base + rank] = off + s;
        remaining -= take;
        found += take;
        if (!pass && __ballot_sync(0xffffffffu, in && (d & VMASK) != target)) break;
      }
    }
    const bool cached = len && A.page_slot[page_of(A, off)] != PAGE_NONE;
    const u64 bytes = 4ull * reads;
    if (cached) hbm += bytes; else link += bytes;
    const u64 total_reads = warp_sum(reads);
    if (lane == 0) {
      if (found) atomicSub(A.live + row, found);
      if (found_out) found_out[i] = found;
      if (defer) {
        // the row's suffix is matched later, once for all its records
        D.rem[i] = remaining;
        if (i == 0 || uv[i - 1].x != row) {
          const u64 old = atomicAdd(D.packed, (1ull << 40) | (u64)(len - srt));
          const uint32_t k = (uint32_t)(old >> 40);
          if (k < D.cap_rows) {
            D.row_u[k] = row;
            D.row_base[k] = old & ((1ull << 40) - 1);
          } else {
            atomicCAS(&ctl->err, 0u, ERR_QUEUE);
          }
        }
      } else {
        if (D.on) D.rem[i] = 0;
        missing += mult[i] - found;
      }
      if (total_reads) atomicAdd(A.page_hits + page_of(A, off + pos), (uint32_t)total_reads);
    }
  }
  link = warp_sum(link);
  hbm = warp_sum(hbm);
  if (lane == 0) {
    if (link) atomicAdd(&ctl->stat[ST_MUT_LINK_BYTES], link);
    if (hbm) atomicAdd(&ctl->stat[ST_MUT_HBM_BYTES], hbm);
    if (count_missing && missing) atomicAdd(&ctl->stat[ST_MISSING], missing);
  }
}

__global__ void tombstone_kernel(Adj A, Tombs T, Ctl *ctl) {
  const uint32_t n = min(*T.count, T.cap);
  if (blockIdx.x == 0 && threadIdx.x == 0 && *T.count > T.cap) atomicCAS(&ctl->err, 0u, ERR_QUEUE);
  u64 hbm = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const u64 p = T.pos[i];
    atomicOr(A.tbits + (p >> 5), 1u << (p & 31));
    hbm += 4;
  }
  hbm = warp_sum(hbm);
  if (lane_id() == 0 && hbm) atomicAdd(&ctl->stat[ST_MUT_HBM_BYTES], hbm);
}

// Gather the live suffix slots of the deferred rows: thread per slot j,
// key (row << 32 | neighbour) (KEY_INF for a deleted slot), value = the
// slot's index in its suffix. Gathered in slot order, so a stable sort keeps
// equal keys in slot order.
__global__ void suffix_gather_kernel(Adj A, DeferDel D, uint32_t nrows, u64 total, u64 *keys,
                                     uint32_t *vals, Ctl *ctl) {
  const uint32_t lane = lane_id();
  const uint32_t bytes = 4u * A.stride;
  u64 link = 0, hbm = 0;
  for (u64 j0 = (u64)blockIdx.x * blockDim.x + threadIdx.x - lane; j0 < total;
       j0 += (u64)gridDim.x * blockDim.x) {  // warp-uniform
    const u64 j = j0 + lane;
    const bool in = j < total;
    uint32_t pg = PAGE_NONE;
    if (in) {
      uint32_t lo = 0, hi = nrows;  // largest k with row_base[k] <= j
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (D.row_base[mid] <= j) lo = mid; else hi = mid;
      }
      const uint32_t u = D.row_u[lo];
      const uint32_t si = (uint32_t)(j - D.row_base[lo]);
      const u64 p = A.off[u] + A.srt[u] + si;
      const uint32_t d = read_dst_rw(A, p);
      pg = page_of(A, p);
      if (A.page_slot[pg] != PAGE_NONE) hbm += bytes; else link += bytes;
      keys[j] = slot_deleted_rw(A, p, d) ? KEY_INF : (((u64)u << 32) | (d & VMASK));
      vals[j] = si;
    }
    const uint32_t pg0 = __shfl_sync(0xffffffffu, pg, 0);
    const unsigned same = __ballot_sync(0xffffffffu, in && pg == pg0);
    if (lane == 0 && same) atomicAdd(A.page_hits + pg0, __popc(same));
    if (in && pg != pg0) atomicAdd(A.page_hits + pg, 1u);
  }
  link = warp_sum(link);
  hbm = warp_sum(hbm);
  if (lane == 0) {
    if (link) atomicAdd(&ctl->stat[ST_MUT_LINK_BYTES], link);
    if (hbm) atomicAdd(&ctl->stat[ST_MUT_HBM_BYTES], hbm);
  }
}

// Records left unmatched by the prefix pass take the first `rem` entries of
// their (row, neighbour) run in the sorted gather: the earliest live suffix
// occurrences, as the scan would have found them.
__global__ void suffix_match_kernel(Adj A, const uint2 *uv, const uint32_t *n_ptr, DeferDel D,
                                    const u64 *keys, const uint32_t *vals, u64 total,
                                    uint32_t *found_out, Ctl *ctl, int count_missing, Tombs T) {
  const uint32_t nrec = *n_ptr;
  u64 missing = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nrec;
       i += gridDim.x * blockDim.x) {
    const uint32_t rem = D.rem[i];
    if (!rem) continue;
    const uint2 e = uv[i];
    const u64 key = ((u64)e.x << 32) | e.y;
    u64 lo = 0, hi = total;  // first index with keys[idx] >= key
    while (lo < hi) {
      const u64 mid = (lo + hi) / 2;
      if (keys[mid] < key) lo = mid + 1; else hi = mid;
    }
    const u64 base = A.off[e.x] + A.srt[e.x];
    uint32_t taken = 0;
    for (u64 j = lo; j < total && keys[j] == key && taken < rem; j++, taken++) {
      const uint32_t slot = atomicAdd(T.count, 1u);
      if (slot < T.cap) T.pos[slot] = base + vals[j];
    }
    if (taken) {
      atomicSub(A.live + e.x, taken);
      if (found_out) found_out[i] += taken;
    }
    missing += rem - taken;
  }
  missing = warp_sum(missing);
  if (lane_id() == 0 && count_missing && missing) atomicAdd(&ctl->stat[ST_MISSING], missing);
}

__device__ __forceinline__ uint32_t next_pow2_u32(uint32_t x) {
  return x <= 1 ? 1u : 1u << (32 - __clz(x - 1));
}

// Warp per row segment: append the segment's occurrences in place when they
// fit. A row that does not fit gets a new power-of-two block (with headroom)
// at the arena tail; its descriptor moves at once, while the copy of the old
// slots and the append are deferred to relocate_copy_kernel and
// relocate_append_kernel, so a large row is copied by many warps instead of
// one.
__global__ void add_rows_kernel(Adj A, const u64 *k, const uint32_t *wv, const uint3 *seg,
                                const uint32_t *n_ptr, Reloc R, Ctl *ctl) {
  const uint32_t lane = lane_id();
  const uint32_t nseg = *n_ptr;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  u64 link = 0, hbm = 0, reloc = 0;
  const uint32_t bytes = 4u * A.stride;
  for (uint32_t i = gw; i < nseg; i += nw) {
    const uint3 sg = seg[i];
    const uint32_t row = sg.x, start = sg.y, count = sg.z;
    const uint32_t len = A.len[row], cap = A.cap[row], srt = A.srt[row];
    const uint32_t live = A.live[row];
    const u64 off = A.off[row];
    if ((u64)len + count <= cap) {
      for (uint32_t j = lane; j < count; j += 32) {
        const bool c = write_slot(A, off + len + j, (uint32_t)k[start + j], wv ? wv[start + j] : 0u);
        link += bytes;
        if (c) hbm += bytes;
      }
      // appends stay in the unsorted suffix (no host-link read here); an
      // empty row takes its sorted run of appends as its sorted prefix
      const uint32_t nsrt = len == 0 ? count : srt;
      if (lane == 0) {
        A.len[row] = len + count;
        A.live[row] = live + count;
        A.srt[row] = nsrt;
      }
      continue;
    }
    if (lane == 0) {
      const u64 need = (u64)len + count;
      const uint32_t ncap = next_pow2_u32((uint32_t)(need + need / 8 + 1));
      const u64 noff = atomicAdd(A.top, (u64)ncap);
      const uint32_t r = atomicAdd(R.n_reloc, 1u);
      const uint32_t nchunk = (len + RELOC_CHUNK - 1) / RELOC_CHUNK;
      const uint32_t cb = atomicAdd(R.n_chunks, nchunk);
      if (noff + ncap > A.arena || r >= R.cap || cb + nchunk > R.chunk_cap) {
        atomicCAS(&ctl->err, 0u, ERR_ARENA);
      } else {
        R.rec[r] = RelocRec{row, i, len, 0u, off, noff};
        for (uint32_t c = 0; c < nchunk; c++) R.chunks[cb + c] = make_uint2(r, c);
        A.off[row] = noff;
        A.cap[row] = ncap;
        reloc++;
      }
    }
  }
  link = warp_sum(link);
  hbm = warp_sum(hbm);
  if (lane == 0) {
    if (link) atomicAdd(&ctl->stat[ST_MUT_LINK_BYTES], link);
    if (hbm) atomicAdd(&ctl->stat[ST_MUT_HBM_BYTES], hbm);
    if (reloc) atomicAdd(&ctl->stat[ST_RELOCATED], reloc);
  }
}

// Warp per RELOC_CHUNK slots of a relocated row: verbatim copy (tombstones
// included, so the sorted prefix and the live count stay valid). Each lane
// keeps RELOC_CHUNK/32 loads in flight before storing.
__global__ void relocate_copy_kernel(Adj A, Reloc R, Ctl *ctl) {
  const uint32_t lane = lane_id();
  const uint32_t nch = min(*R.n_chunks, R.chunk_cap);
  const uint32_t nrec = min(*R.n_reloc, R.cap);
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  constexpr uint32_t PER = RELOC_CHUNK / 32;
  const uint32_t bytes = 4u * A.stride;
  u64 link = 0, hbm = 0;
  for (uint32_t i = gw; i < nch; i += nw) {
    const uint2 ch = R.chunks[i];
    if (ch.x >= nrec) continue;
    const RelocRec rec = R.rec[ch.x];
    const uint32_t b = ch.y * RELOC_CHUNK;
    const uint32_t e = min(rec.len, b + RELOC_CHUNK);
    uint2 v[PER];
#pragma unroll
    for (uint32_t t = 0; t < PER; t++) {
      const uint32_t s = b + t * 32 + lane;
      if (s < e) {
        v[t] = read_pair_rw(A, rec.old_off + s);
        // a slot deleted through the bitmap keeps its deletion as a tombstone bit
        if (slot_deleted_rw(A, rec.old_off + s, v[t].x)) v[t].x |= TOMB;
      }
    }
#pragma unroll
    for (uint32_t t = 0; t < PER; t++) {
      const uint32_t s = b + t * 32 + lane;
      if (s < e) {
        const bool c = write_slot(A, rec.new_off + s, v[t].x, v[t].y);
        link += 2 * bytes;
        if (c) hbm += bytes;
      }
    }
  }
  link = warp_sum(link);
  hbm = warp_sum(hbm);
  if (lane == 0) {
    if (link) atomicAdd(&ctl->stat[ST_MUT_LINK_BYTES], link);
    if (hbm) atomicAdd(&ctl->stat[ST_MUT_HBM_BYTES], hbm);
  }
}

// Warp per relocated row: append its segment after the copied slots.
__global__ void relocate_append_kernel(Adj A, const u64 *k, const uint32_t *wv,
                                       const uint3 *seg, Reloc R) {
  const uint32_t lane = lane_id();
  const uint32_t nrec = min(*R.n_reloc, R.cap);
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = gw; i < nrec; i += nw) {
    const RelocRec rec = R.rec[i];
    const uint3 sg = seg[rec.seg];
    const uint32_t start = sg.y, count = sg.z, len = rec.len;
    for (uint32_t j = lane; j < count; j += 32)
      write_slot(A, rec.new_off + len + j, (uint32_t)k[start + j], wv ? wv[start + j] : 0u);
    if (lane == 0) {
      const uint32_t nsrt = len == 0 ? count : A.srt[rec.row];
      A.srt[rec.row] = nsrt;
      A.len[rec.row] = len + count;
      A.live[rec.row] += count;
    }
  }
}

// Valid insertion records (u,v,w) from the sorted out-keys; invalid ones keep
// u = INF32 so the repair kernel skips them.
__global__ void keys_to_uvw_kernel(const u64 *k, const uint32_t *w, uint32_t cnt, uint3 *out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += gridDim.x * blockDim.x) {
    const u64 key = k[i];
    out[i] = key == KEY_INF ? make_uint3(INF32, INF32, 0)
                            : make_uint3((uint32_t)(key >> 32), (uint32_t)key, w ? w[i] : 0u);
  }
}

// Distinct touched sources (per-vertex batch tag), for PR amends and stats.
__global__ void touched_kernel(const u64 *k, uint32_t cnt, uint32_t *tag, uint32_t epoch,
                               uint32_t *list, uint32_t *n_out, Ctl *ctl) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += gridDim.x * blockDim.x) {
    const u64 key = k[i];
    if (key == KEY_INF) continue;
    const uint32_t u = (uint32_t)(key >> 32);
    if (i > 0 && (uint32_t)(k[i - 1] >> 32) == u) continue;
    if (atomicExch(tag + u, epoch) != epoch) {
      const uint32_t s = atomicAdd(n_out, 1u);
      list[s] = u;
      atomicAdd(&ctl->stat[ST_TOUCHED], 1ull);
    }
  }
}

static int grid_for(u64 threads) {
  u64 b = (threads + BLOCK - 1) / BLOCK;
  if (b < 1) b = 1;
  if (b > 148ull * 32) b = 148ull * 32;
  return (int)b;
}

// Grid of a warp-per-record mutation kernel: the records are in row order
// (sorted by ingest) and the rows in arena order, so the warps in flight work
// on a window of consecutive records; capping the CTAs (ctas > 0) narrows
// that window of the host arena, and the host link serves transactions in a
// narrow window several times faster than ones spread over a multi-GB arena.
static int mut_grid(u64 records, uint32_t ctas) {
  const int g = grid_for(records * 32);
  return ctas ? std::min<int>(g, (int)ctas) : g;
}

cudaError_t launch_prep_keys(const dycg_edge_dev *e, uint32_t cnt, uint32_t n, u64 *kout,
                             u64 *kin, uint32_t *w, u64 *invalid, cudaStream_t s) {
  if (!cnt) return cudaSuccess;
  prep_keys_kernel<<<grid_for(cnt), BLOCK, 0, s>>>(e, cnt, n, kout, kin, w, invalid);
  return cudaGetLastError();
}

cudaError_t sort_keys(void *temp, size_t &temp_bytes, const u64 *in, u64 *out, uint32_t cnt,
                      cudaStream_t s) {
  return cub::DeviceRadixSort::SortKeys(temp, temp_bytes, in, out, (int)cnt, 0, 64, s);
}

cudaError_t sort_pairs(void *temp, size_t &temp_bytes, const u64 *kin, u64 *kout,
                       const uint32_t *vin, uint32_t *vout, uint32_t cnt, cudaStream_t s) {
  return cub::DeviceRadixSort::SortPairs(temp, temp_bytes, kin, kout, vin, vout, (int)cnt, 0,
                                         64, s);
}

size_t unique_runs_temp_bytes(uint32_t cnt) {
  size_t b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, b, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                (int)cnt);
  return b;
}

template <bool ROWS>
static cudaError_t run_starts(const u64 *k, uint32_t cnt, uint32_t *n_out, uint32_t cap,
                              uint32_t *err, const RunScratch &S, cudaStream_t s) {
  cudaMemsetAsync(S.valid, 0, 4, s);
  run_heads_kernel<ROWS><<<grid_for(cnt), BLOCK, 0, s>>>(k, cnt, S.flags, S.valid);
  size_t tb = S.temp_bytes;
  cudaError_t e = cub::DeviceScan::ExclusiveSum(S.temp, tb, S.flags, S.pos, (int)cnt, s);
  if (e != cudaSuccess) return e;
  run_starts_kernel<<<grid_for(cnt), BLOCK, 0, s>>>(cnt, S.flags, S.pos, S.start, n_out, cap, err);
  return cudaGetLastError();
}

cudaError_t launch_unique_runs(const u64 *k, uint32_t cnt, uint2 *uv, uint32_t *mult,
                               uint32_t *n_out, uint32_t cap, uint32_t *err, const RunScratch &S,
                               cudaStream_t s) {
  if (!cnt) return cudaSuccess;
  cudaError_t e = run_starts<false>(k, cnt, n_out, cap, err, S, s);
  if (e != cudaSuccess) return e;
  runs_emit_kernel<<<grid_for(cnt), BLOCK, 0, s>>>(k, S.start, n_out, S.valid, uv, mult);
  return cudaGetLastError();
}

cudaError_t launch_row_segments(const u64 *k, uint32_t cnt, uint3 *seg, uint32_t *n_out,
                                uint32_t cap, uint32_t *err, const RunScratch &S, cudaStream_t s) {
  if (!cnt) return cudaSuccess;
  cudaError_t e = run_starts<true>(k, cnt, n_out, cap, err, S, s);
  if (e != cudaSuccess) return e;
  segs_emit_kernel<<<grid_for(cnt), BLOCK, 0, s>>>(k, S.start, n_out, S.valid, seg);
  return cudaGetLastError();
}

cudaError_t launch_delete_rows(const Adj &A, const uint2 *uv, const uint32_t *mult,
                               const uint32_t *n_ptr, uint32_t max_n, uint32_t *found, Ctl *ctl,
                               int count_missing, const Tombs &T, uint32_t ctas, cudaStream_t s) {
  if (!max_n) return cudaSuccess;
  cudaMemsetAsync(T.count, 0, 4, s);
  DeferDel off{};
  delete_rows_kernel<<<mut_grid(max_n, ctas), BLOCK, 0, s>>>(A, uv, mult, n_ptr, found, ctl,
                                                             count_missing, T, off);
  tombstone_kernel<<<grid_for(max_n), BLOCK, 0, s>>>(A, T, ctl);
  return cudaGetLastError();
}

cudaError_t launch_delete_prefix(const Adj &A, const uint2 *uv, const uint32_t *mult,
                                 const uint32_t *n_ptr, uint32_t max_n, uint32_t *found, Ctl *ctl,
                                 int count_missing, const Tombs &T, const DeferDel &D,
                                 uint32_t ctas, cudaStream_t s) {
  if (!max_n) return cudaSuccess;
  cudaMemsetAsync(T.count, 0, 4, s);
  cudaMemsetAsync(D.packed, 0, 8, s);
  delete_rows_kernel<<<mut_grid(max_n, ctas), BLOCK, 0, s>>>(A, uv, mult, n_ptr, found, ctl,
                                                             count_missing, T, D);
  return cudaGetLastError();
}

size_t delete_sort_temp_bytes(u64 total) {
  size_t b = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, b, (const u64 *)nullptr, (u64 *)nullptr,
                                  (const uint32_t *)nullptr, (uint32_t *)nullptr, (int64_t)total,
                                  0, 64);
  return b;
}

cudaError_t launch_delete_suffix(const Adj &A, const uint2 *uv, const uint32_t *n_ptr,
                                 uint32_t max_n, uint32_t *found, Ctl *ctl, int count_missing,
                                 const Tombs &T, const DeferDel &D, uint32_t nrows, u64 total,
                                 const DeferBufs &B, cudaStream_t s) {
  if (!max_n) return cudaSuccess;
  if (nrows && total) {
    suffix_gather_kernel<<<grid_for(total), BLOCK, 0, s>>>(A, D, nrows, total, B.k_in, B.v_in, ctl);
    size_t tb = B.temp_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(B.temp, tb, B.k_in, B.k_out, B.v_in, B.v_out,
                                                    (int64_t)total, 0, 64, s);
    if (e != cudaSuccess) return e;
    suffix_match_kernel<<<grid_for(max_n), BLOCK, 0, s>>>(A, uv, n_ptr, D, B.k_out, B.v_out, total,
                                                          found, ctl, count_missing, T);
  } else if (nrows) {
    suffix_match_kernel<<<grid_for(max_n), BLOCK, 0, s>>>(A, uv, n_ptr, D, B.k_out, B.v_out, 0,
                                                          found, ctl, count_missing, T);
  }
  tombstone_kernel<<<grid_for(max_n), BLOCK, 0, s>>>(A, T, ctl);
  return cudaGetLastError();
}

cudaError_t launch_add_rows(const Adj &A, const u64 *k, const uint32_t *w, const uint3 *seg,
                            const uint32_t *n_ptr, uint32_t max_n, const Reloc &R, Ctl *ctl,
                            uint32_t ctas, cudaStream_t s) {
  if (!max_n) return cudaSuccess;
  cudaMemsetAsync(R.n_reloc, 0, 4, s);
  cudaMemsetAsync(R.n_chunks, 0, 4, s);
  const uint32_t *wv = A.stride == 2 ? w : nullptr;
  add_rows_kernel<<<mut_grid(max_n, ctas), BLOCK, 0, s>>>(A, k, wv, seg, n_ptr, R, ctl);
  relocate_copy_kernel<<<148 * 16, BLOCK, 0, s>>>(A, R, ctl);
  relocate_append_kernel<<<grid_for((u64)max_n * 32), BLOCK, 0, s>>>(A, k, wv, seg, R);
  return cudaGetLastError();
}

cudaError_t launch_keys_to_uvw(const u64 *k, const uint32_t *w, uint32_t cnt, uint3 *out,
                               cudaStream_t s) {
  if (!cnt) return cudaSuccess;
  keys_to_uvw_kernel<<<grid_for(cnt), BLOCK, 0, s>>>(k, w, cnt, out);
  return cudaGetLastError();
}

cudaError_t launch_touched(const u64 *k, uint32_t cnt, uint32_t *tag, uint32_t epoch,
                           uint32_t *list, uint32_t *n_out, Ctl *ctl, cudaStream_t s) {
  if (!cnt) return cudaSuccess;
  touched_kernel<<<grid_for(cnt), BLOCK, 0, s>>>(k, cnt, tag, epoch, list, n_out, ctl);
  return cudaGetLastError();
}

}  // namespace dycg
