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

// Unique (row, neighbour) runs of a sorted key array with their multiplicity.
__global__ void unique_runs_kernel(const u64 *k, uint32_t cnt, uint2 *uv, uint32_t *mult,
                                   uint32_t *n_out, uint32_t cap, uint32_t *err) {
  const uint32_t lane = lane_id();
  const uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) - lane;
  for (uint32_t i0 = base; i0 < cnt; i0 += gridDim.x * blockDim.x) {
    const uint32_t i = i0 + lane;
    bool head = false;
    u64 key = KEY_INF;
    if (i < cnt) {
      key = k[i];
      head = key != KEY_INF && (i == 0 || k[i - 1] != key);
    }
    uint32_t m = 0;
    if (head) {
      uint32_t j = i + 1;
      while (j < cnt && k[j] == key) j++;
      m = j - i;
    }
    const unsigned hm = __ballot_sync(0xffffffffu, head);
    if (!hm) continue;
    uint32_t slot = 0;
    if (lane == (uint32_t)(__ffs(hm) - 1)) slot = atomicAdd(n_out, (uint32_t)__popc(hm));
    slot = __shfl_sync(0xffffffffu, slot, __ffs(hm) - 1) + __popc(hm & ((1u << lane) - 1));
    if (head) {
      if (slot < cap) {
        uv[slot] = make_uint2((uint32_t)(key >> 32), (uint32_t)key);
        mult[slot] = m;
      } else {
        atomicCAS(err, 0u, ERR_QUEUE);
      }
    }
  }
}

// Row segments (row, first index, count) of a sorted key array.
__global__ void row_segments_kernel(const u64 *k, uint32_t cnt, uint3 *seg, uint32_t *n_out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += gridDim.x * blockDim.x) {
    const u64 key = k[i];
    if (key == KEY_INF) continue;
    const uint32_t row = (uint32_t)(key >> 32);
    if (i > 0 && (uint32_t)(k[i - 1] >> 32) == row) continue;
    uint32_t j = i + 1;
    while (j < cnt && k[j] != KEY_INF && (uint32_t)(k[j] >> 32) == row) j++;
    const uint32_t slot = atomicAdd(n_out, 1u);
    seg[slot] = make_uint3(row, i, j - i);
  }
}

// First index in [lo, hi) of the sorted prefix whose id is >= target
// (32-ary search: each step narrows the window 32-fold with one warp read).
__device__ uint32_t warp_lower_bound(const Adj &A, u64 off, uint32_t lo, uint32_t hi,
                                     uint32_t target, uint32_t &reads) {
  const uint32_t lane = lane_id();
  while (hi - lo > 32) {
    const uint32_t step = (hi - lo + 31) / 32;
    uint32_t pos = lo + (lane + 1) * step - 1;
    if (pos >= hi) pos = hi - 1;
    const uint32_t val = read_dst_rw(A, off + pos) & VMASK;
    reads++;
    const unsigned ge = __ballot_sync(0xffffffffu, val >= target);
    if (!ge) return hi;
    const uint32_t f = __ffs(ge) - 1;
    const uint32_t nlo = lo + f * step;
    const uint32_t nhi = min(lo + (f + 1) * step, hi);
    lo = nlo;
    hi = nhi;
  }
  const uint32_t pos = lo + lane;
  const bool in = pos < hi;
  const uint32_t val = in ? (read_dst_rw(A, off + pos) & VMASK) : 0xFFFFFFFFu;
  if (in) reads++;
  const unsigned ge = __ballot_sync(0xffffffffu, in && val >= target);
  return ge ? lo + __ffs(ge) - 1 : hi;
}

// Warp per unique deletion record: tombstone up to mult live occurrences.
__global__ void delete_rows_kernel(Adj A, const uint2 *uv, const uint32_t *mult,
                                   const uint32_t *n_ptr, uint32_t *found_out, Ctl *ctl,
                                   int count_missing) {
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
    const uint32_t pos = warp_lower_bound(A, off, 0, srt, target, reads);
    for (uint32_t s0 = pos; s0 < srt && remaining; s0 += 32) {
      const uint32_t s = s0 + lane;
      const bool in = s < srt;
      const uint32_t d = in ? read_dst_rw(A, off + s) : 0xFFFFFFFFu;
      reads += in;
      const bool live = in && (d & VMASK) == target && !(d & TOMB);
      const unsigned lm = __ballot_sync(0xffffffffu, live);
      const uint32_t rank = __popc(lm & ((1u << lane) - 1));
      if (live && rank < remaining) write_dst(A, off + s, d | TOMB);
      const uint32_t take = min((uint32_t)__popc(lm), remaining);
      remaining -= take;
      found += take;
      if (__ballot_sync(0xffffffffu, in && (d & VMASK) != target)) break;
    }
    for (uint32_t s0 = srt; s0 < len && remaining; s0 += 32) {
      const uint32_t s = s0 + lane;
      const bool in = s < len;
      const uint32_t d = in ? read_dst_rw(A, off + s) : 0xFFFFFFFFu;
      reads += in;
      const bool live = in && (d & VMASK) == target && !(d & TOMB);
      const unsigned lm = __ballot_sync(0xffffffffu, live);
      const uint32_t rank = __popc(lm & ((1u << lane) - 1));
      if (live && rank < remaining) write_dst(A, off + s, d | TOMB);
      const uint32_t take = min((uint32_t)__popc(lm), remaining);
      remaining -= take;
      found += take;
    }
    const bool cached = len && A.page_slot[page_of(A, off)] != PAGE_NONE;
    const u64 bytes = 4ull * reads + (lane == 0 ? 4ull * found : 0ull);
    if (cached) hbm += bytes; else link += bytes;
    const u64 total_reads = warp_sum(reads);
    if (lane == 0) {
      if (found) atomicSub(A.live + row, found);
      if (found_out) found_out[i] = found;
      missing += mult[i] - found;
      if (total_reads) atomicAdd(A.page_hits + page_of(A, off), (uint32_t)total_reads);
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

__device__ __forceinline__ uint32_t next_pow2_u32(uint32_t x) {
  return x <= 1 ? 1u : 1u << (32 - __clz(x - 1));
}

// Warp per row segment: append the segment's occurrences, relocating the row
// to a new power-of-two block when it does not fit.
__global__ void add_rows_kernel(Adj A, const u64 *k, const uint32_t *wv, const uint3 *seg,
                                const uint32_t *n_ptr, int with_w, Ctl *ctl) {
  const uint32_t lane = lane_id();
  const uint32_t nseg = *n_ptr;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  u64 link = 0, hbm = 0, reloc = 0;
  const uint32_t bytes = with_w ? 8u : 4u;
  for (uint32_t i = gw; i < nseg; i += nw) {
    const uint3 sg = seg[i];
    const uint32_t row = sg.x, start = sg.y, count = sg.z;
    const uint32_t len = A.len[row], cap = A.cap[row], srt = A.srt[row];
    const uint32_t live = A.live[row];
    const u64 off = A.off[row];
    const uint32_t first_new = (uint32_t)k[start];
    if ((u64)len + count <= cap) {
      for (uint32_t j = lane; j < count; j += 32) {
        const bool c = write_slot(A, off + len + j, (uint32_t)k[start + j],
                                  with_w ? wv[start + j] : 0u, with_w);
        link += bytes;
        if (c) hbm += bytes;
      }
      uint32_t nsrt = srt;
      if (srt == len) {
        const uint32_t last = len ? (read_dst_rw(A, off + len - 1) & VMASK) : 0u;
        if (len == 0 || last <= first_new) nsrt = len + count;
      }
      if (lane == 0) {
        A.len[row] = len + count;
        A.live[row] = live + count;
        A.srt[row] = nsrt;
      }
      continue;
    }
    // relocation
    const uint32_t ncap = max(4u, next_pow2_u32(live + count));
    u64 noff = 0;
    if (lane == 0) noff = atomicAdd(A.top, (u64)ncap);
    noff = __shfl_sync(0xffffffffu, noff, 0);
    if (noff + ncap > A.arena) {
      if (lane == 0) atomicCAS(&ctl->err, 0u, ERR_ARENA);
      continue;
    }
    uint32_t wpos = 0, nsrt = 0, last_val = 0;
    for (uint32_t s0 = 0; s0 < len; s0 += 32) {
      const uint32_t s = s0 + lane;
      const bool in = s < len;
      const uint32_t d = in ? read_dst_rw(A, off + s) : TOMB;
      const uint32_t w = (with_w && in && !(d & TOMB)) ? read_w_rw(A, off + s) : 0u;
      const bool keep = in && !(d & TOMB);
      const unsigned m = __ballot_sync(0xffffffffu, keep);
      const unsigned ms = __ballot_sync(0xffffffffu, keep && s < srt);
      if (keep) {
        const bool c = write_slot(A, noff + wpos + __popc(m & ((1u << lane) - 1)), d, w, with_w);
        link += bytes;
        if (c) hbm += bytes;
      }
      if (in) link += bytes;
      if (m) last_val = __shfl_sync(0xffffffffu, d, 31 - __clz(m)) & VMASK;
      wpos += __popc(m);
      nsrt += __popc(ms);
    }
    for (uint32_t j = lane; j < count; j += 32) {
      const bool c = write_slot(A, noff + wpos + j, (uint32_t)k[start + j],
                                with_w ? wv[start + j] : 0u, with_w);
      link += bytes;
      if (c) hbm += bytes;
    }
    if (nsrt == wpos && (wpos == 0 || last_val <= first_new)) nsrt = wpos + count;
    if (lane == 0) {
      A.off[row] = noff;
      A.cap[row] = ncap;
      A.len[row] = wpos + count;
      A.live[row] = wpos + count;
      A.srt[row] = nsrt;
      reloc++;
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

cudaError_t launch_unique_runs(const u64 *k, uint32_t cnt, uint2 *uv, uint32_t *mult,
                               uint32_t *n_out, uint32_t cap, uint32_t *err, cudaStream_t s) {
  if (!cnt) return cudaSuccess;
  unique_runs_kernel<<<grid_for(cnt), BLOCK, 0, s>>>(k, cnt, uv, mult, n_out, cap, err);
  return cudaGetLastError();
}

cudaError_t launch_row_segments(const u64 *k, uint32_t cnt, uint3 *seg, uint32_t *n_out,
                                cudaStream_t s) {
  if (!cnt) return cudaSuccess;
  row_segments_kernel<<<grid_for(cnt), BLOCK, 0, s>>>(k, cnt, seg, n_out);
  return cudaGetLastError();
}

cudaError_t launch_delete_rows(const Adj &A, const uint2 *uv, const uint32_t *mult,
                               const uint32_t *n_ptr, uint32_t max_n, uint32_t *found, Ctl *ctl,
                               int count_missing, cudaStream_t s) {
  if (!max_n) return cudaSuccess;
  delete_rows_kernel<<<grid_for((u64)max_n * 32), BLOCK, 0, s>>>(A, uv, mult, n_ptr, found, ctl,
                                                                 count_missing);
  return cudaGetLastError();
}

cudaError_t launch_add_rows(const Adj &A, const u64 *k, const uint32_t *w, const uint3 *seg,
                            const uint32_t *n_ptr, uint32_t max_n, int with_w, Ctl *ctl,
                            cudaStream_t s) {
  if (!max_n) return cudaSuccess;
  add_rows_kernel<<<grid_for((u64)max_n * 32), BLOCK, 0, s>>>(A, k, w, seg, n_ptr, with_w, ctl);
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
