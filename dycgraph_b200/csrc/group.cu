// group.cu -- standalone GPU grouping of an update batch, the device form of
// the reference's GroupedUpdateBatch (include/framework/effective_update_batch.h:
// 36-207): records with an endpoint outside the vertex range are dropped and
// counted, the rest are radix-sorted by (u, v), and each distinct (u, v)
// becomes one output record with its multiplicity, in ascending (u, v) order.
// Optional per-segment counts of the distinct records bin them by source into
// the caller's vertex ranges (the reference's SEGMENT ranges).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "../../include/dycg.h"
#include "group.cuh"

namespace dycg {

__global__ void group_keys_kernel(const dycg_edge *e, uint32_t cnt, uint32_t n, u64 *keys,
                                  uint32_t *invalid) {
  uint32_t bad = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += gridDim.x * blockDim.x) {
    const dycg_edge r = e[i];
    const bool ok = r.u < n && r.v < n;
    bad += !ok;
    keys[i] = ok ? (((u64)r.u << 32) | r.v) : KEY_INF;
  }
  for (int o = 16; o; o >>= 1) bad += __shfl_down_sync(0xffffffffu, bad, o);
  if ((threadIdx.x & 31) == 0 && bad) atomicAdd(invalid, bad);
}

__global__ void group_heads_kernel(const u64 *k, uint32_t cnt, uint32_t *head) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += gridDim.x * blockDim.x)
    head[i] = k[i] != KEY_INF && (i == 0 || k[i - 1] != k[i]);
}

// Run heads in key order: the run number o of head i is pos[i]; record its
// first index, emit its (u, v) and bin it into its segment.
__global__ void group_starts_kernel(const u64 *k, const uint32_t *head, const uint32_t *pos,
                                    uint32_t cnt, uint32_t *start, uint32_t *out_uv,
                                    const uint32_t *seg_ends, uint32_t nseg,
                                    uint32_t *seg_counts, uint32_t *counts) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += gridDim.x * blockDim.x) {
    if (i == cnt - 1) counts[0] = pos[i] + head[i];
    if (!head[i]) continue;
    const u64 key = k[i];
    const uint32_t o = pos[i];
    const uint32_t u = (uint32_t)(key >> 32);
    start[o] = i;
    out_uv[2 * o] = u;
    out_uv[2 * o + 1] = (uint32_t)key;
    if (seg_counts && nseg) {
      uint32_t lo = 0, hi = nseg;  // first segment whose end is > u
      while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2;
        if (seg_ends[mid] <= u) lo = mid + 1; else hi = mid;
      }
      if (lo < nseg) atomicAdd(seg_counts + lo, 1u);
    }
  }
}

// Multiplicity of run o = distance to the next run's first index; the last
// run ends at the number of valid keys (invalid ones sort last as KEY_INF).
// One thread per run whatever its length, so a batch of one repeated record
// costs the same as a batch of distinct ones.
__global__ void group_mult_kernel(const uint32_t *start, uint32_t cnt, const uint32_t *counts,
                                  uint32_t *out_mult) {
  const uint32_t runs = counts[0];
  const uint32_t valid = cnt - counts[1];
  for (uint32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < runs;
       o += gridDim.x * blockDim.x) {
    const uint32_t end = o + 1 < runs ? start[o + 1] : valid;
    out_mult[o] = end - start[o];
  }
}

static int grid_for(u64 threads) {
  u64 b = (threads + BLOCK - 1) / BLOCK;
  if (b < 1) b = 1;
  if (b > 148ull * 32) b = 148ull * 32;
  return (int)b;
}

size_t group_temp_bytes(uint32_t n) {
  size_t a = 0, b = 0;
  cub::DeviceRadixSort::SortKeys(nullptr, a, (const u64 *)nullptr, (u64 *)nullptr, (int)n, 0, 64);
  cub::DeviceScan::ExclusiveSum(nullptr, b, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                (int)n);
  return a > b ? a : b;
}

cudaError_t group_run(const dycg_edge *d_records, uint32_t n, uint32_t num_vertices,
                      const uint32_t *seg_ends, uint32_t nseg, uint32_t *out_uv,
                      uint32_t *out_mult, uint32_t *seg_counts, uint32_t *counts,
                      const GroupScratch &S, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(counts, 0, 2 * sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  if (seg_counts && nseg) {
    e = cudaMemsetAsync(seg_counts, 0, (size_t)nseg * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
  }
  if (n == 0) return cudaSuccess;
  group_keys_kernel<<<grid_for(n), BLOCK, 0, s>>>(d_records, n, num_vertices, S.keys_a,
                                                  counts + 1);
  size_t tb = S.temp_bytes;
  e = cub::DeviceRadixSort::SortKeys(S.temp, tb, S.keys_a, S.keys_b, (int)n, 0, 64, s);
  if (e != cudaSuccess) return e;
  group_heads_kernel<<<grid_for(n), BLOCK, 0, s>>>(S.keys_b, n, S.head);
  tb = S.temp_bytes;
  e = cub::DeviceScan::ExclusiveSum(S.temp, tb, S.head, S.pos, (int)n, s);
  if (e != cudaSuccess) return e;
  group_starts_kernel<<<grid_for(n), BLOCK, 0, s>>>(S.keys_b, S.head, S.pos, n, S.start, out_uv,
                                                    seg_ends, nseg, seg_counts, counts);
  group_mult_kernel<<<grid_for(n), BLOCK, 0, s>>>(S.start, n, counts, out_mult);
  return cudaGetLastError();
}

}  // namespace dycg

using namespace dycg;

extern "C" int dycg_group_updates(const dycg_edge *d_records, size_t n, uint32_t num_vertices,
                                  const uint32_t *d_segment_ends, uint32_t num_segments,
                                  uint32_t *d_out_uv, uint32_t *d_out_mult,
                                  uint32_t *d_segment_counts, uint32_t *d_counts,
                                  void *stream) {
  if ((n && (!d_records || !d_out_uv || !d_out_mult)) || !d_counts || n > 0x7FFFFFFFull ||
      (num_segments && !d_segment_ends))
    return DYCG_EINVAL;
  cudaStream_t s = (cudaStream_t)stream;
  GroupScratch S{};
  const uint32_t m = (uint32_t)std::max<size_t>(n, 1);
  S.temp_bytes = group_temp_bytes(m);
  void *base = nullptr;
  const size_t bytes = group_scratch_bytes(m, S.temp_bytes);
  if (cudaMallocAsync(&base, bytes, s) != cudaSuccess) return DYCG_ENOMEM;
  group_carve(base, m, S);
  cudaError_t e = group_run(d_records, (uint32_t)n, num_vertices, d_segment_ends, num_segments,
                            d_out_uv, d_out_mult, d_segment_counts, d_counts, S, s);
  cudaError_t f = cudaFreeAsync(base, s);
  if (e != cudaSuccess || f != cudaSuccess) return DYCG_ECUDA;
  return DYCG_OK;
}
