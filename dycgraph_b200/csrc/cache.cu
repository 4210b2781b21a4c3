// cache.cu -- HBM page cache: hotness scores, top-K admission, eviction and
// page staging.
//
// Replaces the reference's per-vertex edge cache maintenance
// (compute_hot_vertices_sssp / confirm_candidate_batch / evication_cache /
// compact_cache / LoadCache, include/framework/framework.cuh:1264-1567,
// :2978-3061; comp_hotness_sssp, include/framework/variants/driver.cuh:486-515;
// cache_refresh_gate.h:9-31). The unit is a fixed-size page of the host arena
// instead of a vertex row: a page's score is a decayed count of the slots the
// kernels read from it (the reference sums four uint8 activity windows per
// vertex); the resident set is the top-K pages by score (stable: ties go to
// the smaller page id, as the reference's stable CUB sort does,
// tests/hotness_pairing_test.cu:30-55); a refresh happens only when enough
// top-K pages are missing (the refresh gate). Because every write goes to both
// copies, eviction is a page-table update and compaction is never needed.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "internal.h"

namespace dycg {

__global__ void score_kernel(uint32_t *hits, float *score, uint32_t *ids, uint32_t npages,
                             float decay) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npages;
       p += gridDim.x * blockDim.x) {
    score[p] = score[p] * decay + (float)hits[p];
    hits[p] = 0;
    ids[p] = p;
  }
}

// flags in sorted (descending score) order: admit candidates among the top K,
// eviction candidates among the rest.
__global__ void flag_kernel(const uint32_t *ids, const float *sc, uint32_t npages, uint32_t K,
                            float min_score, const uint32_t *page_slot, uint32_t *fa,
                            uint32_t *fe) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npages;
       i += gridDim.x * blockDim.x) {
    const bool top = i < K && sc[i] > 0.f;
    const bool res = page_slot[ids[i]] != PAGE_NONE;
    fa[i] = top && !res && sc[i] >= min_score;
    fe[i] = !top && res;
  }
}

// Admission plan of one maintenance round, computed on the device from the
// flag scans (admit candidates among the top K, eviction candidates among the
// rest) and the free-slot count, so no host round trip sits between ranking
// and staging: the refresh gate skips rounds with fewer than `gate` missing
// top pages, at most `cap` pages are admitted, and only as many resident
// pages are evicted (the lowest ranked first) as the free slots cannot cover.
__global__ void plan_kernel(const uint32_t *sa, const uint32_t *fa, const uint32_t *se,
                            const uint32_t *fe, uint32_t npages, uint32_t gate, uint32_t cap,
                            CachePlan *plan, u64 *stat_loaded, u64 *stat_evicted) {
  if (threadIdx.x || blockIdx.x) return;
  const uint32_t n_admit = npages ? sa[npages - 1] + fa[npages - 1] : 0;
  const uint32_t n_evict = npages ? se[npages - 1] + fe[npages - 1] : 0;
  const uint32_t free0 = plan->free_count;
  uint32_t admit = 0, evict = 0;
  if (n_admit >= gate && n_admit) {
    admit = min(n_admit, cap);
    const uint32_t need = admit > free0 ? admit - free0 : 0u;
    evict = min(n_evict, need);
    admit = min(admit, free0 + evict);
  }
  plan->candidates = n_admit;
  plan->admit = admit;
  plan->evict = evict;
  plan->first_rank = n_evict - evict;
  plan->free_base = free0;
  plan->top = free0 + evict;
  plan->free_count = free0 + evict - admit;
  plan->loaded += admit;
  plan->evicted += evict;
  if (stat_loaded && admit) atomicAdd(stat_loaded, (u64)admit);
  if (stat_evicted && evict) atomicAdd(stat_evicted, (u64)evict);
}

__global__ void evict_kernel(const uint32_t *ids, uint32_t npages, const uint32_t *fe,
                             const uint32_t *se, const CachePlan *plan, uint32_t *page_slot,
                             uint32_t *free_list) {
  const uint32_t evict = plan->evict, first_rank = plan->first_rank, base = plan->free_base;
  if (!evict) return;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npages;
       i += gridDim.x * blockDim.x) {
    if (!fe[i] || se[i] < first_rank) continue;
    const uint32_t p = ids[i];
    free_list[base + (se[i] - first_rank)] = page_slot[p];
    page_slot[p] = PAGE_NONE;
  }
}

__global__ void admit_list_kernel(const uint32_t *ids, uint32_t npages, const uint32_t *fa,
                                  const uint32_t *sa, const CachePlan *plan, uint32_t *admit) {
  const uint32_t limit = plan->admit;
  if (!limit) return;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npages;
       i += gridDim.x * blockDim.x)
    if (fa[i] && sa[i] < limit) admit[sa[i]] = ids[i];
}

// CTA per page: copy the page's slot words from the host arena into its cache
// slot with 16-byte loads, then publish it in the page table. The grid is
// fixed; the page count comes from the plan.
__global__ void fill_kernel(const uint32_t *admit, const CachePlan *plan,
                            const uint32_t *free_list, uint32_t *page_slot, const uint32_t *h_out,
                            const uint32_t *h_in, uint32_t pages_out, uint32_t page_shift,
                            uint32_t stride, uint32_t *cdst) {
  const uint32_t count = plan->admit, free_top = plan->top;
  const u64 words = (u64)stride << page_shift;
  for (uint32_t j = blockIdx.x; j < count; j += gridDim.x) {
    const uint32_t p = admit[j];
    const uint32_t slot = free_list[free_top - 1 - j];
    const bool in_dir = p >= pages_out;
    const u64 first = (u64)(in_dir ? p - pages_out : p) * words;
    const uint4 *sd = reinterpret_cast<const uint4 *>((in_dir ? h_in : h_out) + first);
    uint4 *dd = reinterpret_cast<uint4 *>(cdst + (u64)slot * words);
    for (uint32_t t = threadIdx.x; t < words / 4; t += blockDim.x) dd[t] = sd[t];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) page_slot[p] = slot;
  }
}

static int grid_for(u64 threads) {
  u64 b = (threads + BLOCK - 1) / BLOCK;
  if (b < 1) b = 1;
  if (b > 148ull * 32) b = 148ull * 32;
  return (int)b;
}

cudaError_t cache_rank(CacheWork &W, uint32_t npages, uint32_t K, float decay, float min_score,
                       const uint32_t *page_slot, cudaStream_t s) {
  score_kernel<<<grid_for(npages), BLOCK, 0, s>>>(W.hits, W.score, W.ids, npages, decay);
  size_t bytes = W.temp_bytes;
  cudaError_t e = cub::DeviceRadixSort::SortPairsDescending(
      W.temp, bytes, W.score, W.score_sorted, W.ids, W.ids_sorted, (int)npages, 0, 32, s);
  if (e != cudaSuccess) return e;
  flag_kernel<<<grid_for(npages), BLOCK, 0, s>>>(W.ids_sorted, W.score_sorted, npages, K,
                                                 min_score, page_slot, W.fa, W.fe);
  bytes = W.temp_bytes;
  e = cub::DeviceScan::ExclusiveSum(W.temp, bytes, W.fa, W.sa, (int)npages, s);
  if (e != cudaSuccess) return e;
  bytes = W.temp_bytes;
  e = cub::DeviceScan::ExclusiveSum(W.temp, bytes, W.fe, W.se, (int)npages, s);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

cudaError_t cache_rank_given(CacheWork &W, uint32_t npages, uint32_t K, float min_score,
                             const uint32_t *page_slot, cudaStream_t s) {
  size_t bytes = W.temp_bytes;
  cudaError_t e = cub::DeviceRadixSort::SortPairsDescending(
      W.temp, bytes, W.score, W.score_sorted, W.ids, W.ids_sorted, (int)npages, 0, 32, s);
  if (e != cudaSuccess) return e;
  flag_kernel<<<grid_for(npages), BLOCK, 0, s>>>(W.ids_sorted, W.score_sorted, npages, K,
                                                 min_score, page_slot, W.fa, W.fe);
  bytes = W.temp_bytes;
  e = cub::DeviceScan::ExclusiveSum(W.temp, bytes, W.fa, W.sa, (int)npages, s);
  if (e != cudaSuccess) return e;
  bytes = W.temp_bytes;
  e = cub::DeviceScan::ExclusiveSum(W.temp, bytes, W.fe, W.se, (int)npages, s);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

size_t cache_temp_bytes(uint32_t npages) {
  size_t a = 0, b = 0;
  cub::DeviceRadixSort::SortPairsDescending(nullptr, a, (const float *)nullptr, (float *)nullptr,
                                            (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                            (int)npages, 0, 32);
  cub::DeviceScan::ExclusiveSum(nullptr, b, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                (int)npages);
  return a > b ? a : b;
}

cudaError_t cache_plan(CacheWork &W, uint32_t npages, uint32_t gate, uint32_t cap,
                       u64 *stat_loaded, u64 *stat_evicted, cudaStream_t s) {
  plan_kernel<<<1, 32, 0, s>>>(W.sa, W.fa, W.se, W.fe, npages, gate, cap, W.plan, stat_loaded,
                               stat_evicted);
  return cudaGetLastError();
}

cudaError_t cache_stage(CacheWork &W, uint32_t npages, uint32_t *page_slot, uint32_t *free_list,
                        const CachePages &pg, cudaStream_t s) {
  evict_kernel<<<grid_for(npages), BLOCK, 0, s>>>(W.ids_sorted, npages, W.fe, W.se, W.plan,
                                                  page_slot, free_list);
  admit_list_kernel<<<grid_for(npages), BLOCK, 0, s>>>(W.ids_sorted, npages, W.fa, W.sa, W.plan,
                                                       W.admit);
  fill_kernel<<<148 * 8, BLOCK, 0, s>>>(W.admit, W.plan, free_list, page_slot, pg.h_out, pg.h_in,
                                        pg.pages_out, pg.page_shift, pg.stride, pg.cdst);
  return cudaGetLastError();
}

cudaError_t cache_apply(CacheWork &W, uint32_t npages, uint32_t gate, uint32_t cap,
                        uint32_t *page_slot, uint32_t *free_list, const CachePages &pg,
                        u64 *stat_loaded, u64 *stat_evicted, cudaStream_t s) {
  cudaError_t e = cache_plan(W, npages, gate, cap, stat_loaded, stat_evicted, s);
  if (e != cudaSuccess) return e;
  return cache_stage(W, npages, page_slot, free_list, pg, s);
}

}  // namespace dycg
