// group.cuh -- scratch layout of the update-grouping step (group.cu).
#pragma once
#include "../../include/dycg.h"
#include "common.cuh"

namespace dycg {

struct GroupScratch {
  u64 *keys_a, *keys_b;  // unsorted / sorted (row << 32 | neighbour) keys
  uint32_t *head, *pos;  // run heads and their exclusive prefix
  uint32_t *start;       // first sorted index of every run
  void *temp;            // CUB temporary storage
  size_t temp_bytes;
};

// Lay out the scratch for m records at base (256-byte aligned pieces).
inline void group_carve(void *base, uint32_t m, GroupScratch &S) {
  auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
  char *p = (char *)(((uintptr_t)base + 255) & ~(uintptr_t)255);
  S.keys_a = (u64 *)p;
  p += up((size_t)m * 8);
  S.keys_b = (u64 *)p;
  p += up((size_t)m * 8);
  S.head = (uint32_t *)p;
  p += up((size_t)m * 4);
  S.pos = (uint32_t *)p;
  p += up((size_t)m * 4);
  S.start = (uint32_t *)p;
  p += up((size_t)m * 4);
  S.temp = p;
}

inline size_t group_scratch_bytes(uint32_t m, size_t temp_bytes) {
  auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
  return 256 + 2 * up((size_t)m * 8) + 3 * up((size_t)m * 4) + temp_bytes;
}

size_t group_temp_bytes(uint32_t n);
cudaError_t group_run(const dycg_edge *d_records, uint32_t n, uint32_t num_vertices,
                      const uint32_t *seg_ends, uint32_t nseg, uint32_t *out_uv,
                      uint32_t *out_mult, uint32_t *seg_counts, uint32_t *counts,
                      const GroupScratch &S, cudaStream_t s);

}  // namespace dycg
