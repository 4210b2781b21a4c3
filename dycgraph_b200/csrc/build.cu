// build.cu -- graph construction on the GPU straight into the pinned host
// arenas: synthetic generators (R-MAT, 2D grid with shortcuts), key sort,
// de-duplication, power-of-two block layout (the chunk store's layout,
// include/framework/framework.cuh:1657-1668) and the incoming adjacency
// (the reference builds a CPU reverse index instead,
// include/framework/dynamic_reverse_index.h:46).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "internal.h"

namespace dycg {

static int grid_for(u64 threads) {
  u64 b = (threads + BLOCK - 1) / BLOCK;
  if (b < 1) b = 1;
  if (b > 148ull * 64) b = 148ull * 64;
  return (int)b;
}

__global__ void rmat_keys_kernel(u64 *keys, u64 count, u64 seed, uint32_t scale, uint32_t ta,
                                 uint32_t tab, uint32_t tabc, int symmetrize) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < count;
       i += (u64)gridDim.x * blockDim.x) {
    uint32_t u, v;
    rmat_draw(seed, i, scale, ta, tab, tabc, u, v);
    keys[i] = u == v ? KEY_INF : (((u64)u << 32) | v);
    if (symmetrize) keys[count + i] = u == v ? KEY_INF : (((u64)v << 32) | u);
  }
}

// 4-neighbour grid (both directions) plus random shortcuts within a
// Chebyshev radius, also in both directions.
__global__ void grid_keys_kernel(u64 *keys, uint32_t side, u64 nshort, uint32_t radius,
                                 u64 seed) {
  const u64 nv = (u64)side * side;
  const u64 total = nv * 4 + nshort * 2;
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < total;
       i += (u64)gridDim.x * blockDim.x) {
    u64 key = KEY_INF;
    if (i < nv * 4) {
      const u64 x = i >> 2;
      const uint32_t r = (uint32_t)(x / side), c = (uint32_t)(x % side);
      const uint32_t u = (uint32_t)x;
      switch (i & 3) {
        case 0: if (c + 1 < side) key = ((u64)u << 32) | (u + 1); break;
        case 1: if (c + 1 < side) key = ((u64)(u + 1) << 32) | u; break;
        case 2: if (r + 1 < side) key = ((u64)u << 32) | (u + side); break;
        default: if (r + 1 < side) key = ((u64)(u + side) << 32) | u; break;
      }
    } else {
      const u64 j = (i - nv * 4) >> 1;
      const u64 h = mix64(seed ^ mix64(j + 0x51ED270B));
      const uint32_t u = (uint32_t)(h % nv);
      const int span = 2 * (int)radius + 1;
      const int dr = (int)((h >> 32) % span) - (int)radius;
      const int dc = (int)((h >> 48) % span) - (int)radius;
      const int r = (int)(u / side) + dr, c = (int)(u % side) + dc;
      if ((dr || dc) && r >= 0 && c >= 0 && r < (int)side && c < (int)side) {
        const uint32_t v = (uint32_t)r * side + (uint32_t)c;
        key = (i & 1) ? (((u64)v << 32) | u) : (((u64)u << 32) | v);
      }
    }
    keys[i] = key;
  }
}

__global__ void csr_keys_kernel(const u64 *off, const uint32_t *dst, uint32_t n, u64 *keys) {
  // one thread per vertex row is enough for the loader (rows are copied in order)
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x)
    for (u64 e = off[u]; e < off[u + 1]; e++) keys[e] = ((u64)u << 32) | dst[e];
}

__global__ void swap_keys_kernel(const u64 *in, u64 *out, u64 count) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < count;
       i += (u64)gridDim.x * blockDim.x) {
    const u64 k = in[i];
    out[i] = k == KEY_INF ? KEY_INF : ((k << 32) | (k >> 32));
  }
}

__global__ void unique_flags_kernel(const u64 *k, u64 count, uint32_t *flag, int dedup) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < count;
       i += (u64)gridDim.x * blockDim.x)
    flag[i] = k[i] != KEY_INF && (!dedup || i == 0 || k[i - 1] != k[i]);
}

__global__ void compact_kernel(const u64 *k, const uint32_t *vin, const uint32_t *flag,
                               const u64 *pos, u64 count, u64 *out, uint32_t *vout) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < count;
       i += (u64)gridDim.x * blockDim.x)
    if (flag[i]) {
      out[pos[i]] = k[i];
      if (vin) vout[pos[i]] = vin[i];
    }
}

__global__ void degree_kernel(const u64 *k, u64 m, uint32_t *deg) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < m;
       i += (u64)gridDim.x * blockDim.x)
    atomicAdd(deg + (uint32_t)(k[i] >> 32), 1u);
}

__global__ void caps_kernel(const uint32_t *deg, uint32_t n, u64 *cap64, uint32_t *cap,
                            uint32_t *len, uint32_t *srt, uint32_t *live) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    // power-of-two blocks with headroom: a row of exactly 2^k occurrences
    // still has room to grow before it must move
    const uint32_t d = deg[v];
    const uint32_t need = d + d / 16 + 1;
    const uint32_t c = d == 0 ? 0u : (need <= 1 ? 1u : 1u << (32 - __clz(need - 1)));
    cap64[v] = c;
    cap[v] = c;
    len[v] = d;
    srt[v] = d;
    live[v] = d;
  }
}

// Rows are contiguous in the sorted key array: slot = off[u] + (i - rowstart[u]).
__global__ void scatter_kernel(const u64 *k, const uint32_t *wv, u64 m, const u64 *off,
                               const u64 *rowstart, uint32_t *hwords, uint32_t stride,
                               uint32_t *fence, uint32_t fence_shift, u64 wseed, uint32_t wlo,
                               uint32_t whi, int weight_from_hash, int swapped) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < m;
       i += (u64)gridDim.x * blockDim.x) {
    const u64 key = k[i];
    const uint32_t u = (uint32_t)(key >> 32), v = (uint32_t)key;
    const u64 slot = off[u] + (i - rowstart[u]);
    if (stride == 2) {
      // weights are a property of the directed edge (source, target)
      const uint32_t s = swapped ? v : u, t = swapped ? u : v;
      const uint32_t w = weight_from_hash ? hash_weight(wseed, s, t, wlo, whi) : wv[i];
      *reinterpret_cast<uint2 *>(hwords + slot * 2) = make_uint2(v, w);
    } else {
      hwords[slot] = v;
    }
    if ((slot & ((1ull << fence_shift) - 1)) == 0) fence[slot >> fence_shift] = v;
  }
}

cudaError_t build_gen_rmat(u64 *keys, u64 draws, u64 seed, uint32_t scale, double a, double b,
                           double c, int symmetrize, cudaStream_t s) {
  const double S = (double)(1u << 21);
  const uint32_t ta = (uint32_t)(a * S), tab = (uint32_t)((a + b) * S),
                 tabc = (uint32_t)((a + b + c) * S);
  rmat_keys_kernel<<<grid_for(draws), BLOCK, 0, s>>>(keys, draws, seed, scale, ta, tab, tabc,
                                                     symmetrize);
  return cudaGetLastError();
}

cudaError_t build_gen_grid(u64 *keys, uint32_t side, u64 nshort, uint32_t radius, u64 seed,
                           cudaStream_t s) {
  const u64 total = (u64)side * side * 4 + nshort * 2;
  grid_keys_kernel<<<grid_for(total), BLOCK, 0, s>>>(keys, side, nshort, radius, seed);
  return cudaGetLastError();
}

cudaError_t build_csr_keys(const u64 *off, const uint32_t *dst, uint32_t n, u64 *keys,
                           cudaStream_t s) {
  csr_keys_kernel<<<grid_for(n), BLOCK, 0, s>>>(off, dst, n, keys);
  return cudaGetLastError();
}

cudaError_t build_swap_keys(const u64 *in, u64 *out, u64 count, cudaStream_t s) {
  swap_keys_kernel<<<grid_for(count), BLOCK, 0, s>>>(in, out, count);
  return cudaGetLastError();
}

cudaError_t build_sort(void *temp, size_t &bytes, u64 *k_in, u64 *k_out, uint32_t *v_in,
                       uint32_t *v_out, u64 count, cudaStream_t s) {
  if (v_in)
    return cub::DeviceRadixSort::SortPairs(temp, bytes, k_in, k_out, v_in, v_out, (int64_t)count,
                                           0, 64, s);
  return cub::DeviceRadixSort::SortKeys(temp, bytes, k_in, k_out, (int64_t)count, 0, 64, s);
}

cudaError_t build_scan_u32_to_u64(void *temp, size_t &bytes, const uint32_t *in, u64 *out,
                                  u64 count, cudaStream_t s) {
  return cub::DeviceScan::ExclusiveSum(temp, bytes, in, out, (int64_t)count, s);
}

cudaError_t build_scan_u64(void *temp, size_t &bytes, const u64 *in, u64 *out, u64 count,
                           cudaStream_t s) {
  return cub::DeviceScan::ExclusiveSum(temp, bytes, in, out, (int64_t)count, s);
}

cudaError_t build_unique(const u64 *k, const uint32_t *vin, u64 count, int dedup,
                         uint32_t *flag, u64 *pos, u64 *out, uint32_t *vout, void *temp,
                         size_t temp_bytes, cudaStream_t s) {
  unique_flags_kernel<<<grid_for(count), BLOCK, 0, s>>>(k, count, flag, dedup);
  size_t b = temp_bytes;
  cudaError_t e = cub::DeviceScan::ExclusiveSum(temp, b, flag, pos, (int64_t)count, s);
  if (e != cudaSuccess) return e;
  compact_kernel<<<grid_for(count), BLOCK, 0, s>>>(k, vin, flag, pos, count, out, vout);
  return cudaGetLastError();
}

cudaError_t build_degrees(const u64 *k, u64 m, uint32_t *deg, cudaStream_t s) {
  if (!m) return cudaSuccess;
  degree_kernel<<<grid_for(m), BLOCK, 0, s>>>(k, m, deg);
  return cudaGetLastError();
}

cudaError_t build_caps(const uint32_t *deg, uint32_t n, u64 *cap64, uint32_t *cap,
                       uint32_t *len, uint32_t *srt, uint32_t *live, cudaStream_t s) {
  caps_kernel<<<grid_for(n), BLOCK, 0, s>>>(deg, n, cap64, cap, len, srt, live);
  return cudaGetLastError();
}

cudaError_t build_scatter(const u64 *k, const uint32_t *wv, u64 m, const u64 *off,
                          const u64 *rowstart, uint32_t *hwords, uint32_t stride, uint32_t *fence,
                          uint32_t fence_shift, u64 wseed, uint32_t wlo, uint32_t whi,
                          int weight_from_hash, int swapped, cudaStream_t s) {
  if (!m) return cudaSuccess;
  scatter_kernel<<<grid_for(m), BLOCK, 0, s>>>(k, wv, m, off, rowstart, hwords, stride, fence,
                                               fence_shift, wseed, wlo, whi, weight_from_hash,
                                               swapped);
  return cudaGetLastError();
}

size_t build_temp_bytes(u64 count, bool pairs) {
  size_t a = 0, b = 0, c = 0;
  if (pairs)
    cub::DeviceRadixSort::SortPairs(nullptr, a, (u64 *)nullptr, (u64 *)nullptr,
                                    (uint32_t *)nullptr, (uint32_t *)nullptr, (int64_t)count, 0,
                                    64);
  else
    cub::DeviceRadixSort::SortKeys(nullptr, a, (u64 *)nullptr, (u64 *)nullptr, (int64_t)count, 0,
                                   64);
  cub::DeviceScan::ExclusiveSum(nullptr, b, (const uint32_t *)nullptr, (u64 *)nullptr,
                                (int64_t)count);
  cub::DeviceScan::ExclusiveSum(nullptr, c, (const u64 *)nullptr, (u64 *)nullptr,
                                (int64_t)count);
  return std::max(a, std::max(b, c));
}

// ---- sampling of live edges (workload generation) -----------------------

__global__ void draw_positions_kernel(u64 *pos, u64 count, u64 seed, u64 total) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < count;
       i += (u64)gridDim.x * blockDim.x)
    pos[i] = mix64(seed ^ mix64(i + 0xA24BAED4963EE407ull)) % total;
}

// Resolve a live-edge rank r into (u, v, w): u by binary search over the
// exclusive prefix of live degrees, then the k-th live slot of u's row.
__global__ void resolve_positions_kernel(const u64 *pos, u64 count, const u64 *pre, uint32_t n,
                                         Adj A, uint32_t *out) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < count;
       i += (u64)gridDim.x * blockDim.x) {
    const u64 r = pos[i];
    uint32_t lo = 0, hi = n;  // largest u with pre[u] <= r
    while (hi - lo > 1) {
      const uint32_t mid = lo + (hi - lo) / 2;
      if (pre[mid] <= r) lo = mid; else hi = mid;
    }
    const uint32_t u = lo;
    u64 k = r - pre[u];
    const u64 off = A.off[u];
    const uint32_t len = A.len[u];
    uint32_t v = 0, w = 0;
    if (A.live[u] == len && k < len) {  // no deleted slot: direct index
      const uint2 pr = read_pair_rw(A, off + k);
      v = pr.x & VMASK;
      w = pr.y;
      k = len;  // skip the scan
    }
    for (uint32_t s = 0; s < len && k < len; s++) {
      const uint2 pr = read_pair_rw(A, off + s);
      if (slot_deleted_rw(A, off + s, pr.x)) continue;
      if (k == 0) {
        v = pr.x;
        w = pr.y;
        break;
      }
      k--;
    }
    out[3 * i] = u;
    out[3 * i + 1] = v;
    out[3 * i + 2] = w;
  }
}

// One live out-edge of each given source, uniform over its live slots (up to
// 16 random probes, then a scan); (INF32, INF32, 0) when the row is empty or
// the source is out of range.
__global__ void row_edges_kernel(Adj A, const uint32_t *sources, u64 count, u64 seed, uint32_t n,
                                 uint32_t *out) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < count;
       i += (u64)gridDim.x * blockDim.x) {
    const uint32_t u = sources[i];
    uint32_t v = INF32, w = 0, uu = INF32;
    if (u < n && A.live[u] > 0) {
      const u64 off = A.off[u];
      const uint32_t len = A.len[u];
      bool got = false;
      for (int t = 0; t < 16 && !got; t++) {
        const uint32_t k = (uint32_t)(mix64(seed ^ mix64(i * 16 + t + 1)) % len);
        const uint2 pr = read_pair_rw(A, off + k);
        if (!slot_deleted_rw(A, off + k, pr.x)) {
          v = pr.x & VMASK;
          w = pr.y;
          got = true;
        }
      }
      for (uint32_t k = 0; k < len && !got; k++) {
        const uint2 pr = read_pair_rw(A, off + k);
        if (!slot_deleted_rw(A, off + k, pr.x)) {
          v = pr.x & VMASK;
          w = pr.y;
          got = true;
        }
      }
      if (got) uu = u;
    }
    out[3 * i] = uu;
    out[3 * i + 1] = v;
    out[3 * i + 2] = w;
  }
}

cudaError_t sample_row_edges(const Adj &A, const uint32_t *sources, u64 count, u64 seed,
                             uint32_t n, uint32_t *out, cudaStream_t s) {
  if (!count) return cudaSuccess;
  row_edges_kernel<<<grid_for(count), BLOCK, 0, s>>>(A, sources, count, seed, n, out);
  return cudaGetLastError();
}

cudaError_t sample_draw(u64 *pos, u64 count, u64 seed, u64 total, cudaStream_t s) {
  draw_positions_kernel<<<grid_for(count), BLOCK, 0, s>>>(pos, count, seed, total);
  return cudaGetLastError();
}

cudaError_t sample_resolve(const u64 *pos, u64 count, const u64 *pre, uint32_t n, const Adj &A,
                           uint32_t *out, cudaStream_t s) {
  resolve_positions_kernel<<<grid_for(count), BLOCK, 0, s>>>(pos, count, pre, n, A, out);
  return cudaGetLastError();
}

}  // namespace dycg
