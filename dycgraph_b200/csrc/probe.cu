// probe.cu -- host-link bandwidth measurement used to state the roofline of
// kernels that read the pinned host arena.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/dycg.h"
#include "common.cuh"

namespace dycg {

__global__ void zero_copy_read_kernel(const uint4 *src, u64 n16, unsigned long long *sink) {
  uint32_t acc = 0;
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n16;
       i += (u64)gridDim.x * blockDim.x) {
    const uint4 v = __ldg(src + i);
    acc ^= v.x ^ v.y ^ v.z ^ v.w;
  }
  if (acc == 0x9E3779B9u) atomicAdd(sink, 1ull);  // keeps the loads alive
}

// Random host-link transactions: every thread (op_bytes 4, 8 or 16) or every
// warp (op_bytes 128, one 4-byte word per lane) makes `per` accesses at
// op_bytes-aligned offsets drawn by a hash, reads or writes; the accesses of
// one thread are independent, so many are in flight. Offsets are
// line * op_bytes with line < lines = bytes / op_bytes: always inside the
// buffer.
__global__ void random_ops_kernel(uint8_t *base, u64 lines, uint32_t op_bytes, int write,
                                  uint32_t per, u64 seed, unsigned long long *sink) {
  const u64 tid = blockIdx.x * (u64)blockDim.x + threadIdx.x;
  const bool warp_op = op_bytes == 128;
  const u64 who = warp_op ? tid >> 5 : tid;  // warp-uniform for 128-byte lines
  const uint32_t lane = threadIdx.x & 31;
  uint32_t acc = 0;
#pragma unroll 4
  for (uint32_t i = 0; i < per; i++) {
    const u64 line = mix64(seed ^ (who * per + i)) % lines;
    uint8_t *p = base + line * op_bytes;
    // __ldcv / __stwt: uncached loads and write-through stores, so every
    // access goes over the link
    if (warp_op) {
      unsigned int *q = reinterpret_cast<unsigned int *>(p) + lane;
      if (write) __stwt(q, i);
      else acc ^= __ldcv(q);
    } else if (op_bytes == 16) {
      uint4 *q = reinterpret_cast<uint4 *>(p);
      if (write) {
        __stwt(q, make_uint4(i, i, i, i));
      } else {
        const uint4 v = __ldcv(q);
        acc ^= v.x ^ v.w;
      }
    } else if (op_bytes == 8) {
      uint2 *q = reinterpret_cast<uint2 *>(p);
      if (write) {
        __stwt(q, make_uint2(i, i));
      } else {
        const uint2 v = __ldcv(q);
        acc ^= v.x ^ v.y;
      }
    } else {
      unsigned int *q = reinterpret_cast<unsigned int *>(p);
      if (write) __stwt(q, i);
      else acc ^= __ldcv(q);
    }
  }
  if (acc == 0x9E3779B9u) atomicAdd(sink, 1ull);  // keeps the loads alive
}

// Accesses at the given byte offsets, in the order given (sorted by the
// caller), one per thread (8-byte words) or per warp (128-byte lines); the
// grid strides over them, so the accesses in flight are consecutive ones.
__global__ void sweep_ops_kernel(uint8_t *base, const u64 *off, u64 n, uint32_t op_bytes,
                                 int write, unsigned long long *sink) {
  const u64 tid = blockIdx.x * (u64)blockDim.x + threadIdx.x;
  const u64 nthreads = (u64)gridDim.x * blockDim.x;
  const uint32_t lane = threadIdx.x & 31;
  uint32_t acc = 0;
  if (op_bytes == 128) {
    for (u64 i = tid >> 5; i < n; i += nthreads >> 5) {
      unsigned int *q = reinterpret_cast<unsigned int *>(base + off[i]) + lane;
      if (write) __stwt(q, (uint32_t)i);
      else acc ^= __ldcv(q);
    }
  } else {
    for (u64 i = tid; i < n; i += nthreads) {
      uint2 *q = reinterpret_cast<uint2 *>(base + off[i]);
      if (write) {
        __stwt(q, make_uint2((uint32_t)i, 0u));
      } else {
        const uint2 v = __ldcv(q);
        acc ^= v.x ^ v.y;
      }
    }
  }
  if (acc == 0x9E3779B9u) atomicAdd(sink, 1ull);  // keeps the loads alive
}

}  // namespace dycg

extern "C" int dycg_measure_host_sweep(int device, uint64_t bytes, uint32_t op_bytes, int write,
                                       uint64_t ops, uint32_t ctas, double *ns_per_op) {
  if (op_bytes != 8 && op_bytes != 128) return DYCG_EINVAL;
  if (bytes < (1u << 20) || ops == 0 || ops > (1ull << 28) || ctas == 0 || !ns_per_op)
    return DYCG_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) return DYCG_ENOGPU;
  bytes &= ~127ull;
  // offsets: random lines of op_bytes, sorted ascending (inside the buffer)
  const uint64_t lines = bytes / op_bytes;
  std::vector<uint64_t> off(ops);
  for (uint64_t i = 0; i < ops; i++) off[i] = (dycg::mix64(0x5EED5ull ^ i) % lines) * op_bytes;
  std::sort(off.begin(), off.end());
  void *h = nullptr, *hd = nullptr;
  uint64_t *d_off = nullptr;
  unsigned long long *sink = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  int rc = DYCG_OK;
  if (cudaHostAlloc(&h, bytes, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess ||
      cudaMalloc(&sink, 8) != cudaSuccess || cudaMalloc(&d_off, ops * 8) != cudaSuccess ||
      cudaHostGetDevicePointer(&hd, h, 0) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
    rc = DYCG_ENOMEM;
  } else {
    memset(h, 1, bytes);
    cudaMemcpyAsync(d_off, off.data(), ops * 8, cudaMemcpyHostToDevice, s);
    float best = 1e30f;
    for (int rep = 0; rep < 4; rep++) {  // the first run warms up
      float ms = 0;
      cudaEventRecord(a, s);
      dycg::sweep_ops_kernel<<<ctas, 256, 0, s>>>((uint8_t *)hd, (const dycg::u64 *)d_off, ops,
                                                  op_bytes, write, sink);
      cudaEventRecord(b, s);
      cudaEventSynchronize(b);
      cudaEventElapsedTime(&ms, a, b);
      if (rep) best = std::min(best, ms);
    }
    if (cudaGetLastError() != cudaSuccess) rc = DYCG_ECUDA;
    *ns_per_op = best * 1e6 / (double)ops;
  }
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (s) cudaStreamDestroy(s);
  if (sink) cudaFree(sink);
  if (d_off) cudaFree(d_off);
  if (h) cudaFreeHost(h);
  return rc;
}

extern "C" int dycg_measure_host_random(int device, uint64_t bytes, uint32_t op_bytes, int write,
                                        uint64_t ops, double *ns_per_op) {
  if (op_bytes != 4 && op_bytes != 8 && op_bytes != 16 && op_bytes != 128) return DYCG_EINVAL;
  if (bytes < (1u << 20) || ops == 0 || !ns_per_op) return DYCG_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) return DYCG_ENOGPU;
  bytes &= ~127ull;
  void *h = nullptr, *hd = nullptr;
  unsigned long long *sink = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  int rc = DYCG_OK;
  if (cudaHostAlloc(&h, bytes, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess ||
      cudaMalloc(&sink, 8) != cudaSuccess || cudaHostGetDevicePointer(&hd, h, 0) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
    rc = DYCG_ENOMEM;
  } else {
    memset(h, 1, bytes);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const uint32_t blocks = (uint32_t)sms * 8, threads = 256;
    const uint64_t actors =
        op_bytes == 128 ? (uint64_t)blocks * threads / 32 : (uint64_t)blocks * threads;
    const uint32_t per = (uint32_t)std::min<uint64_t>((ops + actors - 1) / actors, 1u << 20);
    const uint64_t lines = bytes / op_bytes;
    float best = 1e30f;
    for (int rep = 0; rep < 4; rep++) {  // the first run warms up
      float ms = 0;
      cudaEventRecord(a, s);
      dycg::random_ops_kernel<<<blocks, threads, 0, s>>>((uint8_t *)hd, lines, op_bytes, write,
                                                        per, 0x5EEDull + rep, sink);
      cudaEventRecord(b, s);
      cudaEventSynchronize(b);
      cudaEventElapsedTime(&ms, a, b);
      if (rep) best = std::min(best, ms);
    }
    if (cudaGetLastError() != cudaSuccess) rc = DYCG_ECUDA;
    *ns_per_op = best * 1e6 / ((double)actors * per);
  }
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (s) cudaStreamDestroy(s);
  if (sink) cudaFree(sink);
  if (h) cudaFreeHost(h);
  return rc;
}

extern "C" int dycg_measure_host_link(int device, uint64_t bytes, double *h2d_gbs,
                                      double *zero_copy_gbs) {
  if (bytes < (1u << 20)) return DYCG_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) return DYCG_ENOGPU;
  bytes &= ~15ull;
  void *h = nullptr, *d = nullptr, *hd = nullptr;
  unsigned long long *sink = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  int rc = DYCG_OK;
  if (cudaHostAlloc(&h, bytes, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess ||
      cudaMalloc(&d, bytes) != cudaSuccess || cudaMalloc(&sink, 8) != cudaSuccess ||
      cudaHostGetDevicePointer(&hd, h, 0) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
    rc = DYCG_ENOMEM;
  } else {
    memset(h, 1, bytes);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    float best_copy = 1e30f, best_zc = 1e30f;
    for (int rep = 0; rep < 6; rep++) {
      float ms = 0;
      cudaEventRecord(a, s);
      cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s);
      cudaEventRecord(b, s);
      cudaEventSynchronize(b);
      cudaEventElapsedTime(&ms, a, b);
      if (rep) best_copy = std::min(best_copy, ms);
      cudaEventRecord(a, s);
      dycg::zero_copy_read_kernel<<<sms * 8, 256, 0, s>>>((const uint4 *)hd, bytes / 16, sink);
      cudaEventRecord(b, s);
      cudaEventSynchronize(b);
      cudaEventElapsedTime(&ms, a, b);
      if (rep) best_zc = std::min(best_zc, ms);
    }
    if (cudaGetLastError() != cudaSuccess) rc = DYCG_ECUDA;
    if (h2d_gbs) *h2d_gbs = bytes / (best_copy * 1e6);
    if (zero_copy_gbs) *zero_copy_gbs = bytes / (best_zc * 1e6);
  }
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (s) cudaStreamDestroy(s);
  if (sink) cudaFree(sink);
  if (d) cudaFree(d);
  if (h) cudaFreeHost(h);
  return rc;
}
