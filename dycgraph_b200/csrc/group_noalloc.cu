// group_noalloc.cu -- dycg_group_updates_noalloc: the update-grouping step with
// its scratch in a fixed, file-scope device array, for callers that cannot
// allocate device memory at call time.
//
// Who needs it: code running where a cudaMalloc is not allowed or not safe --
// inside a region that must not synchronise the device (cudaMalloc may), in a
// process whose device memory is already fully reserved by another allocator
// or pool, or in a host component that must not own GPU allocations at all.
// Those callers still pass their own input and output buffers.
//
// Limits and sharing: the array holds at most DYCG_GROUP_NOALLOC_MAX_RECORDS
// records' scratch (about 10 MiB) and stays allocated on every GPU that loads
// the library until the process exits. Every call uses the same array and
// leaves its contents behind, so calls that overlap on the GPU (different
// streams without ordering, or different host threads) race and must not be
// issued concurrently; calls ordered on one stream are safe.
//
// Set-up: the host-side name of a __device__ array is only a stand-in and must
// never be handed to a kernel, so a call resolves the array's device address
// with cudaGetSymbolAddress on the current device. The first call on a device
// does this set-up and should come before any stream capture. Later calls
// resolve it again whenever their stream is not capturing, so the address
// stays valid after a device reset has reloaded the module.
#include <cstdio>
#include <mutex>

#include "../../include/dycg.h"
#include "group.cuh"

namespace {

constexpr uint32_t kMax = DYCG_GROUP_NOALLOC_MAX_RECORDS;
constexpr size_t kTemp = 4u << 20;  // CUB sort/scan temporary storage
constexpr size_t kUp8 = ((size_t)kMax * 8 + 255) & ~(size_t)255;
constexpr size_t kUp4 = ((size_t)kMax * 4 + 255) & ~(size_t)255;
constexpr size_t kBytes = 256 + 2 * kUp8 + 3 * kUp4 + kTemp;

__device__ __align__(256) unsigned char g_group_scratch[kBytes];

std::mutex g_mu;
void *g_addr[128] = {};  // device address of g_group_scratch, per device ordinal
int g_temp_ok = -1;      // CUB's storage need for kMax records fits kTemp (checked once)

}  // namespace

extern "C" int dycg_group_updates_noalloc(const dycg_edge *d_records, size_t n,
                                          uint32_t num_vertices, const uint32_t *d_segment_ends,
                                          uint32_t num_segments, uint32_t *d_out_uv,
                                          uint32_t *d_out_mult, uint32_t *d_segment_counts,
                                          uint32_t *d_counts, void *stream) {
  if ((n && (!d_records || !d_out_uv || !d_out_mult)) || !d_counts ||
      (num_segments && !d_segment_ends))
    return DYCG_EINVAL;
  if (n > kMax) {
    std::fprintf(stderr,
                 "dycg_group_updates_noalloc: %zu records exceed the fixed scratch capacity "
                 "of %u records; use dycg_group_updates or split the batch\n",
                 n, kMax);
    return DYCG_ECAPACITY;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return DYCG_ENOGPU;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing((cudaStream_t)stream, &cap) != cudaSuccess) return DYCG_ECUDA;
  void *base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (g_temp_ok < 0) {
      // a build whose CUB needs more temporary storage than the array holds is
      // a configuration error, not an oversized batch
      g_temp_ok = dycg::group_temp_bytes(kMax) <= kTemp ? 1 : 0;
      if (!g_temp_ok)
        std::fprintf(stderr,
                     "dycg_group_updates_noalloc: CUB needs %zu bytes of temporary storage "
                     "for %u records, more than the fixed %zu (kTemp); rebuild with a larger "
                     "kTemp\n",
                     dycg::group_temp_bytes(kMax), kMax, kTemp);
    }
    if (!g_temp_ok) return DYCG_ESTATE;
    if (cap == cudaStreamCaptureStatusNone) {
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_group_scratch);
      if (e != cudaSuccess || !p) return DYCG_ECUDA;
      g_addr[dev] = p;
    } else if (!g_addr[dev]) {
      std::fprintf(stderr,
                   "dycg_group_updates_noalloc: the first call on a device must not be "
                   "captured (the scratch address is resolved outside capture)\n");
      return DYCG_ESTATE;
    }
    base = g_addr[dev];
  }
  dycg::GroupScratch S{};
  S.temp_bytes = kTemp;
  dycg::group_carve(base, kMax, S);
  const cudaError_t e =
      dycg::group_run(d_records, (uint32_t)n, num_vertices, d_segment_ends, num_segments,
                      d_out_uv, d_out_mult, d_segment_counts, d_counts, S, (cudaStream_t)stream);
  return e == cudaSuccess ? DYCG_OK : DYCG_ECUDA;
}
