// waitcheck.cu -- failure detection of the persistent kernels' bounded waits,
// exercised without a GPU fault: a cooperative launch in which one block
// never arrives at the grid barrier (it waits, bounded, on a flag that nothing
// sets), so every other block's barrier wait runs out, records ERR_BARRIER and
// returns; the host reads the status, and a second launch on the same context
// in which every block arrives must complete cleanly.
#include <cuda_runtime.h>

#include "../../include/dycg.h"
#include "frontier.cuh"

namespace dycg {

__global__ void wait_check_kernel(Ctl *ctl, const uint32_t *never, int absent, u64 limit_ns) {
  if (absent && blockIdx.x == 0) {
    // the absent block: a bounded wait on a flag that nothing sets
    if (threadIdx.x == 0) {
      const u64 t0 = globaltimer_ns();
      while (*(volatile const uint32_t *)never == 0u && globaltimer_ns() - t0 < limit_ns)
        __nanosleep(1000);
    }
    return;
  }
  grid_sync(ctl, 0, limit_ns);
}

}  // namespace dycg

extern "C" int dycg_check_bounded_wait(int device, uint32_t limit_ms, uint32_t *status_absent,
                                       uint32_t *status_all) {
  if (!status_absent || !status_all || limit_ms == 0 || limit_ms > 10000) return DYCG_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) return DYCG_ENOGPU;
  dycg::Ctl *ctl = nullptr;
  uint32_t *never = nullptr;
  int rc = DYCG_OK;
  if (cudaMalloc(&ctl, sizeof(dycg::Ctl)) != cudaSuccess ||
      cudaMalloc(&never, sizeof(uint32_t)) != cudaSuccess) {
    rc = DYCG_ENOMEM;
  } else {
    const dycg::u64 limit_ns = (dycg::u64)limit_ms * 1000000ull;
    uint32_t *out[2] = {status_absent, status_all};
    for (int absent = 1; absent >= 0 && rc == DYCG_OK; absent--) {
      // 8 co-resident blocks (cooperative launch), a fresh control block
      if (cudaMemset(ctl, 0, sizeof(dycg::Ctl)) != cudaSuccess ||
          cudaMemset(never, 0, sizeof(uint32_t)) != cudaSuccess) {
        rc = DYCG_ECUDA;
        break;
      }
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(8);
      cfg.blockDim = dim3(128);
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeCooperative;
      attr[0].val.cooperative = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      const dycg::Ctl *cc = ctl;
      if (cudaLaunchKernelEx(&cfg, dycg::wait_check_kernel, ctl, (const uint32_t *)never, absent,
                             limit_ns) != cudaSuccess ||
          cudaDeviceSynchronize() != cudaSuccess ||
          cudaMemcpy(out[1 - absent], &cc->err, sizeof(uint32_t), cudaMemcpyDeviceToHost) !=
              cudaSuccess)
        rc = DYCG_ECUDA;
    }
  }
  if (ctl) cudaFree(ctl);
  if (never) cudaFree(never);
  return rc;
}
