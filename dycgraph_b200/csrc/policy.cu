// policy.cu -- learned cache admission: per-page features, a BF16 MLP served
// and trained by the kernels below, and the per-snapshot bookkeeping that
// records access traces.
//
// No reference counterpart: the reference admits rows by a decayed activity
// count (include/framework/variants/driver.cuh:486-515, comp_hotness_sssp),
// which stays here as the hotness policy (cache.cu) and as the yardstick.
//
// Unit: one cache page (2^page_shift adjacency slots). Features per page
// (POLICY_F = 8, BF16):
//   0    log1p(slot reads of the page so far in this snapshot: its mutation)
//   1-2  log1p(slot reads of the page in each of the last two snapshots)
//   3    log1p(decayed read score: score * 0.75 + reads, per snapshot -- the
//        hotness policy's ranking signal)
//   4    log1p(update records of the current batch whose row starts in the
//        page, at the row's place after the mutation)
//   5    min(snapshots since the page was last read, 16) / 16
//   6    log1p(rows starting in the page) / 8
//   7    log1p(longest row starting in the page) / 16
// Target: log1p(slot reads of the page during the current snapshot and the
// next POLICY_HORIZON - 1 ones), so pages rank by near-future value. The
// network is POLICY_F -> 64 -> 64 -> 1, ReLU, BF16 weights and inputs, FP32
// accumulation and FP32 master weights; loss = mean squared error.
//
// The MLP is 4.7K multiply-adds per page. Inference runs every snapshot over
// every page (1.85M pages at R-MAT 27, ~9 GMAC): it runs on the 5th-generation
// tensor cores (tcgen05.mma, 128-page tiles, accumulators in tensor memory),
// where the FP32-FMA version took ~1.2 ms per snapshot. Training (forward,
// backward and the gradient sums over samples) runs on them too.
#include <cuda_bf16.h>

#include <atomic>

#include "common.cuh"
#include "internal.h"

namespace dycg {

namespace {

constexpr int F = POLICY_F, H = POLICY_H;
constexpr int OFF_W1 = 0, OFF_B1 = F * H, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
              OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + H;
static_assert(OFF_B3 + 1 == POLICY_PARAMS, "parameter layout");

__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

int grid_for(u64 threads) {
  u64 b = (threads + BLOCK - 1) / BLOCK;
  if (b < 1) b = 1;
  if (b > 148ull * 32) b = 148ull * 32;
  return (int)b;
}

}  // namespace

// ---- features ----------------------------------------------------------------

// Rows starting in each page and the longest of them (one arena). Rows laid
// out in vertex order share pages, so a warp whose lanes all land in one page
// adds once.
__global__ void page_rows_kernel(const u64 *off, const uint32_t *len, uint32_t n,
                                 uint32_t page_base, uint32_t page_shift, uint32_t *rows,
                                 uint32_t *maxlen, const uint32_t *period) {
  if (period && period[0] % period[1]) return;  // not a refresh snapshot
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t v0 = blockIdx.x * blockDim.x + threadIdx.x - lane; v0 < n;
       v0 += gridDim.x * blockDim.x) {  // warp-uniform
    const uint32_t v = v0 + lane;
    const uint32_t l = v < n ? len[v] : 0;
    const uint32_t p = l ? page_base + (uint32_t)(off[v] >> page_shift) : 0xFFFFFFFFu;
    const uint32_t p0 = __shfl_sync(0xffffffffu, p, 0);
    const bool uni = __all_sync(0xffffffffu, p == p0 || p == 0xFFFFFFFFu) && p0 != 0xFFFFFFFFu;
    if (uni) {
      const unsigned has = __ballot_sync(0xffffffffu, l != 0);
      uint32_t m = l;
      for (int o = 16; o; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
      if (lane == 0) {
        atomicAdd(rows + p0, (uint32_t)__popc(has));
        atomicMax(maxlen + p0, m);
      }
    } else if (l) {
      atomicAdd(rows + p, 1u);
      atomicMax(maxlen + p, l);
    }
  }
}

// Update records per page: each sorted batch key (row << 32 | neighbour) names
// the row it touches in this arena.
__global__ void page_delta_kernel(const u64 *keys, uint32_t cnt, const u64 *off,
                                  uint32_t page_base, uint32_t page_shift, uint32_t *delta) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const u64 k = keys[i];
    if (k == KEY_INF) continue;
    atomicAdd(delta + page_base + (uint32_t)(off[(uint32_t)(k >> 32)] >> page_shift), 1u);
  }
}

__global__ void features_kernel(const uint32_t *hits, const float *hist, const uint8_t *age,
                                const uint32_t *delta, const uint32_t *rows,
                                const uint32_t *maxlen, uint32_t npages, __nv_bfloat16 *x) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npages;
       p += gridDim.x * blockDim.x) {
    float f[F];
    f[0] = log1pf((float)hits[p]);
    f[1] = hist[p];
    f[2] = hist[1ull * npages + p];
    f[3] = log1pf(hist[3ull * npages + p]);
    f[4] = log1pf((float)delta[p]);
    f[5] = fminf((float)age[p], 16.f) / 16.f;
    f[6] = log1pf((float)rows[p]) / 8.f;
    f[7] = log1pf((float)maxlen[p]) / 16.f;
    __align__(16) __nv_bfloat16 o[F];
    for (int k = 0; k < F; k++) o[k] = __float2bfloat16_rn(f[k]);
    *reinterpret_cast<uint4 *>(x + (u64)p * F) = *reinterpret_cast<const uint4 *>(o);
  }
}

// End of a snapshot: shift this snapshot's page reads into the history,
// decay the read score, update ages, add the reads to the raw training
// targets of the traced snapshots whose horizon covers this one (target[j],
// up to POLICY_HORIZON of them), and clear the counters (unless the hotness
// policy still has to read them).
__global__ void history_kernel(uint32_t *hits, float *hist, uint8_t *age, uint32_t npages,
                               TargetRefs tg, bool clear) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npages;
       p += gridDim.x * blockDim.x) {
    const uint32_t h = hits[p];
    hist[2ull * npages + p] = hist[1ull * npages + p];
    hist[1ull * npages + p] = hist[p];
    hist[p] = log1pf((float)h);
    hist[3ull * npages + p] = hist[3ull * npages + p] * 0.75f + (float)h;
    age[p] = h ? 0 : (uint8_t)min(255, age[p] + 1);
    for (int j = 0; j < POLICY_HORIZON; j++)
      if (tg.t[j]) tg.t[j][p] += (float)h;
    if (clear) hits[p] = 0;
  }
}

__global__ void log1p_kernel(const float *in, float *out, u64 n) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    out[i] = log1pf(in[i]);
}

// ---- inference -----------------------------------------------------------------

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // lo in the low half
  return *reinterpret_cast<uint32_t *>(&v);
}

// ---- inference on the 5th-generation tensor cores (tcgen05) ---------------------

// A CTA of 4 warps serves 128 pages per tile: layer 1 and layer 2 are
// tcgen05.mma products (M = 128 pages, N = 64 hidden units, K = 16 per
// instruction, BF16 operands from shared memory, FP32 accumulators in tensor
// memory), issued by one thread; each thread then reads its page's row of
// the accumulator back with tcgen05.ld (warp w owns tensor-memory lanes
// 32w..32w+31) for the bias / ReLU epilogue, the BF16 hi + lo split of the
// layer-1 activations (both parts go through layer 2, so the activations keep
// FP32-level precision: h = hi + lo to ~2^-17 relative, while a single BF16
// rounding missed the float64 oracle's tolerance by 60-190x) and the final
// FP32 dot product. Operands sit in shared
// memory in the no-swizzle K-major layout of 8-row x 16-byte core matrices:
// element (row, k) of an operand with KC chunks of 8 along K lives at
// ((row / 8) * KC + k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2 bytes, so the
// descriptor's leading byte offset (next core matrix along K) is 128 and its
// stride byte offset (next 8 rows) is KC * 128.
namespace tc {
constexpr uint32_t M = 128, N = 64;
constexpr uint32_t SM_A1 = 0;                  // 128 x 16 (KC 2): 4 KB
constexpr uint32_t SM_B1 = SM_A1 + 4096;       // 64 x 16 (KC 2): 2 KB
constexpr uint32_t SM_A2H = SM_B1 + 2048;      // 128 x 64 (KC 8): 16 KB
constexpr uint32_t SM_A2L = SM_A2H + 16384;    // 16 KB
constexpr uint32_t SM_B2 = SM_A2L + 16384;     // 64 x 64 (KC 8): 8 KB
constexpr uint32_t SM_BIAS = SM_B2 + 8192;     // b1, b2, W3 (BF16-rounded, FP32): 768 B
constexpr uint32_t SM_BAR = SM_BIAS + 768;     // mbarrier (8 B) + tensor-memory address (4 B)
constexpr uint32_t SM_BYTES = SM_BAR + 16;
// idesc: D FP32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1), both
// K-major, N >> 3 in bits 17-22, M >> 4 in bits 24-28
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);

__device__ __forceinline__ uint32_t off(uint32_t row, uint32_t k, uint32_t kc) {
  return ((row >> 3) * kc + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2;
}
// shared-memory matrix descriptor: start >> 4 (bits 0-13), leading byte
// offset >> 4 (bits 16-29), stride byte offset >> 4 (bits 32-45), version 1
// (bits 46-47), no swizzle (bits 61-63 = 0)
__device__ __forceinline__ u64 sdesc(uint32_t saddr, uint32_t sbo) {
  return (u64)((saddr >> 4) & 0x3FFF) | ((u64)(128 >> 4) << 16) | ((u64)((sbo >> 4) & 0x3FFF) << 32) |
         (1ull << 46);
}
__device__ __forceinline__ void mma(uint32_t d_tmem, u64 a, u64 b, uint32_t accumulate,
                                    uint32_t idesc = IDESC) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
      :
      : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u));
}
__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(bar)
               : "memory");
}
// bounded wait on the mbarrier's phase; false when the limit ran out
__device__ __forceinline__ bool wait(uint32_t bar, uint32_t phase) {
  const u64 t0 = globaltimer_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
    if (globaltimer_ns() - t0 > 1000000000ull) return false;
  }
}
// 32 FP32 columns of this thread's tensor-memory lane (warp-collective)
__device__ __forceinline__ void ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
      "%28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}
// 64 FP32 columns of this thread's tensor-memory lane, in two 32-column loads
__device__ __forceinline__ void ld64(uint32_t taddr, float (&v)[64]) {
  ld32(taddr, v);
  ld32(taddr + 32, v + 32);
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
}  // namespace tc

__global__ void __launch_bounds__(128, 4) mlp_infer_tc_kernel(const __nv_bfloat16 *x, uint32_t n,
                                                              const float *params, float *score,
                                                              uint32_t *ids, uint32_t *err) {
  extern __shared__ __align__(1024) uint8_t sm_tc[];
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm_tc);
  const uint32_t bar = sbase + tc::SM_BAR;
  uint32_t *taddr_slot = reinterpret_cast<uint32_t *>(sm_tc + tc::SM_BAR + 8);
  // the weights as the B operands (N = hidden unit, K = input), BF16; the
  // padding columns 8..15 of layer 1 are zero; biases and W3 in registers
  for (uint32_t i = tid; i < tc::N * 16; i += blockDim.x) {
    const uint32_t nn = i / 16, k = i % 16;
    const float wv = k < (uint32_t)F ? params[OFF_W1 + k * H + nn] : 0.f;
    *reinterpret_cast<__nv_bfloat16 *>(sm_tc + tc::SM_B1 + tc::off(nn, k, 2)) = __float2bfloat16_rn(wv);
  }
  for (uint32_t i = tid; i < tc::N * (uint32_t)H; i += blockDim.x) {
    const uint32_t nn = i / H, k = i % H;
    *reinterpret_cast<__nv_bfloat16 *>(sm_tc + tc::SM_B2 + tc::off(nn, k, 8)) =
        __float2bfloat16_rn(params[OFF_W2 + k * H + nn]);
  }
  float *bias = reinterpret_cast<float *>(sm_tc + tc::SM_BIAS);  // b1[64], b2[64], W3[64]
  for (uint32_t i = tid; i < 3 * (uint32_t)H; i += blockDim.x)
    bias[i] = bf(params[(i < (uint32_t)H ? OFF_B1 : i < 2u * H ? OFF_B2 - H : OFF_W3 - 2 * H) + i]);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {  // 128 tensor-memory columns: layer 1 in 0..63, layer 2 in 64..127
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" ::"r"(
        sbase + tc::SM_BAR + 8));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *taddr_slot;
  const uint32_t lane_base = (32 * warp) << 16;  // this warp's tensor-memory lanes
  const float b3 = bf(params[OFF_B3]);
  uint32_t phase = 0;
  bool ok = true;
  const uint32_t tiles = (n + tc::M - 1) / tc::M;
  for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    const uint32_t row = tile * tc::M + tid;
    // A1: this page's 8 BF16 features, zero padding to K = 16
    {
      uint4 f = make_uint4(0, 0, 0, 0);
      if (row < n) f = __ldg(reinterpret_cast<const uint4 *>(x) + row);
      *reinterpret_cast<uint4 *>(sm_tc + tc::SM_A1 + tc::off(tid, 0, 2)) = f;
      *reinterpret_cast<uint4 *>(sm_tc + tc::SM_A1 + tc::off(tid, 8, 2)) = make_uint4(0, 0, 0, 0);
    }
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (tid == 0) {
      tc::mma(tmem, tc::sdesc(sbase + tc::SM_A1, 256), tc::sdesc(sbase + tc::SM_B1, 256), 0);
      tc::commit(bar);
    }
    ok = tc::wait(bar, phase);
    phase ^= 1;
    tc::fence_after();
    float v[64];
    tc::ld64(tmem + lane_base, v);
    // layer-1 epilogue: bias, ReLU, BF16 hi + lo parts as the A operands of layer 2
#pragma unroll
    for (int h = 0; h < H; h += 8) {
      uint32_t hw[4], lw[4];
#pragma unroll
      for (int e = 0; e < 8; e += 2) {
        const float a0 = fmaxf(v[h + e] + bias[h + e], 0.f);
        const float a1 = fmaxf(v[h + e + 1] + bias[h + e + 1], 0.f);
        const float h0 = bf(a0), h1 = bf(a1);
        hw[e / 2] = pack2(h0, h1);
        lw[e / 2] = pack2(a0 - h0, a1 - h1);
      }
      *reinterpret_cast<uint4 *>(sm_tc + tc::SM_A2H + tc::off(tid, h, 8)) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
      *reinterpret_cast<uint4 *>(sm_tc + tc::SM_A2L + tc::off(tid, h, 8)) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    }
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (tid == 0 && ok) {
#pragma unroll
      for (uint32_t s = 0; s < (uint32_t)H / 16; s++) {
        const uint32_t kb = s * 256;  // 16 K-elements = two core matrices along K
        tc::mma(tmem + tc::N, tc::sdesc(sbase + tc::SM_A2H + kb, 1024),
                tc::sdesc(sbase + tc::SM_B2 + kb, 1024), s > 0);
        tc::mma(tmem + tc::N, tc::sdesc(sbase + tc::SM_A2L + kb, 1024),
                tc::sdesc(sbase + tc::SM_B2 + kb, 1024), 1);
      }
      tc::commit(bar);
    }
    if (ok) ok = tc::wait(bar, phase);
    phase ^= 1;
    tc::fence_after();
    tc::ld64(tmem + lane_base + tc::N, v);
    float y = 0.f;
#pragma unroll
    for (int h = 0; h < H; h++)
      y = fmaf(fmaxf(v[h] + bias[H + h], 0.f), bias[2 * H + h], y);
    if (row < n) {
      score[row] = y + b3;
      if (ids) ids[row] = row;
    }
    tc::fence_before();
    __syncthreads();  // every lane's reads of the accumulators are done before the next tile
    tc::fence_after();
  }
  if (!ok && err && tid == 0) atomicCAS(err, 0u, ERR_BARRIER);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(tmem));
}

// ---- training on the 5th-generation tensor cores ----------------------------------

// One CTA of 4 warps per SM, 128 samples per tile (thread t = sample t of the
// tile = tensor-memory lane t). Per tile, four tcgen05.mma products with FP32
// accumulators in tensor memory, each followed by a per-thread epilogue:
//   Z1 = X W1             (M 128 samples, N 64, K 16: the 8 features padded)
//   Z2 = H1 W2            (N 64, K 64; H1 as BF16 hi + lo)
//   G1 = dH2 W2^T         (N 64, K 64; dH2 as hi + lo) -> dH1 = G1 * [H1 > 0]
//   G  = A B              (M 128, N 208, K 128 samples), accumulated over the
//                          CTA's tiles, where the rows of A are H1^T (64), X^T
//                          (8), a row of ones and dy^T, and the columns of B are
//                          dH2 (64), dH1 (64), H2 (64) and a column of ones:
//                          G[H1^T][dH2] = dW2, G[X^T][dH1] = dW1,
//                          G[ones][dH2 | dH1] = db2 | db1,
//                          G[dy^T][H2 | ones] = dW3 | db3.
// FP32 operands (activations, gradients) enter as BF16 hi + lo parts, and G
// sums hi*hi + hi*lo + lo*hi, so products keep ~2^-16 relative precision, as
// the FP32 FMA formulation it replaces; X, ones and the BF16-rounded weights
// are exact in BF16. Operand layout and descriptors as in the inference
// kernel (no-swizzle K-major core matrices).
namespace tt {
constexpr uint32_t TS = 128, GN = 208;        // samples per tile; columns of G
constexpr uint32_t KG = TS / 8;                // core-matrix chunks along G's K
constexpr uint32_t SM_A1 = 0;                  // X: 128 x 16 (KC 2), 4 KB
constexpr uint32_t SM_B1 = 4096;               // W1 as [n = hidden][k = feature], 2 KB
constexpr uint32_t SM_AH = SM_B1 + 2048;       // H1, then dH2: 128 x 64 hi (KC 8), 16 KB
constexpr uint32_t SM_AL = SM_AH + 16384;      // ... lo
constexpr uint32_t SM_B2F = SM_AL + 16384;     // W2 as [n = out][k = in], 8 KB
constexpr uint32_t SM_B2B = SM_B2F + 8192;     // W2 as [n = in][k = out], 8 KB
constexpr uint32_t SM_GAH = SM_B2B + 8192;     // A of G: 128 x 128 (KC 16) hi, 32 KB
constexpr uint32_t SM_GAL = SM_GAH + 32768;    // ... lo
constexpr uint32_t SM_GBH = SM_GAL + 32768;    // B of G: 208 x 128 (KC 16) hi, 52 KB
constexpr uint32_t SM_GBL = SM_GBH + GN * TS * 2;  // ... lo
constexpr uint32_t SM_BIAS = SM_GBL + GN * TS * 2;  // b1, b2, W3, b3 (FP32)
constexpr uint32_t SM_BAR = SM_BIAS + 784;     // mbarrier + tensor-memory address
constexpr uint32_t SM_BYTES = SM_BAR + 16;
static_assert(SM_BYTES <= 232448, "shared memory per block");
// rows of A and columns (rows of the K-major B) of G
constexpr uint32_t A_H1 = 0, A_X = 64, A_ONE = 72, A_DY = 73;
constexpr uint32_t B_DH2 = 0, B_DH1 = 64, B_H2 = 128, B_ONE = 192;
// tensor-memory columns: Z1 / G1 in 0..63, Z2 in 64..127, G in 128..335
constexpr uint32_t T_Z1 = 0, T_Z2 = 64, T_G = 128, T_COLS = 512;
constexpr uint32_t ID64 = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
constexpr uint32_t IDG = (1u << 4) | (1u << 7) | (1u << 10) | ((GN >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void put(uint8_t *sm, uint32_t base, uint32_t row, uint32_t k,
                                    uint32_t kc, __nv_bfloat16 v) {
  *reinterpret_cast<__nv_bfloat16 *>(sm + base + tc::off(row, k, kc)) = v;
}
// v as BF16 hi + lo at (row, k) of the hi and lo copies of an operand
__device__ __forceinline__ void put2(uint8_t *sm, uint32_t hi, uint32_t lo, uint32_t row,
                                     uint32_t k, uint32_t kc, float v) {
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  put(sm, hi, row, k, kc, h);
  put(sm, lo, row, k, kc, __float2bfloat16_rn(v - __bfloat162float(h)));
}
// 64 values of this thread's sample as hi + lo rows of a sample-major operand
__device__ __forceinline__ void put_row(uint8_t *sm, uint32_t t, const float (&v)[64]) {
#pragma unroll
  for (int h = 0; h < 64; h += 8) {
    uint32_t hw[4], lw[4];
#pragma unroll
    for (int e = 0; e < 8; e += 2) {
      const float h0 = bf(v[h + e]), h1 = bf(v[h + e + 1]);
      hw[e / 2] = pack2(h0, h1);
      lw[e / 2] = pack2(v[h + e] - h0, v[h + e + 1] - h1);
    }
    *reinterpret_cast<uint4 *>(sm + SM_AH + tc::off(t, h, 8)) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    *reinterpret_cast<uint4 *>(sm + SM_AL + tc::off(t, h, 8)) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
  }
}
// all threads' shared-memory operand writes visible to the tensor core, then
// one thread issues; the caller waits on the mbarrier
__device__ __forceinline__ void publish() {
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
}
}  // namespace tt

// Loss and gradient over samples: sample s of the pass is row idx(s) of x
// (idx = identity, or a seeded draw when sample_seed != 0 and total > 0).
// Gradients (FP32, w.r.t. the BF16-rounded parameters) and the summed squared
// error are added into grad[] and *loss. scale multiplies the gradient
// (2/batch for a mean).
__global__ void __launch_bounds__(128, 1)
    mlp_grad_tc_kernel(const __nv_bfloat16 *x, const float *y, uint64_t total, uint32_t count,
                       uint64_t sample_seed, const float *params, float scale, float *grad,
                       float *loss, uint32_t *err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  const uint32_t t = threadIdx.x, warp = t >> 5;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
  const uint32_t bar = sbase + tt::SM_BAR;
  uint32_t *taddr_slot = reinterpret_cast<uint32_t *>(sm + tt::SM_BAR + 8);
  // operands that do not change: zeros everywhere (padding rows and columns,
  // the lo parts of exact values), the weights, the two rows of ones
  for (uint32_t i = t * 16; i < tt::SM_BIAS; i += 128 * 16)
    *reinterpret_cast<uint4 *>(sm + i) = make_uint4(0, 0, 0, 0);
  __syncthreads();
  for (uint32_t i = t; i < 64 * (uint32_t)F; i += 128) {
    const uint32_t nn = i / F, k = i % F;
    tt::put(sm, tt::SM_B1, nn, k, 2, __float2bfloat16_rn(params[OFF_W1 + k * H + nn]));
  }
  for (uint32_t i = t; i < (uint32_t)(H * H); i += 128) {
    const uint32_t a = i / H, b = i % H;  // W2[a][b]: input a, output b
    const __nv_bfloat16 w = __float2bfloat16_rn(params[OFF_W2 + i]);
    tt::put(sm, tt::SM_B2F, b, a, 8, w);
    tt::put(sm, tt::SM_B2B, a, b, 8, w);
  }
  tt::put(sm, tt::SM_GAH, tt::A_ONE, t, tt::KG, __float2bfloat16_rn(1.f));
  tt::put(sm, tt::SM_GBH, tt::B_ONE, t, tt::KG, __float2bfloat16_rn(1.f));
  float *bias = reinterpret_cast<float *>(sm + tt::SM_BIAS);  // b1[64], b2[64], W3[64], b3
  for (uint32_t i = t; i < 3 * (uint32_t)H; i += 128)
    bias[i] = bf(params[(i < (uint32_t)H ? OFF_B1 : i < 2u * H ? OFF_B2 - H : OFF_W3 - 2 * H) + i]);
  if (t == 0) {
    bias[3 * H] = bf(params[OFF_B3]);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     sbase + tt::SM_BAR + 8),
                 "n"(tt::T_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tt::publish();
  const uint32_t tmem = *taddr_slot;
  const uint32_t lane_base = (32 * warp) << 16;  // this warp's tensor-memory lanes
  const float *b1 = bias, *b2 = bias + H, *w3 = bias + 2 * H;
  const float b3 = bias[3 * H];
  uint32_t phase = 0;
  bool ok = true;
  float lsum = 0.f;
  const uint32_t tiles = (count + tt::TS - 1) / tt::TS;
  uint32_t done = 0;  // tiles this CTA accumulated into G
  for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x, done++) {
    const uint32_t s0 = tile * tt::TS;
    const bool valid = t < min(tt::TS, count - s0);
    // inputs: X row into A1, X^T into G's A, the target
    uint4 xf = make_uint4(0, 0, 0, 0);
    float target = 0.f;
    if (valid) {
      u64 r = s0 + t;
      if (sample_seed) r = mix64(sample_seed ^ mix64(r)) % total;
      xf = __ldg(reinterpret_cast<const uint4 *>(x) + r);
      target = y[r];
    }
    *reinterpret_cast<uint4 *>(sm + tt::SM_A1 + tc::off(t, 0, 2)) = xf;
    {
      const __nv_bfloat16 *xv = reinterpret_cast<const __nv_bfloat16 *>(&xf);
#pragma unroll
      for (int k = 0; k < F; k++) tt::put(sm, tt::SM_GAH, tt::A_X + k, t, tt::KG, xv[k]);
    }
    tt::publish();
    if (t == 0) {
      tc::mma(tmem + tt::T_Z1, tc::sdesc(sbase + tt::SM_A1, 256), tc::sdesc(sbase + tt::SM_B1, 256),
              0, tt::ID64);
      tc::commit(bar);
    }
    ok = tc::wait(bar, phase);
    phase ^= 1;
    tc::fence_after();
    // layer 1: H1 = relu(Z1 + b1), its sign mask, H1 as A of layer 2, H1^T in G's A
    float v[64];
    u64 mask1 = 0;
    tc::ld64(tmem + lane_base + tt::T_Z1, v);
#pragma unroll
    for (int i = 0; i < H; i++) {
      v[i] = fmaxf(v[i] + b1[i], 0.f);
      if (v[i] > 0.f) mask1 |= 1ull << i;
      tt::put2(sm, tt::SM_GAH, tt::SM_GAL, tt::A_H1 + i, t, tt::KG, v[i]);
    }
    tt::put_row(sm, t, v);
    tt::publish();
    if (t == 0 && ok) {
#pragma unroll
      for (uint32_t s = 0; s < (uint32_t)H / 16; s++) {
        const uint32_t kb = s * 256;
        tc::mma(tmem + tt::T_Z2, tc::sdesc(sbase + tt::SM_AH + kb, 1024),
                tc::sdesc(sbase + tt::SM_B2F + kb, 1024), s > 0, tt::ID64);
        tc::mma(tmem + tt::T_Z2, tc::sdesc(sbase + tt::SM_AL + kb, 1024),
                tc::sdesc(sbase + tt::SM_B2F + kb, 1024), 1, tt::ID64);
      }
      tc::commit(bar);
    }
    if (ok) ok = tc::wait(bar, phase);
    phase ^= 1;
    tc::fence_after();
    // layer 2 and output: H2, y, dy; dH2 = dy W3 [H2 > 0]
    tc::ld64(tmem + lane_base + tt::T_Z2, v);
    float out = b3;
#pragma unroll
    for (int j = 0; j < H; j++) {
      v[j] = fmaxf(v[j] + b2[j], 0.f);
      out = fmaf(v[j], w3[j], out);
    }
    const float d = out - target;
    const float dy = valid ? scale * d : 0.f;
    if (valid) lsum = fmaf(d, d, lsum);
    tt::put2(sm, tt::SM_GAH, tt::SM_GAL, tt::A_DY, t, tt::KG, dy);
#pragma unroll
    for (int j = 0; j < H; j++) {
      tt::put2(sm, tt::SM_GBH, tt::SM_GBL, tt::B_H2 + j, t, tt::KG, v[j]);
      v[j] = v[j] > 0.f ? dy * w3[j] : 0.f;
      tt::put2(sm, tt::SM_GBH, tt::SM_GBL, tt::B_DH2 + j, t, tt::KG, v[j]);
    }
    tt::put_row(sm, t, v);  // dH2 as A of G1 (layer 2's MMAs are complete)
    tt::publish();
    if (t == 0 && ok) {
#pragma unroll
      for (uint32_t s = 0; s < (uint32_t)H / 16; s++) {
        const uint32_t kb = s * 256;
        tc::mma(tmem + tt::T_Z1, tc::sdesc(sbase + tt::SM_AH + kb, 1024),
                tc::sdesc(sbase + tt::SM_B2B + kb, 1024), s > 0, tt::ID64);
        tc::mma(tmem + tt::T_Z1, tc::sdesc(sbase + tt::SM_AL + kb, 1024),
                tc::sdesc(sbase + tt::SM_B2B + kb, 1024), 1, tt::ID64);
      }
      tc::commit(bar);
    }
    if (ok) ok = tc::wait(bar, phase);
    phase ^= 1;
    tc::fence_after();
    // dH1 = G1 [H1 > 0] into G's B
    tc::ld64(tmem + lane_base + tt::T_Z1, v);
#pragma unroll
    for (int i = 0; i < H; i++)
      tt::put2(sm, tt::SM_GBH, tt::SM_GBL, tt::B_DH1 + i, t, tt::KG,
               (mask1 >> i) & 1ull ? v[i] : 0.f);
    tt::publish();
    if (t == 0 && ok) {
#pragma unroll
      for (uint32_t s = 0; s < tt::TS / 16; s++) {
        const uint32_t kb = s * 256;
        const u64 ah = tc::sdesc(sbase + tt::SM_GAH + kb, tt::KG * 128);
        const u64 al = tc::sdesc(sbase + tt::SM_GAL + kb, tt::KG * 128);
        const u64 bh = tc::sdesc(sbase + tt::SM_GBH + kb, tt::KG * 128);
        const u64 bl = tc::sdesc(sbase + tt::SM_GBL + kb, tt::KG * 128);
        tc::mma(tmem + tt::T_G, ah, bh, done > 0 || s > 0, tt::IDG);
        tc::mma(tmem + tt::T_G, ah, bl, 1, tt::IDG);
        tc::mma(tmem + tt::T_G, al, bh, 1, tt::IDG);
      }
      tc::commit(bar);
    }
    if (ok) ok = tc::wait(bar, phase);  // the next tile rewrites G's operands
    phase ^= 1;
    tc::fence_after();
  }
  // G's rows to the gradient: warps 0-1 hold dW2, warp 2 dW1, the biases, dW3
  if (ok && done) {
    float g[32];
    if (warp < 2) {
#pragma unroll
      for (uint32_t c = 0; c < 64; c += 32) {
        tc::ld32(tmem + lane_base + tt::T_G + tt::B_DH2 + c, g);
#pragma unroll
        for (int j = 0; j < 32; j++) atomicAdd(grad + OFF_W2 + t * H + c + j, g[j]);
      }
    } else if (warp == 2) {
      for (uint32_t c = 0; c < 224; c += 32) {  // G columns 0..223 (208.. unused)
        tc::ld32(tmem + lane_base + tt::T_G + c, g);
#pragma unroll
        for (int j = 0; j < 32; j++) {
          const uint32_t col = c + j;
          if (t >= tt::A_X && t < tt::A_X + F && col >= tt::B_DH1 && col < tt::B_DH1 + H)
            atomicAdd(grad + OFF_W1 + (t - tt::A_X) * H + (col - tt::B_DH1), g[j]);
          else if (t == tt::A_ONE && col < tt::B_DH1)
            atomicAdd(grad + OFF_B2 + col, g[j]);
          else if (t == tt::A_ONE && col < tt::B_H2)
            atomicAdd(grad + OFF_B1 + (col - tt::B_DH1), g[j]);
          else if (t == tt::A_DY && col >= tt::B_H2 && col < tt::B_ONE)
            atomicAdd(grad + OFF_W3 + (col - tt::B_H2), g[j]);
          else if (t == tt::A_DY && col == tt::B_ONE)
            atomicAdd(grad + OFF_B3, g[j]);
        }
      }
    }
  }
  for (int o = 16; o; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
  if ((t & 31) == 0 && lsum != 0.f) atomicAdd(loss, lsum);
  if (!ok && err && t == 0) atomicCAS(err, 0u, ERR_BARRIER);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "n"(tt::T_COLS));
}

// Adam on the FP32 master parameters; clears the gradient.
__global__ void adam_kernel(float *p, float *g, float *m, float *v, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < POLICY_PARAMS;
       i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    m[i] = b1 * m[i] + (1.f - b1) * gi;
    v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
    p[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
    g[i] = 0.f;
  }
}

// ---- launchers -----------------------------------------------------------------

size_t mlp_grad_smem() { return tt::SM_BYTES; }

// Clears the row-layout features on refresh snapshots (period[0] % period[1]
// == 0); the refresh decision is read on the device so it survives graph
// replay.
__global__ void page_rows_clear_kernel(uint32_t *rows, uint32_t *maxlen, uint32_t npages,
                                       const uint32_t *period) {
  if (period[0] % period[1]) return;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npages;
       p += gridDim.x * blockDim.x) {
    rows[p] = 0;
    maxlen[p] = 0;
  }
}

__global__ void period_step_kernel(uint32_t *period) {
  if (threadIdx.x == 0 && blockIdx.x == 0) period[0]++;
}

cudaError_t launch_page_rows(const u64 *off, const uint32_t *len, uint32_t n, uint32_t page_base,
                             uint32_t page_shift, uint32_t *rows, uint32_t *maxlen,
                             const uint32_t *period, cudaStream_t s) {
  page_rows_kernel<<<grid_for(n), BLOCK, 0, s>>>(off, len, n, page_base, page_shift, rows, maxlen,
                                                 period);
  return cudaGetLastError();
}

cudaError_t launch_page_rows_clear(uint32_t *rows, uint32_t *maxlen, uint32_t npages,
                                   const uint32_t *period, cudaStream_t s) {
  page_rows_clear_kernel<<<grid_for(npages), BLOCK, 0, s>>>(rows, maxlen, npages, period);
  return cudaGetLastError();
}

cudaError_t launch_period_step(uint32_t *period, cudaStream_t s) {
  period_step_kernel<<<1, 32, 0, s>>>(period);
  return cudaGetLastError();
}

cudaError_t launch_page_delta(const u64 *keys, uint32_t cnt, const u64 *off, uint32_t page_base,
                              uint32_t page_shift, uint32_t *delta, cudaStream_t s) {
  if (!cnt) return cudaSuccess;
  page_delta_kernel<<<grid_for(cnt), BLOCK, 0, s>>>(keys, cnt, off, page_base, page_shift, delta);
  return cudaGetLastError();
}

cudaError_t launch_features(const uint32_t *hits, const float *hist, const uint8_t *age,
                            const uint32_t *delta, const uint32_t *rows, const uint32_t *maxlen,
                            uint32_t npages, void *x, cudaStream_t s) {
  features_kernel<<<grid_for(npages), BLOCK, 0, s>>>(hits, hist, age, delta, rows, maxlen, npages,
                                                     (__nv_bfloat16 *)x);
  return cudaGetLastError();
}

cudaError_t launch_history(uint32_t *hits, float *hist, uint8_t *age, uint32_t npages,
                           const TargetRefs &tg, bool clear, cudaStream_t s) {
  history_kernel<<<grid_for(npages), BLOCK, 0, s>>>(hits, hist, age, npages, tg, clear);
  return cudaGetLastError();
}

cudaError_t launch_log1p(const float *in, float *out, u64 n, cudaStream_t s) {
  log1p_kernel<<<grid_for(n), BLOCK, 0, s>>>(in, out, n);
  return cudaGetLastError();
}

cudaError_t launch_mlp_infer(const void *x, uint32_t n, const float *params, float *score,
                             uint32_t *ids, uint32_t *err, cudaStream_t s) {
  if (!n) return cudaSuccess;
  const uint32_t tiles = (n + tc::M - 1) / tc::M;
  // up to 4 CTAs per SM (4 x 128 tensor-memory columns = all 512), so an SM
  // overlaps the MMA and epilogue latencies of four tiles
  const int grid = (int)std::min<uint32_t>(tiles, 148u * 4);
  mlp_infer_tc_kernel<<<grid, 128, tc::SM_BYTES, s>>>((const __nv_bfloat16 *)x, n, params, score,
                                                      ids, err);
  return cudaGetLastError();
}
cudaError_t launch_mlp_grad(const void *x, const float *y, uint64_t total, uint32_t count,
                            uint64_t sample_seed, const float *params, float scale, float *grad,
                            float *loss, uint32_t *err, cudaStream_t s) {
  // the shared-memory opt-in is a per-device setting: once per device used
  constexpr int kMaxDevices = 64;
  static std::atomic<bool> attr[kMaxDevices];
  const size_t smem = mlp_grad_smem();
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices || !attr[dev].load(std::memory_order_acquire)) {
    e = cudaFuncSetAttribute(mlp_grad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < kMaxDevices) attr[dev].store(true, std::memory_order_release);
  }
  if (!count) return cudaSuccess;
  // one CTA per SM (223 KB of shared memory, 512 tensor-memory columns); every
  // CTA gets at least one tile
  const uint32_t tiles = (count + tt::TS - 1) / tt::TS;
  const int grid = (int)std::min<uint32_t>(tiles, 148);
  mlp_grad_tc_kernel<<<grid, 128, smem, s>>>((const __nv_bfloat16 *)x, y, total, count,
                                             sample_seed, params, scale, grad, loss, err);
  return cudaGetLastError();
}

cudaError_t launch_adam(float *p, float *g, float *m, float *v, float lr, uint32_t step,
                        cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  adam_kernel<<<(POLICY_PARAMS + BLOCK - 1) / BLOCK, BLOCK, 0, s>>>(p, g, m, v, lr, b1, b2, 1e-8f,
                                                                    c1, c2);
  return cudaGetLastError();
}

}  // namespace dycg
