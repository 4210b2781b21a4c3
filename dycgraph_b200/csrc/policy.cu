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
// every page (1.85M pages at R-MAT 27, ~9 GMAC): it runs on the tensor cores
// (mma.sync BF16 tiles of 16 pages), where the FP32-FMA version took ~1.2 ms
// per snapshot. Training runs once per trained network on FP32 FMA tiles.
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

// Parameters into shared memory, BF16-rounded (the precision the MLP runs at).
__device__ __forceinline__ void load_params(const float *p, float *s) {
  for (int i = threadIdx.x; i < POLICY_PARAMS; i += blockDim.x) s[i] = bf(p[i]);
  __syncthreads();
}

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

// Tensor-core fragments (mma.sync, BF16 operands, FP32 accumulation). In a
// warp, g = lane / 4 and t = lane % 4; a 16 x K A fragment holds rows g and
// g + 8, columns 2t, 2t + 1 (and 2t + 8, 2t + 9 for K = 16); a K x 8 B
// fragment holds rows 2t, 2t + 1 (and 2t + 8, 2t + 9) of column g; the 16 x 8
// FP32 accumulator holds rows g and g + 8, columns 2t and 2t + 1.
__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // lo in the low half
  return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ void mma_k8(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t b0) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(b0));
}

__device__ __forceinline__ void mma_k16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                        uint32_t b1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

constexpr int IB = 128;  // inference block: 4 warps

// score[p] = MLP(x[p]); ids[p] = p (for the admission sort). A warp runs 16
// pages per tile: layer 1 as eight m16n8k8 products (K = the 8 features),
// layer 2 as m16n8k16 products over the 64 hidden units, layer 3 as an FP32
// dot product reduced over each lane quad. The first layer's FP32 outputs are
// split into BF16 hi + lo parts (h = hi + lo to ~2^-17 relative) and both parts
// go through layer 2, so activations keep FP32-level precision while the
// operands stay BF16; the weight fragments live in registers for the whole
// kernel.
__global__ void __launch_bounds__(IB, 3) mlp_infer_kernel(const __nv_bfloat16 *x, uint32_t n,
                                                          const float *params, float *score,
                                                          uint32_t *ids) {
  __shared__ __align__(16) float w[POLICY_PARAMS];
  load_params(params, w);
  const uint32_t lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  uint32_t b1f[8];
#pragma unroll
  for (int j = 0; j < 8; j++)
    b1f[j] = pack2(w[OFF_W1 + (2 * t) * H + 8 * j + g], w[OFF_W1 + (2 * t + 1) * H + 8 * j + g]);
  uint32_t b2f[4][8][2];
#pragma unroll
  for (int kk = 0; kk < 4; kk++)
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int k0 = 16 * kk + 2 * t, c = OFF_W2 + 8 * j + g;
      b2f[kk][j][0] = pack2(w[c + k0 * H], w[c + (k0 + 1) * H]);
      b2f[kk][j][1] = pack2(w[c + (k0 + 8) * H], w[c + (k0 + 9) * H]);
    }
  const float b3 = w[OFF_B3];
  const uint32_t *xw = reinterpret_cast<const uint32_t *>(x);  // F = 8 BF16 = 4 words per page
  const uint32_t tiles = (n + 15) / 16;
  const uint32_t nwarps = gridDim.x * (IB / 32);
  uint32_t tile = (blockIdx.x * IB + threadIdx.x) >> 5;
  auto load_row = [&](uint32_t r) { return r < n ? __ldg(xw + (u64)r * 4 + t) : 0u; };
  uint32_t na0 = load_row(tile * 16 + g), na1 = load_row(tile * 16 + g + 8);
  for (; tile < tiles; tile += nwarps) {
    const uint32_t a0 = na0, a1 = na1;
    const uint32_t r0 = tile * 16 + g, r1 = r0 + 8;
    if (tile + nwarps < tiles) {  // next tile's inputs in flight during this one
      na0 = load_row(r0 + nwarps * 16);
      na1 = load_row(r1 + nwarps * 16);
    }
    float c2[8][4];
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const float2 b = *reinterpret_cast<const float2 *>(&w[OFF_B2 + 8 * j + 2 * t]);
      c2[j][0] = b.x, c2[j][1] = b.y, c2[j][2] = b.x, c2[j][3] = b.y;
    }
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
      // hidden units 16kk .. 16kk+15 of layer 1 = the A fragment of layer 2
      uint32_t hi[4], lo[4];
#pragma unroll
      for (int half = 0; half < 2; half++) {
        const int j1 = 2 * kk + half;
        const float2 b = *reinterpret_cast<const float2 *>(&w[OFF_B1 + 8 * j1 + 2 * t]);
        float c[4] = {b.x, b.y, b.x, b.y};
        mma_k8(c, a0, a1, b1f[j1]);
        float h[4], r[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const float v = fmaxf(c[e], 0.f);
          h[e] = bf(v);
          r[e] = v - h[e];  // exact in FP32
        }
        hi[2 * half] = pack2(h[0], h[1]);
        hi[2 * half + 1] = pack2(h[2], h[3]);
        lo[2 * half] = pack2(r[0], r[1]);
        lo[2 * half + 1] = pack2(r[2], r[3]);
      }
#pragma unroll
      for (int j = 0; j < 8; j++) {
        mma_k16(c2[j], hi, b2f[kk][j][0], b2f[kk][j][1]);
        mma_k16(c2[j], lo, b2f[kk][j][0], b2f[kk][j][1]);
      }
    }
    float y0 = 0.f, y1 = 0.f;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const float2 w3 = *reinterpret_cast<const float2 *>(&w[OFF_W3 + 8 * j + 2 * t]);
      y0 = fmaf(fmaxf(c2[j][0], 0.f), w3.x, y0);
      y0 = fmaf(fmaxf(c2[j][1], 0.f), w3.y, y0);
      y1 = fmaf(fmaxf(c2[j][2], 0.f), w3.x, y1);
      y1 = fmaf(fmaxf(c2[j][3], 0.f), w3.y, y1);
    }
    y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
    y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
    y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
    y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
    if (t == 0) {
      if (r0 < n) score[r0] = y0 + b3;
      if (r1 < n) score[r1] = y1 + b3;
    }
    if (ids && lane < 16 && tile * 16 + lane < n) ids[tile * 16 + lane] = tile * 16 + lane;
  }
}

// ---- training ------------------------------------------------------------------

constexpr int TS = 128;     // samples per tile
constexpr int HP = H + 1;   // padded activation row (bank-conflict free)

// Loss and gradient over samples: sample s of the pass is row idx(s) of x
// (idx = identity, or a seeded draw when sample_seed != 0 and total > 0).
// Gradients (FP32, w.r.t. the BF16-rounded parameters) and the summed squared
// error are added into grad[] and *loss. scale multiplies the gradient
// (2/batch for a mean).
__global__ void __launch_bounds__(BLOCK) mlp_grad_kernel(const __nv_bfloat16 *x, const float *y,
                                                         uint64_t total, uint32_t count,
                                                         uint64_t sample_seed, const float *params,
                                                         float scale, float *grad, float *loss) {
  extern __shared__ float sm[];
  float *w = sm;                          // POLICY_PARAMS
  float *X = w + POLICY_PARAMS;           // TS x F
  float *A1 = X + TS * F;                 // TS x HP: H1, then dH1
  float *A2 = A1 + TS * HP;               // TS x HP: H2, then dH2
  float *T = A2 + TS * HP;                // TS: target, then dy
  load_params(params, w);
  const int t = threadIdx.x;
  float gW2[H * H / BLOCK] = {}, gW1[F * H / BLOCK] = {};
  float gb1 = 0, gb2 = 0, gW3 = 0, gb3 = 0, lsum = 0;
  const uint32_t tiles = (count + TS - 1) / TS;
  for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const uint32_t s0 = tile * TS;
    const int ns = (int)min((uint32_t)TS, count - s0);
    // load inputs and targets
    for (int e = t; e < TS * F; e += BLOCK) {
      const int s = e / F, k = e % F;
      float v = 0.f;
      if (s < ns) {
        u64 r = s0 + s;
        if (sample_seed) r = mix64(sample_seed ^ mix64(r)) % total;
        v = __bfloat162float(x[r * F + k]);
        if (k == 0) T[s] = y[r];
      }
      X[s * F + k] = v;
    }
    __syncthreads();
    // H1 = relu(X W1 + b1)
    for (int e = t; e < TS * H; e += BLOCK) {
      const int s = e / H, i = e % H;
      float a = w[OFF_B1 + i];
#pragma unroll
      for (int k = 0; k < F; k++) a = fmaf(X[s * F + k], w[OFF_W1 + k * H + i], a);
      A1[s * HP + i] = fmaxf(a, 0.f);
    }
    __syncthreads();
    // H2 = relu(H1 W2 + b2)
    for (int e = t; e < TS * H; e += BLOCK) {
      const int s = e / H, j = e % H;
      float a = w[OFF_B2 + j];
      for (int i = 0; i < H; i++) a = fmaf(A1[s * HP + i], w[OFF_W2 + i * H + j], a);
      A2[s * HP + j] = fmaxf(a, 0.f);
    }
    __syncthreads();
    // y = H2 W3 + b3; dy = scale * (y - target)
    if (t < TS) {
      float d = 0.f;
      if (t < ns) {
        float a = w[OFF_B3];
        for (int j = 0; j < H; j++) a = fmaf(A2[t * HP + j], w[OFF_W3 + j], a);
        d = a - T[t];
        lsum += d * d;
      }
      T[t] = scale * d;
    }
    __syncthreads();
    // gW3, gb3 (need H2), then dH2 in place
    if (t < H) {
      float a = 0.f;
      for (int s = 0; s < ns; s++) a = fmaf(A2[s * HP + t], T[s], a);
      gW3 += a;
    }
    if (t == 0)
      for (int s = 0; s < ns; s++) gb3 += T[s];
    __syncthreads();
    for (int e = t; e < TS * H; e += BLOCK) {
      const int s = e / H, j = e % H;
      A2[s * HP + j] = A2[s * HP + j] > 0.f ? T[s] * w[OFF_W3 + j] : 0.f;
    }
    __syncthreads();
    // gW2[i][j] += sum_s H1[s][i] dH2[s][j]; gb2[j] += sum_s dH2[s][j]
#pragma unroll
    for (int r = 0; r < H * H / BLOCK; r++) {
      const int e = t + r * BLOCK, i = e / H, j = e % H;
      float a = 0.f;
      for (int s = 0; s < ns; s++) a = fmaf(A1[s * HP + i], A2[s * HP + j], a);
      gW2[r] += a;
    }
    if (t < H) {
      float a = 0.f;
      for (int s = 0; s < ns; s++) a += A2[s * HP + t];
      gb2 += a;
    }
    __syncthreads();
    // dH1 = mask(H1) * (dH2 W2^T), in place
    for (int e = t; e < TS * H; e += BLOCK) {
      const int s = e / H, i = e % H;
      float a = 0.f;
      if (A1[s * HP + i] > 0.f)
        for (int j = 0; j < H; j++) a = fmaf(A2[s * HP + j], w[OFF_W2 + i * H + j], a);
      A1[s * HP + i] = a;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < F * H / BLOCK; r++) {
      const int e = t + r * BLOCK, k = e / H, i = e % H;
      float a = 0.f;
      for (int s = 0; s < ns; s++) a = fmaf(X[s * F + k], A1[s * HP + i], a);
      gW1[r] += a;
    }
    if (t < H) {
      float a = 0.f;
      for (int s = 0; s < ns; s++) a += A1[s * HP + t];
      gb1 += a;
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < H * H / BLOCK; r++) atomicAdd(grad + OFF_W2 + t + r * BLOCK, gW2[r]);
#pragma unroll
  for (int r = 0; r < F * H / BLOCK; r++) atomicAdd(grad + OFF_W1 + t + r * BLOCK, gW1[r]);
  if (t < H) {
    atomicAdd(grad + OFF_B1 + t, gb1);
    atomicAdd(grad + OFF_B2 + t, gb2);
    atomicAdd(grad + OFF_W3 + t, gW3);
  }
  if (t == 0) atomicAdd(grad + OFF_B3, gb3);
  for (int o = 16; o; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
  if ((t & 31) == 0 && lsum != 0.f) atomicAdd(loss, lsum);
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

size_t mlp_grad_smem() {
  return sizeof(float) * (POLICY_PARAMS + TS * F + 2 * TS * HP + TS);
}

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
                             uint32_t *ids, cudaStream_t s) {
  const u64 warps = ((u64)n + 15) / 16;
  const int grid = (int)std::max<u64>(1, std::min<u64>((warps + 3) / 4, 148ull * 3));
  mlp_infer_kernel<<<grid, IB, 0, s>>>((const __nv_bfloat16 *)x, n, params, score, ids);
  return cudaGetLastError();
}

cudaError_t launch_mlp_grad(const void *x, const float *y, uint64_t total, uint32_t count,
                            uint64_t sample_seed, const float *params, float scale, float *grad,
                            float *loss, cudaStream_t s) {
  // the shared-memory opt-in is a per-device setting: once per device used
  constexpr int kMaxDevices = 64;
  static std::atomic<bool> attr[kMaxDevices];
  const size_t smem = mlp_grad_smem();
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices || !attr[dev].load(std::memory_order_acquire)) {
    e = cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < kMaxDevices) attr[dev].store(true, std::memory_order_release);
  }
  const uint32_t tiles = (count + TS - 1) / TS;
  const int grid = (int)std::max<uint32_t>(1, std::min<uint32_t>(tiles, 148 * 2));
  mlp_grad_kernel<<<grid, BLOCK, smem, s>>>((const __nv_bfloat16 *)x, y, total, count,
                                            sample_seed, params, scale, grad, loss);
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
