// pr.cu -- signed-residual PageRank on the paged adjacency, one persistent
// cooperative kernel per phase group.
//
// Semantics follow the reference's pr::Runtime (include/framework/pr_residual.cuh):
// unnormalised ranks x = (1-alpha) + alpha * P^T x with dangling mass dropped;
// a vertex is in the frontier while |r| > epsilon (Frontier::Add :21-30);
// Consume (:54-71) moves r into x; Scatter (:74-100) pushes
// alpha * delta / degree along every live occurrence with FP32 atomics. A
// batch amends r by -alpha*x[u]/deg_old(u) over the old rows of the touched
// sources before the topology changes and by +alpha*x[u]/deg_new(u) over the
// new rows after (Engine::UpdatePageRank, framework.cuh:2692-2736), then
// converges for at most max_rounds rounds; unfinished work carries over.
#include "frontier.cuh"
#include "internal.h"

namespace dycg {

struct PrParams {
  Adj out;
  float *x;
  float *r;
  float *delta;
  uint32_t *queued;
  uint32_t *q[2];
  const uint32_t *sources;  // touched sources (amend)
  const uint32_t *n_sources;
  Tiles tiles;
  Ctl *ctl;
  uint32_t n;
  uint32_t cur;             // queue holding the frontier
  uint32_t phases;          // PR_AMEND and/or PR_CONVERGE
  float sign;               // amend sign
  float eps;
  float alpha;
  uint32_t max_rounds;
  u64 timeout_ns;
};

// Frontier::Add: enqueue on crossing epsilon.
__device__ __forceinline__ bool pr_add(const PrParams *P, uint32_t dst, float c) {
  const float old = atomicAdd(P->r + dst, c);
  const float nv = old + c;
  if (!isfinite(nv)) atomicCAS(&P->ctl->err, 0u, ERR_NONFINITE);
  return fabsf(old) <= P->eps && fabsf(nv) > P->eps && atomicCAS(P->queued + dst, 0u, 1u) == 0u;
}

struct AmendOp {
  const PrParams *P;
  uint32_t *outq;
  uint32_t *outc;
  struct Row {
    float c;
  };
  __device__ bool begin(uint32_t u, Row &row) {
    const uint32_t deg = P->out.live[u];
    const float xu = P->x[u];
    if (!deg || xu == 0.f) return false;
    row.c = P->sign * P->alpha * xu / (float)deg;
    return true;
  }
  __device__ void edge(uint32_t, uint32_t y, uint32_t, bool valid, Row &row, Acc &acc) {
    bool want = false;
    if (valid) {
      want = pr_add(P, y, row.c);
      acc.improved++;
    }
    warp_append(outq, outc, P->n, want, y, &P->ctl->err);
  }
  __device__ void end(uint32_t, Row &) {}
};

struct ScatterOp {
  const PrParams *P;
  uint32_t *outq;
  uint32_t *outc;
  struct Row {
    float c;
  };
  __device__ bool begin(uint32_t v, Row &row) {
    const float d = P->delta[v];
    const uint32_t deg = P->out.live[v];
    if (d == 0.f || !deg) return false;
    row.c = P->alpha * d / (float)deg;
    return true;
  }
  __device__ void edge(uint32_t, uint32_t y, uint32_t, bool valid, Row &row, Acc &acc) {
    bool want = false;
    if (valid) {
      want = pr_add(P, y, row.c);
      acc.improved++;
    }
    warp_append(outq, outc, P->n, want, y, &P->ctl->err);
  }
  __device__ void end(uint32_t, Row &) {}
};

__global__ void __launch_bounds__(BLOCK) pr_kernel(PrParams P) {
  Ctl *ctl = P.ctl;
  Acc acc = {0, 0, 0, 0, 0};
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t gstride = gridDim.x * blockDim.x;
  uint32_t cur = P.cur;
  if (P.phases & PR_AMEND) {
    AmendOp op{&P, P.q[cur], &ctl->q_count[cur]};
    if (!expand_rows<false>(P.out, P.sources, *P.n_sources, op, acc, P.tiles, ctl, 0,
                            P.timeout_ns))
      goto done;
  } else {
    if (!grid_sync(ctl, 0, P.timeout_ns)) goto done;
  }
  if (P.phases & PR_CONVERGE) {
    for (uint32_t round = 0; round < P.max_rounds; round++) {
      const uint32_t cnt = *(volatile uint32_t *)&ctl->snap_q[cur];
      if (cnt == 0) break;
      // Consume
      for (uint32_t i = gtid; i < cnt; i += gstride) {
        const uint32_t v = P.q[cur][i];
        const float rv = P.r[v];
        P.queued[v] = 0;
        if (!isfinite(rv) || !isfinite(P.x[v])) atomicCAS(&ctl->err, 0u, ERR_NONFINITE);
        if (fabsf(rv) > P.eps) {
          P.x[v] += rv;
          P.r[v] = 0.f;
          P.delta[v] = rv;
        } else {
          P.delta[v] = 0.f;
        }
      }
      if (!grid_sync(ctl, cur ? SYNC_RESET_Q0 : SYNC_RESET_Q1, P.timeout_ns)) goto done;
      // Scatter
      ScatterOp op{&P, P.q[cur ^ 1], &ctl->q_count[cur ^ 1]};
      if (!expand_rows<false>(P.out, P.q[cur], cnt, op, acc, P.tiles, ctl,
                              cur ? SYNC_RESET_Q1 : SYNC_RESET_Q0, P.timeout_ns))
        goto done;
      cur ^= 1;
      if (gtid == 0) ctl->waves = round + 1;
    }
  }
done:
  acc.flush(ctl);
  if (gtid == 0) {
    ctl->pad[0] = cur;
    ctl->pad[1] = *(volatile uint32_t *)&ctl->q_count[cur];
  }
}

__global__ void pr_init_kernel(float *x, float *r, uint32_t *queued, uint32_t *q0, uint32_t n,
                               float base, Ctl *ctl) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += gridDim.x * blockDim.x) {
    x[v] = 0.f;
    r[v] = base;
    queued[v] = 1;
    q0[v] = v;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->q_count[0] = n;
}

cudaError_t launch_pr(const PrLaunch &L, cudaStream_t s) {
  PrParams P;
  P.out = L.out;
  P.x = L.x;
  P.r = L.r;
  P.delta = L.delta;
  P.queued = L.queued;
  P.q[0] = L.q0;
  P.q[1] = L.q1;
  P.sources = L.sources;
  P.n_sources = L.n_sources;
  P.tiles = Tiles{L.tiles, L.tile_cap};
  P.ctl = L.ctl;
  P.n = L.n;
  P.cur = L.cur;
  P.phases = L.phases;
  P.sign = L.sign;
  P.eps = L.eps;
  P.alpha = L.alpha;
  P.max_rounds = L.max_rounds;
  P.timeout_ns = L.timeout_ns;
  static int blocks_per_sm = -1;
  if (blocks_per_sm < 0) {
    cudaError_t e =
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, pr_kernel, BLOCK, 0);
    if (e != cudaSuccess) return e;
  }
  void *args[] = {&P};
  return cudaLaunchCooperativeKernel((const void *)pr_kernel, blocks_per_sm * L.num_sms, BLOCK,
                                     args, 0, s);
}

cudaError_t launch_pr_init(float *x, float *r, uint32_t *queued, uint32_t *q0, uint32_t n,
                           float base, Ctl *ctl, cudaStream_t s) {
  const int grid = (int)std::min<u64>((n + BLOCK - 1) / BLOCK + 1, 148ull * 16);
  pr_init_kernel<<<grid, BLOCK, 0, s>>>(x, r, queued, q0, n, base, ctl);
  return cudaGetLastError();
}

}  // namespace dycg
