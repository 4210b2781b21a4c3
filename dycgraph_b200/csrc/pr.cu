// pr.cu -- signed-residual PageRank on the paged adjacency, one persistent
// cooperative kernel per phase group.
//
// Semantics follow the reference's pr::Runtime (include/framework/pr_residual.cuh):
// unnormalised ranks x = (1-alpha) + alpha * P^T x with dangling mass dropped;
// a vertex is in the frontier while |r| > epsilon (Frontier::Add :21-30);
// Consume (:54-71) moves r into x; Scatter (:74-100) pushes
// alpha * delta / degree along every live occurrence with FP32 atomics. A
// batch changes r by what the reference's two amend passes add up to
// (Engine::UpdatePageRank, framework.cuh:2692-2736: -alpha*x[u]/deg_old(u)
// over the old row of every touched source before the topology changes,
// +alpha*x[u]/deg_new(u) over the new row after), then converges for at most
// max_rounds rounds; unfinished work carries over. The sum is pushed in one
// pass after the mutation: every live occurrence of the new row gets
// alpha*x[u]*(1/deg_new - 1/deg_old), an inserted occurrence another
// alpha*x[u]/deg_old, a deleted one -alpha*x[u]/deg_old. The residuals are
// the same sums (with one rounding instead of two per kept occurrence), but
// a row whose degree did not change pushes nothing, and a kept neighbour gets
// a push ~deg times smaller, so far fewer vertices cross epsilon only to be
// cancelled by the second pass. deg_old is saved per touched source (in the
// delta array, free between snapshots) before the mutation.
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
  const uint2 *del_uv;      // distinct deleted (u, v) pairs and occurrences found
  const uint32_t *del_found;
  const uint32_t *n_del;
  const uint3 *add_uvw;     // inserted occurrences (u >= n: invalid record)
  uint32_t n_add;
  Tiles tiles;
  Ctl *ctl;
  uint32_t n;
  uint32_t cur;             // queue holding the frontier
  uint32_t phases;          // PR_AMEND and/or PR_CONVERGE
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

// Pushes c to UNROLL targets per lane: the atomics first (independent, in
// flight together), then Frontier::Add's crossing test on each result.
template <int U>
__device__ __forceinline__ void push_batch(const PrParams *P, uint32_t *outq, uint32_t *outc,
                                           const uint32_t (&y)[U], const bool (&valid)[U], float c,
                                           Acc &acc) {
  float old[U];
#pragma unroll
  for (int u = 0; u < U; u++) old[u] = valid[u] ? atomicAdd(P->r + y[u], c) : 0.f;
#pragma unroll
  for (int u = 0; u < U; u++) {
    bool want = false;
    if (valid[u]) {
      const float nv = old[u] + c;
      if (!isfinite(nv)) atomicCAS(&P->ctl->err, 0u, ERR_NONFINITE);
      want = fabsf(old[u]) <= P->eps && fabsf(nv) > P->eps &&
             atomicCAS(P->queued + y[u], 0u, 1u) == 0u;
      acc.improved++;
    }
    warp_append(outq, outc, P->n, want, y[u], &P->ctl->err);
  }
}

__device__ __forceinline__ uint32_t old_degree(const PrParams *P, uint32_t u) {
  return __float_as_uint(P->delta[u]);
}

// The kept-occurrence share of the amend over a touched source's new row.
struct AmendOp {
  const PrParams *P;
  uint32_t *outq;
  uint32_t *outc;
  struct Row {
    float c;
  };
  __device__ bool begin(uint32_t u, Row &row) {
    const uint32_t dn = P->out.live[u], dold = old_degree(P, u);
    const float xu = P->x[u];
    if (!dn || dn == dold || xu == 0.f) return false;
    // alpha x (1/dn - 1/dold) = alpha x (dold - dn) / (dn dold), or alpha x / dn
    row.c = dold ? P->alpha * xu * ((float)((int64_t)dold - (int64_t)dn) /
                                    ((float)dn * (float)dold))
                 : P->alpha * xu / (float)dn;
    return row.c != 0.f;
  }
  static constexpr int kBatch = 1;
  template <int U>
  __device__ void edges(uint32_t, const uint32_t (&y)[U], const bool (&valid)[U], Row &row,
                        Acc &acc) {
    push_batch(P, outq, outc, y, valid, row.c, acc);
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
  static constexpr int kBatch = 1;
  template <int U>
  __device__ void edges(uint32_t, const uint32_t (&y)[U], const bool (&valid)[U], Row &row,
                        Acc &acc) {
    push_batch(P, outq, outc, y, valid, row.c, acc);
  }
  __device__ void end(uint32_t, Row &) {}
};

// The per-occurrence shares of the amend: -alpha x[u]/deg_old for each
// deleted occurrence, +alpha x[u]/deg_old for each inserted one (together with
// the row pass that makes it alpha x[u]/deg_new). Appends into q[cur].
__device__ void amend_records(const PrParams &P, uint32_t cur, Acc &acc) {
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t gstride = gridDim.x * blockDim.x;
  uint32_t *q = P.q[cur], *qc = &P.ctl->q_count[cur];
  const uint32_t nd = *P.n_del;
  for (uint32_t i = gtid; i < nd; i += gstride) {
    const uint32_t f = P.del_found[i];
    bool want = false;
    const uint2 e = P.del_uv[i];
    if (f) {
      const uint32_t dold = old_degree(&P, e.x);
      const float xu = P.x[e.x];
      if (dold && xu != 0.f) {
        want = pr_add(&P, e.y, -P.alpha * xu * (float)f / (float)dold);
        acc.improved++;
      }
    }
    warp_append(q, qc, P.n, want, e.y, &P.ctl->err);
  }
  for (uint32_t i = gtid; i < P.n_add; i += gstride) {
    const uint3 e = P.add_uvw[i];
    bool want = false;
    if (e.x < P.n && e.y < P.n) {
      const uint32_t dold = old_degree(&P, e.x);
      const float xu = P.x[e.x];
      if (dold && xu != 0.f) {
        want = pr_add(&P, e.y, P.alpha * xu / (float)dold);
        acc.improved++;
      }
    }
    warp_append(q, qc, P.n, want, e.y, &P.ctl->err);
  }
}

__global__ void __launch_bounds__(BLOCK) pr_kernel(PrParams P) {
  Ctl *ctl = P.ctl;
  Acc acc = {0, 0, 0, 0, 0};
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t gstride = gridDim.x * blockDim.x;
  uint32_t cur = P.cur;
  if (P.phases & PR_AMEND) {
    amend_records(P, cur, acc);
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
  P.del_uv = L.del_uv;
  P.del_found = L.del_found;
  P.n_del = L.n_del;
  P.add_uvw = L.add_uvw;
  P.n_add = L.n_add;
  P.tiles = Tiles{L.tiles, L.tile_cap};
  P.ctl = L.ctl;
  P.n = L.n;
  P.cur = L.cur;
  P.phases = L.phases;
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

// deg_old of every touched source, kept in the delta array until the amend
__global__ void pr_old_degree_kernel(const uint32_t *sources, const uint32_t *n_sources,
                                     const uint32_t *live, float *delta) {
  const uint32_t cnt = *n_sources;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += gridDim.x * blockDim.x) {
    const uint32_t u = sources[i];
    delta[u] = __uint_as_float(live[u]);
  }
}

cudaError_t launch_pr_old_degree(const uint32_t *sources, const uint32_t *n_sources,
                                 uint32_t max_sources, const uint32_t *live, float *delta,
                                 cudaStream_t s) {
  if (!max_sources) return cudaSuccess;
  const int grid = (int)std::min<u64>((max_sources + BLOCK - 1) / BLOCK, 148ull * 16);
  pr_old_degree_kernel<<<grid, BLOCK, 0, s>>>(sources, n_sources, live, delta);
  return cudaGetLastError();
}

cudaError_t launch_pr_init(float *x, float *r, uint32_t *queued, uint32_t *q0, uint32_t n,
                           float base, Ctl *ctl, cudaStream_t s) {
  const int grid = (int)std::min<u64>((n + BLOCK - 1) / BLOCK + 1, 148ull * 16);
  pr_init_kernel<<<grid, BLOCK, 0, s>>>(x, r, queued, q0, n, base, ctl);
  return cudaGetLastError();
}

}  // namespace dycg
