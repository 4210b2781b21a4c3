/*
 * oracle.c -- CPU oracle for the streaming delta-repair path (test
 * infrastructure only; see oracle.h). Parity anchored on the reference's own
 * fixtures and Python oracles (tests/golden), and on the reference's
 * topology_replay tool compiled from its sources (oracle/Makefile).
 *
 * Reference citations are paths inside MriMouse/DyCGraph.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Mutable multigraph rows with the chunk store's occurrence semantics:
 * include/groute/graphs/source_local_chunk_store.h. Each source owns one
 * block of power-of-two capacity; a block that overflows is rewritten to a
 * new block at the arena tail (:823-893). */
typedef struct adj_t {
  uint32_t n;
  uint64_t *off;
  uint32_t *len;
  uint32_t *cap;
  uint32_t *dst;
  uint32_t *w; /* NULL unless weights are stored */
  uint64_t top, arena;
} adj_t;

struct orc {
  uint32_t algo, wmode, source, symmetric;
  double eps, alpha;
  uint32_t max_rounds;
  int threads;
  uint32_t n;
  adj_t out, in;
  uint32_t *val, *par;
  uint8_t *flag; /* reset / queued marks */
  uint32_t *queue;
  double *x, *r;
  uint32_t *pr_front;
  uint64_t pr_count;
  orc_stats st;
};

static uint64_t next_pow2(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

uint32_t orc_rule_weight(uint32_t algo, uint32_t u, uint32_t v) {
  /* include/framework/variants/api.cuh:26-28 (SSSP), BFS weight 1,
   * samples/hybrid_cc/hybrid_cc.cu:66-72 (CC weight 0). */
  if (algo == ORC_BFS) return 1;
  if (algo == ORC_CC) return 0;
  return (uint32_t)(((uint64_t)u + v) % 128 + 1);
}

static inline uint32_t edge_w(const orc *o, const adj_t *a, uint64_t slot,
                              uint32_t u, uint32_t v) {
  if (o->algo == ORC_SSSP && o->wmode == ORC_WEIGHT_STORED) return a->w[slot];
  return orc_rule_weight(o->algo, u, v);
}

static void adj_free(adj_t *a) {
  free(a->off);
  free(a->len);
  free(a->cap);
  free(a->dst);
  free(a->w);
  memset(a, 0, sizeof(*a));
}

static int adj_reserve(adj_t *a, uint64_t need) {
  if (a->top + need <= a->arena) return 0;
  uint64_t ncap = a->arena * 2;
  if (ncap < a->top + need) ncap = a->top + need + (1u << 20);
  uint32_t *nd = (uint32_t *)realloc(a->dst, ncap * sizeof(uint32_t));
  if (!nd) return -1;
  a->dst = nd;
  if (a->w) {
    uint32_t *nw = (uint32_t *)realloc(a->w, ncap * sizeof(uint32_t));
    if (!nw) return -1;
    a->w = nw;
  }
  a->arena = ncap;
  return 0;
}

/* Rows are laid out in vertex order with power-of-two capacities and the
 * reference's +12.5% (min 2^20) headroom (include/framework/framework.cuh:
 * 1657-1668). */
static int adj_build(adj_t *a, uint32_t n, const uint64_t *off, const uint32_t *dst,
                     const uint32_t *w, int store_w) {
  memset(a, 0, sizeof(*a));
  a->n = n;
  a->off = (uint64_t *)malloc(sizeof(uint64_t) * (n + 1ull));
  a->len = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1ull));
  a->cap = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1ull));
  if (!a->off || !a->len || !a->cap) return -1;
  uint64_t total = 0;
  for (uint32_t v = 0; v < n; v++) {
    uint64_t d = off[v + 1] - off[v];
    a->off[v] = total;
    a->len[v] = (uint32_t)d;
    a->cap[v] = d ? (uint32_t)next_pow2(d) : 0;
    total += a->cap[v];
  }
  uint64_t head = total / 8;
  if (head < (1u << 20)) head = 1u << 20;
  a->arena = total + head;
  a->top = total;
  a->dst = (uint32_t *)malloc(sizeof(uint32_t) * a->arena);
  if (!a->dst) return -1;
  if (store_w) {
    a->w = (uint32_t *)malloc(sizeof(uint32_t) * a->arena);
    if (!a->w) return -1;
  }
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t v = 0; v < (int64_t)n; v++) {
    uint64_t d = off[v + 1] - off[v];
    if (!d) continue;
    memcpy(a->dst + a->off[v], dst + off[v], d * sizeof(uint32_t));
    if (store_w) {
      if (w)
        memcpy(a->w + a->off[v], w + off[v], d * sizeof(uint32_t));
      else
        for (uint64_t i = 0; i < d; i++) a->w[a->off[v] + i] = 1;
    }
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Grouped topology mutation: the chunk store's per-source phase
 * (source_local_chunk_store.h:220-406). For every source, each distinct
 * destination requested r times removes its first r live occurrences in slot
 * order (BuildDeletionPlan :685-739); survivors keep their order
 * (CompactSourceInPlace :769-821); additions are appended in request order;
 * a row that outgrows its block moves to a new power-of-two block. */

static int cmp_u64(const void *a, const void *b) {
  uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return x < y ? -1 : x > y;
}

static int cmp_u32(const void *a, const void *b) {
  uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return x < y ? -1 : x > y;
}

typedef struct group_t {
  uint32_t row;
  uint64_t dbeg, dend; /* into sorted delete keys */
  uint64_t abeg, aend; /* into sorted add keys */
} group_t;

/* by_dst: mutate the incoming rows (row = v, neighbour = u). */
static int adj_mutate(orc *o, adj_t *a, const orc_edge *dels, size_t nd,
                      const orc_edge *adds, size_t na, int by_dst,
                      uint64_t *missing, uint64_t *touched, uint64_t *changed,
                      uint8_t *del_ok) {
  uint32_t n = a->n;
  uint64_t *dk = (uint64_t *)malloc(sizeof(uint64_t) * (nd + 1));
  uint64_t *ak = (uint64_t *)malloc(sizeof(uint64_t) * (na + 1));
  if (!dk || !ak) return -1;
  size_t ndv = 0, nav = 0;
  for (size_t i = 0; i < nd; i++) {
    uint32_t r = by_dst ? dels[i].v : dels[i].u;
    if (dels[i].u >= n || dels[i].v >= n) continue;
    dk[ndv++] = ((uint64_t)r << 32) | (uint64_t)i;
  }
  for (size_t i = 0; i < na; i++) {
    uint32_t r = by_dst ? adds[i].v : adds[i].u;
    if (adds[i].u >= n || adds[i].v >= n) continue;
    ak[nav++] = ((uint64_t)r << 32) | (uint64_t)i;
  }
  qsort(dk, ndv, sizeof(uint64_t), cmp_u64);
  qsort(ak, nav, sizeof(uint64_t), cmp_u64);
  /* merge into per-row groups */
  group_t *g = (group_t *)malloc(sizeof(group_t) * (ndv + nav + 1));
  if (!g) return -1;
  size_t ng = 0, i = 0, j = 0;
  while (i < ndv || j < nav) {
    uint32_t ri = i < ndv ? (uint32_t)(dk[i] >> 32) : 0xFFFFFFFFu;
    uint32_t rj = j < nav ? (uint32_t)(ak[j] >> 32) : 0xFFFFFFFFu;
    uint32_t r = ri < rj ? ri : rj;
    group_t gg = {r, i, i, j, j};
    while (i < ndv && (uint32_t)(dk[i] >> 32) == r) i++;
    while (j < nav && (uint32_t)(ak[j] >> 32) == r) j++;
    gg.dend = i;
    gg.aend = j;
    g[ng++] = gg;
  }
  /* capacity for relocations, reserved before the parallel pass */
  uint64_t extra = 0;
  for (size_t k = 0; k < ng; k++) {
    uint64_t fin = (uint64_t)a->len[g[k].row] + (g[k].aend - g[k].abeg);
    if (fin > a->cap[g[k].row]) extra += next_pow2(fin);
  }
  if (adj_reserve(a, extra)) return -1;
  uint64_t miss = 0, chg = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : miss, chg)
  for (int64_t k = 0; k < (int64_t)ng; k++) {
    const group_t *gg = &g[k];
    uint32_t row = gg->row;
    uint64_t base = a->off[row];
    uint32_t deg = a->len[row];
    uint64_t nreq = gg->dend - gg->dbeg;
    uint64_t removed = 0;
    if (nreq) {
      /* requested destinations, sorted, with counts */
      uint32_t *req = (uint32_t *)malloc(sizeof(uint32_t) * nreq);
      uint32_t *cnt = (uint32_t *)calloc(nreq, sizeof(uint32_t));
      uint32_t *got = (uint32_t *)calloc(nreq, sizeof(uint32_t));
      uint8_t *kill = deg ? (uint8_t *)calloc(deg, 1) : NULL;
      for (uint64_t t = 0; t < nreq; t++) {
        const orc_edge *e = &dels[(uint32_t)dk[gg->dbeg + t]];
        req[t] = by_dst ? e->u : e->v;
      }
      qsort(req, nreq, sizeof(uint32_t), cmp_u32);
      uint64_t nu = 0;
      for (uint64_t t = 0; t < nreq; t++) {
        if (nu && req[nu - 1] == req[t]) {
          cnt[nu - 1]++;
        } else {
          req[nu] = req[t];
          cnt[nu] = 1;
          nu++;
        }
      }
      for (uint32_t s = 0; s < deg && removed < nreq; s++) {
        uint32_t d = a->dst[base + s];
        uint64_t lo = 0, hi = nu;
        while (lo < hi) {
          uint64_t mid = (lo + hi) / 2;
          if (req[mid] < d) lo = mid + 1; else hi = mid;
        }
        if (lo < nu && req[lo] == d && got[lo] < cnt[lo]) {
          got[lo]++;
          kill[s] = 1;
          removed++;
        }
      }
      if (removed) {
        uint32_t wpos = 0;
        for (uint32_t s = 0; s < deg; s++) {
          if (kill[s]) continue;
          a->dst[base + wpos] = a->dst[base + s];
          if (a->w) a->w[base + wpos] = a->w[base + s];
          wpos++;
        }
        deg = wpos;
      }
      /* which requests matched: walk the requests in order, hand out the
       * matched counts per destination (request order within the row) */
      if (del_ok) {
        for (uint64_t t = 0; t < nreq; t++) {
          uint32_t idx = (uint32_t)dk[gg->dbeg + t];
          const orc_edge *e = &dels[idx];
          uint32_t d = by_dst ? e->u : e->v;
          uint64_t lo = 0, hi = nu;
          while (lo < hi) {
            uint64_t mid = (lo + hi) / 2;
            if (req[mid] < d) lo = mid + 1; else hi = mid;
          }
          if (got[lo]) {
            got[lo]--;
            del_ok[idx] = 1;
          }
        }
      }
      miss += nreq - removed;
      free(req);
      free(cnt);
      free(got);
      free(kill);
    }
    uint64_t nadd = gg->aend - gg->abeg;
    if (nadd) {
      uint64_t fin = (uint64_t)deg + nadd;
      if (fin > a->cap[row]) {
        uint64_t ncap = next_pow2(fin);
        uint64_t nb = __atomic_fetch_add(&a->top, ncap, __ATOMIC_RELAXED);
        memcpy(a->dst + nb, a->dst + base, (size_t)deg * sizeof(uint32_t));
        if (a->w) memcpy(a->w + nb, a->w + base, (size_t)deg * sizeof(uint32_t));
        a->off[row] = nb;
        a->cap[row] = (uint32_t)ncap;
        base = nb;
      }
      for (uint64_t t = 0; t < nadd; t++) {
        const orc_edge *e = &adds[(uint32_t)ak[gg->abeg + t]];
        a->dst[base + deg] = by_dst ? e->u : e->v;
        if (a->w) a->w[base + deg] = e->w;
        deg++;
      }
    }
    if (removed || nadd) chg++;
    a->len[row] = deg;
  }
  if (missing) *missing = miss;
  if (touched) *touched = ng;
  if (changed) *changed = chg;
  free(dk);
  free(ak);
  free(g);
  return 0;
}

/* ------------------------------------------------------------------------ */

orc *orc_create(uint32_t algo, uint32_t weight_mode, uint32_t source,
                uint32_t symmetric, double epsilon, double alpha,
                uint32_t max_rounds, int threads) {
  orc *o = (orc *)calloc(1, sizeof(orc));
  if (!o) return NULL;
  o->algo = algo;
  o->wmode = weight_mode;
  o->source = source;
  o->symmetric = symmetric;
  o->eps = epsilon;
  o->alpha = alpha;
  o->max_rounds = max_rounds;
  o->threads = threads;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  return o;
}

void orc_destroy(orc *o) {
  if (!o) return;
  adj_free(&o->out);
  adj_free(&o->in);
  free(o->val);
  free(o->par);
  free(o->flag);
  free(o->queue);
  free(o->x);
  free(o->r);
  free(o->pr_front);
  free(o);
}

static int stored(const orc *o) {
  return o->algo == ORC_SSSP && o->wmode == ORC_WEIGHT_STORED;
}

int orc_load_csr(orc *o, uint32_t n, const uint64_t *off, const uint32_t *dst,
                 const uint32_t *w) {
  o->n = n;
  if (adj_build(&o->out, n, off, dst, w, stored(o))) return -1;
  if (!o->symmetric && o->algo != ORC_PR) {
    /* incoming rows: the reference's reverse index
     * (include/framework/dynamic_reverse_index.h:46 Build). */
    uint64_t m = off[n];
    uint64_t *ioff = (uint64_t *)calloc(n + 1ull, sizeof(uint64_t));
    uint32_t *isrc = (uint32_t *)malloc(sizeof(uint32_t) * (m + 1));
    uint32_t *iw = w ? (uint32_t *)malloc(sizeof(uint32_t) * (m + 1)) : NULL;
    if (!ioff || !isrc) return -1;
    for (uint64_t e = 0; e < m; e++) ioff[dst[e] + 1]++;
    for (uint32_t v = 0; v < n; v++) ioff[v + 1] += ioff[v];
    uint64_t *fill = (uint64_t *)malloc(sizeof(uint64_t) * (n + 1ull));
    memcpy(fill, ioff, sizeof(uint64_t) * n);
    for (uint32_t u = 0; u < n; u++)
      for (uint64_t e = off[u]; e < off[u + 1]; e++) {
        uint64_t p = fill[dst[e]]++;
        isrc[p] = u;
        if (iw) iw[p] = w[e];
      }
    int rc = adj_build(&o->in, n, ioff, isrc, iw, stored(o));
    free(ioff);
    free(isrc);
    free(iw);
    free(fill);
    if (rc) return -1;
  }
  o->val = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1ull));
  o->par = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1ull));
  o->flag = (uint8_t *)calloc(n + 1ull, 1);
  o->queue = (uint32_t *)malloc(sizeof(uint32_t) * (n + 2ull));
  if (!o->val || !o->par || !o->flag || !o->queue) return -1;
  if (o->algo == ORC_PR) {
    o->x = (double *)calloc(n + 1ull, sizeof(double));
    o->r = (double *)calloc(n + 1ull, sizeof(double));
    o->pr_front = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1ull));
    if (!o->x || !o->r || !o->pr_front) return -1;
  }
  return 0;
}

static const adj_t *in_rows(const orc *o) {
  return o->symmetric ? &o->out : &o->in;
}

/* ---- SSSP / BFS / CC state ------------------------------------------- */

static uint32_t init_value(const orc *o, uint32_t v) {
  /* reset_affected_values (include/framework/variants/driver.cuh:448-463):
   * CC seeds every vertex with its own id; SSSP/BFS start unreachable. */
  if (o->algo == ORC_CC) return v;
  return ORC_INF;
}

/* FIFO label-correcting closure from the queued vertices: the CPU twin of
 * the insertion closure (include/framework/framework.cuh:5303-5349; the
 * GPU form is RunExactGpuClosure :504-616 with AccumulateBuffer,
 * samples/hybrid_sssp/hybrid_sssp.cu:125-145). flag[] marks queued. */
static void push_closure(orc *o, uint64_t head, uint64_t tail) {
  const adj_t *a = &o->out;
  uint32_t n = o->n;
  uint32_t *q = o->queue;
  while (head != tail) {
    uint32_t x = q[head];
    head = (head + 1) % (n + 1ull);
    o->flag[x] = 0;
    uint32_t dx = o->val[x];
    if (dx == ORC_INF) continue;
    o->st.expanded++;
    uint64_t b = a->off[x];
    for (uint32_t s = 0; s < a->len[x]; s++) {
      uint32_t y = a->dst[b + s];
      uint64_t cand = (uint64_t)dx + edge_w(o, a, b + s, x, y);
      o->st.edges_scanned++;
      if (cand < o->val[y]) {
        o->val[y] = (uint32_t)cand;
        o->par[y] = x;
        if (!o->flag[y]) {
          o->flag[y] = 1;
          q[tail] = y;
          tail = (tail + 1) % (n + 1ull);
        }
      }
    }
  }
}

/* Initial solve (Engine::Start, include/framework/framework.cuh:1963-2005):
 * every vertex at its initial value, the seeds (the source, or every vertex
 * for CC) queued, then the closure. */
static void solve_from_scratch(orc *o) {
  uint32_t n = o->n;
  uint64_t tail = 0;
  memset(o->flag, 0, n);
  for (uint32_t v = 0; v < n; v++) {
    o->val[v] = init_value(o, v);
    o->par[v] = ORC_INF;
  }
  if (o->algo == ORC_CC) {
    uint64_t head = 0;
    /* every vertex is a seed: one pass over all rows, then the closure */
    for (uint32_t x = 0; x < n; x++) {
      uint32_t dx = o->val[x];
      const adj_t *a = &o->out;
      uint64_t b = a->off[x];
      for (uint32_t s = 0; s < a->len[x]; s++) {
        uint32_t y = a->dst[b + s];
        if (dx < o->val[y]) {
          o->val[y] = dx;
          o->par[y] = x;
          if (!o->flag[y]) {
            o->flag[y] = 1;
            o->queue[tail] = y;
            tail = (tail + 1) % (n + 1ull);
          }
        }
      }
    }
    push_closure(o, head, tail);
    return;
  }
  if (o->source < n) {
    o->val[o->source] = 0;
    o->queue[0] = o->source;
    o->flag[o->source] = 1;
    push_closure(o, 0, 1);
  }
}

/* ---- PageRank (include/framework/pr_residual.cuh) --------------------- */

static void pr_add(orc *o, uint32_t dst, double c) {
  /* Frontier::Add (pr_residual.cuh:21-30): enqueue on crossing epsilon. */
  double old = o->r[dst];
  double nv = old + c;
  o->r[dst] = nv;
  if (fabs(old) <= o->eps && fabs(nv) > o->eps && !o->flag[dst]) {
    o->flag[dst] = 1;
    o->pr_front[o->pr_count++] = dst;
  }
}

static void pr_scatter(orc *o, uint32_t src, double value) {
  /* Scatter (pr_residual.cuh:74-100): alpha * value / degree per occurrence. */
  const adj_t *a = &o->out;
  uint32_t deg = a->len[src];
  if (!deg || value == 0) return;
  double c = o->alpha * value / deg;
  uint64_t b = a->off[src];
  o->st.expanded++;
  for (uint32_t s = 0; s < deg; s++) {
    pr_add(o, a->dst[b + s], c);
    o->st.edges_scanned++;
  }
}

static void pr_converge(orc *o) {
  /* Runtime::Converge (pr_residual.cuh:171-187): Consume then Scatter per
   * round, at most max_rounds rounds; unfinished work carries over. */
  uint32_t *cur = (uint32_t *)malloc(sizeof(uint32_t) * (o->n + 1ull));
  double *delta = (double *)malloc(sizeof(double) * (o->n + 1ull));
  uint32_t rounds = 0;
  while (o->pr_count && rounds < o->max_rounds) {
    uint64_t cnt = o->pr_count;
    memcpy(cur, o->pr_front, cnt * sizeof(uint32_t));
    o->pr_count = 0;
    for (uint64_t i = 0; i < cnt; i++) {
      uint32_t v = cur[i];
      double r = o->r[v];
      o->flag[v] = 0;
      delta[i] = 0;
      if (fabs(r) > o->eps) {
        o->x[v] += r;
        o->r[v] = 0;
        delta[i] = r;
      }
    }
    for (uint64_t i = 0; i < cnt; i++)
      if (delta[i] != 0) pr_scatter(o, cur[i], delta[i]);
    rounds++;
  }
  o->st.pr_rounds += rounds;
  free(cur);
  free(delta);
}

int orc_init(orc *o) {
  memset(&o->st, 0, sizeof(o->st));
  if (o->algo == ORC_PR) {
    /* Initialize (pr_residual.cuh:44-53): x = 0, r = 0.15, all queued. */
    for (uint32_t v = 0; v < o->n; v++) {
      o->x[v] = 0;
      o->r[v] = 1.0 - o->alpha;
      o->flag[v] = 1;
      o->pr_front[v] = v;
    }
    o->pr_count = o->n;
    pr_converge(o);
    return 0;
  }
  solve_from_scratch(o);
  return 0;
}

int orc_set_state(orc *o, const uint32_t *values, const uint32_t *parents,
                  const double *ranks, const double *residuals) {
  uint32_t n = o->n;
  if (o->algo == ORC_PR) {
    if (ranks) memcpy(o->x, ranks, sizeof(double) * n);
    if (residuals) memcpy(o->r, residuals, sizeof(double) * n);
    o->pr_count = 0;
    memset(o->flag, 0, n);
    for (uint32_t v = 0; v < n; v++)
      if (fabs(o->r[v]) > o->eps) {
        o->flag[v] = 1;
        o->pr_front[o->pr_count++] = v;
      }
    return 0;
  }
  if (values) memcpy(o->val, values, sizeof(uint32_t) * n);
  if (parents) memcpy(o->par, parents, sizeof(uint32_t) * n);
  return 0;
}

/* Weight of the first live occurrence of (u,v), for stored weights. */
static uint32_t lookup_w(const orc *o, uint32_t u, uint32_t v, int *found) {
  const adj_t *a = &o->out;
  uint64_t b = a->off[u];
  for (uint32_t s = 0; s < a->len[u]; s++)
    if (a->dst[b + s] == v) {
      *found = 1;
      return edge_w(o, a, b + s, u, v);
    }
  *found = 0;
  return stored(o) ? 1 : orc_rule_weight(o->algo, u, v);
}

/* IsDeletionDependency: SSSP/BFS default rule
 * (include/framework/variants/api.cuh:42-49), CC rule
 * (samples/hybrid_cc/hybrid_cc.cu:60-63). */
static int is_dependency(const orc *o, uint32_t src, uint32_t dst, uint32_t w) {
  uint32_t sv = o->val[src], dv = o->val[dst];
  if (o->algo == ORC_CC) return src != dst && sv == dv && dv < dst;
  uint64_t cand = (uint64_t)sv + w;
  uint32_t p = o->par[dst];
  int tight = 0;
  if (p != ORC_INF && o->val[p] != ORC_INF) {
    int f;
    uint32_t pw = lookup_w(o, p, dst, &f);
    tight = (uint64_t)o->val[p] + pw == (uint64_t)dv;
  }
  return p == src || (sv != ORC_INF && cand == (uint64_t)dv && !tight);
}

/* Deletion phase: reset_del_edges (driver.cuh:401-441), the invalidation
 * closure over the pre-deletion rows (framework.cuh:4890-4913 with
 * PushFunctorDB_Del, push_functor.h:1180-1213), reset_affected_values
 * (driver.cuh:448-463), the topology deletion (framework.cuh:2572), then
 * the pull repair until no change (CPU twin framework.cuh:3975-4022 of
 * GpuAffectedPullRelax :189-263, loop :4313-4353). */
static int delete_phase(orc *o, const orc_edge *dels, size_t nd) {
  uint32_t n = o->n;
  uint64_t na = 0; /* affected count, stored in queue[0..na) */
  memset(o->flag, 0, n);
  for (size_t i = 0; i < nd; i++) {
    uint32_t u = dels[i].u, v = dels[i].v;
    if (u >= n || v >= n) continue;
    int f;
    uint32_t w = lookup_w(o, u, v, &f);
    if (!is_dependency(o, u, v, w)) continue;
    if (o->flag[v]) continue;
    if (o->algo != ORC_CC && v == o->source) continue;
    o->flag[v] = 1;
    o->par[v] = ORC_INF;
    o->queue[na++] = v;
  }
  for (uint64_t h = 0; h < na; h++) {
    uint32_t x = o->queue[h];
    const adj_t *a = &o->out;
    uint64_t b = a->off[x];
    o->st.expanded++;
    for (uint32_t s = 0; s < a->len[x]; s++) {
      uint32_t y = a->dst[b + s];
      o->st.edges_scanned++;
      if (o->flag[y]) continue;
      if (o->algo != ORC_CC && y == o->source) continue;
      if (!is_dependency(o, x, y, edge_w(o, a, b + s, x, y))) continue;
      o->flag[y] = 1;
      o->par[y] = ORC_INF;
      o->queue[na++] = y;
    }
  }
  o->st.affected += na;
  for (uint64_t h = 0; h < na; h++) {
    uint32_t v = o->queue[h];
    o->val[v] = init_value(o, v);
    o->par[v] = ORC_INF;
  }
  uint64_t miss = 0, touched = 0, changed = 0;
  if (adj_mutate(o, &o->out, dels, nd, NULL, 0, 0, &miss, &touched, &changed, NULL))
    return -1;
  if (!o->symmetric && adj_mutate(o, &o->in, dels, nd, NULL, 0, 1, NULL, NULL, NULL, NULL))
    return -1;
  o->st.missing_deletes += miss;
  o->st.touched_sources += touched;
  o->st.changed_sources += changed;
  const adj_t *in = in_rows(o);
  for (;;) {
    uint64_t changes = 0;
    o->st.pull_iterations++;
    for (uint64_t h = 0; h < na; h++) {
      uint32_t v = o->queue[h];
      uint32_t best = o->val[v];
      uint32_t bp = o->par[v];
      uint64_t b = in->off[v];
      for (uint32_t s = 0; s < in->len[v]; s++) {
        uint32_t x = in->dst[b + s];
        uint32_t xv = o->val[x];
        o->st.edges_scanned++;
        if (xv == ORC_INF) continue;
        uint64_t cand = (uint64_t)xv + edge_w(o, in, b + s, x, v);
        if (cand < best || (cand == best && (bp == ORC_INF || x < bp))) {
          best = (uint32_t)cand;
          bp = x;
        }
      }
      if (best < o->val[v]) changes++;
      if (bp != ORC_INF && best <= o->val[v]) {
        o->val[v] = best;
        o->par[v] = bp;
      }
    }
    if (!changes) break;
    if (o->st.pull_iterations > (uint64_t)na + 2) return -2;
  }
  memset(o->flag, 0, n);
  return 0;
}

/* Insertion phase: topology addition (framework.cuh:2549-2570), seeds
 * (SeedAddedEdgeFrontier :297-370), then the closure (:3706-3709). */
static int insert_phase(orc *o, const orc_edge *adds, size_t na) {
  uint32_t n = o->n;
  uint64_t touched = 0, changed = 0;
  if (adj_mutate(o, &o->out, NULL, 0, adds, na, 0, NULL, &touched, &changed, NULL))
    return -1;
  if (!o->symmetric && adj_mutate(o, &o->in, NULL, 0, adds, na, 1, NULL, NULL, NULL, NULL))
    return -1;
  o->st.touched_sources += touched;
  o->st.changed_sources += changed;
  memset(o->flag, 0, n);
  uint64_t tail = 0;
  for (size_t i = 0; i < na; i++) {
    uint32_t u = adds[i].u, v = adds[i].v;
    if (u >= n || v >= n) continue;
    if (o->val[u] == ORC_INF) continue;
    uint32_t w = stored(o) ? adds[i].w : orc_rule_weight(o->algo, u, v);
    uint64_t cand = (uint64_t)o->val[u] + w;
    if (cand < o->val[v]) {
      o->val[v] = (uint32_t)cand;
      o->par[v] = u;
      if (!o->flag[v]) {
        o->flag[v] = 1;
        o->queue[tail] = v;
        tail = (tail + 1) % (n + 1ull);
      }
    }
  }
  push_closure(o, 0, tail);
  return 0;
}

/* Records with an endpoint outside [0, n): the replay tool rejects such
 * additions and counts them (src/topology_replay.cpp:165-167); here both
 * phases drop and count them. */
static uint64_t count_invalid(const orc *o, const orc_edge *e, size_t k) {
  uint64_t c = 0;
  for (size_t i = 0; i < k; i++) c += (e[i].u >= o->n || e[i].v >= o->n);
  return c;
}

/* PR batch: Engine::UpdatePageRank (include/framework/framework.cuh:
 * 2692-2736): Amend(-1) on the old rows of touched sources, mutate,
 * Amend(+1) on the new rows, Converge. */
static int pr_batch(orc *o, const orc_edge *dels, size_t nd, const orc_edge *adds,
                    size_t na) {
  uint32_t n = o->n;
  uint32_t *src = (uint32_t *)malloc(sizeof(uint32_t) * (nd + na + 1));
  size_t ns = 0;
  for (size_t i = 0; i < nd; i++)
    if (dels[i].u < n && dels[i].v < n) src[ns++] = dels[i].u;
  for (size_t i = 0; i < na; i++)
    if (adds[i].u < n && adds[i].v < n) src[ns++] = adds[i].u;
  qsort(src, ns, sizeof(uint32_t), cmp_u32);
  size_t nu = 0;
  for (size_t i = 0; i < ns; i++)
    if (!nu || src[nu - 1] != src[i]) src[nu++] = src[i];
  for (size_t i = 0; i < nu; i++) pr_scatter(o, src[i], -o->x[src[i]]);
  uint64_t miss = 0, touched = 0, changed = 0;
  if (adj_mutate(o, &o->out, dels, nd, adds, na, 0, &miss, &touched, &changed, NULL))
    return -1;
  o->st.missing_deletes += miss;
  o->st.touched_sources += touched;
  o->st.changed_sources += changed;
  for (size_t i = 0; i < nu; i++) pr_scatter(o, src[i], o->x[src[i]]);
  free(src);
  pr_converge(o);
  return 0;
}

int orc_delete_edges(orc *o, const orc_edge *dels, size_t nd) {
  memset(&o->st, 0, sizeof(o->st));
  o->st.invalid_updates = count_invalid(o, dels, nd);
  if (o->algo == ORC_PR) return pr_batch(o, dels, nd, NULL, 0);
  return delete_phase(o, dels, nd);
}

int orc_insert_edges(orc *o, const orc_edge *adds, size_t na) {
  memset(&o->st, 0, sizeof(o->st));
  o->st.invalid_updates = count_invalid(o, adds, na);
  if (o->algo == ORC_PR) return pr_batch(o, NULL, 0, adds, na);
  return insert_phase(o, adds, na);
}

int orc_apply_batch(orc *o, const orc_edge *dels, size_t nd, const orc_edge *adds,
                    size_t na) {
  memset(&o->st, 0, sizeof(o->st));
  o->st.invalid_updates = count_invalid(o, dels, nd) + count_invalid(o, adds, na);
  if (o->algo == ORC_PR) return pr_batch(o, dels, nd, adds, na);
  orc_stats keep;
  if (delete_phase(o, dels, nd)) return -1;
  keep = o->st;
  if (insert_phase(o, adds, na)) return -1;
  (void)keep;
  return 0;
}

int orc_mutate(orc *o, const orc_edge *dels, size_t nd, const orc_edge *adds,
               size_t na) {
  memset(&o->st, 0, sizeof(o->st));
  o->st.invalid_updates = count_invalid(o, dels, nd) + count_invalid(o, adds, na);
  uint64_t miss = 0, touched = 0, changed = 0;
  if (adj_mutate(o, &o->out, dels, nd, adds, na, 0, &miss, &touched, &changed, NULL))
    return -1;
  if (o->in.n && adj_mutate(o, &o->in, dels, nd, adds, na, 1, NULL, NULL, NULL, NULL))
    return -1;
  o->st.missing_deletes = miss;
  o->st.touched_sources = touched;
  o->st.changed_sources = changed;
  return 0;
}

int orc_values(const orc *o, uint32_t *values, uint32_t *parents) {
  if (values) memcpy(values, o->val, sizeof(uint32_t) * o->n);
  if (parents) memcpy(parents, o->par, sizeof(uint32_t) * o->n);
  return 0;
}

int orc_ranks(const orc *o, double *ranks, double *residuals) {
  if (o->algo != ORC_PR) return -1;
  if (ranks) memcpy(ranks, o->x, sizeof(double) * o->n);
  if (residuals) memcpy(residuals, o->r, sizeof(double) * o->n);
  return 0;
}

void orc_last_stats(const orc *o, orc_stats *s) { *s = o->st; }
uint64_t orc_nodes(const orc *o) { return o->n; }

uint64_t orc_live_edges(const orc *o) {
  uint64_t m = 0;
  for (uint32_t v = 0; v < o->n; v++) m += o->out.len[v];
  return m;
}

int orc_export_csr(const orc *o, uint64_t *off, uint32_t *dst, uint32_t *w) {
  const adj_t *a = &o->out;
  uint64_t p = 0;
  for (uint32_t v = 0; v < o->n; v++) {
    off[v] = p;
    uint64_t b = a->off[v];
    for (uint32_t s = 0; s < a->len[v]; s++, p++) {
      if (dst) dst[p] = a->dst[b + s];
      if (w) w[p] = a->w ? a->w[b + s] : orc_rule_weight(o->algo, v, a->dst[b + s]);
    }
  }
  off[o->n] = p;
  return 0;
}

uint64_t orc_row_degree(const orc *o, uint32_t v) { return v < o->n ? o->out.len[v] : 0; }

/* HashSequence over the sorted row (include/framework/topology_replay.h:46-66). */
uint64_t orc_row_multiset_hash(const orc *o, uint32_t v) {
  uint32_t d = o->out.len[v];
  uint32_t *tmp = (uint32_t *)malloc(sizeof(uint32_t) * (d + 1));
  memcpy(tmp, o->out.dst + o->out.off[v], sizeof(uint32_t) * d);
  qsort(tmp, d, sizeof(uint32_t), cmp_u32);
  uint64_t h = 1469598103934665603ULL;
  for (uint32_t i = 0; i < d; i++) {
    h ^= (uint64_t)tmp[i];
    h *= 1099511628211ULL;
  }
  h ^= (uint64_t)d;
  h *= 1099511628211ULL;
  free(tmp);
  return h;
}

/* ------------------------------------------------------------------------ */
/* From-scratch static recomputes. */

typedef struct heap_t {
  uint64_t *k;
  size_t n, cap;
} heap_t;

static void heap_push(heap_t *h, uint64_t key) {
  if (h->n == h->cap) {
    h->cap = h->cap ? h->cap * 2 : 1024;
    h->k = (uint64_t *)realloc(h->k, h->cap * sizeof(uint64_t));
  }
  size_t i = h->n++;
  h->k[i] = key;
  while (i) {
    size_t p = (i - 1) / 2;
    if (h->k[p] <= h->k[i]) break;
    uint64_t t = h->k[p];
    h->k[p] = h->k[i];
    h->k[i] = t;
    i = p;
  }
}

static uint64_t heap_pop(heap_t *h) {
  uint64_t top = h->k[0];
  h->k[0] = h->k[--h->n];
  size_t i = 0;
  for (;;) {
    size_t l = 2 * i + 1, r = l + 1, s = i;
    if (l < h->n && h->k[l] < h->k[s]) s = l;
    if (r < h->n && h->k[r] < h->k[s]) s = r;
    if (s == i) break;
    uint64_t t = h->k[s];
    h->k[s] = h->k[i];
    h->k[i] = t;
    i = s;
  }
  return top;
}

/* Dijkstra with (distance << 32 | vertex) heap keys; distances that reach
 * 2^32 - 1 are treated as unreachable (the reference's 32-bit state). */
int orc_static_sssp(uint32_t n, const uint64_t *off, const uint32_t *dst,
                    const uint32_t *w, uint32_t weight_mode, uint32_t source,
                    uint32_t *dist) {
  for (uint32_t v = 0; v < n; v++) dist[v] = ORC_INF;
  if (source >= n) return 0;
  heap_t h = {0, 0, 0};
  dist[source] = 0;
  heap_push(&h, (uint64_t)source);
  while (h.n) {
    uint64_t k = heap_pop(&h);
    uint32_t u = (uint32_t)k, du = (uint32_t)(k >> 32);
    if (du != dist[u]) continue;
    for (uint64_t e = off[u]; e < off[u + 1]; e++) {
      uint32_t v = dst[e];
      uint32_t wt = weight_mode == ORC_WEIGHT_STORED ? w[e]
                                                      : orc_rule_weight(ORC_SSSP, u, v);
      uint64_t c = (uint64_t)du + wt;
      if (c < dist[v]) {
        dist[v] = (uint32_t)c;
        heap_push(&h, (c << 32) | v);
      }
    }
  }
  free(h.k);
  return 0;
}

/* FIFO BFS levels from source (the from-scratch oracle of
 * tests/bfs_dynamic_smoke.py:16-40, its unweighted branch :33-40). */
int orc_static_bfs(uint32_t n, const uint64_t *off, const uint32_t *dst,
                   uint32_t source, uint32_t *level) {
  for (uint32_t v = 0; v < n; v++) level[v] = ORC_INF;
  if (source >= n) return 0;
  uint32_t *q = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1ull));
  uint64_t head = 0, tail = 0;
  level[source] = 0;
  q[tail++] = source;
  while (head < tail) {
    uint32_t u = q[head++];
    for (uint64_t e = off[u]; e < off[u + 1]; e++) {
      uint32_t v = dst[e];
      if (level[v] == ORC_INF) {
        level[v] = level[u] + 1;
        q[tail++] = v;
      }
    }
  }
  free(q);
  return 0;
}

/* Directed min-label: every vertex gets the smallest id that reaches it
 * (flood from starts in increasing id order, as tests/cc_dynamic_smoke.py's
 * oracle does). */
int orc_static_cc(uint32_t n, const uint64_t *off, const uint32_t *dst,
                  uint32_t *label) {
  uint8_t *seen = (uint8_t *)calloc(n + 1ull, 1);
  uint32_t *st = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1ull));
  for (uint32_t s = 0; s < n; s++) {
    if (seen[s]) continue;
    uint64_t top = 0;
    st[top++] = s;
    seen[s] = 1;
    while (top) {
      uint32_t u = st[--top];
      label[u] = s;
      for (uint64_t e = off[u]; e < off[u + 1]; e++) {
        uint32_t v = dst[e];
        if (!seen[v]) {
          seen[v] = 1;
          st[top++] = v;
        }
      }
    }
  }
  free(seen);
  free(st);
  return 0;
}

/* FP64 Jacobi power iteration x = (1-alpha) + alpha * P^T x, dangling mass
 * dropped, multiplicity counted (tests/pr_dynamic_smoke.py oracle,
 * samples/hybrid_pr/hybrid_pr_host.cu:15-33). Stops when the L1 change is
 * below n * tol. Returns the iteration count, or -1 without convergence. */
int orc_static_pr(uint32_t n, const uint64_t *off, const uint32_t *dst,
                  double alpha, double tol, uint32_t max_iter, double *x) {
  double *y = (double *)malloc(sizeof(double) * (n + 1ull));
  for (uint32_t v = 0; v < n; v++) x[v] = 0;
  for (uint32_t it = 1; it <= max_iter; it++) {
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)n; v++) y[v] = 1.0 - alpha;
    for (uint32_t u = 0; u < n; u++) {
      uint64_t d = off[u + 1] - off[u];
      if (!d) continue;
      double c = alpha * x[u] / (double)d;
      for (uint64_t e = off[u]; e < off[u + 1]; e++) y[dst[e]] += c;
    }
    double diff = 0;
    for (uint32_t v = 0; v < n; v++) diff += fabs(x[v] - y[v]);
    memcpy(x, y, sizeof(double) * n);
    if (diff < (double)n * tol) {
      free(y);
      return (int)it;
    }
  }
  free(y);
  return -1;
}

uint64_t orc_bellman_check(uint32_t n, const uint64_t *off, const uint32_t *dst,
                           const uint32_t *w, uint32_t algo, uint32_t weight_mode,
                           uint32_t source, const uint32_t *dist,
                           uint64_t *missing) {
  /* CheckBellmanRelaxed (samples/hybrid_sssp/hybrid_sssp.cu:228-281). */
  uint8_t *tight = (uint8_t *)calloc(n + 1ull, 1);
  if (algo != ORC_CC && source < n) tight[source] = 1;
  uint64_t relax = 0;
  for (uint32_t u = 0; u < n; u++) {
    if (algo == ORC_CC) tight[u] |= dist[u] == u;
    if (dist[u] == ORC_INF) continue;
    for (uint64_t e = off[u]; e < off[u + 1]; e++) {
      uint32_t v = dst[e];
      uint32_t wt = (algo == ORC_SSSP && weight_mode == ORC_WEIGHT_STORED)
                        ? w[e]
                        : orc_rule_weight(algo, u, v);
      uint64_t c = (uint64_t)dist[u] + wt;
      if (dist[v] != ORC_INF && c == dist[v]) tight[v] = 1;
      if (c < dist[v]) relax++;
    }
  }
  uint64_t miss = 0;
  for (uint32_t v = 0; v < n; v++)
    if (dist[v] != ORC_INF && !tight[v]) miss++;
  if (missing) *missing = miss;
  free(tight);
  return relax;
}

/* DistanceChecksum (samples/hybrid_sssp/hybrid_sssp.cu:335-347): FNV-style
 * fold over the reachable vertices. */
uint64_t orc_distance_checksum(const uint32_t *values, uint32_t n) {
  uint64_t c = 1469598103934665603ull;
  for (uint32_t v = 0; v < n; v++) {
    if (values[v] == ORC_INF) continue;
    c ^= (uint64_t)v + 0x9e3779b97f4a7c15ull + ((uint64_t)values[v] << 6) +
         ((uint64_t)values[v] >> 2);
    c *= 1099511628211ull;
  }
  return c;
}
