/*
 * gen.c -- CPU workload synthesis for the oracle side of the benchmark (test
 * infrastructure only): the same counter-based R-MAT draws and seeded edge
 * weights as the GPU loader (restated here so the CPU reference needs no GPU
 * code), a two-pass parallel CSR build, and a parallel label-correcting
 * static solve used only to set up large cases.
 */
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"

typedef unsigned long long u64;

/* SplitMix64 finalizer (Steele, Lea, Flood 2014). */
static inline u64 mix64(u64 z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static inline uint32_t hash_weight(u64 seed, uint32_t u, uint32_t v, uint32_t lo, uint32_t hi) {
  u64 r = mix64(seed ^ mix64(((u64)u << 32) | v));
  return lo + (uint32_t)(r % (u64)(hi - lo + 1));
}

static inline void rmat_draw(u64 seed, u64 idx, uint32_t scale, uint32_t ta, uint32_t tab,
                             uint32_t tabc, uint32_t *u, uint32_t *v) {
  uint32_t uu = 0, vv = 0;
  for (uint32_t level = 0; level < scale; level += 3) {
    u64 r = mix64(seed ^ mix64(idx * 0x9E3779B97F4A7C15ull + level + 1));
    for (uint32_t j = 0; j < 3 && level + j < scale; j++) {
      uint32_t x = (uint32_t)(r >> (21 * j)) & ((1u << 21) - 1);
      uint32_t bu = x >= tab;
      uint32_t bv = (x >= ta && x < tab) || x >= tabc;
      uu = (uu << 1) | bu;
      vv = (vv << 1) | bv;
    }
  }
  *u = uu;
  *v = vv;
}

#define WSEED_SALT 0x5745494748545321ull

void orc_gen_rmat_edges(uint32_t scale, double a, double b, double c, uint64_t seed,
                        uint64_t first, uint64_t count, uint32_t wlo, uint32_t whi,
                        orc_edge *out) {
  const double S = (double)(1u << 21);
  const uint32_t ta = (uint32_t)(a * S), tab = (uint32_t)((a + b) * S),
                 tabc = (uint32_t)((a + b + c) * S);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)count; i++) {
    uint32_t u, v;
    rmat_draw(seed, first + (u64)i, scale, ta, tab, tabc, &u, &v);
    out[i].u = u;
    out[i].v = v;
    out[i].w = hash_weight(seed ^ WSEED_SALT, u, v, wlo, whi);
  }
}

static int cmp_u32(const void *x, const void *y) {
  uint32_t a = *(const uint32_t *)x, b = *(const uint32_t *)y;
  return a < b ? -1 : a > b;
}

/* De-duplicated R-MAT CSR without self-loops, rows sorted; with symmetrize,
 * every draw (u, v) also yields (v, u) (the library's symmetrised R-MAT).
 * Arrays are malloc'd; release with orc_free. Returns 0 on success. */
int orc_rmat_csr(uint32_t scale, uint32_t ef, double a, double b, double c, uint64_t seed,
                 uint32_t wlo, uint32_t whi, int with_w, int symmetrize, uint64_t **off_out,
                 uint32_t **dst_out, uint32_t **w_out, uint64_t *m_out) {
  const uint32_t n = 1u << scale;
  const u64 draws = (u64)ef << scale;
  const double S = (double)(1u << 21);
  const uint32_t ta = (uint32_t)(a * S), tab = (uint32_t)((a + b) * S),
                 tabc = (uint32_t)((a + b + c) * S);
  uint32_t *deg = (uint32_t *)calloc(n + 1ull, sizeof(uint32_t));
  uint64_t *off = (uint64_t *)malloc(sizeof(uint64_t) * (n + 1ull));
  if (!deg || !off) return -1;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)draws; i++) {
    uint32_t u, v;
    rmat_draw(seed, (u64)i, scale, ta, tab, tabc, &u, &v);
    if (u != v) {
      __atomic_fetch_add(&deg[u], 1u, __ATOMIC_RELAXED);
      if (symmetrize) __atomic_fetch_add(&deg[v], 1u, __ATOMIC_RELAXED);
    }
  }
  u64 s = 0;
  for (uint32_t v = 0; v < n; v++) {
    off[v] = s;
    s += deg[v];
  }
  off[n] = s;
  uint32_t *dst = (uint32_t *)malloc(sizeof(uint32_t) * (s + 1));
  uint64_t *cur = (uint64_t *)malloc(sizeof(uint64_t) * (n + 1ull));
  if (!dst || !cur) return -1;
  memcpy(cur, off, sizeof(uint64_t) * n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)draws; i++) {
    uint32_t u, v;
    rmat_draw(seed, (u64)i, scale, ta, tab, tabc, &u, &v);
    if (u != v) {
      dst[__atomic_fetch_add(&cur[u], 1ull, __ATOMIC_RELAXED)] = v;
      if (symmetrize) dst[__atomic_fetch_add(&cur[v], 1ull, __ATOMIC_RELAXED)] = u;
    }
  }
  free(cur);
  /* sort + unique each row in place */
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < (int64_t)n; v++) {
    uint32_t *row = dst + off[v];
    uint32_t d = deg[v];
    if (d > 1) qsort(row, d, sizeof(uint32_t), cmp_u32);
    uint32_t k = 0;
    for (uint32_t i = 0; i < d; i++)
      if (!k || row[k - 1] != row[i]) row[k++] = row[i];
    deg[v] = k;
  }
  /* compact */
  uint64_t *noff = (uint64_t *)malloc(sizeof(uint64_t) * (n + 1ull));
  s = 0;
  for (uint32_t v = 0; v < n; v++) {
    noff[v] = s;
    s += deg[v];
  }
  noff[n] = s;
  uint32_t *ndst = (uint32_t *)malloc(sizeof(uint32_t) * (s + 1));
  uint32_t *nw = with_w ? (uint32_t *)malloc(sizeof(uint32_t) * (s + 1)) : NULL;
  if (!noff || !ndst || (with_w && !nw)) return -1;
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < (int64_t)n; v++) {
    memcpy(ndst + noff[v], dst + off[v], sizeof(uint32_t) * deg[v]);
    if (nw)
      for (uint32_t i = 0; i < deg[v]; i++)
        nw[noff[v] + i] = hash_weight(seed ^ WSEED_SALT, (uint32_t)v, ndst[noff[v] + i], wlo, whi);
  }
  free(dst);
  free(off);
  free(deg);
  *off_out = noff;
  *dst_out = ndst;
  *w_out = nw;
  *m_out = s;
  return 0;
}

void orc_free(void *p) { free(p); }

/* Parallel label-correcting SSSP/BFS (frontier waves, 64-bit CAS-min on
 * (distance << 32 | parent + 1)): set-up of large cases only. */
int orc_parallel_sssp(uint32_t n, const uint64_t *off, const uint32_t *dst, const uint32_t *w,
                      uint32_t algo, uint32_t weight_mode, uint32_t source, uint32_t *dist,
                      uint32_t *parent) {
  u64 *key = (u64 *)malloc(sizeof(u64) * (n + 1ull));
  uint32_t *fr = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1ull));
  uint32_t *nx = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1ull));
  uint32_t *tag = (uint32_t *)calloc(n + 1ull, sizeof(uint32_t));
  if (!key || !fr || !nx || !tag) return -1;
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)n; v++) key[v] = ~0ull;
  if (source >= n) goto out;
  key[source] = 0;
  fr[0] = source;
  u64 fc = 1;
  uint32_t wave = 0;
  while (fc) {
    wave++;
    u64 nc = 0;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)fc; i++) {
      const uint32_t x = fr[i];
      const uint32_t dx = (uint32_t)(__atomic_load_n(&key[x], __ATOMIC_RELAXED) >> 32);
      for (uint64_t e = off[x]; e < off[x + 1]; e++) {
        const uint32_t y = dst[e];
        uint32_t wt = 1;
        if (algo == ORC_SSSP)
          wt = weight_mode == ORC_WEIGHT_STORED ? w[e] : (uint32_t)(((u64)x + y) % 128 + 1);
        const u64 c = (u64)dx + wt;
        if (c >= 0xFFFFFFFFull) continue;
        const u64 cand = (c << 32) | (x + 1u);
        u64 old = __atomic_load_n(&key[y], __ATOMIC_RELAXED);
        int lowered = 0;
        while (cand < old) {
          if (__atomic_compare_exchange_n(&key[y], &old, cand, 0, __ATOMIC_RELAXED,
                                          __ATOMIC_RELAXED)) {
            lowered = (old >> 32) > c;
            break;
          }
        }
        if (lowered && __atomic_exchange_n(&tag[y], wave, __ATOMIC_RELAXED) != wave) {
          u64 p = __atomic_fetch_add(&nc, 1ull, __ATOMIC_RELAXED);
          nx[p] = y;
        }
      }
    }
    uint32_t *t = fr;
    fr = nx;
    nx = t;
    fc = nc;
  }
out:
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)n; v++) {
    const u64 k = key[v];
    dist[v] = (uint32_t)(k >> 32);
    parent[v] = (dist[v] == 0xFFFFFFFFu || (uint32_t)k == 0) ? 0xFFFFFFFFu : (uint32_t)k - 1;
  }
  free(key);
  free(fr);
  free(nx);
  free(tag);
  return 0;
}
