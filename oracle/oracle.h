/*
 * oracle.h -- CPU oracle for the streaming delta-repair path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker: the parity tests,
 * the smoke entry and the CPU-baseline leg of the benchmark call it; the
 * product path (libdycg) never links, loads or calls it.
 *
 * Two independent references live here:
 *  1. A restatement of the reference engine's per-snapshot repair
 *     (MriMouse/DyCGraph): chunk-store mutation semantics, deletion seeding,
 *     dependency invalidation, pull repair, insertion closure and signed
 *     residual PageRank. Each function cites the reference file:line it
 *     follows.
 *  2. From-scratch static recomputes of every result (Dijkstra, FIFO BFS,
 *     directed min-label flood, FP64 Jacobi PageRank) and the reference's
 *     checksums, used to check 1. and the GPU engine.
 */
#ifndef DYCG_ORACLE_H
#define DYCG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_SSSP 0
#define ORC_BFS 1
#define ORC_CC 2
#define ORC_PR 3

#define ORC_WEIGHT_HASH128 0
#define ORC_WEIGHT_STORED 1

#define ORC_INF 0xFFFFFFFFu

typedef struct orc_edge {
  uint32_t u, v, w;
} orc_edge;

typedef struct orc_stats {
  uint64_t missing_deletes;
  uint64_t invalid_updates;
  uint64_t touched_sources;
  uint64_t changed_sources;
  uint64_t affected;
  uint64_t pull_iterations;
  uint64_t expanded;
  uint64_t edges_scanned;
  uint64_t pr_rounds;
} orc_stats;

typedef struct orc orc;

orc *orc_create(uint32_t algo, uint32_t weight_mode, uint32_t source,
                uint32_t symmetric, double epsilon, double alpha,
                uint32_t max_rounds, int threads);
void orc_destroy(orc *o);
int orc_load_csr(orc *o, uint32_t n, const uint64_t *off, const uint32_t *dst,
                 const uint32_t *w);
/* Static solve of the initial graph (Dijkstra / BFS / min-label flood /
 * residual PageRank from r = 0.15). */
int orc_init(orc *o);
/* Import a result state instead of solving (values/parents or ranks/residuals). */
int orc_set_state(orc *o, const uint32_t *values, const uint32_t *parents,
                  const double *ranks, const double *residuals);

int orc_delete_edges(orc *o, const orc_edge *dels, size_t nd);
int orc_insert_edges(orc *o, const orc_edge *adds, size_t na);
int orc_apply_batch(orc *o, const orc_edge *dels, size_t nd,
                    const orc_edge *adds, size_t na);
/* Topology only (no result repair), all deletes then all adds. */
int orc_mutate(orc *o, const orc_edge *dels, size_t nd, const orc_edge *adds,
               size_t na);

int orc_values(const orc *o, uint32_t *values, uint32_t *parents);
int orc_ranks(const orc *o, double *ranks, double *residuals);
void orc_last_stats(const orc *o, orc_stats *s);
uint64_t orc_nodes(const orc *o);
uint64_t orc_live_edges(const orc *o);
/* Live outgoing adjacency as CSR (offsets n+1; dst/w live_edges entries). */
int orc_export_csr(const orc *o, uint64_t *off, uint32_t *dst, uint32_t *w);
/* Live degree and multiset hash (FNV over sorted destinations) of a row. */
uint64_t orc_row_degree(const orc *o, uint32_t v);
uint64_t orc_row_multiset_hash(const orc *o, uint32_t v);

/* ---- static recomputes (graph given as CSR) ---------------------------- */
int orc_static_sssp(uint32_t n, const uint64_t *off, const uint32_t *dst,
                    const uint32_t *w, uint32_t weight_mode, uint32_t source,
                    uint32_t *dist);
int orc_static_bfs(uint32_t n, const uint64_t *off, const uint32_t *dst,
                   uint32_t source, uint32_t *level);
int orc_static_cc(uint32_t n, const uint64_t *off, const uint32_t *dst,
                  uint32_t *label);
int orc_static_pr(uint32_t n, const uint64_t *off, const uint32_t *dst,
                  double alpha, double tol, uint32_t max_iter, double *x);

/* Bellman relaxation check of a distance vector against a CSR: returns the
 * number of relaxable edges; *missing gets vertices with no tight witness. */
uint64_t orc_bellman_check(uint32_t n, const uint64_t *off, const uint32_t *dst,
                           const uint32_t *w, uint32_t algo, uint32_t weight_mode,
                           uint32_t source, const uint32_t *dist,
                           uint64_t *missing);

/* ---- workload synthesis for the CPU side of the benchmark (gen.c) ------- */
void orc_gen_rmat_edges(uint32_t scale, double a, double b, double c, uint64_t seed,
                        uint64_t first, uint64_t count, uint32_t wlo, uint32_t whi,
                        orc_edge *out);
int orc_rmat_csr(uint32_t scale, uint32_t ef, double a, double b, double c, uint64_t seed,
                 uint32_t wlo, uint32_t whi, int with_w, int symmetrize, uint64_t **off,
                 uint32_t **dst,
                 uint32_t **w, uint64_t *m);
void orc_free(void *p);
int orc_parallel_sssp(uint32_t n, const uint64_t *off, const uint32_t *dst, const uint32_t *w,
                      uint32_t algo, uint32_t weight_mode, uint32_t source, uint32_t *dist,
                      uint32_t *parent);

/* samples/hybrid_sssp/hybrid_sssp.cu:335-347 (DistanceChecksum). */
uint64_t orc_distance_checksum(const uint32_t *values, uint32_t n);

/* Weight of (u,v): HASH128 rule, unit for BFS, zero for CC. */
uint32_t orc_rule_weight(uint32_t algo, uint32_t u, uint32_t v);

#ifdef __cplusplus
}
#endif
#endif
