/*
 * dycg.h -- C ABI of the B200 streaming delta-repair engine.
 *
 * One engine handle owns one graph (a paged adjacency held in pinned, mapped
 * host memory, with an HBM page cache capped by a byte budget), the per-vertex
 * results of one algorithm (SSSP, BFS, directed min-label CC or PageRank) and
 * the CUDA stream everything runs on. After every snapshot of edge deletions
 * and insertions the engine repairs the results incrementally on the GPU.
 *
 * Conventions
 *  - Every function returns an int status: DYCG_OK (0) or a negative DYCG_E*
 *    code. Nothing aborts the process; after an error, dycg_last_error() holds
 *    a one-line description and the handle stays usable for gather/destroy.
 *  - Input arrays are borrowed for the duration of the call only. Output
 *    buffers are allocated by the caller.
 *  - One host thread per handle; calls on one handle are not re-entrant.
 *  - Vertex ids are uint32 and must be < 2^31 (bit 31 of an adjacency slot
 *    marks a deleted occurrence).
 *
 * Each entry point cites the reference interface it replaces
 * (MriMouse/DyCGraph, paths relative to that project).
 */
#ifndef DYCG_H
#define DYCG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define DYCG_OK 0
#define DYCG_EINVAL (-1)      /* bad argument                                 */
#define DYCG_ECUDA (-2)       /* a CUDA runtime call failed                   */
#define DYCG_ENOMEM (-3)      /* host or device allocation failed             */
#define DYCG_ESTATE (-4)      /* call out of order (e.g. batch before init)   */
#define DYCG_ECAPACITY (-5)   /* adjacency arena or a queue is exhausted      */
#define DYCG_ELIMIT (-6)      /* a bounded device loop hit its iteration cap  */
#define DYCG_EIO (-7)         /* file could not be read or parsed             */
#define DYCG_ENOGPU (-8)      /* no CUDA device is available                  */

/* ---- algorithms (the reference's four hybrid_* operators) -------------- */
#define DYCG_ALGO_SSSP 0      /* samples/hybrid_sssp/hybrid_sssp.cu:51-204     */
#define DYCG_ALGO_BFS 1       /* samples/hybrid_bfs/hybrid_bfs.cu (weight 1)   */
#define DYCG_ALGO_CC 2        /* samples/hybrid_cc/hybrid_cc.cu:51-200         */
#define DYCG_ALGO_PR 3        /* samples/hybrid_pr/hybrid_pr.cu:36-124         */

/* ---- edge weights (SSSP) ----------------------------------------------- */
/* HASH128: w(u,v) = (u+v) % 128 + 1, the reference's TraversalEdgeWeight
 * (include/framework/variants/api.cuh:26-28); file weights are ignored.
 * STORED: every adjacency slot carries the weight given at load/insert time.
 *   A deletion record matches an occurrence by (u, v) alone, as in the
 *   reference; its w is ignored. When parallel occurrences of (u, v) carry
 *   different weights, which one a deletion removes is not specified, so
 *   results can depend on it. Giving every occurrence of (u, v) the same
 *   weight (the loaders and the benchmark hash it from (seed, u, v)) keeps
 *   results independent of it. */
#define DYCG_WEIGHT_HASH128 0
#define DYCG_WEIGHT_STORED 1

/* ---- cache admission policy -------------------------------------------- */
#define DYCG_CACHE_NONE 0     /* no page is staged in HBM (reference -cache=0) */
#define DYCG_CACHE_HOTNESS 1  /* decayed per-page access counts, top-K pages   */
#define DYCG_CACHE_LEARNED 2  /* BF16 MLP ranks pages before each repair        */

#define DYCG_INFINITY 0xFFFFFFFFu /* unreachable distance / no parent        */

/* One update record, layout-compatible with the reference's 12-byte
 * WEdgePair<uint32_t> (include/framework/edgepair.h:17-31). */
typedef struct dycg_edge {
  uint32_t u;
  uint32_t v;
  uint32_t w;
} dycg_edge;

typedef struct dycg_options {
  uint32_t algo;          /* DYCG_ALGO_*                                      */
  uint32_t weight_mode;   /* DYCG_WEIGHT_* (SSSP only)                        */
  uint32_t source;        /* SSSP/BFS root (reference -source_node)           */
  uint32_t segments;      /* reference -SEGMENT, accepted for compatibility:   */
                          /* the engine's unit of storage, caching and update */
                          /* binning is the page (2^page_shift slots); the    */
                          /* per-segment binning is dycg_group_updates's      */
  uint64_t hbm_graph_budget_bytes; /* cap on adjacency bytes resident in HBM  */
  uint32_t cache_policy;  /* DYCG_CACHE_*                                     */
  uint32_t symmetric;     /* 1: graph and every batch are symmetric, the      */
                          /* incoming adjacency aliases the outgoing one      */
  float epsilon;          /* PR push threshold (reference -error)             */
  float alpha;            /* PR damping factor (0.85)                         */
  uint32_t max_rounds;    /* PR rounds per batch (reference -pr_max_rounds)   */
  int32_t device;         /* CUDA device ordinal                              */
  uint32_t page_shift;    /* log2 of adjacency slots per cache page (0: 12)   */
  uint32_t ordered_delta; /* SSSP/BFS/CC: 0 = unordered closure; d > 0 = each  */
                          /* wave expands only values < wave min + d (the    */
                          /* reference's ordered schedule, for high-diameter */
                          /* graphs; 1 is exact-min order for BFS and CC)    */
  uint32_t arena_headroom_permille; /* spare arena slots for row growth, per   */
                          /* mille of the loaded slots (0: 125, the reference's */
                          /* 1/8; at least 2^20 slots either way)              */
  uint32_t frontier_queue; /* single-source repair: DYCG_QUEUE_STATIC (0) or   */
                          /* DYCG_QUEUE_CLAIMED, how warps share a wave's rows */
                          /* (the batched form's scheme is tuned, see          */
                          /* dycg_tune_query_mapping)                          */
  uint32_t mutation_ctas; /* CTAs of the deletion / append kernels (0: one    */
                          /* per SM). They take a snapshot's records in row   */
                          /* order, so fewer CTAs in flight keep their host   */
                          /* transactions in a narrower window of the arena,  */
                          /* which the host link serves faster                */
  uint32_t reserved[3];
} dycg_options;

/* Per-call counters. Byte counts are algorithmic: every adjacency slot read
 * or written is charged once, to the host link when its page is not resident
 * in HBM and to HBM otherwise. */
typedef struct dycg_batch_stats {
  uint64_t deletions;          /* delete records received                    */
  uint64_t insertions;         /* insert records received                    */
  uint64_t missing_deletes;    /* deletes that matched no live occurrence    */
  uint64_t invalid_updates;    /* records with an endpoint >= n              */
  uint64_t touched_sources;    /* distinct sources of valid records          */
  uint64_t relocated_rows;     /* rows moved to a larger block               */
  uint64_t affected;           /* vertices invalidated by deletions          */
  uint64_t expanded;           /* row expansions in the repair closures      */
  uint64_t edges_scanned;      /* adjacency slots read by the repair         */
  uint64_t improvements;       /* successful relaxations / residual pushes   */
  uint64_t waves;              /* frontier waves (all closures)              */
  uint64_t link_bytes;         /* adjacency bytes read/written over the host link */
  uint64_t hbm_adj_bytes;      /* adjacency bytes read/written in the HBM cache   */
  uint64_t state_bytes;        /* vertex-state bytes read/written (HBM)      */
  uint64_t cache_pages_loaded; /* pages staged into HBM by maintenance       */
  uint64_t cache_pages_evicted;
  uint64_t kernel_launches;    /* CUDA kernels launched by the call          */
  double ms_ingest;            /* device time per stage (CUDA events)        */
  double ms_mutate;
  double ms_repair;
  double ms_cache;
  double ms_total;
  uint64_t mutate_link_bytes;  /* mutation kernels' share of link_bytes      */
  uint64_t mutate_hbm_bytes;   /* mutation kernels' share of hbm_adj_bytes    */
  /* time inside the repair kernel per phase (SSSP/BFS/CC: one source, or
     the batched many-query form; zero for PageRank and per-query repairs) */
  double ms_phase_invalidate;  /* deletion seeds + invalidation waves        */
  double ms_phase_pull;        /* reset + pull over in-rows                  */
  double ms_phase_seed;        /* frontier + insertion seeds                 */
  double ms_phase_closure;     /* push closure waves                         */
  uint64_t reserved[2];
} dycg_batch_stats;

typedef struct dycg_graph_info {
  uint64_t nodes;
  uint64_t live_edges;
  uint64_t arena_slots;        /* slots allocated in the host arena          */
  uint64_t arena_used;         /* slots handed out (rows + relocations)      */
  uint64_t pages;              /* pages over both adjacency directions       */
  uint64_t cache_slots;        /* pages the HBM budget can hold              */
  uint64_t cached_pages;       /* pages resident now                         */
  uint64_t host_bytes;         /* pinned host bytes held by the arenas       */
  uint64_t device_bytes;       /* device bytes held by the engine            */
  uint32_t page_shift;
  uint32_t has_incoming;       /* 1 if a separate incoming adjacency exists  */
  uint64_t reserved[6];
} dycg_graph_info;

typedef struct dycg_engine dycg_engine;

/* Fill *opt with the reference's defaults (SSSP, HASH128, source 0,
 * SEGMENT 1, no cache, epsilon 1e-6, alpha 0.85, 100 rounds). */
int dycg_options_default(dycg_options *opt);

/* Replaces Engine::Engine(AlgoType) + SetOptions
 * (include/framework/framework.cuh:1158, :1245). */
int dycg_create(const dycg_options *opt, dycg_engine **out);

/* Releases every device and pinned host allocation of the handle. */
void dycg_destroy(dycg_engine *e);

/* Replaces Engine::LoadGraph (include/framework/framework.cuh:1569-1798):
 * builds the outgoing (and, unless symmetric, incoming) adjacency from a host
 * CSR. offsets has n+1 entries; w may be NULL (weights then follow the weight
 * mode). Rows keep their multiset of occurrences (duplicates are kept). */
int dycg_load_graph_csr(dycg_engine *e, uint32_t n, const uint64_t *offsets,
                        const uint32_t *dst, const uint32_t *w);

/* Replaces Context's market_big reader (src/utils/parser.cpp:296-406): text
 * lines "u v [w]"; n = max(max id + 1, min_nodes). */
int dycg_load_graph_file(dycg_engine *e, const char *path, uint32_t min_nodes,
                         int weighted);

/* Binary CSR graph file (replaces the market_big text parse,
 * src/utils/parser.cpp:296-406, for large graphs): little-endian
 *   char magic[8] = "DYCGCSR1"; uint64 n; uint64 m; uint64 flags (bit 0: weights)
 *   uint64 offsets[n+1]; uint32 dst[m]; uint32 w[m] (when bit 0 is set)
 * read with one pass over a memory map. */
int dycg_load_graph_binary(dycg_engine *e, const char *path);

/* Converts a text edge list, read exactly as dycg_load_graph_file reads it
 * (the market_big parse it replaces, src/utils/parser.cpp:296-406), into the
 * binary CSR file above, so that large graphs are parsed once and later load
 * from a memory map. Host only (no GPU needed). */
int dycg_convert_graph_text(const char *text_path, const char *binary_path, uint32_t min_nodes,
                            int weighted);

/* Synthetic workloads built on the GPU straight into the engine. R-MAT:
 * 2^scale vertices, edge_factor*2^scale draws with quadrant probabilities
 * (a,b,c,1-a-b-c), self-loops and duplicates removed; weights uniform in
 * [wlo,whi] as a hash of (seed,u,v). symmetrize adds the reverse of every
 * edge before de-duplication. */
int dycg_load_graph_rmat(dycg_engine *e, uint32_t scale, uint32_t edge_factor,
                         double a, double b, double c, uint64_t seed,
                         uint32_t wlo, uint32_t whi, int symmetrize);

/* 2D grid side x side, 4-neighbour edges in both directions, plus
 * shortcut_permille/1000 * side^2 random shortcuts within radius (Chebyshev),
 * inserted in both directions; weights uniform in [wlo,whi]. */
int dycg_load_graph_grid(dycg_engine *e, uint32_t side, uint32_t shortcut_permille,
                         uint32_t radius, uint64_t seed, uint32_t wlo, uint32_t whi);

/* Replaces Engine::InitGraph + Engine::Start / StartPageRank
 * (include/framework/framework.cuh:1803, :1963-2005, :2681) and the initial
 * compute_hot_vertices/confirm_candidate_batch/LoadCache sequence
 * (samples/hybrid_sssp/hybrid_sssp.cu:412-416): static solve on the GPU,
 * then the first cache admission. */
int dycg_init(dycg_engine *e);

/* Replaces Engine::del_edge (include/framework/framework.cuh:2595-2618 ->
 * update_tree_del :4811-4957): remove one occurrence per record, repair. */
int dycg_delete_edges(dycg_engine *e, const dycg_edge *dels, size_t nd,
                      dycg_batch_stats *stats);

/* Replaces Engine::add_edge (include/framework/framework.cuh:2419 ->
 * update_tree_add :3525-3756): append each record, repair. */
int dycg_insert_edges(dycg_engine *e, const dycg_edge *adds, size_t na,
                      dycg_batch_stats *stats);

/* Replaces Engine::compute_hot_vertices_sssp + confirm_candidate_batch +
 * CacheRefreshRequired + evication_cache + compact_cache + LoadCache
 * (include/framework/framework.cuh:1264-1567, :2978-3061). */
int dycg_cache_maintenance(dycg_engine *e, dycg_batch_stats *stats);

/* One snapshot: all deletions, then all insertions (the reference's order,
 * include/framework/topology_replay.h:71-72), one fused repair, then cache
 * maintenance -- the unit the reference's batch timer measures
 * (samples/hybrid_sssp/hybrid_sssp.cu:444-548). PR follows
 * Engine::UpdatePageRank (include/framework/framework.cuh:2692-2736).
 * Host arrays; the copies to the device are part of the call. */
int dycg_apply_batch(dycg_engine *e, const dycg_edge *dels, size_t nd,
                     const dycg_edge *adds, size_t na, dycg_batch_stats *stats);

/* Size the per-batch buffers for snapshots of up to max_records deletions
 * (and as many insertions) ahead of time, the way the reference sizes its
 * mapped update arrays from the update file before replay
 * (include/framework/framework.cuh:2387-2412 get_update_file). Without it the
 * buffers grow on the first larger batch, inside that call. After dycg_init
 * in the batched many-query form it also captures the replay graphs of every
 * batch-size class up to max_records (see dycg_apply_batches). */
int dycg_reserve_batch(dycg_engine *e, size_t max_records);

/* Same as dycg_apply_batch with the records already in device memory. */
int dycg_apply_batch_device(dycg_engine *e, const dycg_edge *d_dels, size_t nd,
                            const dycg_edge *d_adds, size_t na,
                            dycg_batch_stats *stats);

/* Replaces Engine::GatherValue/GatherParent (include/framework/framework.cuh:
 * 4959-4984). values/parents: n entries each (either may be NULL). SSSP/BFS:
 * distance/level, DYCG_INFINITY if unreachable; CC: label; parent is
 * DYCG_INFINITY for roots and unreachable vertices. */
int dycg_gather(dycg_engine *e, uint32_t *values, uint32_t *parents);

/* PR: ranks x and residuals r (n floats each, either may be NULL). */
int dycg_gather_ranks(dycg_engine *e, float *ranks, float *residuals);

/* Current live row of v (outgoing, or incoming when incoming != 0), in slot
 * order; *deg receives the live degree even when it exceeds cap. */
int dycg_get_row(dycg_engine *e, uint32_t v, int incoming, uint32_t *dst,
                 uint32_t *w, uint32_t cap, uint32_t *deg);

/* Whole live outgoing adjacency as CSR (offsets n+1, dst/w live_edges). */
int dycg_export_csr(dycg_engine *e, uint64_t *offsets, uint32_t *dst, uint32_t *w);

int dycg_graph_info_get(dycg_engine *e, dycg_graph_info *info);

/* Sample `count` distinct live edges uniformly (by occurrence) from the
 * current outgoing adjacency, with their weights; deterministic in seed. */
int dycg_sample_edges(dycg_engine *e, uint64_t count, uint64_t seed, dycg_edge *out);

/* R-MAT edge draws (no de-duplication), computed on the host; identical to
 * the draws dycg_load_graph_rmat makes for the same arguments at indices
 * [first, first+count). Used for insertion batches. */
int dycg_gen_rmat_edges(uint32_t scale, double a, double b, double c, uint64_t seed,
                        uint64_t first, uint64_t count, uint32_t wlo, uint32_t whi,
                        dycg_edge *out);

/* Weight of edge (u,v) under the seeded uniform rule used by the loaders. */
uint32_t dycg_hash_weight(uint64_t seed, uint32_t u, uint32_t v, uint32_t wlo,
                          uint32_t whi);

/* Measurement helper (no reference counterpart): host-link bandwidth on
 * `device` with a `bytes`-sized pinned buffer -- a host-to-device copy-engine
 * transfer and a kernel reading the mapped buffer zero-copy with 16-byte
 * loads (best of 5 each, GB/s). */
int dycg_measure_host_link(int device, uint64_t bytes, double *h2d_gbs, double *zero_copy_gbs);

/* Failure-detection check (no reference counterpart): every wait of the
 * persistent repair kernels (grid barriers, worklist waits) is bounded by a
 * time limit after which the kernel records an error status and returns, so
 * a rank or block that never arrives is reported to the host instead of
 * hanging the GPU. This runs the library's grid barrier in a cooperative
 * launch of 8 blocks in which block 0 never arrives (it waits, bounded, on a
 * flag that nothing sets): *status_absent receives the status the waiting
 * blocks recorded (1, the barrier time-limit error, expected); then a launch
 * in which every block arrives runs on the same context: *status_all (0
 * expected). limit_ms in [1, 10000]. */
int dycg_check_bounded_wait(int device, uint32_t limit_ms, uint32_t *status_absent,
                            uint32_t *status_all);

/* Measurement helper (no reference counterpart): cost of random host-link
 * transactions on `device` -- `ops` reads (write = 0) or writes of op_bytes
 * (4, 8 or 16 per thread, or 128 per warp) at random aligned offsets of a
 * `bytes`-sized pinned, mapped buffer, many in flight; *ns_per_op is the
 * device time per access (best of 3 after a warm-up). The bound of kernels
 * that touch rows of a multi-GB arena at random. */
int dycg_measure_host_random(int device, uint64_t bytes, uint32_t op_bytes, int write,
                             uint64_t ops, double *ns_per_op);

/* Measurement helper (no reference counterpart): the same accesses as
 * dycg_measure_host_random (op_bytes 8 per thread or 128 per warp, reads or
 * writes, `ops` random aligned offsets of a `bytes`-sized pinned buffer) but
 * issued in ascending address order by `ctas` CTAs of 256 threads taking
 * them in turn, the way the mutation kernels take their row-ordered records:
 * the warps in flight then touch a narrow window of the buffer. Needs
 * ops * 8 bytes of device memory for the sorted offsets. */
int dycg_measure_host_sweep(int device, uint64_t bytes, uint32_t op_bytes, int write,
                            uint64_t ops, uint32_t ctas, double *ns_per_op);

/* Replaces GroupedUpdateBatch (include/framework/effective_update_batch.h:
 * 36-207) as a standalone device step. Device pointers throughout; stream is a
 * cudaStream_t (NULL = default stream). Records with an endpoint >=
 * num_vertices are dropped; the rest are sorted by (u, v) and each distinct
 * (u, v) is written once, in ascending order, as d_out_uv[2i], d_out_uv[2i+1]
 * with its multiplicity d_out_mult[i] (outputs sized n). d_counts[0] = distinct
 * records, d_counts[1] = dropped records. When num_segments > 0, the distinct
 * records are also counted per source segment: segment s holds sources in
 * [d_segment_ends[s-1], d_segment_ends[s]) (ends ascending). Scratch memory is
 * allocated on the stream and released before the call returns. */
int dycg_group_updates(const dycg_edge *d_records, size_t n, uint32_t num_vertices,
                       const uint32_t *d_segment_ends, uint32_t num_segments,
                       uint32_t *d_out_uv, uint32_t *d_out_mult, uint32_t *d_segment_counts,
                       uint32_t *d_counts, void *stream);

/* dycg_group_updates without any allocation -- no counterpart in the
 * reference. Same inputs, outputs and results as dycg_group_updates, for
 * callers that cannot allocate device memory at call time (code that must not
 * synchronise the device, processes whose device memory is held by another
 * allocator, hosts that must not own GPU allocations). Its scratch is a fixed
 * file-scope device array sized for DYCG_GROUP_NOALLOC_MAX_RECORDS records
 * (about 11 MiB, held on every GPU that loads the library until exit); larger
 * batches return DYCG_ECAPACITY. All calls share that array: calls that
 * overlap on the GPU race, calls ordered on one stream are safe. The first
 * call on a device looks up the array's device address and should come
 * before any stream capture; later calls whose stream is not capturing look
 * it up again, so a device reset leaves no stale address behind. */
#define DYCG_GROUP_NOALLOC_MAX_RECORDS 262144u
int dycg_group_updates_noalloc(const dycg_edge *d_records, size_t n, uint32_t num_vertices,
                               const uint32_t *d_segment_ends, uint32_t num_segments,
                               uint32_t *d_out_uv, uint32_t *d_out_mult,
                               uint32_t *d_segment_counts, uint32_t *d_counts, void *stream);

/* ---- many-query forms (SSSP/BFS) ---------------------------------------
 * The reference engine holds one source per engine (Engine::InitGraph(src),
 * include/framework/framework.cuh:1803); these calls let one engine keep the
 * results of up to DYCG_MAX_QUERIES sources over one graph, repaired together
 * after every snapshot by dycg_apply_batch / dycg_delete_edges /
 * dycg_insert_edges. No reference counterpart.
 *  BATCHED: one repair launch per snapshot for all queries; results stored
 *           vertex-major, so a row read serves every query active on it.
 *  PER_QUERY: the single-source repair launched once per query (the plain
 *           per-query path, kept for comparison); results query-major.
 * Call after loading and before dycg_init. sources: count ids < n. */
#define DYCG_MAX_QUERIES 256u
#define DYCG_QUERIES_BATCHED 0u
#define DYCG_QUERIES_PER_QUERY 1u
int dycg_set_queries(dycg_engine *e, const uint32_t *sources, uint32_t count, uint32_t mode);

/* Batched form's work mapping. A row of len slots active in act queries is
 * expanded with lanes over queries (one edge at a time) when
 * 4*act >= qratio*min(len, 32), else with lanes over slots (the active queries
 * in turn); qratio 0 always maps lanes to queries. Rows whose work exceeds
 * `heavy` warp iterations are split into tile-slot pieces processed by whole
 * CTAs (tile >= 1024). Defaults: qratio 4, heavy 64, tile 4096. The mapping
 * changes speed only, never results. */
int dycg_set_query_mapping(dycg_engine *e, uint32_t qratio, uint32_t heavy, uint32_t tile);

/* One work mapping of the batched form and the repair time it took. */
typedef struct dycg_query_mapping {
  uint32_t qratio;
  uint32_t heavy;
  uint32_t tile;
  uint32_t pull_qratio;  /* the mapping rule's ratio for the pull phase       */
  uint32_t queue;        /* frontier-queue scheme, DYCG_QUEUE_*               */
  float repair_ms;
} dycg_query_mapping;

/* Frontier-queue schemes of the batched form: how a wave's frontier items
 * (vertices with per-query masks) are queued and shared by the warps of the
 * repair launch. STATIC: warp w takes items w, w + warps, ... (no shared
 * counter); CLAIMED: warps claim items one at a time from a counter of the
 * wave, so warps that drew long rows do not hold the wave's barrier.
 * RANGES (a flag, combined with either): each wave queue is cut into 64
 * regions by vertex range and read region by region, so the warps in flight
 * read rows from a narrow window of the host arena (fewer address
 * translations per host transaction) instead of from all of it.
 * ASYNC (a flag; RANGES is then ignored): the invalidation and the push
 * closure run without waves: a vertex whose masks gain bits is appended to a
 * ring unless it already waits there, and every warp takes ring items in
 * turn until none is left and none is being processed (label-correcting
 * order, same fixpoint); heavy rows are split into tile items. The pull
 * phase (one pass) keeps the static or claimed distribution. */
#define DYCG_QUEUE_STATIC 0u
#define DYCG_QUEUE_CLAIMED 1u
#define DYCG_QUEUE_RANGES 2u
#define DYCG_QUEUE_ASYNC 4u
int dycg_set_query_queue(dycg_engine *e, uint32_t scheme);

/* Autotuner of the batched form's work mapping (no reference counterpart):
 * applies one snapshot like dycg_apply_batch, but repairs it once per
 * candidate mapping (qratio in {2,4,8,2^20} x heavy in {4,8,16,64,256} with the
 * pull phase on the same ratio, then the best of those with the pull phase's
 * ratio in {0,1,2,8}, then the best so far with query-lane tiles of
 * {1024,4096,16384} slots, then the best so far under the other
 * frontier-queue schemes: static, claimed, ranges, claimed + ranges, async,
 * async + claimed), each from the same saved state, keeps the fastest
 * mapping for later snapshots
 * and leaves the state of one ordinary repair. Needs HBM for one extra copy
 * of the query results while it runs. tried (cap entries, may be NULL)
 * receives the candidates with their repair times; *n_tried their count. */
int dycg_tune_query_mapping(dycg_engine *e, const dycg_edge *dels, size_t nd,
                            const dycg_edge *adds, size_t na, dycg_query_mapping *tried,
                            uint32_t cap, uint32_t *n_tried, dycg_batch_stats *stats);

/* Many snapshots in one call, in order (the reference's sample drivers loop
 * over batches one call each, samples/hybrid_sssp/hybrid_sssp.cu:444-548).
 * The records of snapshot i follow those of snapshot i-1: del_counts[i]
 * deletions in dels, add_counts[i] insertions in adds. stats: one entry per
 * snapshot, or NULL. In the batched many-query form each snapshot is one
 * replay of a CUDA graph (ingest, mutation, learned admission when that
 * policy is set, repair, cache maintenance) captured once per batch size
 * class (powers of two >= 1024; records are padded with out-of-range entries
 * that ingest drops), with no host synchronisation between snapshots; the
 * admission plan is computed on the device. Per-stage times are then not
 * split (ms_total per snapshot, ms_repair from the repair kernel's own
 * stamps). Other forms, and an engine still recording policy traces, apply
 * the snapshots one by one. */
int dycg_apply_batches(dycg_engine *e, const dycg_edge *dels, const uint64_t *del_counts,
                       const dycg_edge *adds, const uint64_t *add_counts, uint32_t snapshots,
                       dycg_batch_stats *stats);

/* Same as dycg_apply_batches with the records already in device memory. */
int dycg_apply_batches_device(dycg_engine *e, const dycg_edge *d_dels,
                              const uint64_t *del_counts, const dycg_edge *d_adds,
                              const uint64_t *add_counts, uint32_t snapshots,
                              dycg_batch_stats *stats);

/* Results of query q (values/parents as dycg_gather; n entries each, either
 * may be NULL). With queries set, dycg_gather returns query 0. */
int dycg_gather_query(dycg_engine *e, uint32_t q, uint32_t *values, uint32_t *parents);

/* ---- learned cache admission (no reference counterpart) -------------------
 * The reference admits rows by a decayed activity count
 * (include/framework/variants/driver.cuh:486-515); that is DYCG_CACHE_HOTNESS
 * here. DYCG_CACHE_LEARNED ranks every cache page with a small MLP
 * (DYCG_POLICY_FEATURES -> 64 -> 64 -> 1, ReLU, BF16 weights and inputs, FP32
 * accumulation) after a snapshot's mutation, from per-page features (page
 * reads of the mutation just done and of the last two snapshots, the decayed
 * read score, update records of this batch whose row starts in the page,
 * snapshots since the last read, rows starting in the page and the longest of
 * them -- these two refreshed every 8 snapshots), and stages the pages it
 * predicts to be read most before the repair, when the predicted reads over
 * the horizon cover at least half the page's slots (half its fill over the
 * host link), up to cache pages/256 per snapshot. Which pages are cached never changes results.
 * The network predicts log1p(page reads over this snapshot and the next
 * two) and is trained on traces the engine records, by the library's own
 * forward/backward and Adam kernels on the GPU; one of its history features
 * is the hotness policy's decayed read score. */
#define DYCG_POLICY_FEATURES 8
#define DYCG_POLICY_HIDDEN 64
#define DYCG_POLICY_PARAMS 4801 /* W1[8x64] b1[64] W2[64x64] b2[64] W3[64] b3, FP32 */

typedef struct dycg_policy_report {
  uint64_t samples;      /* trace samples used (pages x complete snapshots)    */
  uint64_t steps;        /* optimizer steps                                    */
  float loss_before;     /* mean squared error over all samples, before/after   */
  float loss_after;
  float ms;              /* device time of the training call                    */
  uint32_t reserved[5];
} dycg_policy_report;

/* Switch between DYCG_CACHE_HOTNESS and DYCG_CACHE_LEARNED (needs a page
 * cache: a non-zero budget and a policy other than NONE at create). */
int dycg_set_cache_policy(dycg_engine *e, uint32_t policy);

/* Record the features of the next `snapshots` snapshot calls and their page
 * reads (over each snapshot and the two after it), under whatever policy is
 * active, as the training set; 0 drops the traces. Training uses the traced
 * snapshots whose two following snapshots have also run. */
int dycg_policy_trace(dycg_engine *e, uint32_t snapshots);

/* Train the network on the recorded traces with Adam (lr), minibatches of
 * `batch` samples drawn with a seed, epochs x samples / batch steps. */
int dycg_policy_train(dycg_engine *e, uint32_t epochs, float lr, uint32_t batch,
                      uint64_t seed, dycg_policy_report *report);

/* Read / replace the FP32 master parameters (DYCG_POLICY_PARAMS floats). */
int dycg_policy_params(dycg_engine *e, float *params);
int dycg_policy_set_params(dycg_engine *e, const float *params);

/* Standalone network kernels on device buffers (stream = cudaStream_t or
 * NULL): x = n rows of DYCG_POLICY_FEATURES bf16 values, params FP32 (used
 * rounded to bf16). dycg_mlp_infer writes n predictions; dycg_mlp_loss_grad
 * adds the summed squared error over n rows against y into *d_loss and its
 * gradient w.r.t. the parameters into d_grad (both must start at zero). */
int dycg_mlp_infer(const void *d_x, uint32_t n, const float *d_params, float *d_out,
                   void *stream);
int dycg_mlp_loss_grad(const void *d_x, const float *d_y, uint32_t n, const float *d_params,
                       float *d_grad, float *d_loss, void *stream);

/* For each source, one live out-edge drawn uniformly (deterministic in seed);
 * {DYCG_INFINITY, DYCG_INFINITY, 0} for a source without live edges. Used to
 * draw deletions with skewed endpoints. */
int dycg_sample_row_edges(dycg_engine *e, const uint32_t *sources, uint64_t count,
                          uint64_t seed, dycg_edge *out);

/* cudaStream_t the engine launches on (for CUDA-event timing by callers).
 * Like every call other than the snapshot calls, it first makes that stream
 * wait for the engine's side-stream work of earlier calls (the hotness
 * policy's page staging), so an event recorded on the stream afterwards
 * covers all the work of those calls. */
int dycg_stream(dycg_engine *e, void **stream);

/* Copy of the last error message into buf (always NUL-terminated). */
int dycg_last_error(dycg_engine *e, char *buf, size_t len);

/* Library version string. */
const char *dycg_version(void);

#ifdef __cplusplus
}
#endif
#endif /* DYCG_H */
