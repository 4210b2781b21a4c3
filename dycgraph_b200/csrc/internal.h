// internal.h -- launcher declarations shared between the kernel files and the
// host engine.
#pragma once
#include <algorithm>
#include <cstddef>
#include <cstdint>

#include "common.cuh"

namespace dycg {

struct dycg_edge_dev {
  uint32_t u, v, w;
};

constexpr uint32_t PH_DELETE = 1, PH_INSERT = 2, PH_CLOSE = 4;
constexpr uint32_t PR_AMEND = 1, PR_CONVERGE = 2;

struct RepairLaunch {
  Adj out, in;
  u64 *key;
  uint32_t *mark, *wtag, *aff, *q0, *q1;
  uint4 *tiles;
  uint32_t tile_cap;
  Ctl *ctl;
  const uint2 *del_uv;
  const uint32_t *del_found;
  const uint32_t *n_del_ptr;
  const uint3 *add_uvw;
  uint32_t n_add;
  uint32_t n, source, epoch, tag_base, phases, max_waves;
  uint32_t delta;  // ordered closure bucket width (0: unordered)
  uint32_t *q2;
  uint32_t *tag_dev;  // optional device wave-tag counter (replaces tag_base)
  u64 timeout_ns;
  uint32_t algo;
  bool stored;
  int num_sms;
  uint32_t sched;     // frontier items: 0 static, 1 claimed one at a time
};
cudaError_t launch_repair(const RepairLaunch &L, cudaStream_t s);
cudaError_t launch_init_state(uint32_t algo, u64 *key, uint32_t n, uint32_t source,
                              uint32_t *q0, Ctl *ctl, cudaStream_t s);

// Batched repair of Q = 32*nb queries over one graph (multi.cu).
constexpr uint32_t MULTI_MAX_BLOCKS = 8;   // up to 256 queries
constexpr uint32_t MULTI_MIN_TILE = 1024;  // smallest tile (sizes the tile queue)
struct MultiLaunch {
  Adj out, in;
  u64 *key;                     // n * Q, vertex-major
  uint32_t *affm, *inew0, *inew1, *nmask0, *nmask1, *cmask;  // n * nb each
  uint32_t *mark, *wtag, *aff, *q0, *q1;
  uint4 *tiles;
  uint32_t tile_cap;
  Ctl *ctl;
  uint32_t *seq;                // device {epoch, next wave tag}, advanced by each launch
  const uint2 *del_uv;
  const uint32_t *del_found;
  const uint32_t *n_del_ptr;
  const uint3 *add_uvw;
  uint32_t n_add;
  uint32_t n, nb, phases, max_waves;
  uint32_t qratio;              // query lanes when 4*active >= qratio*min(len,32)
  uint32_t pull_qratio;         // the same rule for the pull phase
  uint32_t heavy;               // rows with more work (warp iterations) are tiled
  uint32_t tile;                // tile size, in slots
  uint32_t sched;               // frontier-queue scheme (DYCG_QUEUE_* bits): claimed items,
                                // range-ordered wave queues, asynchronous worklist
  u64 *ring;                    // asynchronous worklist ring (ring_cap items)
  uint32_t ring_cap;
  uint32_t *inq;                // per vertex: an item waits in the ring
  uint32_t *pool;               // mask records of split heavy rows (pool_cap x nb words)
  uint32_t pool_cap;
  u64 timeout_ns;
  uint32_t algo;
  bool stored;
  int num_sms;
};
cudaError_t launch_multi(const MultiLaunch &L, cudaStream_t s);
cudaError_t launch_multi_init(u64 *key, uint32_t n, uint32_t nb, const uint32_t *sources,
                              uint32_t *nmask0, uint32_t *q0, uint32_t *wtag, const uint32_t *seq,
                              Ctl *ctl, uint32_t sched, cudaStream_t s);
// values/parents of query q out of the vertex-major (Q = 32*nb) or
// query-major (Q = 0: key already offset to the query) key array
cudaError_t launch_multi_gather(const u64 *key, uint32_t n, uint32_t Q, uint32_t q,
                                uint32_t *values, uint32_t *parents, cudaStream_t s);

struct PrLaunch {
  Adj out;
  float *x, *r, *delta;
  uint32_t *queued, *q0, *q1;
  const uint32_t *sources, *n_sources;  // touched sources
  const uint2 *del_uv;                   // distinct deleted pairs, occurrences found
  const uint32_t *del_found, *n_del;
  const uint3 *add_uvw;                  // inserted occurrences
  uint32_t n_add;
  uint4 *tiles;
  uint32_t tile_cap;
  Ctl *ctl;
  uint32_t n, cur, phases;
  float eps, alpha;
  uint32_t max_rounds;
  u64 timeout_ns;
  int num_sms;
};
cudaError_t launch_pr(const PrLaunch &L, cudaStream_t s);
cudaError_t launch_pr_old_degree(const uint32_t *sources, const uint32_t *n_sources,
                                 uint32_t max_sources, const uint32_t *live, float *delta,
                                 cudaStream_t s);
cudaError_t launch_pr_init(float *x, float *r, uint32_t *queued, uint32_t *q0, uint32_t n,
                           float base, Ctl *ctl, cudaStream_t s);

// ingest + mutation
cudaError_t launch_prep_keys(const dycg_edge_dev *e, uint32_t cnt, uint32_t n, u64 *kout,
                             u64 *kin, uint32_t *w, u64 *invalid, cudaStream_t s);
cudaError_t sort_keys(void *temp, size_t &temp_bytes, const u64 *in, u64 *out, uint32_t cnt,
                      cudaStream_t s);
cudaError_t sort_pairs(void *temp, size_t &temp_bytes, const u64 *kin, u64 *kout,
                       const uint32_t *vin, uint32_t *vout, uint32_t cnt, cudaStream_t s);
// Scratch of the run finder (per batch capacity; temp = CUB scan storage).
struct RunScratch {
  uint32_t *flags, *pos, *start, *valid;
  void *temp;
  size_t temp_bytes;
};
size_t unique_runs_temp_bytes(uint32_t cnt);
cudaError_t launch_unique_runs(const u64 *k, uint32_t cnt, uint2 *uv, uint32_t *mult,
                               uint32_t *n_out, uint32_t cap, uint32_t *err, const RunScratch &S,
                               cudaStream_t s);
cudaError_t launch_row_segments(const u64 *k, uint32_t cnt, uint3 *seg, uint32_t *n_out,
                                uint32_t cap, uint32_t *err, const RunScratch &S, cudaStream_t s);
// Deleted occurrences found by the read-only search, written afterwards.
struct Tombs {
  u64 *pos;
  uint32_t *count;
  uint32_t cap;
};
// ctas: CTAs of the warp-per-record mutation kernels (0: one warp per record,
// up to the grid cap)
cudaError_t launch_delete_rows(const Adj &A, const uint2 *uv, const uint32_t *mult,
                               const uint32_t *n_ptr, uint32_t max_n, uint32_t *found, Ctl *ctl,
                               int count_missing, const Tombs &T, uint32_t ctas, cudaStream_t s);
// Deletions in rows whose unsorted suffix exceeds DEFER_SUFFIX slots are
// matched by sort-merge (gather the live suffix slots once, stable sort by
// (row, neighbour), binary search per record) instead of a suffix scan per
// record, whose cost grows with (records in the row) x (suffix length).
constexpr uint32_t DEFER_SUFFIX = 1024;
struct DeferDel {
  bool on;
  uint32_t *rem;       // per record: occurrences left after the sorted-prefix pass
  u64 *packed;         // (deferred rows << 40) | suffix slots reserved
  uint32_t *row_u;     // deferred rows, in reservation order
  u64 *row_base;       // first gather index of each deferred row
  uint32_t cap_rows;
};
struct DeferBufs {
  u64 *k_in, *k_out;
  uint32_t *v_in, *v_out;
  void *temp;
  size_t temp_bytes;
};
// pass over the sorted prefixes (and short suffixes); long suffixes deferred
cudaError_t launch_delete_prefix(const Adj &A, const uint2 *uv, const uint32_t *mult,
                                 const uint32_t *n_ptr, uint32_t max_n, uint32_t *found, Ctl *ctl,
                                 int count_missing, const Tombs &T, const DeferDel &D,
                                 uint32_t ctas, cudaStream_t s);
size_t delete_sort_temp_bytes(u64 total);
// sort-merge of the deferred suffixes (total gathered slots, nrows rows), then
// the tombstones of all found occurrences
cudaError_t launch_delete_suffix(const Adj &A, const uint2 *uv, const uint32_t *n_ptr,
                                 uint32_t max_n, uint32_t *found, Ctl *ctl, int count_missing,
                                 const Tombs &T, const DeferDel &D, uint32_t nrows, u64 total,
                                 const DeferBufs &B, cudaStream_t s);

// Relocation bookkeeping for rows that outgrow their block.
constexpr uint32_t RELOC_CHUNK = 1024;
struct RelocRec {
  uint32_t row, seg, len, pad;
  u64 old_off, new_off;
};
struct Reloc {
  RelocRec *rec;
  uint2 *chunks;
  uint32_t *n_reloc, *n_chunks;
  uint32_t cap, chunk_cap;
};
cudaError_t launch_add_rows(const Adj &A, const u64 *k, const uint32_t *w, const uint3 *seg,
                            const uint32_t *n_ptr, uint32_t max_n, const Reloc &R, Ctl *ctl,
                            uint32_t ctas, cudaStream_t s);
cudaError_t launch_keys_to_uvw(const u64 *k, const uint32_t *w, uint32_t cnt, uint3 *out,
                               cudaStream_t s);
cudaError_t launch_touched(const u64 *k, uint32_t cnt, uint32_t *tag, uint32_t epoch,
                           uint32_t *list, uint32_t *n_out, Ctl *ctl, cudaStream_t s);

// cache
// Device-resident admission state: the free-slot count and the plan of the
// last maintenance round (cache.cu plan_kernel), so that ranking, eviction
// and staging run without a host round trip (inside captured graphs too).
struct CachePlan {
  uint32_t free_count;   // free cache slots: free_list[0, free_count)
  uint32_t candidates;   // last round: top-K pages not resident
  uint32_t admit, evict; // last round: pages staged / evicted
  uint32_t first_rank;   // last round: first evicted rank among the candidates
  uint32_t free_base;    // last round: free count before eviction
  uint32_t top;          // last round: free count after eviction
  uint32_t pad;
  u64 loaded, evicted;   // totals
};
struct CacheWork {
  uint32_t *hits;        // == page_hits
  float *score, *score_sorted;
  uint32_t *ids, *ids_sorted, *fa, *fe, *sa, *se, *admit;
  void *temp;
  size_t temp_bytes;
  CachePlan *plan;       // device
  CachePlan *h_plan;     // pinned host copy (read after a synchronisation)
};
struct CachePages {
  const uint32_t *h_out, *h_in;  // host arena words (device-mapped)
  uint32_t pages_out, page_shift, stride;
  uint32_t *cdst;
};
size_t cache_temp_bytes(uint32_t npages);
cudaError_t cache_rank(CacheWork &W, uint32_t npages, uint32_t K, float decay, float min_score,
                       const uint32_t *page_slot, cudaStream_t s);
// plan (refresh gate, at most cap admissions), evict, stage; admissions and
// evictions are also added to the optional device counters. cache_plan and
// cache_stage are its two halves (the staging may run on another stream,
// ordered after the plan).
cudaError_t cache_plan(CacheWork &W, uint32_t npages, uint32_t gate, uint32_t cap,
                       u64 *stat_loaded, u64 *stat_evicted, cudaStream_t s);
cudaError_t cache_stage(CacheWork &W, uint32_t npages, uint32_t *page_slot, uint32_t *free_list,
                        const CachePages &pg, cudaStream_t s);
cudaError_t cache_apply(CacheWork &W, uint32_t npages, uint32_t gate, uint32_t cap,
                        uint32_t *page_slot, uint32_t *free_list, const CachePages &pg,
                        u64 *stat_loaded, u64 *stat_evicted, cudaStream_t s);

// cache given precomputed scores (W.score, W.ids filled): sort, flags, counts
cudaError_t cache_rank_given(CacheWork &W, uint32_t npages, uint32_t K, float min_score,
                             const uint32_t *page_slot, cudaStream_t s);

// learned admission policy (policy.cu)
constexpr int POLICY_F = 8, POLICY_H = 64;
constexpr int POLICY_PARAMS = POLICY_F * POLICY_H + POLICY_H + POLICY_H * POLICY_H + POLICY_H +
                              POLICY_H + 1;
size_t mlp_grad_smem();
// Row-layout features (rows starting in each page, longest of them). With
// period = {counter, every}: only when counter % every == 0 (device values).
cudaError_t launch_page_rows(const u64 *off, const uint32_t *len, uint32_t n, uint32_t page_base,
                             uint32_t page_shift, uint32_t *rows, uint32_t *maxlen,
                             const uint32_t *period, cudaStream_t s);
cudaError_t launch_page_rows_clear(uint32_t *rows, uint32_t *maxlen, uint32_t npages,
                                   const uint32_t *period, cudaStream_t s);
cudaError_t launch_period_step(uint32_t *period, cudaStream_t s);
cudaError_t launch_page_delta(const u64 *keys, uint32_t cnt, const u64 *off, uint32_t page_base,
                              uint32_t page_shift, uint32_t *delta, cudaStream_t s);
cudaError_t launch_features(const uint32_t *hits, const float *hist, const uint8_t *age,
                            const uint32_t *delta, const uint32_t *rows, const uint32_t *maxlen,
                            uint32_t npages, void *x, cudaStream_t s);
constexpr int POLICY_HORIZON = 3;  // training target: reads over this many snapshots
struct TargetRefs {
  float *t[POLICY_HORIZON];  // raw targets receiving this snapshot's reads (or null)
};
cudaError_t launch_history(uint32_t *hits, float *hist, uint8_t *age, uint32_t npages,
                           const TargetRefs &tg, bool clear, cudaStream_t s);
cudaError_t launch_log1p(const float *in, float *out, u64 n, cudaStream_t s);
// tcgen05 inference; err (optional) receives ERR_BARRIER if a tensor-core
// completion wait ran out
cudaError_t launch_mlp_infer(const void *x, uint32_t n, const float *params, float *score,
                             uint32_t *ids, uint32_t *err, cudaStream_t s);
// tcgen05 loss and gradient; err (optional) as for inference
cudaError_t launch_mlp_grad(const void *x, const float *y, uint64_t total, uint32_t count,
                            uint64_t sample_seed, const float *params, float scale, float *grad,
                            float *loss, uint32_t *err, cudaStream_t s);
cudaError_t launch_adam(float *p, float *g, float *m, float *v, float lr, uint32_t step,
                        cudaStream_t s);
cudaError_t sample_row_edges(const Adj &A, const uint32_t *sources, u64 count, u64 seed,
                             uint32_t n, uint32_t *out, cudaStream_t s);

// build
cudaError_t build_gen_rmat(u64 *keys, u64 draws, u64 seed, uint32_t scale, double a, double b,
                           double c, int symmetrize, cudaStream_t s);
cudaError_t build_gen_grid(u64 *keys, uint32_t side, u64 nshort, uint32_t radius, u64 seed,
                           cudaStream_t s);
cudaError_t build_csr_keys(const u64 *off, const uint32_t *dst, uint32_t n, u64 *keys,
                           cudaStream_t s);
cudaError_t build_swap_keys(const u64 *in, u64 *out, u64 count, cudaStream_t s);
cudaError_t build_sort(void *temp, size_t &bytes, u64 *k_in, u64 *k_out, uint32_t *v_in,
                       uint32_t *v_out, u64 count, cudaStream_t s);
cudaError_t build_scan_u32_to_u64(void *temp, size_t &bytes, const uint32_t *in, u64 *out,
                                  u64 count, cudaStream_t s);
cudaError_t build_scan_u64(void *temp, size_t &bytes, const u64 *in, u64 *out, u64 count,
                           cudaStream_t s);
cudaError_t build_unique(const u64 *k, const uint32_t *vin, u64 count, int dedup,
                         uint32_t *flag, u64 *pos, u64 *out, uint32_t *vout, void *temp,
                         size_t temp_bytes, cudaStream_t s);
cudaError_t build_degrees(const u64 *k, u64 m, uint32_t *deg, cudaStream_t s);
cudaError_t build_caps(const uint32_t *deg, uint32_t n, u64 *cap64, uint32_t *cap,
                       uint32_t *len, uint32_t *srt, uint32_t *live, cudaStream_t s);
cudaError_t build_scatter(const u64 *k, const uint32_t *wv, u64 m, const u64 *off,
                          const u64 *rowstart, uint32_t *hwords, uint32_t stride, uint32_t *fence,
                          uint32_t fence_shift, u64 wseed, uint32_t wlo, uint32_t whi,
                          int weight_from_hash, int swapped, cudaStream_t s);
size_t build_temp_bytes(u64 count, bool pairs);
cudaError_t sample_draw(u64 *pos, u64 count, u64 seed, u64 total, cudaStream_t s);
cudaError_t sample_resolve(const u64 *pos, u64 count, const u64 *pre, uint32_t n, const Adj &A,
                           uint32_t *out, cudaStream_t s);

}  // namespace dycg
