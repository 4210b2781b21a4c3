// engine.h -- host-side engine behind the C ABI (include/dycg.h).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/dycg.h"
#include "internal.h"

namespace dycg {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// A text edge list parsed on the host (shared by Engine::load_file and the
// text-to-binary converter).
struct TextGraph {
  uint32_t n = 0;
  uint64_t m = 0;
  std::vector<uint64_t> off;
  std::vector<uint32_t> dst, w;
};
TextGraph parse_text_graph(const char *path, uint32_t min_nodes, int weighted);

// One adjacency direction: a pinned, mapped host arena plus its descriptors.
struct Arena {
  uint32_t *h_dst = nullptr;  // host address of the slot words
  uint32_t *d_dst = nullptr;  // device-mapped address of the same words
  uint32_t stride = 1;        // words per slot: 1 (id) or 2 (id, weight)
  uint32_t fence_shift = 5;   // one fence per 128 bytes of slots
  uint32_t *tbits = nullptr;  // HBM deletion bitmap
  u64 slots = 0;
  uint32_t pages = 0, page_base = 0;
  u64 *off = nullptr;
  uint32_t *len = nullptr, *cap = nullptr, *srt = nullptr, *live = nullptr;
  u64 *top = nullptr;
  uint32_t *fence = nullptr;  // HBM fence index (id of every 32nd slot)
};

class Engine {
 public:
  explicit Engine(const dycg_options &opt);
  ~Engine();

  void load_csr(uint32_t n, const uint64_t *off, const uint32_t *dst, const uint32_t *w);
  void load_file(const char *path, uint32_t min_nodes, int weighted);
  void load_binary(const char *path);
  void load_rmat(uint32_t scale, uint32_t ef, double a, double b, double c, uint64_t seed,
                 uint32_t wlo, uint32_t whi, int symmetrize);
  void load_grid(uint32_t side, uint32_t permille, uint32_t radius, uint64_t seed, uint32_t wlo,
                 uint32_t whi);
  void init();
  // mode: 0 fused batch, 1 deletions only, 2 insertions only
  void apply(const dycg_edge *dels, size_t nd, const dycg_edge *adds, size_t na, bool device_ptrs,
             int mode, bool maintenance, dycg_batch_stats *stats);
  void cache_maintenance(bool initial, dycg_batch_stats *stats);
  void reserve_batch(size_t max_records);
  void gather(uint32_t *values, uint32_t *parents);
  void gather_ranks(float *ranks, float *residuals);
  void get_row(uint32_t v, int incoming, uint32_t *dst, uint32_t *w, uint32_t cap, uint32_t *deg);
  void export_csr(uint64_t *off, uint32_t *dst, uint32_t *w);
  void info(dycg_graph_info *out);
  void sample_edges(uint64_t count, uint64_t seed, dycg_edge *out);
  // many-query forms (SSSP/BFS): set after loading, before init
  void set_queries(const uint32_t *sources, uint32_t count, uint32_t mode);
  void set_query_mapping(uint32_t qratio, uint32_t heavy, uint32_t tile);
  void set_query_queue(uint32_t scheme);
  void gather_query(uint32_t q, uint32_t *values, uint32_t *parents);
  void tune(const dycg_edge *dels, size_t nd, const dycg_edge *adds, size_t na,
            dycg_query_mapping *tried, uint32_t cap, uint32_t *n_tried, dycg_batch_stats *stats);
  void apply_batches(const dycg_edge *dels, const uint64_t *nd, const dycg_edge *adds,
                     const uint64_t *na, uint32_t count, bool device_ptrs, dycg_batch_stats *stats);
  uint32_t queries() const { return nq_; }
  // learned cache admission
  void set_cache_policy(uint32_t policy);
  void policy_trace(uint32_t snapshots);
  void policy_train(uint32_t epochs, float lr, uint32_t batch, uint64_t seed,
                    dycg_policy_report *rep);
  void policy_params(float *out);
  void policy_set_params(const float *in);
  void sample_row_edges(const uint32_t *sources, uint64_t count, uint64_t seed, dycg_edge *out);
  cudaStream_t stream() const { return st_; }
  // make the engine stream wait for side-stream page staging (every call
  // that reads adjacency or the page table starts with this)
  void join() { join_staging(); }

  std::string last_error;
  bool failed = false;

 private:
  void check_loaded() const;
  void build_from_sorted_keys(u64 *keys, uint32_t *wv, u64 m, bool weight_from_hash, u64 wseed,
                              uint32_t wlo, uint32_t whi, u64 *scratch_keys, uint32_t *scratch_w);
  void build_direction(Arena &A, const u64 *keys, const uint32_t *wv, u64 m, bool weight_from_hash,
                       u64 wseed, uint32_t wlo, uint32_t whi, bool swapped);
  void finish_load();
  void ensure_batch(size_t cnt);
  Adj adj(const Arena &A) const;
  void sync_check(const char *where);
  void fill_stats(dycg_batch_stats *s, float ms[4]);
  void enqueue_snapshot(const dycg_edge_dev *d_dels, size_t nd, const dycg_edge_dev *d_adds,
                        size_t na, bool capture);
  void tune_repair(uint32_t nd, uint32_t na, u64 timeout);
  struct SnapshotGraph {
    cudaGraphExec_t exec;
    uint64_t kernels;
  };
  const SnapshotGraph &graph_for(uint32_t cls);
  void drop_graphs();
  void policy_alloc();
  void delete_direction(const Adj &A, const uint2 *uv, const uint32_t *mult,
                        const uint32_t *n_ptr, uint32_t nd, uint32_t *found, int count_missing,
                        bool capture);
  void policy_prefetch(size_t nd, size_t na, bool capture);
  void hotness_round(bool initial, bool side = false);
  void join_staging();
  void maintenance_device();
  void init_queries(u64 timeout);
  void repair_queries(uint32_t nd, uint32_t na, u64 timeout);
  MultiLaunch multi_launch(uint32_t phases, uint32_t n_add, u64 timeout);
  void *dmalloc(size_t bytes);
  void dfree_all();

  dycg_options opt_;
  int dev_ = 0, num_sms_ = 148;
  uint32_t mut_ctas_ = 148;  // CTAs of the warp-per-record mutation kernels
  cudaStream_t st_ = nullptr;
  cudaEvent_t ev_[6] = {};
  // side stream of the hotness path's page staging (eviction, admission list,
  // fills), overlapped with the next call's staging and ingest; joined
  // before anything reads the page table or the cached pages again
  cudaStream_t fst_ = nullptr;
  cudaEvent_t fev_[2] = {};
  bool staging_ = false;
  uint32_t n_ = 0;
  bool loaded_ = false, inited_ = false, has_in_ = false, stored_ = false;
  Arena out_, in_;
  std::vector<void *> dallocs_;
  std::vector<void *> hallocs_;

  // cache
  uint32_t page_shift_ = 12, npages_ = 0, cache_slots_ = 0;
  uint32_t *page_slot_ = nullptr, *page_hits_ = nullptr, *cdst_ = nullptr, *free_list_ = nullptr;
  CacheWork cwk_{};
  u64 index_bytes_ = 0;

  // vertex state
  u64 *key_ = nullptr;
  uint32_t *mark_ = nullptr, *wtag_ = nullptr, *aff_ = nullptr, *q0_ = nullptr, *q1_ = nullptr,
           *q2_ = nullptr, *touch_ = nullptr;
  uint4 *tiles_ = nullptr;
  uint32_t tile_cap_ = 0;
  Ctl *ctl_ = nullptr, *h_ctl_ = nullptr;
  float *x_ = nullptr, *r_ = nullptr, *delta_ = nullptr;
  uint32_t *queued_ = nullptr;
  uint32_t pr_cur_ = 0, pr_count_ = 0;
  uint32_t epoch_ = 0, tag_base_ = 1, touch_epoch_ = 0;

  // many-query forms: batched (one launch, vertex-major keys) or per query
  // (one single-source launch per query, query-major keys)
  uint32_t nq_ = 0, qmode_ = 0, qnb_ = 0;
  uint32_t *d_sources_ = nullptr;
  std::vector<uint32_t> sources_;
  u64 *qkey_ = nullptr;
  uint32_t *affm_ = nullptr, *inew_[2] = {}, *nmask_[2] = {}, *cmask_ = nullptr;
  uint32_t *seq_ = nullptr, *h_seq_ = nullptr;  // device {epoch, next wave tag}
  Ctl *qctl_ = nullptr, *h_qctl_ = nullptr;     // per-query control blocks
  uint4 *mtiles_ = nullptr;
  uint32_t mtile_cap_ = 0;
  // asynchronous worklist of the batched form (DYCG_QUEUE_ASYNC)
  u64 *aring_ = nullptr;
  uint32_t aring_cap_ = 0, apool_cap_ = 0;
  uint32_t *ainq_ = nullptr, *apool_ = nullptr;
  uint32_t qratio_ = 4, heavy_ = 64, tile_ = 4096, pull_qratio_ = 4, sched_ = 0;
  u64 qbytes_ = 0;
  bool tune_ = false;
  std::vector<dycg_query_mapping> tried_;
  // multi-snapshot replay: one graph per padded batch-size class
  std::map<uint32_t, SnapshotGraph> graphs_;
  std::vector<cudaEvent_t> bev_;
  Ctl *h_bctl_ = nullptr;
  uint32_t bctl_cap_ = 0;
  void *h_rec_ = nullptr, *d_rec_ = nullptr;
  u64 hrec_bytes_ = 0;

  // learned cache admission (policy.cu): features, history, network, traces
  uint32_t policy_ = 0;
  void *feat_ = nullptr;
  float *hist_ = nullptr;
  uint8_t *age_ = nullptr;
  uint32_t *prows_ = nullptr, *pmax_ = nullptr, *pdelta_ = nullptr;
  float *params_ = nullptr, *grad_ = nullptr, *adam_m_ = nullptr, *adam_v_ = nullptr,
        *ploss_ = nullptr;
  uint32_t adam_step_ = 0;
  void *tx_ = nullptr;
  float *ty_ = nullptr;
  uint32_t trace_cap_ = 0, trace_n_ = 0, trace_post_ = 0;
  bool trace_pending_ = false, prefetched_ = false;
  uint32_t learned_cap_div_ = 256;
  uint32_t *pperiod_ = nullptr;  // device {snapshot counter, refresh period} of the layout features
  cudaEvent_t pev_[2] = {};
  u64 policy_bytes_ = 0;

  // batch buffers
  size_t bcap_ = 0;
  u64 *k_tmp_out_ = nullptr, *k_tmp_in_ = nullptr, *k_del_out_ = nullptr, *k_del_in_ = nullptr,
      *k_add_out_ = nullptr, *k_add_in_ = nullptr;
  uint32_t *w_tmp_ = nullptr, *w_add_out_ = nullptr, *w_add_in_ = nullptr;
  uint2 *uv_out_ = nullptr, *uv_in_ = nullptr;
  uint32_t *mult_out_ = nullptr, *mult_in_ = nullptr, *found_out_ = nullptr;
  uint3 *seg_out_ = nullptr, *seg_in_ = nullptr, *add_uvw_ = nullptr;
  uint32_t *touched_ = nullptr, *counts_ = nullptr;
  RunScratch runs_{};  // run finder scratch (unique deletions, row segments)
  Reloc reloc_{};
  Tombs tombs_{};
  DeferDel defer_{};
  void ensure_defer(u64 slots);
  DeferBufs dbufs_{};
  u64 dbuf_cap_ = 0;
  u64 *h_dpacked_ = nullptr;  // pinned
  dycg_edge_dev *d_edges_ = nullptr;
  dycg_edge *h_stage_ = nullptr;
  void *cub_temp_ = nullptr;
  size_t cub_bytes_ = 0;
  std::vector<void *> batch_allocs_;
  uint64_t launches_ = 0;
};

}  // namespace dycg
