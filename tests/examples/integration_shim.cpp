// The reference-side C++ shim of the integration guide, kept here so the
// CPU suite compiles it against include/dycg.h.
// dycg_engine_shim.h -- drop-in for the subset of sepgraph::engine::Engine the samples use.
#include "dycg.h"
#include <stdexcept>
#include <string>
#include <vector>

class DycgEngine {
 public:
  explicit DycgEngine(uint32_t algo, uint32_t source, uint64_t hbm_budget_bytes) {
    dycg_options o; dycg_options_default(&o);
    o.algo = algo; o.source = source;
    o.hbm_graph_budget_bytes = hbm_budget_bytes;
    o.cache_policy = hbm_budget_bytes ? DYCG_CACHE_HOTNESS : DYCG_CACHE_NONE;
    check(dycg_create(&o, &e_), "dycg_create");
  }
  ~DycgEngine() { dycg_destroy(e_); }
  void LoadGraph(const char* market_big_path) {            // Engine::LoadGraph :1569
    check(dycg_load_graph_file(e_, market_big_path, 0, 0), "LoadGraph");
  }
  void Start() { check(dycg_init(e_), "Start"); }          // InitGraph + Start :1803/:1963
  void del_edge(const dycg_edge* d, size_t n) {            // Engine::del_edge :2595
    check(dycg_delete_edges(e_, d, n, &last_), "del_edge");
  }
  void add_edge(const dycg_edge* a, size_t n) {            // Engine::add_edge :2419
    check(dycg_insert_edges(e_, a, n, &last_), "add_edge");
  }
  void LoadCache() { check(dycg_cache_maintenance(e_, &last_), "LoadCache"); }  // :1264-1567
  void Gather(std::vector<uint32_t>& value, std::vector<uint32_t>& parent, size_t n) {
    value.resize(n); parent.resize(n);                     // GatherValue/GatherParent :4959
    check(dycg_gather(e_, value.data(), parent.data()), "Gather");
  }
  const dycg_batch_stats& stats() const { return last_; }
 private:
  void check(int rc, const char* what) {
    if (rc == DYCG_OK) return;
    char buf[256]; dycg_last_error(e_, buf, sizeof buf);
    throw std::runtime_error(std::string(what) + ": " + buf);  // the reference aborted here
  }
  dycg_engine* e_ = nullptr;
  dycg_batch_stats last_{};
};
