/* The C example of the README, as a function (compiled by
 * tests/test_abi_layout_cpu.py against include/dycg.h). */
#include "dycg.h"
int example(const dycg_edge *dels, size_t nd, const dycg_edge *adds, size_t na,
            uint32_t *dist, uint32_t *parent) {
dycg_options o; dycg_options_default(&o);
o.algo = DYCG_ALGO_SSSP; o.hbm_graph_budget_bytes = 4ull << 30; o.cache_policy = DYCG_CACHE_HOTNESS;
dycg_engine *e; dycg_create(&o, &e);
dycg_load_graph_binary(e, "graph.bin");
dycg_init(e);                                  /* static solve on the GPU */
dycg_batch_stats st;
dycg_apply_batch(e, dels, nd, adds, na, &st);  /* deletions, insertions, repair, cache */
dycg_gather(e, dist, parent);
dycg_destroy(e);
  return 0;
}
