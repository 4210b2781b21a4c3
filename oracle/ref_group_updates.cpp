// ref_group_updates -- TEST INFRASTRUCTURE: runs the reference's own update
// grouping (sepgraph::topology::GroupedUpdateBatch,
// include/framework/effective_update_batch.h:36-207, compiled from the
// reference checkout by oracle/Makefile into oracle/_ref/) on a batch read
// from stdin, and prints each source group, so the tests can pin the grouping
// restatement that checks dycg_group_updates against the reference itself.
//
// stdin:  "nd na" then nd lines "u v" (deletions) and na lines "u v" (additions)
// stdout: per source group, in the class's order:
//           "S <source>"
//           "D <dst> <dst> ..."   deletions in the class's order
//           "A <dst> <dst> ..."   additions in the class's order
//         then "phases <sources with deletions> <sources with additions>".
#include <cstdio>
#include <framework/effective_update_batch.h>

int main() {
  using namespace sepgraph::topology;
  size_t nd = 0, na = 0;
  if (std::scanf("%zu %zu", &nd, &na) != 2) return 2;
  TopologyMutationBatch batch;
  batch.deletions.resize(nd);
  batch.additions.resize(na);
  for (auto *list : {&batch.deletions, &batch.additions})
    for (auto &m : *list) {
      unsigned long long u = 0, v = 0;
      if (std::scanf("%llu %llu", &u, &v) != 2) return 2;
      m.source = (index_t)u;
      m.destination = (index_t)v;
    }
  GroupedUpdateBatch g(batch);
  for (size_t i = 0; i < g.sources.size(); i++) {
    const SourceMutationView view = g.View(i, UpdatePhase::Mixed);
    std::printf("S %llu\nD", (unsigned long long)g.sources[i]);
    for (index_t v : view.deletions) std::printf(" %llu", (unsigned long long)v);
    std::printf("\nA");
    for (index_t v : view.additions) std::printf(" %llu", (unsigned long long)v);
    std::printf("\n");
  }
  std::printf("phases %zu %zu\n", g.PhaseSize(UpdatePhase::Delete), g.PhaseSize(UpdatePhase::Add));
  return 0;
}
