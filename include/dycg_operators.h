/* dycg_operators.h -- the reference's operator interface as compile-time C++
 * structs (header-only, host and device).
 *
 * Replaces sepgraph::api::AppBase (include/framework/variants/api.cuh:22-174)
 * and the four sample operators (samples/hybrid_sssp/hybrid_sssp.cu:51-204,
 * samples/hybrid_bfs/hybrid_bfs.cu, samples/hybrid_cc/hybrid_cc.cu:51-200,
 * samples/hybrid_pr/hybrid_pr.cu:36-124) with the same names and rules, as
 * static members instead of device virtual functions. libdycg's repair
 * kernels take their edge-weight rule from TraversalEdgeWeight here
 * (ForAlgo<algo>). They keep value and parent in one 64-bit key. SSSP/BFS
 * deletions invalidate by the parent rule (parent == src). CC deletions
 * invalidate by recorded label parents instead of the reference's label test
 * below, and need no rooted witness search. The Python statement of the same
 * traits is dycgraph_b200/operators.py. */
#ifndef DYCG_OPERATORS_H
#define DYCG_OPERATORS_H

#include <stdint.h>

#if defined(__CUDACC__)
#define DYCG_HD __host__ __device__ __forceinline__
#else
#define DYCG_HD inline
#endif

namespace dycg_ops {

constexpr uint32_t kInfinity = 0xFFFFFFFFu;

struct AppBase {
  static constexpr bool kSupportsGpuDeletionRepair = false;
  static constexpr bool kComponentLabels = false;
  static constexpr bool kVertexSeeds = false;
  static constexpr bool kRootedDeletionWitness = false;
  static constexpr bool kSignedResidual = false;
  DYCG_HD static bool NormalizeUndirectedInput() { return false; }
  /* api.cuh:26-28 */
  DYCG_HD static uint32_t TraversalEdgeWeight(uint32_t src, uint32_t dst) {
    return (uint32_t)(((uint64_t)src + dst) % 128u + 1u);
  }
  DYCG_HD static uint32_t DeletionEdgeWeight(uint32_t, uint32_t) { return 1u; }
  /* api.cuh:42-49: dst depends on the deleted edge when src is its parent, or
   * when src's value delivered dst's value as a candidate that is not backed
   * by a tight parent */
  DYCG_HD static bool IsDeletionDependency(uint32_t src, uint32_t, uint32_t src_value,
                                           uint32_t dst_value, uint32_t candidate,
                                           uint32_t parent, bool parent_tight) {
    return parent == src || (src_value != kInfinity && candidate == dst_value && !parent_tight);
  }
  DYCG_HD static uint32_t GetInitValue(uint32_t, uint32_t) { return kInfinity; }
  DYCG_HD static uint32_t GetInitBuffer(uint32_t, uint32_t) { return kInfinity; }
};

struct SSSP : AppBase {
  static constexpr bool kSupportsGpuDeletionRepair = true;
  DYCG_HD static uint32_t DeletionEdgeWeight(uint32_t src, uint32_t dst) {
    return TraversalEdgeWeight(src, dst);
  }
  DYCG_HD static uint32_t GetInitBuffer(uint32_t node, uint32_t source) {
    return node == source ? 0u : kInfinity;
  }
};

struct BFS : SSSP {
  DYCG_HD static uint32_t TraversalEdgeWeight(uint32_t, uint32_t) { return 1u; }
  DYCG_HD static uint32_t DeletionEdgeWeight(uint32_t, uint32_t) { return 1u; }
};

/* directed minimum-label propagation: every vertex seeds its own id */
struct CC : AppBase {
  static constexpr bool kSupportsGpuDeletionRepair = true;
  static constexpr bool kVertexSeeds = true;
  static constexpr bool kRootedDeletionWitness = true;
  DYCG_HD static uint32_t TraversalEdgeWeight(uint32_t, uint32_t) { return 0u; }
  DYCG_HD static uint32_t DeletionEdgeWeight(uint32_t, uint32_t) { return 0u; }
  /* hybrid_cc.cu:60-63 */
  DYCG_HD static bool IsDeletionDependency(uint32_t src, uint32_t dst, uint32_t src_value,
                                           uint32_t dst_value, uint32_t, uint32_t, bool) {
    return src != dst && src_value == dst_value && dst_value < dst;
  }
  DYCG_HD static uint32_t GetInitBuffer(uint32_t node, uint32_t) { return node; }
};

/* unnormalised residual-push PageRank (include/framework/pr_residual.cuh) */
struct PR : AppBase {
  static constexpr bool kSignedResidual = true;
  static constexpr float kAlpha = 0.85f;
  static constexpr float kBase = 0.15f;
};

/* algorithm id (DYCG_ALGO_*) -> operator */
template <uint32_t A> struct ForAlgo;
template <> struct ForAlgo<0> { using type = SSSP; };
template <> struct ForAlgo<1> { using type = BFS; };
template <> struct ForAlgo<2> { using type = CC; };
template <> struct ForAlgo<3> { using type = PR; };

}  // namespace dycg_ops

#endif /* DYCG_OPERATORS_H */
