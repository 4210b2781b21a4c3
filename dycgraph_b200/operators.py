"""Host-side restatement of the reference's operator interface.

sepgraph::api::AppBase (include/framework/variants/api.cuh:22-174) and the
four sample operators define, per algorithm, the edge weight, the initial
value, the deletion-dependency rule and a few traits. On the device these
rules are compiled into libdycg's kernels (rule_weight, reset_key, the
parent test of the repair kernel); this module states them for users and
tests, with the same names.
"""
INF = 0xFFFFFFFF


class AppBase:
    kSupportsGpuDeletionRepair = False
    kComponentLabels = False
    kVertexSeeds = False
    kRootedDeletionWitness = False
    kSignedResidual = False
    algo = None

    @staticmethod
    def NormalizeUndirectedInput():
        return False

    @staticmethod
    def TraversalEdgeWeight(src, dst):
        # api.cuh:26-28
        return (src + dst) % 128 + 1

    @staticmethod
    def DeletionEdgeWeight(src, dst):
        return 1

    @staticmethod
    def IsDeletionDependency(src, dst, source, destination, candidate, parent, parent_tight):
        # api.cuh:42-49
        return parent == src or (source != INF and candidate == destination and not parent_tight)

    @staticmethod
    def GetInitValue(node, source=0):
        return INF


class SSSP(AppBase):
    """samples/hybrid_sssp/hybrid_sssp.cu:51-204"""
    kSupportsGpuDeletionRepair = True
    algo = "sssp"

    @staticmethod
    def DeletionEdgeWeight(src, dst):
        return (src + dst) % 128 + 1

    @staticmethod
    def GetInitBuffer(node, source=0):
        return 0 if node == source else INF


class BFS(SSSP):
    """samples/hybrid_bfs/hybrid_bfs.cu: unit weights."""
    algo = "bfs"

    @staticmethod
    def TraversalEdgeWeight(src, dst):
        return 1

    @staticmethod
    def DeletionEdgeWeight(src, dst):
        return 1


class CC(AppBase):
    """samples/hybrid_cc/hybrid_cc.cu:51-200: directed minimum-label propagation."""
    kSupportsGpuDeletionRepair = True
    kVertexSeeds = True
    kRootedDeletionWitness = True
    algo = "cc"

    @staticmethod
    def TraversalEdgeWeight(src, dst):
        return 0

    @staticmethod
    def DeletionEdgeWeight(src, dst):
        return 0

    @staticmethod
    def IsDeletionDependency(src, dst, source, destination, candidate=None, parent=None,
                             parent_tight=None):
        # hybrid_cc.cu:60-63
        return src != dst and source == destination and destination < dst

    @staticmethod
    def GetInitBuffer(node, source=0):
        return node


class PR(AppBase):
    """samples/hybrid_pr/hybrid_pr.cu:36-124 with include/framework/pr_residual.cuh."""
    kSignedResidual = True
    algo = "pr"
    kAlpha = 0.85
    kBase = 0.15


BY_NAME = {"sssp": SSSP, "bfs": BFS, "cc": CC, "pr": PR}
