"""dycgraph_b200 -- B200-native streaming delta repair (SSSP / BFS / CC / PageRank).

The compute path is libdycg.so (hand-written CUDA for sm_100a behind the C ABI
in include/dycg.h). This package is the host-side mirror of the reference's
engine and operator interface: `Engine` keeps the reference Engine's method
names (LoadGraph, Start, del_edge, add_edge, LoadCache, GatherValue, ...) and
`operators` restates the AppBase traits. There is no CPU fallback: importing
works without a GPU, but creating an engine fails loudly when the library or
a CUDA device is missing.
"""
from .engine import (  # noqa: F401
    Engine, DycgError, BatchStats, GraphInfo, Edge, lib, library_path, edges_array,
    gen_rmat_edges, hash_weight, measure_host_link, measure_host_random, measure_host_sweep, mlp_infer, mlp_loss_grad,
    ALGOS, STATUS, POLICY_F, POLICY_H, POLICY_PARAMS, CTL_BYTES,
)
from . import operators  # noqa: F401

__all__ = ["Engine", "DycgError", "BatchStats", "GraphInfo", "Edge", "lib", "library_path",
           "edges_array", "gen_rmat_edges", "hash_weight", "operators", "ALGOS", "STATUS"]
