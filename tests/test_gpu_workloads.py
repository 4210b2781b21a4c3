"""The benchmark's workload generators on the GPU: the CPU restatements the
reference arm uses (graph, edge sampler) give exactly the engine's graph and
snapshots."""
import numpy as np
import pytest

import dycgraph_b200 as dg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("stored", [True, False])
def test_engine_sampler_matches_its_restatement(stored):
    import bench
    import oracle
    e = dg.Engine("sssp" if stored else "bfs", weight_mode="stored" if stored else "hash128",
                  device=0)
    e.load_rmat(14, 16, seed=9, wlo=1, whi=64)
    n, off, dst, w = oracle.rmat_csr(14, 16, 9, wlo=1, whi=64, with_w=stored)
    o2, d2, w2 = e.csr()
    assert e.n == n and np.array_equal(o2, off) and np.array_equal(d2, dst)
    if stored:
        assert np.array_equal(w2, w)
    smp = bench._engine_sampler(off, dst, w if stored else None)
    for count, seed in ((1, 3), (5000, 17), (60_000, 18)):
        assert np.array_equal(e.sample_edges(count, seed), smp(count, seed)), (count, seed)
    e.close()
