"""Parity at the workloads' full sizes (one snapshot each), against
from-scratch static recomputes on the host cores:

  * road-like grid 4096x4096 + 1% shortcuts within radius 8, HBM graph budget
    256 MB, one 10K-update snapshot (70% of the deletions on grid edges):
    SSSP (weights [1,1000], ordered closure, delta 2048), BFS and CC (ordered,
    delta 1); the library's grid generator equals the host restatement the
    reference arm repairs, edge for edge;
  * R-MAT scale 26 (67.1M vertices, ~1.07B edges), HBM graph budget 4 GB, one
    100K-update snapshot: BFS; CC on the symmetrised graph with symmetric
    updates; PageRank (epsilon 1e-4, FP32) against the FP64 restatement of the
    reference's residual push started from the engine's state, with the
    reference's own acceptance bound and the errors reported.

Bit-exact for levels, distances and labels. Each test prints its figures.
DYCG_CONFIG_SCALE_SHIFT=k shrinks every workload by 2^k vertices (quick
runs); the default is the full size.
"""
import os
import time

import numpy as np
import pytest

import dycgraph_b200 as dg

pytestmark = pytest.mark.gpu
SHIFT = int(os.environ.get("DYCG_CONFIG_SCALE_SHIFT", "0"))
GRID_LOG = 12 - SHIFT // 2
RMAT_SCALE = 26 - SHIFT
SEED = 20261203


def _grid_engine(algo):
    delta = 2048 if algo == "sssp" else 1
    e = dg.Engine(algo, weight_mode="stored" if algo == "sssp" else "hash128",
                  hbm_graph_budget_bytes=256 << 20, ordered_delta=delta, device=0)
    e.load_grid(1 << GRID_LOG, 10, 8, seed=SEED, wlo=1, whi=1000)
    return e


def test_grid_generator_matches_restatement():
    import oracle
    e = _grid_engine("sssp")
    off, dst, w = e.csr()
    n, o2, d2, w2 = oracle.grid_csr(1 << GRID_LOG, 10, 8, SEED, 1, 1000, with_w=True)
    e.close()
    print(f"[GRID-GEN] n={n} m={len(d2)}")
    assert n == len(off) - 1
    assert np.array_equal(off, o2) and np.array_equal(dst, d2) and np.array_equal(w, w2)


@pytest.mark.parametrize("algo", ["sssp", "bfs", "cc"])
def test_grid_snapshot_matches_static_recompute(algo):
    import bench
    import oracle
    e = _grid_engine(algo)
    t0 = time.time()
    e.start()
    t_init = time.time() - t0
    (d, a), = bench.make_batches(GRID_LOG, 1, 5000, 5000, SEED + 17, e.sample_edges, "grid", 1000)
    st = e.apply_batch(d, a)
    vals, _ = e.gather()
    off, dst, w = e.csr()
    n = e.n
    e.close()
    t0 = time.time()
    if algo == "sssp":
        ref = oracle.static_sssp(n, off, dst, w, oracle.WEIGHT_STORED, 0)
    elif algo == "bfs":
        ref = oracle.static_bfs(n, off, dst, 0)
    else:
        ref = oracle.static_cc(n, off, dst)
    print(f"[GRID-{algo.upper()}] n={n} init_s={t_init:.1f} snapshot_ms={st['ms_total']:.1f} "
          f"affected={st['affected']} waves={st['waves']} oracle_s={time.time() - t0:.1f} "
          f"mismatches={int(np.sum(vals != ref))}")
    assert np.array_equal(vals, ref)


def _rmat_engine(algo, **kw):
    e = dg.Engine(algo, weight_mode="hash128", hbm_graph_budget_bytes=4 << 30,
                  symmetric=(algo == "cc"), epsilon=1e-4, device=0, **kw)
    e.load_rmat(RMAT_SCALE, 16, seed=SEED, wlo=1, whi=64, symmetrize=(algo == "cc"))
    e.start()
    return e


def _rmat_snapshot(e, algo):
    import bench
    (d, a), = bench.make_batches(RMAT_SCALE, 1, 50_000, 50_000, SEED + 17, e.sample_edges)
    if algo == "cc":  # symmetric updates on the symmetrised graph
        d = np.concatenate([d, d[:, [1, 0, 2]]])
        a = np.concatenate([a, a[:, [1, 0, 2]]])
    return d, a


@pytest.mark.parametrize("algo", ["bfs", "cc"])
def test_rmat26_snapshot_matches_static_recompute(algo):
    import oracle
    e = _rmat_engine(algo)
    d, a = _rmat_snapshot(e, algo)
    st = e.apply_batch(d, a)
    vals, _ = e.gather()
    off, dst, _ = e.csr()
    n = e.n
    e.close()
    t0 = time.time()
    ref = oracle.static_bfs(n, off, dst, 0) if algo == "bfs" else oracle.static_cc(n, off, dst)
    print(f"[RMAT{RMAT_SCALE}-{algo.upper()}] n={n} m={len(dst)} snapshot_ms={st['ms_total']:.2f} "
          f"affected={st['affected']} oracle_s={time.time() - t0:.1f} "
          f"mismatches={int(np.sum(vals != ref))}")
    assert np.array_equal(vals, ref)


def test_rmat26_pagerank_snapshot_within_reference_bound():
    """The FP64 restatement of the reference's residual push takes the
    engine's ranks and residuals (a from-scratch FP64 solve of a billion-edge
    graph would not fit the run), both repair the same 100K-update snapshot at
    epsilon 1e-4, and the FP32 ranks must be within the sum of the two runs'
    residual bounds |r|_1 / (1 - alpha) (plus FP32 rounding, 1e-4 relative);
    the reference's own L1 bound (n * eps + roundoff) / 0.15
    (samples/hybrid_pr/hybrid_pr_host.cu:47-52) must hold between them too."""
    import oracle
    e = _rmat_engine("pr", max_rounds=100)
    d, a = _rmat_snapshot(e, "pr")
    off, dst, _ = e.csr()
    x0, r0 = e.gather_ranks()
    orc = oracle.Oracle(oracle.PR, e.n, off, dst, None, epsilon=1e-4, alpha=0.85, max_rounds=100,
                        threads=os.cpu_count() or 1)
    orc.set_state(ranks=x0.astype(np.float64), residuals=r0.astype(np.float64))
    del off, dst
    st = e.apply_batch(d, a)
    orc.apply_batch(d, a)
    xg, rg = e.gather_ranks()
    n = e.n
    e.close()
    xo, ro = orc.ranks()
    diff = np.abs(xg.astype(np.float64) - xo)
    bound = (float(np.sum(np.abs(rg.astype(np.float64)))) + float(np.sum(np.abs(ro)))) / 0.15 \
        + 1e-4 * np.abs(xo)
    mass = float(np.sum(np.abs(xo)))
    roundoff = 64 * float(np.finfo(np.float32).eps) * max(1.0, mass)
    l1_bound = (n * 1e-4 + roundoff) / 0.15
    print(f"[RMAT{RMAT_SCALE}-PR] n={n} snapshot_ms={st['ms_total']:.1f} max_abs={diff.max():.3e} "
          f"max_abs_normalized={diff.max() / n:.3e} l1={diff.sum():.3e} l1_bound={l1_bound:.3e} "
          f"max_residual={float(np.abs(rg).max()):.3e}")
    assert (diff <= bound).all()
    assert float(diff.sum()) <= l1_bound
    assert float(np.abs(rg).max()) <= float(np.float32(1e-4)) * 1.0001
