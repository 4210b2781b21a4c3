"""The oracle's host-side workload builders (no GPU): the road-like grid and
the symmetrised R-MAT that the CPU reference arm repairs, the stored-weight
hash they share with the library, and parents derived from static distances."""
import numpy as np
import pytest

import dycgraph_b200 as dg
import oracle


def _edges(n, off, dst):
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(off.astype(np.int64)))
    return src, dst.astype(np.int64)


def test_hash_weights_match_the_library():
    rng = np.random.default_rng(3)
    u = rng.integers(0, 1 << 30, 500)
    v = rng.integers(0, 1 << 30, 500)
    for seed, lo, hi in ((0, 1, 64), (20261203, 1, 1000), ((1 << 64) - 1, 7, 7)):
        got = oracle.hash_weights(seed, u, v, lo, hi)
        want = [dg.engine.hash_weight(seed, int(a), int(b), lo, hi) for a, b in zip(u, v)]
        assert (got == np.array(want)).all()


@pytest.mark.parametrize("side,seed", [(32, 1), (57, 9)])
def test_grid_structure(side, seed):
    n, off, dst, w = oracle.grid_csr(side, 10, 8, seed, 1, 1000)
    assert n == side * side and off[0] == 0 and off[-1] == len(dst) == len(w)
    src, d = _edges(n, off, dst)
    # rows sorted and free of duplicates and self-loops
    key = src * n + d
    assert (np.diff(key) > 0).all() and (src != d).all()
    # every 4-neighbour edge, in both directions
    es = set(key.tolist())
    for u in range(n):
        r, c = divmod(u, side)
        for v, ok in ((u + 1, c + 1 < side), (u + side, r + 1 < side)):
            if ok:
                assert u * n + v in es and v * n + u in es
    # the rest are shortcuts within Chebyshev radius 8, present in both directions
    dr = np.abs(src // side - d // side)
    dc = np.abs(src % side - d % side)
    grid = (dr + dc) == 1
    assert (np.maximum(dr, dc)[~grid] <= 8).all() and (~grid).sum() > 0
    assert all(int(b) * n + int(a) in es for a, b in zip(src[~grid], d[~grid]))
    assert (w == oracle.hash_weights(seed, src, d, 1, 1000)).all()
    assert w.min() >= 1 and w.max() <= 1000
    n2, off2, dst2, _ = oracle.grid_csr(side, 10, 8, seed, 1, 1000)
    assert (off2 == off).all() and (dst2 == dst).all()


def test_symmetrised_rmat_is_the_draws_and_their_reverses():
    n, off, dst, _ = oracle.rmat_csr(11, 8, 4, with_w=False)
    ns, offs, dsts, _ = oracle.rmat_csr(11, 8, 4, with_w=False, symmetrize=True)
    a = set((_edges(n, off, dst)[0] * n + _edges(n, off, dst)[1]).tolist())
    s, d = _edges(ns, offs, dsts)
    b = set((s * n + d).tolist())
    assert b == a | {(x % n) * n + x // n for x in a}


@pytest.mark.parametrize("algo,mode", [(oracle.SSSP, oracle.WEIGHT_STORED),
                                       (oracle.SSSP, oracle.WEIGHT_HASH128),
                                       (oracle.BFS, oracle.WEIGHT_HASH128)])
def test_tight_parents_equal_the_parallel_solver(algo, mode):
    n, off, dst, w = oracle.grid_csr(96, 10, 8, 2, 1, 1000)
    wv = w if mode == oracle.WEIGHT_STORED else None
    v1, p1 = oracle.parallel_sssp(n, off, dst, wv, algo, mode, 0)
    v2 = (oracle.static_sssp(n, off, dst, wv, mode, 0) if algo == oracle.SSSP
          else oracle.static_bfs(n, off, dst, 0))
    assert (v1 == v2).all()
    assert (oracle.tight_parents(n, off, dst, wv, algo, mode, 0, v2) == p1).all()
