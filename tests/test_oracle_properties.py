"""Properties of the CPU oracle on seeded random multigraphs (no GPU).

After every batch the oracle's incremental repair (deletion seeds, invalidation,
pull, insertion closure; residual push for PageRank) must equal a from-scratch
recompute on the mutated graph, and its adjacency must follow the chunk
store's occurrence semantics (include/framework/source_local_chunk_store.h:
685-739: a deletion removes one live occurrence of (u, v), a request without
one is counted as missing; appends add occurrences; all deletions of a batch
come before its insertions). These pin the oracle's repair against its own
static solvers on many more graphs than the golden fixtures hold.
"""
import collections

import numpy as np
import pytest

import oracle


def _w(u, v):
    # stored weights fixed per (u, v), so duplicate occurrences are
    # interchangeable and the occurrence multiset is well defined
    return int((u * 2654435761 + v * 40503) % 64) + 1


def _graph(n, m, rng):
    u = rng.integers(0, n, m)
    v = rng.integers(0, n, m)
    keep = u != v
    edges = [(int(a), int(b), _w(int(a), int(b))) for a, b in zip(u[keep], v[keep])]
    return edges


def _batch(n, live, rng, nd, na):
    """Deletions: live occurrences, repeats of one occurrence, absent pairs and
    out-of-range ids; insertions: new pairs, repeats of live pairs, invalid ids."""
    pool = list(live.elements())
    dels = [pool[i] for i in rng.choice(len(pool), size=min(nd, len(pool)), replace=False)]
    dels += dels[:3]  # second request for the same occurrence
    dels += [(int(a), int(b), _w(int(a), int(b))) for a, b in rng.integers(0, n, (4, 2)) if a != b]
    dels += [(n + 3, 0, 1)]
    adds = [(int(a), int(b), _w(int(a), int(b))) for a, b in rng.integers(0, n, (na, 2)) if a != b]
    adds += pool[:5]  # parallel occurrences of live edges
    adds += [(0, n, 1)]
    return dels, adds


def _apply_counter(live, dels, adds, n):
    missing = 0
    for u, v, w in dels:
        if u >= n or v >= n:
            continue
        if live[(u, v, w)] > 0:
            live[(u, v, w)] -= 1
            if not live[(u, v, w)]:
                del live[(u, v, w)]
        else:
            missing += 1
    for u, v, w in adds:
        if u < n and v < n:
            live[(u, v, w)] += 1
    return missing


def _rows(off, dst, w, n):
    c = collections.Counter()
    for u in range(n):
        for k in range(int(off[u]), int(off[u + 1])):
            c[(u, int(dst[k]), int(w[k]))] += 1
    return c


def _static(algo, n, off, dst, w, mode):
    if algo == oracle.SSSP:
        return oracle.static_sssp(n, off, dst, w, mode, 0)
    if algo == oracle.BFS:
        return oracle.static_bfs(n, off, dst, 0)
    return oracle.static_cc(n, off, dst)


@pytest.mark.parametrize("algo,mode", [(oracle.SSSP, oracle.WEIGHT_HASH128),
                                       (oracle.SSSP, oracle.WEIGHT_STORED),
                                       (oracle.BFS, oracle.WEIGHT_HASH128),
                                       (oracle.CC, oracle.WEIGHT_HASH128)])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_incremental_repair_equals_recompute(algo, mode, seed):
    rng = np.random.default_rng(seed * 10 + algo)
    n = 150
    # CC on a sparse graph, so that batches split and merge labelled regions
    m, k = (200, 20) if algo == oracle.CC else (600, 40)
    edges = _graph(n, m, rng)
    off, dst, w = oracle.csr_from_edges(n, edges)
    orc = oracle.Oracle(algo, n, off, dst, w if mode == oracle.WEIGHT_STORED else None,
                        weight_mode=mode, source=0)
    orc.init()
    live = collections.Counter(edges)
    for _ in range(6):
        dels, adds = _batch(n, live, rng, k, k)
        want_missing = _apply_counter(live, dels, adds, n)
        orc.apply_batch(dels, adds)
        st = orc.stats()
        assert st["invalid_updates"] == 2
        assert st["missing_deletes"] == want_missing
        o, d, ww = orc.csr()
        got = _rows(o, d, ww, n) if mode == oracle.WEIGHT_STORED else \
            collections.Counter({(a, b, _w(a, b)): c for (a, b, _), c in _rows(o, d, ww, n).items()})
        assert got == live
        vals, par = orc.values()
        ref = _static(algo, n, o, d, ww if mode == oracle.WEIGHT_STORED else None, mode)
        assert (vals == ref).all()
        if algo == oracle.CC:
            continue
        # every reachable non-root vertex names a parent through a live, tight edge
        for v in range(1, n):
            if vals[v] == oracle.INF:
                assert par[v] == oracle.INF
                continue
            p = int(par[v])
            row = [(int(d[j]), int(ww[j])) for j in range(int(o[p]), int(o[p + 1]))]
            if algo == oracle.BFS:
                assert any(x == v for x, _ in row) and vals[p] + 1 == vals[v]
            elif mode == oracle.WEIGHT_STORED:
                assert any(x == v and vals[p] + wt == vals[v] for x, wt in row)
            else:
                assert any(x == v for x, _ in row) and vals[p] + (p + v) % 128 + 1 == vals[v]


def test_batch_of_only_missing_or_invalid_records_changes_nothing():
    rng = np.random.default_rng(5)
    n = 80
    edges = _graph(n, 300, rng)
    off, dst, w = oracle.csr_from_edges(n, edges)
    orc = oracle.Oracle(oracle.SSSP, n, off, dst, source=0)
    orc.init()
    before = orc.values()[0].copy()
    present = set((a, b) for a, b, _ in edges)
    absent = [(a, b, 1) for a in range(n) for b in range(n) if a != b and (a, b) not in present][:10]
    orc.apply_batch(absent + [(n, 1, 1)], [(1, n + 7, 1)])
    st = orc.stats()
    assert st["missing_deletes"] == 10 and st["invalid_updates"] == 2
    assert (orc.values()[0] == before).all()
    assert orc.live_edges() == len(edges)


@pytest.mark.parametrize("seed", [1, 2])
def test_incremental_pagerank_matches_power_iteration(seed):
    rng = np.random.default_rng(seed)
    n = 120
    edges = _graph(n, 500, rng)
    off, dst, _ = oracle.csr_from_edges(n, edges)
    orc = oracle.Oracle(oracle.PR, n, off, dst, epsilon=1e-12, max_rounds=1_000_000)
    orc.init()
    live = collections.Counter(edges)
    for _ in range(4):
        dels, adds = _batch(n, live, rng, 30, 30)
        _apply_counter(live, dels, adds, n)
        orc.apply_batch(dels, adds)
        o, d, _ = orc.csr()
        x, r = orc.ranks()
        ref = oracle.static_pr(n, o, d)
        # residual push to a per-vertex threshold of 1e-12: the remaining error
        # is bounded by |r|_1 / (1 - alpha)
        bound = float(np.sum(np.abs(r))) / 0.15 + 1e-9 * np.abs(ref) + 1e-12
        assert (np.abs(x - ref) <= bound).all(), float(np.max(np.abs(x - ref) - bound))
