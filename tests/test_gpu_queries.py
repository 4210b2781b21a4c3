"""GPU parity of the many-query forms (dycg_set_queries): after the static
solve and after every snapshot, each query's distances / levels must equal a
from-scratch static recompute (Dijkstra / FIFO BFS from that query's source)
on the oracle's copy of the graph, bit for bit, and every parent must be a
live, tight in-edge. The batched form and the per-query form must agree."""
import numpy as np
import pytest

import dycgraph_b200 as dg
import oracle
from tests import cases

pytestmark = pytest.mark.gpu

INF = 0xFFFFFFFF
ALGO = {"sssp": oracle.SSSP, "bfs": oracle.BFS}


def static(algo, n, off, dst, w, stored, src):
    if algo == "bfs":
        return oracle.static_bfs(n, off, dst, src)
    return oracle.static_sssp(n, off, dst, w if stored else None,
                              oracle.WEIGHT_STORED if stored else oracle.WEIGHT_HASH128, src)


def tight_parents(algo, stored, off, dst, w, vals, par, src):
    """Count reachable non-source vertices whose parent is not a live tight in-edge."""
    n = len(vals)
    rows = np.repeat(np.arange(n), np.diff(off).astype(np.int64))
    weight = {}
    for u, v, x in zip(rows.tolist(), dst.tolist(), w.tolist()):
        wt = x if stored else cases.rule_w(ALGO[algo], u, v)
        weight.setdefault((u, v), set()).add(wt)
    bad = 0
    for v in range(n):
        if vals[v] == INF:
            bad += par[v] != INF
            continue
        if v == src:
            continue
        p = int(par[v])
        ok = p < n and any(int(vals[p]) + x == int(vals[v]) for x in weight.get((p, v), ()))
        bad += not ok
    return bad


def run_queries(algo, nq, mode, scale=10, batches=3, nd=300, na=300, seed=7, stored=False,
                budget=0, qratio=4, heavy=64, tile=4096, split=False, ef=8,
                parent_every=16, queue=None):
    n, off, dst, w = cases.small_rmat(scale, ef, seed)
    rng = np.random.default_rng(seed)
    # sources: distinct vertices with out-edges (plus vertex 0)
    cand = np.nonzero(np.diff(off) > 0)[0]
    sources = np.unique(np.concatenate([[0], rng.choice(cand, size=min(nq, len(cand)), replace=False)]))[:nq]
    sources = rng.permutation(sources)
    e = dg.Engine(algo, weight_mode="stored" if stored else "hash128",
                  hbm_graph_budget_bytes=budget, page_shift=8)
    e.load_csr(n, off, dst, w if stored else None)
    e.set_queries(sources, mode)
    if mode == "batched":
        e.set_query_mapping(qratio, heavy, tile)
        if queue is not None:
            e.set_query_queue(queue)
    e.start()
    orc = oracle.Oracle(ALGO[algo], n, off, dst, w if stored else None,
                        weight_mode=oracle.WEIGHT_STORED if stored else oracle.WEIGHT_HASH128)
    cur = (off, dst, w)

    def check(tag, parents):
        o, d, ww = cur
        for q, s in enumerate(sources):
            vals, par = e.gather_query(q)
            ref = static(algo, n, o, d, ww, stored, int(s))
            assert (vals == ref).all(), (tag, q, int(s), int(np.sum(vals != ref)))
            if parents and q % parent_every == 0:
                assert tight_parents(algo, stored, o, d, ww, vals, par, int(s)) == 0, (tag, q)

    check("init", True)
    for bi in range(batches):
        dels, adds = cases.random_batch(n, cur[0], cur[1], cur[2], nd, na, seed * 100 + bi)
        if not stored:
            dels = [(u, v, cases.rule_w(ALGO[algo], u, v)) for u, v, _ in dels]
            adds = [(u, v, cases.rule_w(ALGO[algo], u, v)) for u, v, _ in adds]
        if split:
            e.delete_edges(dels)
            orc.mutate(dels, [])
            cur = orc.csr()
            check(("delete", bi), False)
            e.insert_edges(adds)
            orc.mutate([], adds)
        else:
            e.apply_batch(dels, adds)
            orc.mutate(dels, adds)
        cur = orc.csr()
        check(bi, bi == batches - 1)
    return e, sources


@pytest.mark.parametrize("mode", ["batched", "per_query"])
@pytest.mark.parametrize("algo,stored", [("sssp", False), ("sssp", True), ("bfs", False)])
def test_queries_match_static(algo, stored, mode):
    run_queries(algo, 40, mode, stored=stored)


@pytest.mark.parametrize("qratio,heavy", [(0, 64), (1 << 20, 64), (4, 1), (4, 1 << 30)])
def test_batched_work_mappings(qratio, heavy):
    # qratio 0: every row on query lanes; 2^20: every row on edge lanes;
    # heavy 1: every row tiled (CTA splits); 2^30: no row tiled
    run_queries("sssp", 64, "batched", stored=True, qratio=qratio, heavy=heavy, seed=9)


@pytest.mark.parametrize("queue", ["static", "claimed", "ranges", "claimed+ranges", "async",
                                   "async+claimed"])
def test_batched_frontier_queue_schemes(queue):
    # every frontier-queue scheme (static or claimed items, plain or
    # range-ordered wave queues) gives the static recompute's results, heavy
    # rows and tiles included
    run_queries("sssp", 64, "batched", scale=12, ef=16, batches=2, nd=800, na=800, seed=21,
                stored=True, heavy=4, tile=1024, queue=queue, parent_every=32)


def test_batched_256_queries_split_phases():
    run_queries("bfs", 256, "batched", scale=9, batches=2, split=True, seed=11, parent_every=64)


def test_batched_few_queries_single_block():
    run_queries("sssp", 3, "batched", batches=3, seed=13)


def test_batched_heavy_rows_tiles_cached():
    # scale 14 R-MAT hubs exceed the 1024-slot heavy threshold: tile phase, HBM cache on
    n, off, dst, _ = cases.small_rmat(14, 16, 17)
    assert int(np.max(np.diff(off))) > 2 * 1024
    for qratio in (0, 1 << 20):
        run_queries("sssp", 32, "batched", scale=14, ef=16, batches=2, nd=1500, na=1500,
                    seed=17, stored=True, budget=1 << 20, qratio=qratio, heavy=64,
                    tile=1024, parent_every=32)


def test_batched_equals_per_query():
    a, src = run_queries("sssp", 24, "batched", batches=2, seed=19, stored=True)
    b, _ = run_queries("sssp", 24, "per_query", batches=2, seed=19, stored=True)
    for q in range(len(src)):
        assert (a.gather_query(q)[0] == b.gather_query(q)[0]).all()
    # with queries set, dycg_gather returns query 0
    assert (a.gather()[0] == a.gather_query(0)[0]).all()


def test_query_argument_errors():
    n, off, dst, w = cases.small_rmat(8, 4, 3)
    e = dg.Engine("sssp")
    e.load_csr(n, off, dst)
    for bad in ([], list(range(257))):
        with pytest.raises(dg.DycgError):
            e.set_queries(np.array(bad, np.uint32))
    with pytest.raises(dg.DycgError):
        e.set_queries([n])
    with pytest.raises(dg.DycgError):
        e.set_query_mapping(4, 0, 4096)
    with pytest.raises(dg.DycgError):
        e.set_query_mapping(4, 64, 512)
    e.set_queries([0, 1, 2])
    with pytest.raises(dg.DycgError):
        e.set_queries([0])
    e.start()
    with pytest.raises(dg.DycgError):
        e.gather_query(3)
    cc = dg.Engine("cc")
    cc.load_csr(n, off, dst)
    with pytest.raises(dg.DycgError):
        cc.set_queries([0])


def _engine_and_sources(scale, nq, seed, stored=True, mode="batched", budget=0):
    n, off, dst, w = cases.small_rmat(scale, 8, seed)
    rng = np.random.default_rng(seed)
    cand = np.nonzero(np.diff(off) > 0)[0]
    sources = rng.choice(cand, size=nq, replace=False).astype(np.uint32)
    e = dg.Engine("sssp", weight_mode="stored" if stored else "hash128",
                  hbm_graph_budget_bytes=budget, page_shift=8)
    e.load_csr(n, off, dst, w if stored else None)
    e.set_queries(sources, mode)
    e.start()
    return e, (n, off, dst, w), sources


def _check_all(e, n, csr_, sources):
    o, d, ww = csr_
    for q, s in enumerate(sources):
        ref = oracle.static_sssp(n, o, d, ww, oracle.WEIGHT_STORED, int(s))
        assert (e.gather_query(q)[0] == ref).all(), q


def test_tune_mapping_keeps_results():
    e, (n, off, dst, w), src = _engine_and_sources(11, 48, 23)
    orc = oracle.Oracle(oracle.SSSP, n, off, dst, w, weight_mode=oracle.WEIGHT_STORED)
    cur = (off, dst, w)
    dels, adds = cases.random_batch(n, *cur, 600, 600, 2301)
    tried = e.tune_query_mapping(dels, adds)
    orc.mutate(dels, adds)
    cur = orc.csr()
    # 20 (qratio x heavy) + 3-4 pull ratios + 2-3 tile sizes + 5 frontier-queue schemes
    assert 20 < len(tried) <= 32 and all(t["repair_ms"] > 0 for t in tried)
    assert {t["heavy"] for t in tried} >= {4, 8, 16, 64, 256}
    assert {t["tile"] for t in tried} == {1024, 4096, 16384}
    assert {t["queue"] for t in tried} == {0, 1, 2, 3, 4, 5}
    _check_all(e, n, cur, src)
    for bi in range(2):  # later snapshots under the kept mapping
        dels, adds = cases.random_batch(n, *cur, 400, 400, 2310 + bi)
        e.apply_batch(dels, adds)
        orc.mutate(dels, adds)
        cur = orc.csr()
    _check_all(e, n, cur, src)


@pytest.mark.parametrize("mode", ["batched", "per_query"])
def test_apply_batches_replay_matches_one_by_one(mode):
    # uneven snapshot sizes across three padding classes, classes replayed twice
    a, (n, off, dst, w), src = _engine_and_sources(11, 40, 29, mode=mode)
    b, _, _ = _engine_and_sources(11, 40, 29, mode=mode)
    orc = oracle.Oracle(oracle.SSSP, n, off, dst, w, weight_mode=oracle.WEIGHT_STORED)
    cur = (off, dst, w)
    for rnd, sizes in enumerate([(5, 700, 1500), (3000, 1, 900)]):
        snaps = []
        for i, sz in enumerate(sizes):
            dels, adds = cases.random_batch(n, *cur, sz // 2, sz - sz // 2, 2900 + 10 * rnd + i)
            snaps.append((dels, adds))
            orc.mutate(dels, adds)
            cur = orc.csr()
        stats = a.apply_batches(snaps)
        one = [b.apply_batch(d, ad) for d, ad in snaps]
        assert len(stats) == len(snaps)
        for s, o, (d, ad) in zip(stats, one, snaps):
            assert s["deletions"] == len(d) and s["insertions"] == len(ad)
            assert s["invalid_updates"] == 0
            assert s["missing_deletes"] == o["missing_deletes"]
            assert s["ms_total"] > 0
        _check_all(a, n, cur, src)
        for q in range(len(src)):
            assert (a.gather_query(q)[0] == b.gather_query(q)[0]).all()


def test_apply_batches_invalid_records_and_empty_snapshots():
    e, (n, off, dst, w), src = _engine_and_sources(10, 32, 31)
    orc = oracle.Oracle(oracle.SSSP, n, off, dst, w, weight_mode=oracle.WEIGHT_STORED)
    dels, adds = cases.random_batch(n, off, dst, w, 50, 50, 3101)
    bad = [(n + 5, 1, 3), (2, n, 4)]
    stats = e.apply_batches([([], []), (dels, adds + bad), ([], [])])
    assert stats[1]["invalid_updates"] == 2 and stats[0]["invalid_updates"] == 0
    orc.mutate(dels, adds)
    _check_all(e, n, orc.csr(), src)


@pytest.mark.parametrize("policy", ["hotness", "learned"])
def test_replayed_snapshots_with_cache_admission_inside_the_graph(policy):
    """Snapshots replayed from captured graphs with the cache admission
    (hotness round after the repair, or the learned admission between the
    mutation and the repair, with its page history) recorded inside each
    graph: results equal the static recompute and the one-by-one engine's, and
    pages are admitted along the way."""
    a, (n, off, dst, w), src = _engine_and_sources(12, 32, 37, budget=2 << 20)
    b, _, _ = _engine_and_sources(12, 32, 37, budget=2 << 20)
    if policy == "learned":
        # a network that predicts log1p(reads) = 10 for every page (above the
        # admission threshold log1p(64)), so pages are admitted every snapshot
        p = np.zeros(dg.POLICY_PARAMS, np.float32)
        p[-1] = 10.0
        a.policy_set_params(p)
        a.set_cache_policy("learned")
    orc = oracle.Oracle(oracle.SSSP, n, off, dst, w, weight_mode=oracle.WEIGHT_STORED)
    cur = (off, dst, w)
    loaded = 0
    for rnd in range(3):
        snaps = []
        for i, sz in enumerate((900, 2500, 40)):
            dels, adds = cases.random_batch(n, *cur, sz // 2, sz - sz // 2, 3700 + 10 * rnd + i)
            snaps.append((dels, adds))
            orc.mutate(dels, adds)
            cur = orc.csr()
        stats = a.apply_batches(snaps)
        loaded += sum(s["cache_pages_loaded"] for s in stats)
        for d, ad in snaps:
            b.apply_batch(d, ad)
    _check_all(a, n, cur, src)
    for q in range(len(src)):
        assert (a.gather_query(q)[0] == b.gather_query(q)[0]).all()
    info = a.info()
    assert 0 < info["cached_pages"] <= info["cache_slots"]
    if policy == "learned":
        assert loaded > 0
