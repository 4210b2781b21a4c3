"""The CPU oracle against the reference's own golden vectors (no GPU)."""
import numpy as np
import pytest

import oracle
from tests import cases


def _phase_checksums(algo, case):
    n = case["n"]
    off, dst, _ = cases.csr(n, case["graph"])
    orc = oracle.Oracle(algo, n, off, dst, source=0)
    orc.init()
    out = []
    for b in case["batches"]:
        orc.delete_edges(cases.triples(b["dels"], algo))
        out.append(("delete", oracle.checksum(orc.values()[0])))
        orc.insert_edges(cases.triples(b["adds"], algo))
        out.append(("batch", oracle.checksum(orc.values()[0])))
    return out, orc


@pytest.mark.parametrize("algo,name", [(oracle.BFS, "bfs"), (oracle.SSSP, "sssp")])
def test_smoke_bfs_sssp_phase_checksums(algo, name):
    case = cases.load("smoke_bfs_sssp.json")
    got, orc = _phase_checksums(algo, case)
    want = [(e["phase"], e["checksum"]) for e in case["expected"][name]]
    assert got == want
    vals, par = orc.values()
    assert list(vals) == case["final_values"][name]
    # parents are tight witnesses of existing edges
    off, dst, _ = orc.csr()
    for v in range(case["n"]):
        if v == 0 or vals[v] == oracle.INF:
            continue
        p = int(par[v])
        row = dst[int(off[p]):int(off[p + 1])]
        assert v in row
        assert vals[p] + cases.rule_w(algo, p, v) == vals[v]


def test_smoke_cc_phase_checksums():
    case = cases.load("smoke_cc.json")
    got, orc = _phase_checksums(oracle.CC, case)
    want = [(e["phase"], e["checksum"]) for e in case["expected"]]
    assert got == want
    assert list(orc.values()[0]) == case["final_labels"]


def test_static_recompute_matches_golden():
    case = cases.load("smoke_bfs_sssp.json")
    n = case["n"]
    edges = {tuple(e) for e in case["graph"]}
    for b in case["batches"]:
        edges -= {tuple(e) for e in b["dels"]}
        edges |= {tuple(e) for e in b["adds"]}
    off, dst, _ = cases.csr(n, sorted(edges))
    assert list(oracle.static_bfs(n, off, dst, 0)) == case["final_values"]["bfs"]
    assert list(oracle.static_sssp(n, off, dst, None, oracle.WEIGHT_HASH128, 0)) == \
        case["final_values"]["sssp"]


def test_pr_smoke_static_and_incremental():
    case = cases.load("smoke_pr.json")
    n = case["n"]
    off, dst, _ = cases.csr(n, case["graph"])
    x0 = oracle.static_pr(n, off, dst)
    assert np.max(np.abs(x0 - np.array(case["initial_ranks"]))) < 1e-9
    eps = 1e-9
    orc = oracle.Oracle(oracle.PR, n, off, dst, epsilon=eps, max_rounds=100000)
    orc.init()
    for b in case["batches"]:
        orc.apply_batch(cases.triples(b["dels"]), cases.triples(b["adds"]))
    x, r = orc.ranks()
    fin = np.array(case["final_ranks"])
    # residual push leaves |r| <= eps per vertex: error <= sum|r| / (1 - alpha)
    bound = np.sum(np.abs(r)) / 0.15 + 1e-9
    assert np.max(np.abs(x - fin)) <= bound
    sx = oracle.static_pr(n, *orc.csr()[:2])
    assert np.max(np.abs(sx - fin)) < 1e-9


def test_pr_probe_reference_ranks():
    case = cases.load("pr_probe.json")
    ref = np.array(case["reference_ranks"])
    n = len(ref)
    off, dst, _ = cases.csr(n, case["graph"])
    batches = cases.replay_batches(case["updates"], case["sizes"])
    orc = oracle.Oracle(oracle.PR, n, off, dst, epsilon=1e-10, max_rounds=100000)
    orc.init()
    for dels, adds in batches:
        orc.apply_batch(cases.triples(dels), cases.triples(adds))
    x, _ = orc.ranks()
    assert np.max(np.abs(x - ref)) < 1e-8
    off2, dst2, _ = orc.csr()
    assert np.max(np.abs(oracle.static_pr(n, off2, dst2) - ref)) < 1e-9


def test_topology_replay_fixture():
    case = cases.load("topology_replay.json")
    # n spans the update ids too (the replay model accepts dst 5)
    n = 1 + max(max(max(e) for e in case["graph"]), max(max(u, v) for _, u, v in case["updates"]))
    off, dst, _ = cases.csr(n, case["graph"])
    orc = oracle.Oracle(oracle.SSSP, n, off, dst)
    batches = cases.replay_batches(case["updates"], case["sizes"])
    for bi, (dels, adds) in enumerate(batches):
        orc.mutate(cases.triples(dels), cases.triples(adds))
        st = orc.stats()
        want = case["replay_batches"][bi]
        assert st["missing_deletes"] == want["missing_deletes"]
        assert orc.live_edges() == want["graph_edges"]
        assert st["changed_sources"] == want["changed_sources"]
        for s in case["replay_sources"]:
            if s["batch"] == bi:
                assert orc.row_degree(s["source"]) == s["after_degree"]
                assert orc.row_multiset_hash(s["source"]) == s["multiset_hash"]


def test_grouping_checker_matches_the_reference_grouping():
    """group_ref, the restatement tests/test_gpu_group.py checks
    dycg_group_updates against, groups every batch exactly as the reference's
    GroupedUpdateBatch does: per source (ascending), the same multiset of
    deletion and of addition destinations, and the same number of sources per
    phase. (The reference also keeps arrival order inside a source; the
    device grouping sorts by destination, which changes no repair result.)"""
    import collections
    from tests.test_gpu_group import group_ref
    case = cases.load("group_updates.json")
    assert len(case["batches"]) == 6
    for b in case["batches"]:
        nv = b["num_vertices"]
        ends = np.array([nv], np.uint32)
        want = {s: (collections.Counter(d), collections.Counter(a)) for s, d, a in b["groups"]}
        assert [g[0] for g in b["groups"]] == sorted(want)
        got = {}
        for phase, recs in ((0, b["dels"]), (1, b["adds"])):
            rec = np.asarray(recs, np.uint32).reshape(-1, 2)
            rec = np.concatenate([rec, np.ones((len(rec), 1), np.uint32)], 1)
            keys, mult, invalid, _ = group_ref(rec, nv, ends)
            assert invalid == 0
            for k, m in zip(keys.tolist(), mult.tolist()):
                got.setdefault(k >> 32, (collections.Counter(), collections.Counter()))[phase][
                    k & 0xFFFFFFFF] += m
        assert got == want
        assert b["phases"] == [sum(1 for d, _ in want.values() if d),
                               sum(1 for _, a in want.values() if a)]
        # the reference keeps arrival order inside a source (stable grouping)
        for s, d, a in b["groups"]:
            assert d == [v for u, v in b["dels"] if u == s]
            assert a == [v for u, v in b["adds"] if u == s]


def test_deletion_repair_matches_the_reference_verifier():
    """SSSP deletion phases (rule weights) whose repaired distances the
    reference's own CPU verifier (src/i16_repair_oracle.cpp: Dijkstra over the
    affected subgraph seeded from its boundary) accepted when the fixture was
    made: the oracle invalidates the same dependency closure and repairs it to
    the same distances, and the verifier caught the planted wrong distance."""
    case_file = cases.load("i16_repair.json")
    inf = oracle.INF
    for c in case_file["cases"]:
        n = c["n"]
        off, dst, _ = oracle.csr_from_edges(n, [(a, b, 1) for a, b in c["graph"]])
        orc = oracle.Oracle(oracle.SSSP, n, off, dst, source=c["source"])
        orc.init()
        for s in c["snapshots"]:
            rep = s["report"]
            assert rep["state"] == "passed" and rep["distance_mismatches"] == 0
            assert rep["external_state_changes"] == 0 and rep["affected"] == len(s["affected"])
            _, par = orc.values()
            dels = [(u, v, 1) for u, v in s["dels"]]
            # the dependency closure under the deleted tree edges
            children = {}
            for x in range(n):
                if par[x] != inf:
                    children.setdefault(int(par[x]), []).append(x)
            aff = {v for u, v, _ in dels if v != c["source"] and par[v] == u}
            stack = list(aff)
            while stack:
                for ch in children.get(stack.pop(), ()):
                    if ch not in aff:
                        aff.add(ch)
                        stack.append(ch)
            assert sorted(aff) == s["affected"]
            orc.delete_edges(dels)
            assert orc.stats()["affected"] == len(aff)
            vals, _ = orc.values()
            assert [int(vals[x]) for x in s["affected"]] == s["after"]
            if "planted_report" in s:
                assert s["planted_report"]["distance_mismatches"] == 1


def test_random_multigraph_stream_matches_the_reference_chunk_store():
    """A seeded multigraph with parallel edges and self-loops, and an update
    stream with repeated, absent and parallel records, replayed by the oracle:
    per batch the same missing deletions and edge count as the reference's
    replay model and its chunk store, the same changed-source count as the
    chunk store (a source that lost or gained an occurrence,
    source_local_chunk_store.h:291-311), and per touched source the same degree
    and multiset hash as the replay model's dump. (The replay model counts a
    source as changed only when its row's digest differs, so a deletion and
    re-insertion that restore the same sequence counts there as unchanged:
    the two reference tools differ by one source in two of this stream's six
    batches.)"""
    case = cases.load("replay_random.json")
    n = 1 + max(max(max(e) for e in case["graph"]),
                max(max(u, v) for _, u, v in case["updates"]))
    off, dst, _ = cases.csr(n, case["graph"])
    orc = oracle.Oracle(oracle.SSSP, n, off, dst)
    batches = cases.replay_batches(case["updates"], case["sizes"])
    assert len(batches) == len(case["replay_batches"]) == len(case["chunk_store_batches"]) == 6
    sources = {}
    for s in case["replay_sources"]:
        sources.setdefault(s["batch"], []).append(s)
    for bi, (dels, adds) in enumerate(batches):
        orc.mutate(cases.triples(dels), cases.triples(adds))
        st = orc.stats()
        for want in (case["replay_batches"][bi], case["chunk_store_batches"][bi]):
            assert st["missing_deletes"] == want["missing_deletes"], (bi, want)
            assert orc.live_edges() == want["graph_edges"], (bi, want)
        assert st["changed_sources"] == case["chunk_store_batches"][bi]["changed_sources"], bi
        assert st["changed_sources"] - case["replay_batches"][bi]["changed_sources"] in (0, 1)
        assert len(sources[bi]) == case["replay_batches"][bi]["touched_sources"]
        for s in sources[bi]:
            assert orc.row_degree(s["source"]) == s["after_degree"]
            assert orc.row_multiset_hash(s["source"]) == s["multiset_hash"]
