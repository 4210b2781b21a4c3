"""Randomised cross-checks against the reference's own code, run live (no GPU).

oracle/Makefile compiles a few of the reference's CPU tools into oracle/_ref/
when the reference checkout is present (the update grouping driver, the
topology replay model, the chunk store replay). Where they are built, these
tests draw fresh seeded batches and streams and compare the grouping checker
and the oracle's mutation with the reference's output; elsewhere they skip
(the committed fixtures in tests/golden/ carry a fixed sample of the same).
"""
import collections
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
from tests import cases

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


def _tool(name):
    path = os.path.join(REF, name)
    if not os.access(path, os.X_OK):
        pytest.skip(f"oracle/_ref/{name} not built (no reference checkout here)")
    return path


@pytest.mark.parametrize("seed", range(12))
def test_grouping_checker_matches_reference_grouping_live(seed):
    from tests.test_gpu_group import group_ref
    tool = _tool("group_updates")
    rng = np.random.default_rng(seed)
    nv = int(rng.integers(2, 3000))
    nd, na = (int(x) for x in rng.integers(0, 3000, 2))
    if seed == 0:
        nd, na = 3000, 2500  # above the reference's radix-sort threshold (4096 records)
    dels = np.stack([(nv * rng.random(nd) ** 2).astype(np.int64), rng.integers(0, nv, nd)], 1)
    adds = np.stack([(nv * rng.random(na) ** 2).astype(np.int64), rng.integers(0, nv, na)], 1)
    text = f"{nd} {na}\n" + "".join(f"{u} {v}\n" for u, v in np.concatenate([dels, adds]))
    out = subprocess.run([tool], input=text, check=True, capture_output=True, text=True).stdout
    want, phases = {}, None
    for line in out.splitlines():
        f = line.split()
        if f[0] == "S":
            cur = want.setdefault(int(f[1]), [collections.Counter(), collections.Counter()])
        elif f[0] in ("D", "A"):
            cur[0 if f[0] == "D" else 1].update(int(x) for x in f[1:])
        else:
            phases = [int(f[1]), int(f[2])]
    got = {}
    ends = np.array([nv], np.uint32)
    for ph, recs in ((0, dels), (1, adds)):
        rec = np.concatenate([recs, np.ones((len(recs), 1), np.int64)], 1).astype(np.uint32)
        keys, mult, invalid, _ = group_ref(rec, nv, ends)
        assert invalid == 0
        for k, m in zip(keys.tolist(), mult.tolist()):
            got.setdefault(k >> 32, [collections.Counter(), collections.Counter()])[ph][
                k & 0xFFFFFFFF] += m
    assert got == want
    assert phases == [sum(1 for d, _ in want.values() if d), sum(1 for _, a in want.values() if a)]


def _stream(rng, n, m, nb):
    graph = [[int(rng.integers(n)), int(rng.integers(n))] for _ in range(m)]
    graph += graph[: m // 10]
    live = [tuple(e) for e in graph]
    updates, sizes = [], []
    for _ in range(nb):
        k = int(rng.integers(5, 80))
        dels = [list(live[int(rng.integers(len(live)))]) for _ in range(k)]
        dels += dels[:3] + [[int(rng.integers(n)), int(rng.integers(n))] for _ in range(5)]
        adds = [[int(rng.integers(n)), int(rng.integers(n))] for _ in range(k)]
        adds += [list(live[int(rng.integers(len(live)))]) for _ in range(4)]
        recs = [("d", u, v) for u, v in dels] + [("a", u, v) for u, v in adds]
        rng.shuffle(recs)
        updates += recs
        sizes.append((len(adds), len(dels)))
        live += [tuple(e) for e in adds]
    return graph, updates, sizes


def _run(tool, tmp_path, graph, updates, sizes, *extra):
    (tmp_path / "g.txt").write_text("".join(f"{u} {v}\n" for u, v in graph))
    (tmp_path / "u.txt").write_text("".join(f"{t} {u} {v} 1\n" for t, u, v in updates))
    (tmp_path / "s.txt").write_text("".join(f"{a} {d}\n" for a, d in sizes))
    return subprocess.run([tool, "--graph", str(tmp_path / "g.txt"), "--updates",
                           str(tmp_path / "u.txt"), "--batch-sizes", str(tmp_path / "s.txt"),
                           *extra], check=True, capture_output=True, text=True).stdout


def _fields(text, tag):
    return [dict((k, int(v)) for k, v in re.findall(r"(\w+)=(\d+)(?=\s|$)", ln))
            for ln in text.splitlines() if ln.startswith(tag)]


@pytest.mark.parametrize("seed", range(4))
def test_oracle_mutation_matches_reference_chunk_store_live(seed, tmp_path):
    topo_tool, chunk_tool = _tool("topology_replay"), _tool("chunk_store_replay")
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(20, 300))
    graph, updates, sizes = _stream(rng, n, int(rng.integers(50, 1500)), 5)
    topo = _run(topo_tool, tmp_path, graph, updates, sizes, "--dump-sources")
    chunk = _run(chunk_tool, tmp_path, graph, updates, sizes, "--pageable")
    tb, src = _fields(topo, "[TOPOLOGY-REPLAY-BATCH]"), _fields(topo, "[TOPOLOGY-REPLAY-SOURCE]")
    cb = _fields(chunk, "[CHUNK-STORE-BATCH]")
    nn = 1 + max(max(max(e) for e in graph), max(max(u, v) for _, u, v in updates))
    off, dst, _ = cases.csr(nn, graph)
    orc = oracle.Oracle(oracle.SSSP, nn, off, dst)
    for bi, (dels, adds) in enumerate(cases.replay_batches(updates, sizes)):
        orc.mutate(cases.triples(dels), cases.triples(adds))
        st = orc.stats()
        for want in (tb[bi], cb[bi]):
            assert st["missing_deletes"] == want["missing_deletes"]
            assert orc.live_edges() == want["graph_edges"]
        assert st["changed_sources"] == cb[bi]["changed_sources"]
        for s in (s for s in src if s["batch"] == bi):
            assert orc.row_degree(s["source"]) == s["after_degree"]
            assert orc.row_multiset_hash(s["source"]) == s["multiset_hash"]
