"""Randomised cross-checks against the reference's own code, run live (no GPU).

oracle/Makefile compiles a few of the reference's CPU tools into oracle/_ref/
when the reference checkout is present (the update grouping driver, the
topology replay model, the chunk store replay, the deletion-repair verifier).
Where they are built, these tests draw fresh seeded batches, streams and
deletion phases and compare the grouping checker, the oracle's mutation and
its deletion repair with the reference's output; elsewhere they skip (the
committed fixtures in tests/golden/ carry a fixed sample of the same).
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


def _make_golden():
    import importlib.util
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "make_golden.py")
    spec = importlib.util.spec_from_file_location("make_golden", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("seed", range(3))
def test_deletion_repair_passes_reference_verifier_live(seed, tmp_path):
    """Fresh deletion phases repaired by the oracle, each checked by the
    reference's CPU verifier (Dijkstra over the affected subgraph seeded from
    its boundary): no distance mismatch, no change outside the affected set."""
    import json
    tool = _tool("i16_repair_oracle")
    mg = _make_golden()
    rng = np.random.default_rng(500 + seed)
    n = int(rng.integers(50, 400))
    m = int(rng.integers(3, 9)) * n
    u, v = rng.integers(0, n, m), rng.integers(0, n, m)
    off, dst, _ = oracle.csr_from_edges(n, [(int(a), int(b), 1) for a, b in zip(u, v) if a != b])
    orc = oracle.Oracle(oracle.SSSP, n, off, dst, source=0)
    orc.init()
    for b in range(3):
        vals0, par0 = orc.values()
        o, d, _ = orc.csr()
        src = np.repeat(np.arange(n), np.diff(o.astype(np.int64)))
        pick = rng.choice(len(d), size=min(len(d), 30), replace=False)
        dels = [(int(src[i]), int(d[i]), 1) for i in pick]
        aff = mg.i16_affected(n, par0, dels, 0)
        orc.delete_edges(dels)
        assert orc.stats()["affected"] == len(aff)
        vals1, par1 = orc.values()
        o, d, _ = orc.csr()
        src = np.repeat(np.arange(n), np.diff(o.astype(np.int64)))
        idx = {x: i for i, x in enumerate(aff)}
        inc = [[] for _ in aff]
        for s_, t_ in zip(src.tolist(), d.tolist()):
            if t_ in idx:
                inc[idx[t_]].append(s_)
        inc_off = np.zeros(len(aff) + 1, np.uint64)
        inc_off[1:] = np.cumsum([len(x) for x in inc])
        flat = [s_ for row in inc for s_ in row]
        listed = sorted(set(aff) | set(flat))
        inf = oracle.INF
        before = [(x, inf, inf, inf) if x in idx else (x, int(vals0[x]), int(vals0[x]), int(par0[x]))
                  for x in listed]
        after = [(x, int(vals1[x]), int(vals1[x]), int(par1[x])) for x in listed]
        mg.i16_snapshot(tmp_path / "s.bin", b, 0, n, aff, inc_off, flat, before, after)
        r = subprocess.run([tool, str(tmp_path / "s.bin"), str(tmp_path / "r.json")],
                           capture_output=True, text=True)
        rep = json.loads(r.stdout)
        assert r.returncode == 0 and rep["distance_mismatches"] == 0, rep
        assert rep["external_state_changes"] == 0


def test_reference_tool_fixtures_regenerate_identically(tmp_path):
    """The committed fixtures made with the reference's own tools come back
    byte for byte when regenerated from the reference checkout."""
    import sys
    ref = os.environ.get("DYCG_REFERENCE", "")
    if not ref or not os.path.exists(os.path.join(ref, "tests", "bfs_dynamic_smoke.py")):
        pytest.skip("no reference checkout named by DYCG_REFERENCE")
    for name in ("group_updates", "i16_repair_oracle", "chunk_store_replay"):
        _tool(name)
    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    names = ["group_updates.json", "i16_repair.json", "replay_random.json"]
    subprocess.run([sys.executable, os.path.join(golden, "make_golden.py"), "--ref", ref,
                    "--out", str(tmp_path), "--only", *names], check=True, capture_output=True)
    for name in names:
        assert (tmp_path / name).read_bytes() == open(os.path.join(golden, name), "rb").read(), name
