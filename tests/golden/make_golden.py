"""Generate the golden fixtures in tests/golden/ from the reference's own tests.

Run where the reference checkout is present, naming it with --ref or the
DYCG_REFERENCE environment variable:

    python tests/golden/make_golden.py --ref <reference checkout>

What it records (all small JSON, committed):
  smoke_bfs_sssp.json  -- the graph/update stream that tests/bfs_dynamic_smoke.py
                          and tests/i22_ordered_insertion_test.py build, with
                          per-phase distance checksums from that file's own
                          oracle() (FIFO BFS and Dijkstra, weight (u+v)%128+1).
  smoke_cc.json        -- tests/cc_dynamic_smoke.py's multigraph and 20 batches
                          (6 random ones from its seed), checksums from its
                          directed-reachability oracle().
  smoke_pr.json        -- tests/pr_dynamic_smoke.py's graph and batches with the
                          FP64 Jacobi ranks from its oracle().
  pr_probe.json        -- paper/evaluation/audit_20261004/pr_probe: graph,
                          updates, sizes and the FP64 reference ranks stored in
                          its result.json.
  topology_replay.json -- tests/fixtures/topology_replay_* with the output of
                          the reference's topology_replay tool (built from the
                          reference sources by oracle/Makefile).
  i16_repair.json      -- seeded SSSP deletion phases repaired by the oracle and
                          checked by the reference's own CPU verifier
                          (src/i16_repair_oracle.cpp, built by oracle/Makefile):
                          graph, deletions, affected set, repaired distances and
                          the verifier's report, plus one planted mistake that
                          it must catch.
  replay_random.json   -- a seeded random multigraph and update stream (repeated
                          pairs, absent deletions, self-loops) replayed by the
                          reference's topology_replay (per-source degrees and
                          multiset hashes) and by its chunk store through
                          chunk_store_replay --pageable (per-batch counts).
  group_updates.json   -- seeded update batches grouped by the reference's own
                          GroupedUpdateBatch (effective_update_batch.h, driven
                          by oracle/ref_group_updates.cpp, built by
                          oracle/Makefile): per source, its deletions and
                          additions in the class's order.
The reference is only read here; nothing at test time touches it.
"""
import argparse
import importlib.util
import json
import os
import random
import re
import subprocess
import sys
from collections import Counter
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent


def load_module(path, name):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def bfs_sssp_case(ref):
    """The n=2048 stream of bfs_dynamic_smoke.py:59-77 (also i22:49-68)."""
    mod = load_module(ref / "tests/bfs_dynamic_smoke.py", "ref_bfs_smoke")
    n = 2048
    edges = {(u, (u + 1) % n) for u in range(n)}
    edges |= {(u, 1024) for u in range(1024)} | {(0, 0), (0, 2), (1, 3)}
    graph = sorted(edges)
    deleted = [(0, 1024), (20, 21), (700, 701), (1200, 1201)]
    added = [(1, 1900), (500, 1700), (900, 2000), (3, 1500)]
    batches, expect = [], {"bfs": [], "sssp": []}
    for dels, adds in [(deleted, added), (added, deleted), (deleted, added)]:
        for u, v in dels:
            edges.remove((u, v))
        for algo, weighted in (("bfs", False), ("sssp", True)):
            expect[algo].append({"phase": "delete", "checksum": mod.oracle(edges, n, weighted)[1]})
        for u, v in adds:
            edges.add((u, v))
        for algo, weighted in (("bfs", False), ("sssp", True)):
            expect[algo].append({"phase": "batch", "checksum": mod.oracle(edges, n, weighted)[1]})
        batches.append({"dels": [list(e) for e in dels], "adds": [list(e) for e in adds]})
    final = {algo: mod.oracle(edges, n, algo == "sssp")[0] for algo in ("bfs", "sssp")}
    return {"n": n, "source": 0, "graph": [list(e) for e in graph], "batches": batches,
            "expected": expect, "final_values": final,
            "origin": "tests/bfs_dynamic_smoke.py:59-77 oracle() :16-44"}


def cc_case(ref):
    """The n=256 multigraph and batches of cc_dynamic_smoke.py:58-88."""
    mod = load_module(ref / "tests/cc_dynamic_smoke.py", "ref_cc_smoke")
    nodes = 256
    base = [(0, 0), (11, 11), (255, 255)]
    base += [(0, 1), (1, 2), (2, 0), (2, 3), (3, 4), (4, 5), (5, 3)]
    base += [(8, 9), (8, 9), (130, 140), (140, 150), (150, 130)]
    base += [(u, u + 1) for u in range(160, 200)]
    base += [(31, 30), (32, 30), (40, 41), (41, 42), (42, 41)]
    base += [(0, 220), (220, 210), (210, 211), (211, 210)]
    base += [(50, 51), (50, 52), (51, 53), (52, 53), (53, 54), (54, 53)]
    base += [(60, 61), (60, 62), (61, 63), (62, 63), (63, 64), (64, 63)]
    original = Counter(base)
    graph = []
    for (u, v), count in sorted(original.items()):
        graph += [[u, v]] * count
    batches = [([], []), ([(2, 3), (40, 41), (220, 210)], []), ([(0, 1)], []),
               ([(8, 9)], []), ([(8, 9)], [(5, 8)]),
               ([(3, 4), (3, 5)], [(2, 4), (9, 130)]),
               ([(180, 181)], [(150, 190)]),
               ([(210, 211), (11, 11)], [(10, 11)]),
               ([], [(5, 8)]), ([(5, 8)], [(2, 3)])]
    batches += [([(51, 53)], []), ([(50, 52), (61, 63), (62, 63)], []),
                ([], [(49, 53)]), ([(49, 53)], [])]
    rng = random.Random(20260923)
    for _ in range(6):
        batches.append(([(rng.randrange(nodes), rng.randrange(nodes)) for _ in range(8)],
                        [(rng.randrange(nodes), rng.randrange(nodes)) for _ in range(8)]))
    edges = original.copy()
    expect, out = [], []
    for deleted, added in batches:
        for u, v in deleted:
            edges[u, v] = max(0, edges[u, v] - 1)
        expect.append({"phase": "delete", "checksum": mod.oracle(edges, nodes)[1]})
        for u, v in added:
            edges[u, v] += 1
        expect.append({"phase": "batch", "checksum": mod.oracle(edges, nodes)[1]})
        out.append({"dels": [list(e) for e in deleted], "adds": [list(e) for e in added]})
    return {"n": nodes, "graph": graph, "batches": out, "expected": expect,
            "final_labels": mod.oracle(edges, nodes)[0],
            "origin": "tests/cc_dynamic_smoke.py:58-88 oracle() :17-41"}


def pr_case(ref):
    """The n=4096 graph and batches of pr_dynamic_smoke.py:44-64."""
    mod = load_module(ref / "tests/pr_dynamic_smoke.py", "ref_pr_smoke")
    n = 4096
    base = [(0, 1), (1, 2), (2, 0), (3, 4), (4, 3), (8, 9), (8, 9), (10, 10), (n - 1, n - 1)]
    base += [(20, v) for v in range(21, 1800)]
    base += [(v, 20) for v in range(21, 1800)]
    base += [(v, v + 1) for v in range(2000, 2020)]
    original = Counter(base)
    batches = [([], []), ([(2, 0)], []), ([], [(2, 3)]),
               ([(3, 4)], [(3, 4)]), ([(8, 9)], []),
               ([(8, 9), (10, 10)], [(9, 8)]),
               ([(20, v) for v in range(21, 1800, 3)], [(20, 2000), (2020, 20)]),
               ([(2000, 2001), (4000, 4001)], [(0, 8), (3, 10)]),
               ([], [(10, 10), (10, 3), (8, 9), (8, 9)]),
               ([(20, 2000), (2020, 20)], [(2000, 2001)])]
    edges = original.copy()
    out = []
    for deleted, added in batches:
        for u, v in deleted:
            edges[u, v] = max(0, edges[u, v] - 1)
        for u, v in added:
            edges[u, v] += 1
        out.append({"dels": [list(e) for e in deleted], "adds": [list(e) for e in added]})
    return {"n": n, "graph": [list(e) for e in sorted(base)], "batches": out,
            "initial_ranks": mod.oracle(original, n), "final_ranks": mod.oracle(edges, n),
            "origin": "tests/pr_dynamic_smoke.py:44-64 oracle() :16-31"}


def read_pairs(path):
    rows = []
    for line in Path(path).read_text().splitlines():
        parts = line.split()
        if len(parts) >= 2:
            rows.append([int(parts[0]), int(parts[1])])
    return rows


def read_updates(path):
    rows = []
    for line in Path(path).read_text().splitlines():
        parts = line.split()
        if len(parts) >= 3:
            rows.append([parts[0], int(parts[1]), int(parts[2])])
    return rows


def read_sizes(path):
    return [[int(x) for x in line.split()[:2]] for line in Path(path).read_text().splitlines()
            if line.strip()]


def pr_probe_case(ref):
    d = ref / "paper/evaluation/audit_20261004/pr_probe"
    result = json.loads((d / "result.json").read_text())
    return {"graph": read_pairs(d / "graph"), "updates": read_updates(d / "updates"),
            "sizes": read_sizes(d / "sizes"), "reference_ranks": result["reference"],
            "gpu_max_error": result["results"][0]["max_error"],
            "origin": "paper/evaluation/audit_20261004/pr_probe (result.json 'reference')"}


def topology_case(ref):
    fx = ref / "tests/fixtures"
    subprocess.run(["make", "-s", "-C", str(REPO / "oracle"), f"REF={ref}"], check=True)
    tool = REPO / "oracle/_ref/topology_replay"
    text = subprocess.run([str(tool), "--graph", str(fx / "topology_replay_graph.txt"),
                           "--updates", str(fx / "topology_replay_updates.txt"),
                           "--batch-sizes", str(fx / "topology_replay_batch_sizes.txt"),
                           "--dump-sources"], check=True, capture_output=True, text=True).stdout
    batches = [dict((k, int(v)) for k, v in re.findall(r"(\w+)=(\d+)", line))
               for line in text.splitlines() if line.startswith("[TOPOLOGY-REPLAY-BATCH]")]
    sources = [dict((k, int(v)) for k, v in re.findall(r"(\w+)=(\d+)", line))
               for line in text.splitlines() if line.startswith("[TOPOLOGY-REPLAY-SOURCE]")]
    return {"graph": read_pairs(fx / "topology_replay_graph.txt"),
            "updates": read_updates(fx / "topology_replay_updates.txt"),
            "sizes": read_sizes(fx / "topology_replay_batch_sizes.txt"),
            "replay_batches": batches, "replay_sources": sources,
            "ctest_regex": "batch=1 additions=1 deletions=1 touched_sources=2 changed_sources=1 "
                           "missing_deletes=1 invalid_additions=0 graph_edges=6",
            "origin": "tests/fixtures/topology_replay_*, CMakeLists.txt:134-145, "
                      "src/topology_replay.cpp"}


def group_case(ref):
    """Seeded batches with skewed sources, repeated (u, v) pairs and both
    phases; one batch above 4096 records takes the class's radix-sort path."""
    subprocess.run(["make", "-s", "-C", str(REPO / "oracle"), f"REF={ref}"], check=True)
    tool = REPO / "oracle/_ref/group_updates"
    rng = random.Random(20261203)
    out = []
    for nd, na, nv in ((0, 0, 8), (1, 0, 8), (0, 3, 8), (40, 25, 16), (300, 200, 64),
                       (2600, 1600, 1 << 12)):
        def draw(k):
            # squared uniform: low ids are hot, so sources repeat
            return [[int(nv * rng.random() ** 2), rng.randrange(nv)] for _ in range(k)]
        dels, adds = draw(nd), draw(na)
        dels += dels[:nd // 10]  # repeated deletion requests
        adds += adds[:na // 10]  # parallel insertions
        text = f"{len(dels)} {len(adds)}\n" + "".join(f"{u} {v}\n" for u, v in dels + adds)
        res = subprocess.run([str(tool)], input=text, check=True, capture_output=True,
                             text=True).stdout.splitlines()
        groups, phases = [], None
        for line in res:
            f = line.split()
            if f[0] == "S":
                groups.append([int(f[1]), [], []])
            elif f[0] == "D":
                groups[-1][1] = [int(x) for x in f[1:]]
            elif f[0] == "A":
                groups[-1][2] = [int(x) for x in f[1:]]
            else:
                phases = [int(f[1]), int(f[2])]
        out.append({"num_vertices": nv, "dels": dels, "adds": adds, "groups": groups,
                    "phases": phases})
    return {"batches": out,
            "origin": "include/framework/effective_update_batch.h:36-207 GroupedUpdateBatch "
                      "(Mixed view per source; PhaseSize(Delete/Add))"}


I16_INF = 0xFFFFFFFF


def i16_affected(n, par, dels, source):
    """The deletion-dependency closure: heads of deleted tree edges (parent ==
    tail) and every vertex below them in the parent forest."""
    children = {}
    for x in range(n):
        if par[x] != I16_INF:
            children.setdefault(int(par[x]), []).append(x)
    aff = {v for u, v, _ in dels if v != source and par[v] == u}
    stack = list(aff)
    while stack:
        for c in children.get(stack.pop(), ()):
            if c not in aff:
                aff.add(c)
                stack.append(c)
    return sorted(aff)


def i16_snapshot(path, batch, source, n, affected, inc_off, inc, before, after):
    """The verifier's binary snapshot (include/framework/i16_repair_snapshot.h:
    magic, version 1, infinity, weight rule 1 = (u+v)%128+1, then the
    vectors)."""
    import struct
    import numpy as np
    with open(path, "wb") as f:
        f.write(struct.pack("<QIII", 0x4931365354415445, 1, I16_INF, 1))
        f.write(struct.pack("<III", batch, source, n))
        for arr, dt in ((affected, np.uint32), (inc_off, np.uint64), (inc, np.uint32)):
            a = np.ascontiguousarray(arr, dt)
            f.write(struct.pack("<Q", len(a)) + a.tobytes())
        for st in (before, after):
            a = np.ascontiguousarray(st, np.uint32).reshape(-1, 4)
            f.write(struct.pack("<Q", len(a)) + a.tobytes())


def i16_case(ref):
    import tempfile
    import numpy as np
    sys.path.insert(0, str(REPO))
    import oracle
    subprocess.run(["make", "-s", "-C", str(REPO / "oracle"), f"REF={ref}"], check=True)
    tool = REPO / "oracle/_ref/i16_repair_oracle"
    cases_out = []
    with tempfile.TemporaryDirectory() as td:
        def verify(*snap):
            i16_snapshot(f"{td}/s.bin", *snap)
            r = subprocess.run([str(tool), f"{td}/s.bin", f"{td}/r.json"], capture_output=True,
                               text=True)
            rep = json.loads(r.stdout)
            return {k: rep[k] for k in ("state", "affected", "incoming", "boundary",
                                        "seed_vertices", "improvements", "distance_mismatches",
                                        "external_state_changes")}
        for seed in (1, 2):
            rng = np.random.default_rng(seed)
            n, m = 300, 2400
            u, v = rng.integers(0, n, m), rng.integers(0, n, m)
            edges = [[int(a), int(b)] for a, b in zip(u, v) if a != b]
            off, dst, _ = oracle.csr_from_edges(n, [(a, b, 1) for a, b in edges])
            orc = oracle.Oracle(oracle.SSSP, n, off, dst, source=0)
            orc.init()
            snaps = []
            for b in range(4):
                vals0, par0 = orc.values()
                o, d, _ = orc.csr()
                src = np.repeat(np.arange(n), np.diff(o.astype(np.int64)))
                pick = rng.choice(len(d), size=40, replace=False)
                dels = [(int(src[i]), int(d[i]), 1) for i in pick]
                aff = i16_affected(n, par0, dels, 0)
                orc.delete_edges(dels)
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
                before = [(x, I16_INF, I16_INF, I16_INF) if x in idx else
                          (x, int(vals0[x]), int(vals0[x]), int(par0[x])) for x in listed]
                after = [(x, int(vals1[x]), int(vals1[x]), int(par1[x])) for x in listed]
                snap = {"dels": [[a, b_] for a, b_, _ in dels], "affected": aff,
                        "oracle_affected": int(orc.stats()["affected"]),
                        "after": [int(vals1[x]) for x in aff],
                        "report": verify(b, 0, n, aff, inc_off, flat, before, after)}
                if seed == 1 and b == 0:
                    # planted mistake (in the oracle's output, on the CPU): one
                    # finite affected distance raised by one
                    k = next(i for i, x in enumerate(listed) if x in idx and after[i][1] != I16_INF)
                    bad = list(after)
                    bad[k] = (bad[k][0], bad[k][1] + 1, bad[k][2] + 1, bad[k][3])
                    snap["planted_report"] = verify(b, 0, n, aff, inc_off, flat, before, bad)
                snaps.append(snap)
            cases_out.append({"n": n, "source": 0, "graph": edges, "snapshots": snaps})
    return {"cases": cases_out, "weight_rule": "(u+v)%128+1",
            "origin": "src/i16_repair_oracle.cpp + include/framework/i16_repair_snapshot.h"}


def replay_random_case(ref):
    import tempfile
    subprocess.run(["make", "-s", "-C", str(REPO / "oracle"), f"REF={ref}"], check=True)
    rng = random.Random(20261204)
    n = 400
    graph = [[rng.randrange(n), rng.randrange(n)] for _ in range(2500)]
    graph += graph[:200]                                   # parallel occurrences
    graph += [[v, v] for v in range(0, n, 97)]             # self-loops
    live = [tuple(e) for e in graph]
    updates, sizes = [], []
    for _ in range(6):
        dels = [list(live[rng.randrange(len(live))]) for _ in range(60)]
        dels += dels[:5]                                       # second request, same pair
        dels += [[rng.randrange(n), rng.randrange(n)] for _ in range(10)]  # mostly absent
        adds = [[rng.randrange(n), rng.randrange(n)] for _ in range(60)]
        adds += [list(live[rng.randrange(len(live))]) for _ in range(10)]  # parallel
        recs = [("d", u, v) for u, v in dels] + [("a", u, v) for u, v in adds]
        rng.shuffle(recs)                                      # the Loader splits by type
        updates += recs
        sizes.append([len(adds), len(dels)])
        live += [tuple(e) for e in adds]
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        (td / "g.txt").write_text("".join(f"{u} {v}\n" for u, v in graph))
        (td / "u.txt").write_text("".join(f"{t} {u} {v} 1\n" for t, u, v in updates))
        (td / "s.txt").write_text("".join(f"{a} {d}\n" for a, d in sizes))
        args = ["--graph", str(td / "g.txt"), "--updates", str(td / "u.txt"),
                "--batch-sizes", str(td / "s.txt")]
        topo = subprocess.run([str(REPO / "oracle/_ref/topology_replay"), *args,
                               "--dump-sources"], check=True, capture_output=True,
                              text=True).stdout
        chunk = subprocess.run([str(REPO / "oracle/_ref/chunk_store_replay"), *args,
                                "--pageable"], check=True, capture_output=True, text=True).stdout

    def rows(text, tag, keys=None):
        out = []
        for line in text.splitlines():
            if line.startswith(tag):
                d = dict((k, int(v)) for k, v in re.findall(r"(\w+)=(\d+)(?=\s|$)", line))
                out.append({k: d[k] for k in keys} if keys else d)
        return out
    count_keys = ["batch", "touched_sources", "changed_sources", "missing_deletes",
                  "invalid_additions", "graph_edges"]
    return {"graph": graph, "updates": [list(r) for r in updates], "sizes": sizes,
            "replay_batches": rows(topo, "[TOPOLOGY-REPLAY-BATCH]"),
            "replay_sources": rows(topo, "[TOPOLOGY-REPLAY-SOURCE]"),
            "chunk_store_batches": rows(chunk, "[CHUNK-STORE-BATCH]", count_keys),
            "origin": "src/topology_replay.cpp --dump-sources and src/chunk_store_replay.cpp "
                      "--pageable (include/framework/source_local_chunk_store.h) on a seeded "
                      "stream made by tests/golden/make_golden.py"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("DYCG_REFERENCE"),
                    required="DYCG_REFERENCE" not in os.environ,
                    help="reference checkout (default: $DYCG_REFERENCE)")
    ap.add_argument("--only", nargs="*", default=None, help="regenerate only these fixtures")
    ap.add_argument("--out", default=None, help="write here instead of tests/golden/")
    args = ap.parse_args()
    out_dir = Path(args.out) if args.out else HERE
    ref = Path(args.ref)
    if not (ref / "tests/bfs_dynamic_smoke.py").exists():
        sys.exit(f"reference checkout not found at {ref}")
    makers = {"smoke_bfs_sssp.json": bfs_sssp_case, "smoke_cc.json": cc_case,
              "smoke_pr.json": pr_case, "pr_probe.json": pr_probe_case,
              "topology_replay.json": topology_case, "group_updates.json": group_case,
              "i16_repair.json": i16_case, "replay_random.json": replay_random_case}
    cases = {name: make(ref) for name, make in makers.items()
             if args.only is None or name in args.only}
    for name, data in cases.items():
        (out_dir / name).write_text(json.dumps(data, separators=(",", ":")) + "\n")
        print(name, (out_dir / name).stat().st_size, "bytes")


if __name__ == "__main__":
    main()
