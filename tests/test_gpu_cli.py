"""The hybrid_* command-line drop-ins, driven like the reference's smoke scripts
(tests/bfs_dynamic_smoke.py, cc_dynamic_smoke.py, pr_dynamic_smoke.py): same
flags, same update files, checksums parsed from the same log lines."""
import os
import re
import subprocess

import numpy as np
import pytest

from tests import cases

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "dycgraph_b200")


def write_case(tmp, graph, batches):
    (tmp / "graph").write_text("".join(f"{u} {v}\n" for u, v in graph))
    ups, sizes = [], []
    for b in batches:
        ups += [f"d {u} {v} 77\n" for u, v in b["dels"]]
        ups += [f"a {u} {v} 91\n" for u, v in b["adds"]]
        sizes.append(f"{len(b['adds'])} {len(b['dels'])}\n")
    (tmp / "updates").write_text("".join(ups))
    (tmp / "sizes").write_text("".join(sizes))


def run(tool, tmp, extra):
    cmd = [os.path.join(BIN, tool), f"--graphfile={tmp / 'graph'}", f"--updatefile={tmp / 'updates'}",
           f"--update_size={tmp / 'sizes'}", "--format=market_big", "--SEGMENT=32",
           "--n_stream=3", "--hybrid=0", "--check=true", f"--output={tmp / 'out'}"] + extra
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    return p.stdout


@pytest.mark.parametrize("algo", ["bfs", "sssp"])
@pytest.mark.parametrize("cache", [0, 2])
def test_cli_bfs_sssp_smoke(tmp_path, algo, cache):
    case = cases.load("smoke_bfs_sssp.json")
    write_case(tmp_path, case["graph"], case["batches"])
    tag = algo.upper()
    text = run(f"hybrid_{algo}", tmp_path, [f"--cache={cache}", f"--{algo}_max_batches=3",
                                            f"--{algo}_print_checksum=true", "--source_node=0"])
    got = [int(v) for v in re.findall(rf"\[{tag}-(?:DELETE-STAGE|BATCH)-CHECK\][^\n]*distance_checksum=(\d+)", text)]
    assert got == [e["checksum"] for e in case["expected"][algo]]
    assert len(re.findall(rf"\[{tag}-(?:DELETE-STAGE|BATCH)-CHECK\][^\n]* passed ", text)) == 6
    assert len(re.findall(rf"\[P0-TIMER\]\[{tag}\]\[batch \d+\] total_batch: [\d.]+ ms", text)) == 3
    rows = [list(map(int, line.split())) for line in (tmp_path / "out").read_text().splitlines()]
    assert [r[1] for r in rows] == case["final_values"][algo]


def test_cli_cc_smoke(tmp_path):
    case = cases.load("smoke_cc.json")
    write_case(tmp_path, case["graph"], case["batches"])
    text = run("hybrid_cc", tmp_path, ["--cache=2", f"--cc_max_batches={len(case['batches'])}"])
    got = [int(v) for v in re.findall(r"\[CC-(?:DELETE-STAGE|BATCH)-CHECK\][^\n]*label_checksum=(\d+)", text)]
    assert got == [e["checksum"] for e in case["expected"]]
    assert "failed" not in text


def test_cli_pr_smoke(tmp_path):
    case = cases.load("smoke_pr.json")
    write_case(tmp_path, case["graph"], case["batches"])
    text = run("hybrid_pr", tmp_path, ["--cache=2", "--error=1e-7", "--pr_max_rounds=100000",
                                       "--pr_max_batches=99"])
    assert len(re.findall(r"\[PR-BATCH\]", text)) == len(case["batches"])
    x = np.array([float(line.split()[1]) for line in (tmp_path / "out").read_text().splitlines()])
    # the reference's acceptance bound (tests/pr_dynamic_smoke.py:96-98)
    assert float(np.mean(np.abs(x - np.array(case["final_ranks"])))) < 1e-5


def test_cli_binary_formats(tmp_path):
    """The same smoke stream through the binary graph and update files."""
    from dycgraph_b200 import formats
    case = cases.load("smoke_bfs_sssp.json")
    n = case["n"]
    off, dst, _ = cases.csr(n, case["graph"])
    formats.write_graph(tmp_path / "graph", off, dst)
    formats.write_updates(tmp_path / "updates", [
        (np.array([(u, v, 77) for u, v in b["dels"]], np.uint32),
         np.array([(u, v, 91) for u, v in b["adds"]], np.uint32)) for b in case["batches"]])
    cmd = [os.path.join(BIN, "hybrid_sssp"), f"--graphfile={tmp_path / 'graph'}", "--format=binary",
           f"--updatefile={tmp_path / 'updates'}", "--update_format=binary", "--check=true",
           "--sssp_max_batches=3"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    got = [int(v) for v in re.findall(r"\[SSSP-(?:DELETE-STAGE|BATCH)-CHECK\][^\n]*distance_checksum=(\d+)", p.stdout)]
    assert got == [e["checksum"] for e in case["expected"]["sssp"]]
