"""bench.py's reference arm on the CPU (no GPU): the JSON line it prints keeps
the benchmark contract, and under a multi-rank launch only rank 0 works and
prints."""
import json
import os
import subprocess
import sys
import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, **env):
    e = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    e.update(env)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                          env=e, capture_output=True, text=True, timeout=300)


def test_reference_arm_line_keeps_the_contract(tmp_path):
    out = tmp_path / "ref.json"
    p = _run(["--impl", "reference", "--config", "rmat16", "--steps", "2", "--warmup", "3",
              "--json-out", str(out)])
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert json.loads(out.read_text()) == d
    assert d["impl"] == "reference" and d["unit"] == "updates/s" and d["value"] > 0
    assert d["steps"] == 2 and d["warmup"] >= 3 and d["n_gpus"] == 1
    assert d["higher_is_better"] is True and d["scaling"] == "weak" and d["vs_baseline"] is None
    assert d["ms_per_step"] > 0 and "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    # same metric as the library's own arm
    import bench
    assert d["metric"] == bench.METRIC


def test_reference_arm_other_ranks_exit_without_work():
    p = _run(["--impl", "reference", "--config", "rmat16", "--steps", "2", "--warmup", "3"],
             RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    assert p.returncode == 0, p.stderr[-2000:]
    assert not [ln for ln in p.stdout.splitlines() if ln.startswith("{")]


def test_reference_arm_declines_the_learned_form():
    p = _run(["--impl", "reference", "--config", "learned", "--steps", "2", "--warmup", "3"])
    assert p.returncode == 0, p.stderr[-2000:]
    d = json.loads([ln for ln in p.stdout.splitlines() if ln.startswith("{")][-1])
    assert d["impl"] == "reference" and d["unavailable"]


def test_reference_arm_batched_form_charges_every_query():
    p = _run(["--impl", "reference", "--config", "batched", "--scale", "12", "--queries", "8",
              "--batch-max", "5000", "--steps", "3", "--warmup", "3"])
    assert p.returncode == 0, p.stderr[-2000:]
    d = json.loads([ln for ln in p.stdout.splitlines() if ln.startswith("{")][-1])
    import bench
    assert d["value"] > 0 and d["metric"] == bench.METRIC_HEADLINE
    assert "charged 8 times" in d["cpu_baseline"]["sample"] and d["steps"] == 3


class _OracleEngine:
    """Stands in for the GPU engine in the bench's PageRank CPU leg: the
    interface the leg calls (csr, gather_ranks, apply_batch, sample_edges),
    backed by a second oracle whose ranks are handed out in FP32."""

    def __init__(self, n, off, dst):
        import oracle
        self.n = n
        self.o = oracle.Oracle(oracle.PR, n, off, dst, epsilon=1e-4, max_rounds=100)
        self.o.init()

    def csr(self):
        return self.o.csr()

    def gather_ranks(self):
        x, r = self.o.ranks()
        return x.astype("float32"), r.astype("float32")

    def apply_batch(self, d, a):
        self.o.apply_batch(d, a)

    def sample_edges(self, count, seed):
        import numpy as np
        off, dst, _ = self.o.csr()
        pick = np.random.default_rng(seed).choice(len(dst), size=count, replace=False)
        src = np.searchsorted(off, pick, side="right") - 1
        return np.stack([src.astype(np.uint32), dst[pick], np.ones(count, np.uint32)], 1)


def test_pagerank_cpu_leg_reports_the_oracle_comparison():
    import argparse
    import bench
    import oracle
    n, off, dst, _ = oracle.rmat_csr(12, 8, 3, with_w=False)
    eng = _OracleEngine(n, off, dst)
    args = argparse.Namespace(scale=12, seed=5, cpu_baseline_batches=2, config="rmat26")
    out = bench.cpu_baseline_pr(eng, args, 500, 500)
    assert out["value"] > 0 and out["kind"] == "port" and out["cores"] >= 1
    assert out["gpu_within_bound_of_oracle"] is True
    assert out["gpu_vs_oracle_max_abs_normalized"] < 1e-4


def _line(args):
    p = _run(args)
    assert p.returncode == 0, p.stderr[-2000:]
    return json.loads([ln for ln in p.stdout.splitlines() if ln.startswith("{")][-1])


def test_reference_arm_covers_every_algorithm_and_the_grid():
    for algo in ("bfs", "cc", "pr"):
        d = _line(["--impl", "reference", "--config", "rmat16", "--algo", algo, "--steps", "2",
                   "--warmup", "3"])
        assert d["value"] > 0 and algo in d["config"]["workload"], d
    # CC runs on the symmetrised graph with symmetric updates, as the library's arm does
    d = _line(["--impl", "reference", "--config", "rmat16", "--algo", "cc", "--steps", "2",
               "--warmup", "3"])
    assert "symmetrised" in d["config"]["workload"]
    for algo in ("sssp", "bfs"):
        d = _line(["--impl", "reference", "--config", "grid", "--scale", "6", "--batch", "200",
                   "--algo", algo, "--steps", "2", "--warmup", "3"])
        assert d["value"] > 0 and d["config"]["workload"].startswith("grid64x64"), d
    d = _line(["--impl", "reference", "--config", "grid", "--scale", "6", "--algo", "cc",
               "--steps", "2", "--warmup", "3"])
    assert "component" in d["unavailable"]


def test_reference_arm_declines_pagerank_beyond_its_time_bound():
    d = _line(["--impl", "reference", "--config", "rmat26", "--algo", "pr", "--steps", "2",
               "--warmup", "3"])
    assert d["impl"] == "reference" and "PageRank" in d["unavailable"]


def test_grid_snapshots_mix_grid_edges_and_shortcuts():
    import numpy as np
    import bench
    import oracle
    side = 256
    n, off, dst, w = oracle.grid_csr(side, 10, 8, 11, 1, 1000)
    nd, na, nb = 100, 100, 3
    batches = bench.make_batches(8, nb, nd, na, 5, bench._engine_sampler(off, dst, w), "grid", 1000)
    live = set((np.repeat(np.arange(n), np.diff(off.astype(np.int64))) * n + dst).tolist())
    seen = set()
    for d, a in batches:
        assert len(d) == nd and len(a) == na
        du, dv = d[:, 0].astype(np.int64), d[:, 1].astype(np.int64)
        is_grid = (np.abs(du - dv) == 1) | (np.abs(du - dv) == side)
        assert is_grid.sum() == 70
        keys = (du * n + dv).tolist()
        assert set(keys) <= live and not (set(keys) & seen) and len(set(keys)) == nd
        seen |= set(keys)
        au, av = a[:, 0].astype(np.int64), a[:, 1].astype(np.int64)
        assert (au != av).all() and (a[:, 2] >= 1).all() and (a[:, 2] <= 1000).all()
        cheb = np.maximum(np.abs(au // side - av // side), np.abs(au % side - av % side))
        # within radius 8, except a draw that landed on u itself and was moved to u + 1
        assert ((cheb <= 8) | (av == (au + 1) % n)).all()


def test_link_transactions():
    import bench
    b = bench.link_transactions(4_150_000, 0.98, 14.0)
    assert b["transactions_128B"] == 32_422  # ceil(4.15 MB / 128 B)
    assert abs(b["random_cost_ms"] - 32_422 * 14e-6) < 1e-3
    assert abs(b["ns_per_128B_achieved"] - 0.98e6 / 32_422) < 0.01
    assert b["ns_per_random_transaction"] == 14.0
    assert bench.link_transactions(0, 1.0, 14.0)["transactions_128B"] == 0
    assert bench.link_transactions(0, 1.0, 14.0)["ns_per_128B_achieved"] is None
    assert bench.link_transactions(-5.0, 1.0, 14.0)["random_cost_ms"] == 0
    assert bench.link_transactions(1000, 0, 14.0)["ns_per_128B_achieved"] is None


def test_rmat_snapshots_are_disjoint_live_deletions_and_rmat_insertions():
    import numpy as np
    import bench
    import oracle
    n, off, dst, w = oracle.rmat_csr(12, 8, 4)
    nd, na, nb = 200, 150, 4
    batches = bench.make_batches(12, nb, nd, na, 9, bench._engine_sampler(off, dst, w), "rmat26",
                                 rmat_fn=oracle.gen_rmat_edges)
    src = np.repeat(np.arange(n), np.diff(off.astype(np.int64)))
    live = set((src * n + dst).tolist())
    seen = set()
    adds_all = oracle.gen_rmat_edges(12, nb * na, 10)
    for i, (d, a) in enumerate(batches):
        keys = (d[:, 0].astype(np.int64) * n + d[:, 1]).tolist()
        assert len(d) == nd and set(keys) <= live and len(set(keys)) == nd and not set(keys) & seen
        seen |= set(keys)
        assert (a == adds_all[i * na:(i + 1) * na]).all()


def test_clock_samples_inside_the_timed_region_give_median_and_reasons():
    import bench

    class FakeProc:
        def terminate(self):
            pass

        def wait(self, timeout=None):
            return 0

    c = bench.Clocks(0)
    c.proc = FakeProc()
    row = "0, {sm}, 1965, 900.0, 0x0, {hw}, Not Active, Not Active, {cap}"
    c.lines = [(0.5, row.format(sm=1200, hw="Active", cap="Not Active")),     # before the window
               (1.0, row.format(sm=1965, hw="Not Active", cap="Not Active")),
               (1.5, row.format(sm=1950, hw="Not Active", cap="Active")),
               (2.0, row.format(sm=1965, hw="Not Active", cap="Not Active")),
               (3.5, row.format(sm=300, hw="Active", cap="Not Active"))]     # after it
    c.mark(1.0, 2.0)
    out = c.stop()
    assert out["sm_mhz"] == 1965.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"] and out["samples_inside_timed_region"] == 3


def test_engine_sampler_restatement():
    """The reference arm's restatement of the engine's edge sampler draws
    distinct live edges of the CSR, deterministically per seed, in the
    engine's order of draws (counter hash, first occurrences kept)."""
    import bench
    import oracle
    n, off, dst, w = oracle.rmat_csr(10, 8, 3, wlo=1, whi=64, with_w=True)
    smp = bench._engine_sampler(off, dst, w)
    a = smp(3000, 77)
    assert a.shape == (3000, 3)
    assert np.array_equal(a, smp(3000, 77)) and not np.array_equal(a, smp(3000, 78))
    keys = a[:, 0].astype(np.uint64) << np.uint64(32) | a[:, 1].astype(np.uint64)
    assert len(np.unique(keys)) == 3000  # distinct (the graph has no parallel edges)
    for u, v, ww in a[:200]:
        row = dst[off[u]:off[u + 1]]
        k = np.searchsorted(row, v)
        assert row[k] == v and w[int(off[u]) + int(k)] == ww
    # the first draws are the hash of the draw index, as in the engine
    total = np.uint64(len(dst))
    s0 = bench._mix64(np.uint64(77))
    r0 = int(bench._mix64(s0 ^ bench._mix64(np.uint64(0xA24BAED4963EE407))) % total)
    assert a[0, 0] == np.searchsorted(off, r0, side="right") - 1 and a[0, 1] == dst[r0]
