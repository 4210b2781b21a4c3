"""Benchmark: per-snapshot delta repair on an out-of-memory graph.

Headline (default, --config batched): the metric's own comparison,
learned+batched against plain on the same GPU and the same snapshots with
identical results. R-MAT scale 24 (16.8M vertices, edge factor 16, a=.57
b=.19 c=.19, self-loops and duplicates removed, ~263M directed edges),
uint32 weights uniform in [1,64] stored with every adjacency slot, SSSP from
256 seeded sources, the graph held in pinned host memory with its HBM
residency capped at 2 GB, snapshots of log-uniform size in [1K, 1M] updates
(half deletions sampled uniformly from live edges, half R-MAT insertions).
Three engines replay the same snapshots: batched+learned (all queries in one
repair launch per snapshot, snapshots replayed from CUDA graphs, learned
cache admission before each repair), batched+hotness, and plain (the
single-source repair once per query, hotness admission, host-driven).
Synthetic data: the reference's datasets are not available, seeded R-MAT
stands in for them.

One step = one snapshot (deletions, insertions, repair of every query, cache
maintenance).
  value: updates/s of batched+learned with the snapshots' records already
         resident in HBM (dycg_apply_batches_device), CUDA events on the
         engine stream.
  e2e:   the same engine through dycg_apply_batches with host buffers (H2D of
         the records and D2H of the control blocks inside the timed region).
Other configurations (--config rmat26|rmat16|grid|learned) cover the rest of
the workload table with their own lines.
N > 1 GPUs run independent replicas (a snapshot repair does not shard).

`--impl reference` times the reference's repair algorithm on the host cores
(the CPU oracle restatement; the reference's own engine cannot be built here)
on the same workload.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "batch-repair edges/s (updates applied and repaired per second)"
# the headline comparison: the batched many-query form with learned cache
# admission against the plain per-query path with hotness admission
METRIC_HEADLINE = ("batch-repair edges/s & ms/batch: learned+batched vs plain, same GPU, exact "
                   "results")
UNIT = "updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dycg", choices=["dycg", "reference"])
    ap.add_argument("--algo", default="sssp", choices=["sssp", "bfs", "cc", "pr"])
    ap.add_argument("--config", default="batched",
                    choices=["rmat26", "rmat16", "grid", "batched", "learned"],
                    help="batched (default, the headline metric): R-MAT 24, 256 queries, "
                         "batched+learned vs plain on the same snapshots; rmat26: out-of-memory "
                         "R-MAT, one source; rmat16: the small CPU-runnable R-MAT; grid: 4096^2 "
                         "road-like grid; learned: R-MAT 27 Zipf snapshots, learned vs hotness "
                         "vs no cache")
    ap.add_argument("--scale", type=int, default=None)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--batch", type=int, default=None, help="updates per snapshot (50/50)")
    ap.add_argument("--budget-gb", type=float, default=None)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--cpu-baseline-batches", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ordered-delta", type=int, default=None,
                    help="bucketed closure width (default: 0 on R-MAT, on the grid 2048 for SSSP "
                         "and 1 for BFS/CC)")
    ap.add_argument("--json-out", default=None)
    ap.add_argument("--mutation-ctas", type=int, default=0,
                    help="CTAs of the deletion/append kernels (0: the library default)")
    ap.add_argument("--frontier-queue", default="static", choices=["static", "claimed"],
                    help="single-source repair: how warps share a wave's rows")
    ap.add_argument("--page-shift", type=int, default=12,
                    help="log2 adjacency slots per cache page (8-20; single-source and batched "
                         "lines); 20 approximates the reference's SEGMENT-sized chunks")
    ap.add_argument("--queries", type=int, default=256, help="batched config: sources")
    ap.add_argument("--plain-queries", type=int, default=None,
                    help="batched config: queries timed on the per-query path (default all)")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--qratio", type=int, default=4)
    ap.add_argument("--heavy", type=int, default=64)
    ap.add_argument("--tile", type=int, default=4096)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--no-replay", action="store_true")
    ap.add_argument("--tune-batch", type=int, default=100_000)
    ap.add_argument("--trace-snapshots", type=int, default=10)
    ap.add_argument("--train-epochs", type=int, default=3)
    ap.add_argument("--train-lr", type=float, default=2e-3)
    ap.add_argument("--train-batch", type=int, default=8192)
    ap.add_argument("--batch-min", type=int, default=1_000)
    ap.add_argument("--batch-max", type=int, default=1_000_000)
    args = ap.parse_args()
    if args.ordered_delta is None:
        # grid SSSP (weights [1,1000]): delta 2048 took 330 ms per 10K snapshot against
        # 611 ms at 256 (fewer waves, 8% more row expansions)
        args.ordered_delta = 0 if args.config != "grid" else (2048 if args.algo == "sssp" else 1)
    defaults = {"rmat26": (26, 100_000, 4.0), "rmat16": (16, 2_000, 0.0),
                "grid": (12, 10_000, 0.25), "batched": (24, 0, 2.0),
                "learned": (27, 1_000_000, 8.0)}[args.config]
    if args.scale is None:
        args.scale = defaults[0]
    if args.batch is None:
        args.batch = defaults[1]
    if args.budget_gb is None:
        args.budget_gb = defaults[2]
    return args


class Clocks:
    """nvidia-smi samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.window = (0.0, 0.0)

    def start(self):
        """Start sampling and wait for the first sample (the sampler must be
        running when the timed region opens)."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 10:
                time.sleep(0.01)
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, t_begin, t_end):
        self.window = (t_begin, t_end)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.06)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        b, e = self.window
        inside = [ln for t, ln in self.lines if b - 0.05 <= t <= e + 0.05]
        for ln in inside or [ln for _, ln in self.lines[-2:]]:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "samples_inside_timed_region": len(inside)}


# DRAM bytes (read + write) of the dominant kernel per algorithmic HBM byte,
# from one ncu capture on a smaller case of the same workload (the full-size
# workloads hold tens of GB on the device, too large for a multi-metric
# capture); the line's `traffic` scales it by the run's own algorithmic bytes.
# None where no capture was taken.
# batched repair kernel, R-MAT 20 / 256 queries, the two timed launches of
# profiles/ncu_multi_repair_rmat20_q256.md: 2,728 MB DRAM / 589.2 MB algorithmic
NCU_TRAFFIC_RATIO = {("batched", "sssp"): 4.6}

# Random host-link transactions cost about the same whatever their size up to
# 128 bytes (dycg_measure_host_random: random 128-byte reads over an 8 GB
# pinned buffer, measured in the same run). A repair kernel's host-link bytes
# are row scans: consecutive 128-byte lines of one row share an address
# translation and cost less than a random transaction (~3.4 ns within a narrow
# window), so the random cost per 128 bytes is a scale for its time, not a
# lower bound on it.
def link_transactions(link_bytes, launch_ms, ns_per_tx):
    """A launch's host-link bytes in 128-byte transactions: the time they
    would take as random transactions at ns_per_tx each, and the launch's own
    time per 128 bytes."""
    tx = int(np.ceil(max(0.0, float(link_bytes)) / 128.0))
    return {"ns_per_random_transaction": ns_per_tx, "transactions_128B": tx,
            "random_cost_ms": round(tx * ns_per_tx / 1e6, 4),
            "ns_per_128B_achieved": round(launch_ms * 1e6 / tx, 2) if tx and launch_ms > 0
            else None}


def mutation_bound(updates, algo, ms, ns_per_tx):
    """Lower bound on the mutation kernels' time per snapshot: one random host
    transaction per update record (append or deletion window) and adjacency
    direction (two where the incoming adjacency is kept: SSSP/BFS)."""
    dirs = 2 if algo in ("sssp", "bfs") else 1
    tx = int(updates) * dirs
    bound_ms = tx * ns_per_tx / 1e6
    return {"ns_per_transaction": ns_per_tx, "transactions": tx, "bound_ms": round(bound_ms, 4),
            "ns_per_transaction_achieved": round(ms * 1e6 / tx, 2) if tx else None,
            "frac": round(bound_ms / ms, 4) if ms > 0 else None}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def make_batches(scale, total_batches, nd, na, seed, sample_fn, config="rmat26", wmax=64,
                 rmat_fn=None):
    """Deletions: nd distinct live edges per snapshot, disjoint across snapshots
    (sampled once from the initial graph); insertions: R-MAT draws (rmat_fn,
    the library's generator unless given). On the grid: 70% of the deletions
    are 4-neighbour grid edges and 30% shortcuts, and the insertions are new
    shortcuts within radius 8."""
    if config != "grid":
        if rmat_fn is None:
            import dycgraph_b200 as dg
            rmat_fn = dg.gen_rmat_edges
        dels = sample_fn(total_batches * nd, seed)
        adds = rmat_fn(scale, total_batches * na, seed + 1, first=0)
        return [(dels[i * nd:(i + 1) * nd], adds[i * na:(i + 1) * na])
                for i in range(total_batches)]
    side = 1 << scale
    # shortcuts are ~0.5% of the directed edges: sample a pool large enough to
    # hold 30% of every snapshot's deletions as shortcuts
    need = int(total_batches * nd * 0.3 / 0.004) + total_batches * nd
    pool = sample_fn(min(need, 48_000_000), seed)
    du = pool[:, 0].astype(np.int64)
    dv = pool[:, 1].astype(np.int64)
    is_grid = (np.abs(du - dv) == 1) | (np.abs(du - dv) == side)
    g, sc = pool[is_grid], pool[~is_grid]
    ns = min(nd - int(round(nd * 0.7)), len(sc) // total_batches)
    ng = nd - ns
    if len(g) < ng * total_batches:
        raise RuntimeError("not enough grid edges sampled")
    rng = np.random.default_rng(seed + 5)
    n = side * side
    u = rng.integers(0, n, size=total_batches * na)
    dr = rng.integers(-8, 9, size=u.shape[0])
    dc = rng.integers(-8, 9, size=u.shape[0])
    r = np.clip(u // side + dr, 0, side - 1)
    c = np.clip(u % side + dc, 0, side - 1)
    v = r * side + c
    v = np.where(v == u, (u + 1) % n, v)
    w = (np.random.default_rng(seed + 9).integers(1, wmax + 1, size=u.shape[0])).astype(np.uint32)
    adds = np.stack([u.astype(np.uint32), v.astype(np.uint32), w], 1)
    out = []
    for i in range(total_batches):
        d = np.concatenate([g[i * ng:(i + 1) * ng], sc[i * ns:(i + 1) * ns]])
        out.append((d, adds[i * na:(i + 1) * na]))
    return out


def replica_totals(ms, e2e_ms, per_step_updates, K, E, world, device):
    """N GPUs run independent replicas: the job time is the maximum of the
    ranks' device times, the throughput counts every rank's updates."""
    import torch
    t = torch.tensor([ms, e2e_ms], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms, e2e_ms = float(t[0]), float(t[1])
    value = per_step_updates * K * world / (ms / 1e3)
    e2e_value = per_step_updates * E * world / (e2e_ms / 1e3) if E and e2e_ms > 0 else None
    return ms, e2e_ms, value, e2e_value


# ----------------------------------------------------------------------------
def run_dycg(args):
    import torch
    import dycgraph_b200 as dg

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    K, W = args.steps, max(args.warmup, 3)
    E = args.e2e_steps if args.e2e_steps is not None else K
    nd = args.batch // 2
    na = args.batch - nd
    algo = args.algo
    budget = int(args.budget_gb * (1 << 30))

    t0 = time.time()
    eng = dg.Engine(algo, weight_mode="stored" if algo == "sssp" else "hash128",
                    hbm_graph_budget_bytes=budget,
                    symmetric=(algo == "cc" and args.config != "grid"), epsilon=1e-4,
                    device=local, mutation_ctas=args.mutation_ctas,
                    frontier_queue=args.frontier_queue, page_shift=args.page_shift,
                    ordered_delta=args.ordered_delta if algo != "pr" else 0)
    wmax = 1000 if args.config == "grid" else 64
    if args.config == "grid":
        eng.load_grid(1 << args.scale, 10, 8, seed=args.seed, wlo=1, whi=wmax)
    else:
        eng.load_rmat(args.scale, args.edge_factor, seed=args.seed, wlo=1, whi=wmax,
                      symmetrize=(algo == "cc"))
    t_load = time.time() - t0
    t0 = time.time()
    eng.start()
    t_init = time.time() - t0
    info = eng.info()
    batches = make_batches(args.scale, W + K + E, nd, na, args.seed + 17 + 1000 * rank,
                           eng.sample_edges, args.config, wmax)
    if algo == "cc" and args.config != "grid":  # symmetric updates on the symmetrised graph
        batches = [(np.concatenate([d, d[:, [1, 0, 2]]]), np.concatenate([a, a[:, [1, 0, 2]]]))
                   for d, a in batches]
    per_step_updates = sum(len(d) + len(a) for d, a in batches[:1])
    dev_batches = [(torch.from_numpy(d.astype(np.int32)).cuda(), torch.from_numpy(a.astype(np.int32)).cuda())
                   for d, a in batches[:W + K]]
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(eng.stream())

    def dev_step(i, st):
        d, a = dev_batches[i]
        eng.apply_batch_device(d.data_ptr(), d.shape[0], a.data_ptr(), a.shape[0], st)

    stats = dg.BatchStats()
    for i in range(W):
        dev_step(i, stats)
    # timed region: device-resident records
    clocks = Clocks(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    per = []
    t_begin = time.time()
    ev0.record(stream)
    for i in range(W, W + K):
        dev_step(i, stats)
        per.append(stats.as_dict())
    eng.stream()  # the engine stream waits for the last call's side-stream page staging
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks.mark(t_begin, time.time())
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        torch.distributed.barrier()
    # e2e: host buffers through the public C ABI
    e2e_ms = None
    if E:
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(W + K, W + K + E):
            d, a = batches[i]
            eng.apply_batch(d, a)
        eng.stream()
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1)
    ms, e2e_ms, value, e2e_value = replica_totals(ms, e2e_ms or 0.0, per_step_updates, K, E,
                                                  world, "cuda")

    # roofline of the dominant kernel (the persistent repair kernel; one launch
    # per snapshot): algorithmic bytes from the kernel's own counters
    page_bytes = 4 << 12
    page_bytes *= 2 if algo == "sssp" else 1
    rep_ms = np.mean([p["ms_repair"] for p in per])
    rep_link = np.mean([p["link_bytes"] - p["mutate_link_bytes"] - p["cache_pages_loaded"] * page_bytes
                        for p in per])
    rep_hbm = np.mean([p["hbm_adj_bytes"] - p["mutate_hbm_bytes"] - p["cache_pages_loaded"] * page_bytes
                       + p["state_bytes"] for p in per])
    mut_ms = np.mean([p["ms_mutate"] for p in per])
    mut_bytes_link = np.mean([p["mutate_link_bytes"] for p in per])
    mut_bytes_hbm = np.mean([p["mutate_hbm_bytes"] for p in per])
    hbm_peak, peak_kind = peaks()
    link_h2d, link_zc = dg.measure_host_link(local, 1 << 30)
    tx_ns = dg.measure_host_random(local, 8 << 30, 128, False, 1 << 22)
    ach_hbm = rep_hbm / (rep_ms * 1e6)
    ach_link = rep_link / (rep_ms * 1e6)
    t_bound = max(rep_hbm / (hbm_peak * 1e9), rep_link / (link_zc * 1e9))
    roofline = {
        "kernel": f"repair_kernel<{algo}>",
        "bound": "hbm", "achieved": round(ach_hbm, 2), "peak": hbm_peak, "unit": "GB/s",
        "frac": round(ach_hbm / hbm_peak, 5),
        "traffic": (int(NCU_TRAFFIC_RATIO[(args.config, algo)] * rep_hbm)
                    if (args.config, algo) in NCU_TRAFFIC_RATIO else None),
        "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6650 GB/s",
        "algorithmic_bytes_per_launch": {"hbm": int(rep_hbm), "host_link": int(rep_link)},
        "launch_ms": round(float(rep_ms), 4),
        "host_link": {"achieved": round(ach_link, 2), "peak_zero_copy": round(link_zc, 2),
                      "peak_h2d_copy": round(link_h2d, 2), "unit": "GB/s",
                      "frac": round(ach_link / link_zc, 5),
                      "transactions": link_transactions(rep_link, float(rep_ms), tx_ns)},
        "roofline_time_frac": round(t_bound / (rep_ms / 1e3), 5),
        # deletion search + appends: at least one random host transaction per
        # appended occurrence and per deletion record, in each adjacency direction
        "mutation_kernels": {"ms": round(float(mut_ms), 4), "link_bytes": int(mut_bytes_link),
                             "hbm_bytes": int(mut_bytes_hbm),
                             "transaction_bound": mutation_bound(per_step_updates, algo,
                                                                 float(mut_ms), tx_ns)},
    }
    launches = int(sum(p["kernel_launches"] for p in per))
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": round(ms / K, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32" if algo != "pr" else "f32",
        "data": "synthetic (seeded R-MAT; the reference's real graphs are not available)",
        "config": {"workload": (f"grid{1 << args.scale}x{1 << args.scale}+1%shortcuts"
                                if args.config == "grid" else
                                f"rmat{args.scale}-ef{args.edge_factor}") + f" {algo} "
                               f"{args.batch // 1000}K-update snapshots, HBM graph budget "
                               f"{args.budget_gb:g} GB",
                   "vertices": info["nodes"], "edges": info["live_edges"],
                   "updates_per_step": per_step_updates, "deletes_per_step": nd,
                   "inserts_per_step": na, "weights": f"uint32 uniform [1,{wmax}] stored"
                   if algo == "sssp" else "rule", "graph_host_bytes": info["host_bytes"],
                   "cached_pages": info["cached_pages"], "cache_slots": info["cache_slots"],
                   "page_slots": 1 << args.page_shift,
                   "l2": "inputs larger than L2 (graph in pinned host memory, vertex state "
                         f"{info['nodes'] * 40 / 1e9:.1f} GB in HBM)",
                   "parallelism": f"replicas x{world}", "ordered_delta": args.ordered_delta,
                   "load_s": round(t_load, 2),
                   "static_solve_s": round(t_init, 2)},
        "clocks": clk,
        "e2e": {"value": round(e2e_value, 1) if e2e_value else None, "unit": UNIT,
                "h2d_bytes_per_step": per_step_updates * 12, "d2h_bytes_per_step": 256,
                "steps": E},
        "gpu_launches": launches,
        "roofline": roofline,
        "per_step": {k: round(float(np.mean([p[k] for p in per])), 4) for k in
                     ("ms_ingest", "ms_mutate", "ms_repair", "ms_cache", "ms_total", "affected",
                      "expanded", "edges_scanned", "improvements", "waves", "relocated_rows",
                      "missing_deletes", "cache_pages_loaded", "link_bytes", "hbm_adj_bytes",
                      "ms_phase_invalidate", "ms_phase_pull", "ms_phase_seed",
                      "ms_phase_closure")},
    }
    _hb = float(np.sum([p["hbm_adj_bytes"] for p in per]))
    out["per_step"]["adjacency_hit_rate"] = round(
        _hb / max(1.0, _hb + float(np.sum([p["link_bytes"] for p in per]))), 4)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        if algo == "cc" and args.config == "grid":
            out["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(),
                                   "kind": "port", "sample": "not run: " + GRID_CC_CPU_REASON}
        elif algo == "pr":
            out["cpu_baseline"] = cpu_baseline_pr(eng, args, nd, na)
        else:
            out["cpu_baseline"] = cpu_baseline(eng, args, algo, nd, na)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    eng.close()
    return out if rank == 0 else None


def cpu_baseline(eng, args, algo, nd, na):
    """Time the CPU restatement of the reference's repair on a bounded sample
    of the same workload (the next snapshot(s), from the engine's state), and
    check the GPU's results on those snapshots against it."""
    import oracle
    t0 = time.time()
    off, dst, w = eng.csr()
    vals, par = eng.gather()
    threads = os.cpu_count() or 1
    orc = oracle.Oracle({"sssp": oracle.SSSP, "bfs": oracle.BFS, "cc": oracle.CC}[algo],
                        eng.n, off, dst, w if algo == "sssp" else None,
                        weight_mode=oracle.WEIGHT_STORED if algo == "sssp" else oracle.WEIGHT_HASH128,
                        symmetric=(algo == "cc"), threads=threads)
    orc.set_state(vals, par)
    del off, dst, w
    setup_s = time.time() - t0
    nb = max(1, args.cpu_baseline_batches)
    batches = make_batches(args.scale, nb, nd, na, args.seed + 999, eng.sample_edges, args.config,
                           1000 if args.config == "grid" else 64)
    cpu_s = 0.0
    parity = True
    for d, a in batches:
        t = time.perf_counter()
        orc.apply_batch(d, a)
        cpu_s += time.perf_counter() - t
        eng.apply_batch(d, a)
        parity &= bool((eng.gather()[0] == orc.values()[0]).all())
    upd = sum(len(d) + len(a) for d, a in batches)
    return {"value": round(upd / cpu_s, 1), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{nb} snapshot(s) of {upd // nb} updates on the same rmat{args.scale} graph "
                      f"and state as the GPU run ({cpu_s:.1f} s CPU; mutation parallel over "
                      f"sources, closures serial as in the reference's CPU-owner mode)",
            "setup_s": round(setup_s, 1), "gpu_matches_oracle": parity}


def cpu_baseline_pr(eng, args, nd, na):
    """PageRank: the CPU restatement of the reference's residual push (FP64)
    takes the engine's ranks and residuals, both repair the next snapshot(s),
    and the GPU's FP32 ranks are compared with the oracle's. Both stop pushing
    at the same per-vertex threshold, so each is within |r|_1 / (1 - alpha) of
    the exact ranks and the two within the sum of their bounds (plus FP32
    rounding, 1e-4 relative)."""
    import oracle
    t0 = time.time()
    off, dst, _ = eng.csr()
    x, r = eng.gather_ranks()
    threads = os.cpu_count() or 1
    orc = oracle.Oracle(oracle.PR, eng.n, off, dst, None, epsilon=1e-4, alpha=0.85,
                        max_rounds=100, threads=threads)
    orc.set_state(ranks=x.astype(np.float64), residuals=r.astype(np.float64))
    del off, dst
    setup_s = time.time() - t0
    nb = max(1, args.cpu_baseline_batches)
    batches = make_batches(args.scale, nb, nd, na, args.seed + 999, eng.sample_edges, args.config)
    cpu_s, err, within, tot = 0.0, 0.0, True, 1.0
    for d, a in batches:
        t = time.perf_counter()
        orc.apply_batch(d, a)
        cpu_s += time.perf_counter() - t
        eng.apply_batch(d, a)
        xg, rg = eng.gather_ranks()
        xo, ro = orc.ranks()
        diff = np.abs(xg.astype(np.float64) - xo)
        bound = (float(np.sum(np.abs(rg.astype(np.float64)))) + float(np.sum(np.abs(ro)))) / 0.15 \
            + 1e-4 * np.abs(xo)
        within &= bool((diff <= bound).all())
        err = max(err, float(diff.max()))
        tot = float(np.sum(xo))
    upd = sum(len(d) + len(a) for d, a in batches)
    return {"value": round(upd / cpu_s, 1), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{nb} snapshot(s) of {upd // nb} updates on the same rmat{args.scale} graph "
                      f"and PageRank state as the GPU run ({cpu_s:.1f} s CPU; FP64 residual push, "
                      f"epsilon 1e-4, at most 100 rounds)",
            "setup_s": round(setup_s, 1), "gpu_within_bound_of_oracle": within,
            "gpu_vs_oracle_max_abs": err, "gpu_vs_oracle_max_abs_normalized": err / tot}


# ----------------------------------------------------------------------------
# PageRank's CPU initial solve costs ~0.45 us per edge on 8 host cores (7.2 s
# at R-MAT 20): above R-MAT 24 it alone would exceed the run's few minutes
REF_PR_MAX_SCALE = 24
# CC on the grid: one deletion near a label root invalidates the whole
# component, and the CPU restatement's unordered label propagation re-walks it
GRID_CC_CPU_REASON = ("the CPU restatement's CC repair re-propagates labels over the whole "
                      "component after a deletion near a label root (45.8 s for one 10K-update "
                      "snapshot of a 1024x1024 grid, all 1.05M vertices affected, 8 host cores); "
                      "a 4096x4096 snapshot exceeds this run's time bound")


_M = (np.uint64(0x9E3779B97F4A7C15), np.uint64(0xBF58476D1CE4E5B9), np.uint64(0x94D049BB133111EB))


def _mix64(z):
    """SplitMix64 finalizer on uint64 arrays (the generators' mixing function)."""
    with np.errstate(over="ignore"):
        z = np.asarray(z, np.uint64) + _M[0]
        z = (z ^ (z >> np.uint64(30))) * _M[1]
        z = (z ^ (z >> np.uint64(27))) * _M[2]
        return z ^ (z >> np.uint64(31))


def _engine_sampler(off, dst, w):
    """The engine's edge sampler (dycg_sample_edges) restated for a host CSR of
    the freshly generated graph, so the reference arm repairs the very
    snapshots the library's arm does: live-edge ranks drawn by a counter hash
    in rounds, the first `count` distinct ranks in draw order kept, each rank
    resolved to its row and slot (every slot is live and rows are in CSR
    order before the first snapshot). Weights are the stored ones, or 0."""
    total = np.uint64(len(dst))

    def sample(count, seed):
        chosen = np.empty(0, np.uint64)
        rnd = 0
        while len(chosen) < count and rnd <= 64:
            need = count - len(chosen)
            draws = need + need // 16 + 64
            with np.errstate(over="ignore"):
                s = _mix64(np.uint64(seed % (1 << 64)) + np.uint64(rnd * 0x9E37))
                i = np.arange(draws, dtype=np.uint64) + np.uint64(0xA24BAED4963EE407)
            pos = _mix64(s ^ _mix64(i)) % total
            allp = np.concatenate([chosen, pos])
            first = np.zeros(len(allp), bool)
            first[np.unique(allp, return_index=True)[1]] = True
            new = pos[first[len(chosen):]]
            chosen = np.concatenate([chosen, new[:need]])
            rnd += 1
        r = chosen.astype(np.int64)
        src = np.searchsorted(off, r, side="right") - 1
        ww = w[r] if w is not None else np.zeros(len(r), np.uint32)
        return np.stack([src.astype(np.uint32), dst[r], ww], 1)
    return sample


def run_reference(args):
    """The reference's repair algorithm (CPU oracle restatement) on host cores,
    on the same workload as the library's arm: the same generated graph
    (R-MAT, symmetrised for CC, or the road-like grid), snapshots of the same
    shape, and the same algorithm settings."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    import oracle
    K, W = args.steps, max(args.warmup, 3)
    nd = args.batch // 2
    na = args.batch - nd
    algo = args.algo
    if args.config == "batched":
        return run_reference_batched(args)
    if args.config == "learned":
        return {"impl": "reference",
                "unavailable": "the reference has no learned admission (a GPU cache policy); the "
                               "learned line compares it with the hotness policy and no cache on "
                               "the same snapshots"}
    if algo == "pr" and (args.config == "grid" or args.scale > REF_PR_MAX_SCALE):
        return {"impl": "reference",
                "unavailable": f"PageRank's CPU initial solve above R-MAT {REF_PR_MAX_SCALE} takes "
                               "longer than this run's time bound (~0.45 us per edge on 8 host "
                               "cores); the library's line carries a PageRank cpu_baseline "
                               "started from the engine's ranks instead"}
    if algo == "cc" and args.config == "grid":
        return {"impl": "reference", "unavailable": GRID_CC_CPU_REASON}
    threads = os.cpu_count() or 1
    t0 = time.time()
    grid = args.config == "grid"
    wmax = 1000 if grid else 64
    sym = algo == "cc" and not grid
    if grid:
        n, off, dst, w = oracle.grid_csr(1 << args.scale, 10, 8, args.seed, 1, wmax,
                                         with_w=(algo == "sssp"))
    else:
        n, off, dst, w = oracle.rmat_csr(args.scale, args.edge_factor, args.seed, wlo=1, whi=wmax,
                                         with_w=(algo == "sssp"), symmetrize=sym)
    code = {"sssp": oracle.SSSP, "bfs": oracle.BFS, "cc": oracle.CC, "pr": oracle.PR}[algo]
    wmode = oracle.WEIGHT_STORED if algo == "sssp" else oracle.WEIGHT_HASH128
    orc = oracle.Oracle(code, n, off, dst, w, weight_mode=wmode, symmetric=sym, epsilon=1e-4,
                        alpha=0.85, max_rounds=100, threads=threads)
    if algo in ("cc", "pr"):
        orc.init()
    elif grid:
        # high diameter: one Dijkstra / BFS pass beats frontier waves by ~50x
        vals = (oracle.static_sssp(n, off, dst, w, wmode, 0) if algo == "sssp"
                else oracle.static_bfs(n, off, dst, 0))
        orc.set_state(vals, oracle.tight_parents(n, off, dst, w, code, wmode, 0, vals))
    else:
        vals, par = oracle.parallel_sssp(n, off, dst, w, code, wmode, 0)
        orc.set_state(vals, par)
    batches = make_batches(args.scale, W + K, nd, na, args.seed + 17, _engine_sampler(off, dst, w),
                           args.config, wmax, rmat_fn=oracle.gen_rmat_edges)
    if sym:  # symmetric updates on the symmetrised graph
        batches = [(np.concatenate([d, d[:, [1, 0, 2]]]), np.concatenate([a, a[:, [1, 0, 2]]]))
                   for d, a in batches]
    del off, dst, w
    setup_s = time.time() - t0
    # a step is a bounded sample: a full snapshot, or a fixed leading slice of
    # its deletions and insertions when a whole one would not fit the run's
    # time bound (~150 s of steps)
    budget = min(20.0, max(1.0, 150.0 / (W + K)))
    frac = 1.0
    t = time.perf_counter()
    orc.apply_batch(*batches[0])
    first = time.perf_counter() - t
    if first > budget:
        frac = max(0.01, budget / first)

    def sample(i):
        d, a = batches[i]
        return d[:max(1, int(len(d) * frac))], a[:max(1, int(len(a) * frac))]
    for i in range(1, W):
        orc.apply_batch(*sample(i))
    steps = [sample(i) for i in range(W, W + K)]
    t = time.perf_counter()
    for d, a in steps:
        orc.apply_batch(d, a)
    el = time.perf_counter() - t
    upd = sum(len(d) + len(a) for d, a in steps)
    value = upd / el
    workload = (f"grid{1 << args.scale}x{1 << args.scale}+1%shortcuts {algo}" if grid else
                f"rmat{args.scale}-ef{args.edge_factor}{' symmetrised' if sym else ''} {algo}")
    per = len(batches[0][0]) + len(batches[0][1])
    sample_desc = (f"{K} steps of {upd // K} updates ({frac:.0%} of a {per}-update snapshot) "
                   f"on {workload}; CPU restatement of the reference's repair (reference "
                   f"engine itself not buildable without its CMake deps)")
    return {"impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT,
            "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": K, "warmup": W,
            "ms_per_step": round(el * 1e3 / K, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if algo == "pr" else "u32",
            "data": "synthetic (seeded " + ("grid)" if grid else "R-MAT)"),
            "config": {"workload": f"{workload} " + (f"{args.batch // 1000}K" if args.batch % 1000 == 0
                                                     else f"{args.batch}") + "-update snapshots",
                       "setup_s": round(setup_s, 1), "first_snapshot_s": round(first, 2)},
            "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": threads,
                             "kind": "port", "sample": sample_desc},
            "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_reference_batched(args):
    """Many sources on one R-MAT graph with the reference's repair on the host
    cores. The reference engine holds one source, so the oracle repairs query
    0's results through the snapshots and the time is charged once per query.
    The graph, the way sources are drawn and the snapshot sizes (log-uniform in
    [batch_min, batch_max]) follow the library's batched arm."""
    import oracle
    K, W = args.steps, max(args.warmup, 3)
    Q = args.queries
    algo = args.algo if args.algo in ("sssp", "bfs") else "sssp"
    threads = os.cpu_count() or 1
    t0 = time.time()
    n, off, dst, w = oracle.rmat_csr(args.scale, args.edge_factor, args.seed, wlo=1, whi=64,
                                     with_w=(algo == "sssp"))
    sample = _engine_sampler(off, dst, w)
    smp = sample(16 * Q, args.seed + 3)
    _, first = np.unique(smp[:, 0], return_index=True)
    sources = smp[np.sort(first), 0][:Q].astype(np.uint32)
    # the library's arm's snapshot sequence: the mapping-tuning snapshot, the
    # traced ones, warm-up, timed and e2e snapshots (same sizes, same records)
    T = args.trace_snapshots
    E = args.e2e_steps if args.e2e_steps is not None else min(K, 8)
    rng = np.random.default_rng(args.seed + 41)
    sizes = np.exp(rng.uniform(np.log(args.batch_min), np.log(args.batch_max), T + W + K))
    sizes = np.maximum(2, sizes.astype(np.int64))
    sizes = np.concatenate([sizes, sizes[T + W:T + W + E]])
    sizes = np.concatenate([[args.tune_batch], sizes])
    nd = sizes // 2
    na = sizes - nd
    dels = sample(int(nd.sum()), args.seed + 17)
    adds = oracle.gen_rmat_edges(args.scale, int(na.sum()), args.seed + 18)
    snaps, i, j = [], 0, 0
    for d_, a_ in zip(nd.tolist(), na.tolist()):
        snaps.append((dels[i:i + d_], adds[j:j + a_]))
        i += d_
        j += a_
    # the snapshots before the library's warm-up ones (mapping tuning, traces)
    # are applied first, untimed, so both arms repair the same graph states
    pre, snaps = snaps[:1 + T], snaps[1 + T:1 + T + W + K]
    code = oracle.SSSP if algo == "sssp" else oracle.BFS
    wmode = oracle.WEIGHT_STORED if algo == "sssp" else oracle.WEIGHT_HASH128
    src0 = int(sources[0])
    orc = oracle.Oracle(code, n, off, dst, w, weight_mode=wmode, source=src0, threads=threads)
    vals, par = oracle.parallel_sssp(n, off, dst, w, code, wmode, src0)
    orc.set_state(vals, par)
    del off, dst, w, dels, adds
    for d, a in pre:
        orc.apply_batch(d, a)
    setup_s = time.time() - t0
    # a step is a bounded sample: the snapshot, or a leading slice of its
    # deletions and insertions sized from the first snapshot's rate so that
    # all steps fit ~150 s
    t = time.perf_counter()
    orc.apply_batch(*snaps[0])
    first = time.perf_counter() - t
    rate = (len(snaps[0][0]) + len(snaps[0][1])) / max(first, 1e-6)
    cap = max(1000, int(rate * 150.0 / (W + K)))

    def step(i):
        d, a = snaps[i]
        return d[:cap // 2], a[:cap - cap // 2]
    for i in range(1, W):
        orc.apply_batch(*step(i))
    steps = [step(i) for i in range(W, W + K)]
    t = time.perf_counter()
    for d, a in steps:
        orc.apply_batch(d, a)
    el = time.perf_counter() - t
    upd = sum(len(d) + len(a) for d, a in steps)
    value = upd / (el * Q)
    full = int(sum(len(d) + len(a) for d, a in snaps[W:W + K]))
    workload = (f"rmat{args.scale}-ef{args.edge_factor} {algo}, {Q} sources, snapshots of "
                f"{args.batch_min}-{args.batch_max} updates (log-uniform)")
    sample_desc = (f"{K} steps, {upd} of their {full} updates (steps capped at {cap} updates), "
                   f"query 0's results repaired by the CPU restatement of the reference's repair "
                   f"and charged {Q} times (the reference engine holds one source)")
    return {"impl": "reference", "metric": METRIC_HEADLINE,
            "value": round(value, 1), "unit": UNIT,
            "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": K, "warmup": W,
            "ms_per_step": round(el * 1e3 * Q / K, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded R-MAT)",
            "config": {"workload": workload, "setup_s": round(setup_s, 1),
                       "first_snapshot_s": round(first, 2)},
            "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": threads,
                             "kind": "port", "sample": sample_desc},
            "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


# ----------------------------------------------------------------------------
def query_snapshots(eng, args, sizes, seed):
    """Snapshots of the given sizes (half deletions, half insertions):
    deletions are distinct live edges of the initial graph, disjoint across
    snapshots; insertions are R-MAT draws with seeded weights."""
    import dycgraph_b200 as dg
    nd = sizes // 2
    na = sizes - nd
    dels = eng.sample_edges(int(nd.sum()), seed)
    adds = dg.gen_rmat_edges(args.scale, int(na.sum()), seed + 1, first=0)
    out, i, j = [], 0, 0
    for d, a in zip(nd.tolist(), na.tolist()):
        out.append((dels[i:i + d], adds[j:j + a]))
        i += d
        j += a
    return out


def run_batched(args):
    """The metric's comparison on the many-query workload: R-MAT scale 24,
    SSSP (or BFS) from `queries` seeded sources, snapshots of log-uniform size
    in [batch_min, batch_max], every query repaired after every snapshot,
    the graph's HBM residency capped at budget_gb. Three engines replay the
    same snapshots from the same graph:
      batched+learned  one repair launch per snapshot for all queries, the
                       snapshots replayed from captured CUDA graphs, pages
                       admitted by the learned policy (trained on the first
                       `trace` snapshots' traces) before each repair;
      batched+hotness  the same with the hotness policy (the learned policy's
                       fallback and yardstick);
      plain            the single-source repair launched once per query,
                       hotness admission, one host-driven call per snapshot.
    `value` is the first; results must be identical across all three."""
    import torch
    import dycgraph_b200 as dg

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    K, W = args.steps, max(args.warmup, 3)
    E = args.e2e_steps if args.e2e_steps is not None else min(K, 8)
    T = args.trace_snapshots
    algo = args.algo if args.algo in ("sssp", "bfs") else "sssp"
    Q = args.queries
    budget = int(args.budget_gb * (1 << 30))
    rng = np.random.default_rng(args.seed + 41 + 1000 * rank)
    sizes = np.exp(rng.uniform(np.log(args.batch_min), np.log(args.batch_max), T + W + K))
    sizes = np.maximum(2, sizes.astype(np.int64))
    # the e2e snapshots (new records) repeat the sizes of the first E timed
    # ones, so e2e and value are rates over the same size mix
    sizes = np.concatenate([sizes, sizes[T + W:T + W + E]])
    # snapshot 0 tunes the work mapping (untimed); all deletions are disjoint
    sizes = np.concatenate([[args.tune_batch], sizes])

    def build():
        eng = dg.Engine(algo, weight_mode="stored" if algo == "sssp" else "hash128",
                        hbm_graph_budget_bytes=budget, cache_policy="hotness", device=local,
                        mutation_ctas=args.mutation_ctas, page_shift=args.page_shift)
        eng.load_rmat(args.scale, args.edge_factor, seed=args.seed, wlo=1, whi=64)
        return eng

    snaps, sources, info = None, None, None
    sample_q = sorted({0, 1, Q // 2, Q - 1})

    def arm(mode, policy, headline):
        """One engine through the whole snapshot sequence; returns timings,
        per-snapshot stats and the sampled queries' values."""
        nonlocal snaps, sources, info
        t0 = time.time()
        eng = build()
        t_load = time.time() - t0
        if snaps is None:
            info = eng.info()
            smp = eng.sample_edges(16 * Q, args.seed + 3)
            _, first = np.unique(smp[:, 0], return_index=True)
            sources = smp[np.sort(first), 0][:Q].astype(np.uint32)
            snaps = query_snapshots(eng, args, sizes, args.seed + 17 + 1000 * rank)
        eng.set_queries(sources, mode)
        eng.set_query_mapping(args.qratio, args.heavy, args.tile)
        t0 = time.time()
        eng.start()
        t_init = time.time() - t0
        tried = []
        if mode == "batched" and not args.no_tune:
            tried = eng.tune_query_mapping(*snaps[0])
        else:
            eng.apply_batch(*snaps[0])
        dev = [(torch.from_numpy(d.astype(np.int32)).cuda(), torch.from_numpy(a.astype(np.int32)).cuda())
               for d, a in snaps[1:1 + T + W + K]]
        st = dg.BatchStats()

        def dev_step(i):
            d, a = dev[i]
            eng.apply_batch_device(d.data_ptr(), d.shape[0], a.data_ptr(), a.shape[0], st)
            return st.as_dict()
        report = None
        if policy == "learned":
            eng.policy_trace(T)
        for i in range(T):
            dev_step(i)
        if policy == "learned":
            report = eng.policy_train(epochs=args.train_epochs, lr=args.train_lr,
                                      batch=args.train_batch, seed=args.seed)
            eng.set_cache_policy("learned")
        for i in range(T, T + W):
            dev_step(i)
        max_records = int(max(max(len(d), len(a)) for d, a in snaps))
        eng.reserve_batch(max_records)
        replay = mode == "batched" and not args.no_replay
        t_nd = [int(dev[i][0].shape[0]) for i in range(T + W, T + W + K)]
        t_na = [int(dev[i][1].shape[0]) for i in range(T + W, T + W + K)]
        if replay:
            t_dels = torch.cat([dev[i][0].reshape(-1) for i in range(T + W, T + W + K)])
            t_adds = torch.cat([dev[i][1].reshape(-1) for i in range(T + W, T + W + K)])
        stream = torch.cuda.ExternalStream(eng.stream())
        clocks = Clocks(local) if headline else None
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        if clocks:
            clocks.start()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        t_begin = time.time()
        ev0.record(stream)
        if replay:
            arr = eng.apply_batches_device(t_dels.data_ptr(), t_nd, t_adds.data_ptr(), t_na)
            per = [arr[i].as_dict() for i in range(K)]
        else:
            per = [dev_step(i) for i in range(T + W, T + W + K)]
        eng.stream()  # the engine stream waits for the last call's side-stream page staging
        ev1.record(stream)
        torch.cuda.synchronize()
        clk = None
        if clocks:
            clocks.mark(t_begin, time.time())
            clk = clocks.stop()
        ms = ev0.elapsed_time(ev1)
        del dev
        # e2e: host records through the public C ABI, copies inside the timed region
        e2e_ms, e2e_upd = 0.0, 0
        host = snaps[1 + T + W + K:]
        if host:
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if replay:
                eng.apply_batches(host)
            else:
                for d, a in host:
                    eng.apply_batch(d, a)
            eng.stream()
            e1.record(stream)
            torch.cuda.synchronize()
            e2e_ms = e0.elapsed_time(e1)
            e2e_upd = int(sum(len(d) + len(a) for d, a in host))
        vals = {q: eng.gather_query(q)[0] for q in sample_q}
        upd = int(sum(t_nd) + sum(t_na))
        link = int(sum(p["link_bytes"] for p in per))
        hbm = int(sum(p["hbm_adj_bytes"] for p in per))
        res = {"mode": mode, "policy": policy, "ms": ms, "per": per, "clk": clk, "vals": vals,
               "upd": upd, "e2e_ms": e2e_ms, "e2e_upd": e2e_upd, "tried": tried,
               "report": report, "load_s": t_load, "init_s": t_init,
               "link_bytes_per_step": link // K, "hbm_adj_bytes_per_step": hbm // K,
               "hit_rate": round(hbm / max(1, hbm + link), 4)}
        return eng, res

    arms = {}
    # the headline engine last: slowdowns of later engines (host memory
    # placement after earlier multi-GB pinned allocations) count against it
    order = ([] if args.no_plain else [("per_query", "hotness")]) + \
            [("batched", "hotness"), ("batched", "learned")]
    cpu = static_ok = None
    for mode, policy in order:
        headline = (mode, policy) == ("batched", "learned")
        eng, res = arm(mode, policy, headline)
        arms[(mode, policy)] = res
        if headline and rank == 0 and world == 1:
            if not args.no_cpu_baseline:
                # from-scratch static recompute of one query on the final graph
                static_ok = query_static_check(eng, algo, int(sources[1]), res["vals"][1])
                cpu = query_cpu_baseline(eng, args, algo, int(sources[0]), Q)
        if headline:
            hl_eng = eng
        else:
            eng.close()
            del eng

    L = arms[("batched", "learned")]
    H = arms[("batched", "hotness")]
    P = arms.get(("per_query", "hotness"))
    t = torch.tensor([L["ms"], L["e2e_ms"], P["ms"] if P else 0.0], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms, e2e_ms, p_ms = float(t[0]), float(t[1]), float(t[2])
    value = L["upd"] * world / (ms / 1e3)
    e2e_value = L["e2e_upd"] * world / (e2e_ms / 1e3) if e2e_ms > 0 else None
    exact = {f"{m}+{p}": all(bool(np.array_equal(r["vals"][q], L["vals"][q])) for q in sample_q)
             for (m, p), r in arms.items() if (m, p) != ("batched", "learned")}
    exact["queries_compared"] = sample_q
    if static_ok is not None:
        exact["static_recompute_query1"] = static_ok
    if cpu is not None:
        exact["incremental_oracle_query0"] = cpu.get("gpu_matches_oracle")

    per = L["per"]
    roofline = batched_roofline(dg, per, K, algo, Q, local)

    def summary(r):
        pp = r["per"]
        return {"value": round(r["upd"] * world / (r["ms"] / 1e3), 1), "unit": UNIT,
                "ms_per_step": round(r["ms"] / K, 4),
                "median_ms_per_step": round(float(np.median([p["ms_total"] for p in pp])), 4),
                "e2e": round(r["e2e_upd"] / (r["e2e_ms"] / 1e3), 1) if r["e2e_ms"] > 0 else None,
                "link_bytes_per_step": r["link_bytes_per_step"],
                "hbm_adj_bytes_per_step": r["hbm_adj_bytes_per_step"], "hit_rate": r["hit_rate"],
                "static_solve_s": round(r["init_s"], 2),
                "gpu_launches": int(sum(p["kernel_launches"] for p in pp)),
                "per_step": {k: round(float(np.mean([p[k] for p in pp])), 4) for k in
                             ("ms_ingest", "ms_mutate", "ms_repair", "ms_cache", "ms_total",
                              "edges_scanned", "cache_pages_loaded")}}
    mapping = min(L["tried"], key=lambda x: x["repair_ms"]) if L["tried"] else \
        {"qratio": args.qratio, "heavy": args.heavy, "tile": args.tile}
    per_step = {k: round(float(np.mean([p[k] for p in per])), 4) for k in
                ("ms_ingest", "ms_mutate", "ms_repair", "ms_cache", "ms_total", "affected",
                 "expanded", "edges_scanned", "improvements", "waves", "missing_deletes",
                 "cache_pages_loaded", "ms_phase_invalidate", "ms_phase_pull", "ms_phase_seed",
                 "ms_phase_closure")}
    out = {
        "metric": METRIC_HEADLINE, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": round(ms / K, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded R-MAT; the reference's real graphs are not available)",
        "config": {"workload": f"rmat{args.scale}-ef{args.edge_factor} {algo}, {Q} queries, "
                               f"snapshots log-uniform in [{args.batch_min}, {args.batch_max}] "
                               f"updates, HBM graph budget {args.budget_gb:g} GB; "
                               "batched+learned vs plain on the same snapshots",
                   "vertices": info["nodes"], "edges": info["live_edges"],
                   "updates_timed": L["upd"],
                   "snapshot_sizes": [int(x) for x in sizes[1 + T + W:1 + T + W + K]],
                   "weights": "uint32 uniform [1,64] stored" if algo == "sssp" else "rule",
                   "page_slots": 1 << args.page_shift,
                   "mapping": {k: mapping.get(k) for k in ("qratio", "heavy", "tile", "pull_qratio",
                                                            "queue")},
                   "mapping_tuned_on": (f"one {args.tune_batch}-update snapshot, "
                                        f"{len(L['tried'])} candidates") if L["tried"] else "not tuned",
                   "replay": "one dycg_apply_batches_device call for the timed snapshots "
                             "(a CUDA graph per batch-size class, cache admission inside it)"
                             if not args.no_replay else "one dycg_apply_batch_device call per snapshot",
                   "learned": f"trained on the traces of snapshots 1-{T} (batched form, hotness "
                              f"policy), then admitting before every repair",
                   "l2": "inputs larger than L2 (graph in pinned host memory, "
                         f"{info['nodes'] * Q * 8 / 1e9:.0f} GB of query state in HBM)",
                   "parallelism": f"replicas x{world}", "load_s": round(L["load_s"], 2),
                   "static_solve_s": round(L["init_s"], 2)},
        "clocks": L["clk"],
        # e2e runs on E snapshots drawn after the timed ones, with the sizes
        # of the first E timed snapshots
        "e2e": {"value": round(e2e_value, 1) if e2e_value else None, "unit": UNIT,
                "h2d_bytes_per_step": int(L["e2e_upd"] * 12 / max(E, 1)),
                "d2h_bytes_per_step": int(sizeof_ctl() * 1), "steps": E,
                "mean_updates_per_step": int(L["e2e_upd"] / max(E, 1)),
                "timed_mean_updates_per_step": int(L["upd"] / max(K, 1)),
                "snapshots": "the e2e steps' own snapshots, drawn after the timed ones, with "
                             "the sizes of the first E timed snapshots"},
        "gpu_launches": int(sum(p["kernel_launches"] for p in per)),
        "roofline": roofline,
        "per_step": per_step,
        "plain": summary(P) if P else None,
        "speedup_vs_plain": round(value / (P["upd"] * world / (p_ms / 1e3)), 2) if P else None,
        "batched_hotness": summary(H),
        "learned_vs_hotness": {"updates_per_s": round(L["upd"] / L["ms"] / (H["upd"] / H["ms"]), 3),
                               "link_bytes": round(H["link_bytes_per_step"] /
                                                   max(1, L["link_bytes_per_step"]), 3),
                               "hit_rate": {"learned": L["hit_rate"], "hotness": H["hit_rate"]}},
        "training": L["report"],
        "results_equal": exact,
        # [qratio, heavy, pull ratio, query-lane tile slots, frontier-queue scheme
        # (DYCG_QUEUE_* bits: 1 claimed, 2 ranges), repair ms] per trial
        "mapping_candidates": [[x["qratio"], x["heavy"], x["pull_qratio"], x["tile"], x["queue"],
                                round(x["repair_ms"], 3)] for x in L["tried"]],
    }
    if cpu:
        out["cpu_baseline"] = cpu
    hl_eng.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return out if rank == 0 else None


def sizeof_ctl():
    """Bytes of the per-snapshot control block read back to the host."""
    import dycgraph_b200 as dg
    return dg.CTL_BYTES


def batched_roofline(dg, per, K, algo, Q, device):
    """Roofline of the batched repair kernel (one launch per snapshot, the
    dominant kernel): algorithmic bytes from the kernel's own counters over
    its own stamped duration, against the HBM peak and the host link measured
    in this run (streaming reads, and random transactions over a multi-GB
    pinned buffer, the way the kernel touches rows of the arena)."""
    page_bytes = (4 << 12) * (2 if algo == "sssp" else 1)
    rep_ms = float(np.sum([p["ms_repair"] for p in per]))
    rep_link = float(np.sum([p["link_bytes"] - p["mutate_link_bytes"]
                             - p["cache_pages_loaded"] * page_bytes for p in per]))
    rep_hbm = float(np.sum([p["hbm_adj_bytes"] - p["mutate_hbm_bytes"]
                            - p["cache_pages_loaded"] * page_bytes + p["state_bytes"] for p in per]))
    hbm_peak, peak_kind = peaks()
    link_h2d, link_zc = dg.measure_host_link(device, 1 << 30)
    tx_ns = dg.measure_host_random(device, 8 << 30, 128, False, 1 << 22)
    ach_hbm = rep_hbm / (rep_ms * 1e6)
    ach_link = rep_link / (rep_ms * 1e6)
    t_bound = max(rep_hbm / (hbm_peak * 1e9), rep_link / (link_zc * 1e9))
    traffic = NCU_TRAFFIC_RATIO.get(("batched", algo))
    return {
        "kernel": f"multi_repair_kernel<{algo}, {Q} queries>",
        "bound": "hbm", "achieved": round(ach_hbm, 2), "peak": hbm_peak, "unit": "GB/s",
        "frac": round(ach_hbm / hbm_peak, 5),
        "traffic": int(traffic * rep_hbm / K) if traffic else None,
        "traffic_note": ("DRAM read+write bytes per launch, scaled from an ncu capture on a "
                         "smaller case by its ratio of DRAM bytes to algorithmic HBM bytes "
                         f"({traffic})" if traffic else "no ncu capture for this workload"),
        "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                       else "fallback 6650 GB/s",
        "algorithmic_bytes_per_launch": {"hbm": int(rep_hbm / K), "host_link": int(rep_link / K)},
        "launch_ms": round(rep_ms / K, 4),
        "host_link": {"achieved": round(ach_link, 2), "peak_zero_copy": round(link_zc, 2),
                      "peak_h2d_copy": round(link_h2d, 2), "unit": "GB/s",
                      "frac": round(ach_link / link_zc, 5),
                      "transactions": link_transactions(rep_link / K, rep_ms / K, tx_ns),
                      "measured_in_run": "streaming and copy-engine GB/s, and ns per random "
                                         "128-byte read over an 8 GB pinned buffer"},
        "roofline_time_frac": round(t_bound / (rep_ms / 1e3), 5),
    }


def query_static_check(eng, algo, source, vals):
    """From-scratch static recompute of one query on the engine's final graph
    (CPU, parallel label-correcting solver) against the GPU's values."""
    import oracle
    off, dst, w = eng.csr()
    code = oracle.SSSP if algo == "sssp" else oracle.BFS
    wmode = oracle.WEIGHT_STORED if algo == "sssp" else oracle.WEIGHT_HASH128
    ref, _ = oracle.parallel_sssp(eng.n, off, dst, w if algo == "sssp" else None, code, wmode,
                                  source)
    return bool(np.array_equal(ref, vals))


def query_cpu_baseline(eng, args, algo, source, Q):
    """The reference repairs one source per engine: time the CPU restatement
    of its repair for query 0 on one sample snapshot and charge it Q times;
    check the GPU's query-0 result on that snapshot against it."""
    import oracle
    threads = os.cpu_count() or 1
    off, dst, w = eng.csr()
    vals, par = eng.gather_query(0)
    code = oracle.SSSP if algo == "sssp" else oracle.BFS
    orc = oracle.Oracle(code, eng.n, off, dst, w if algo == "sssp" else None,
                        weight_mode=oracle.WEIGHT_STORED if algo == "sssp" else oracle.WEIGHT_HASH128,
                        source=source, threads=threads)
    orc.set_state(vals, par)
    del off, dst, w
    (d, a), = query_snapshots(eng, args, np.array([20_000]), args.seed + 999)
    t = time.perf_counter()
    orc.apply_batch(d, a)
    cpu_s = time.perf_counter() - t
    eng.apply_batch(d, a)
    parity = bool((eng.gather_query(0)[0] == orc.values()[0]).all())
    upd = len(d) + len(a)
    return {"value": round(upd / (cpu_s * Q), 1), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"one {upd}-update snapshot repaired for query 0 ({cpu_s:.2f} s CPU), "
                      f"charged {Q} times (one repair per source, as the reference's engine "
                      f"holds one source)",
            "gpu_matches_oracle": parity}


# ----------------------------------------------------------------------------
def zipf_ids(n, count, rng, perm, s=1.1):
    """Vertex ids with Zipf(s)-distributed ranks (rank 1 hottest), scattered by perm."""
    out = np.empty(0, np.int64)
    while len(out) < count:
        k = rng.zipf(s, size=2 * (count - len(out)) + 16)
        out = np.concatenate([out, k[k <= n] - 1])
    return perm[out[:count]].astype(np.uint32)


def zipf_snapshots(eng, count, size, rng, perm, wmax=64):
    """`count` snapshots of `size` updates (half deletions, half insertions)
    whose endpoints are Zipf(1.1) over the vertices, drawn from the engine's
    current graph: insertions draw both endpoints; deletions take a live
    out-edge of a drawn source, each edge at most once across the snapshots
    drawn together."""
    n = eng.n
    nd = size // 2
    cands = []
    for _ in range(count):
        d = eng.sample_row_edges(zipf_ids(n, nd + nd // 2, rng, perm), int(rng.integers(1 << 62)))
        cands.append(d[d[:, 0] != 0xFFFFFFFF])
    keys = np.concatenate([c[:, 0].astype(np.uint64) << np.uint64(32) | c[:, 1].astype(np.uint64)
                           for c in cands])
    first = np.zeros(len(keys), bool)
    first[np.unique(keys, return_index=True)[1]] = True
    out, o = [], 0
    for c in cands:
        d = c[first[o:o + len(c)]][:nd]
        o += len(c)
        u = zipf_ids(n, size - nd, rng, perm)
        v = zipf_ids(n, size - nd, rng, perm)
        keep = u != v
        u, v = u[keep], v[keep]
        # weight from the endpoints, so parallel copies of an edge agree
        w = 1 + (u.astype(np.uint64) * np.uint64(0x9E3779B1) +
                 v.astype(np.uint64) * np.uint64(0x85EBCA77)) % np.uint64(wmax)
        out.append((d, np.stack([u, v, w.astype(np.uint32)], 1).astype(np.uint32)))
    return out


def run_learned(args):
    """Learned cache admission against the hotness and no-cache policies on
    the same snapshots: R-MAT 27 (134M vertices, ~2.1B edges), HBM graph budget
    8 GB, snapshots of 1M Zipf(1.1)-skewed updates; the network is trained on
    the traces of the first `trace` snapshots (hotness policy), then all
    policies repair the same following snapshots."""
    import torch
    import dycgraph_b200 as dg
    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    torch.cuda.set_device(local)
    K, W = args.steps, max(args.warmup, 3)
    E = args.e2e_steps if args.e2e_steps is not None else 3
    T = args.trace_snapshots
    algo = args.algo if args.algo in ("sssp", "pr") else "sssp"
    budget = int(args.budget_gb * (1 << 30))
    snaps = None
    res = {}
    report = None
    # order: the learned engine last, so any slowdown of later engines (host
    # memory placement after earlier multi-GB pinned allocations) counts
    # against it; the first engine draws the snapshots all of them replay
    for policy in ("none", "hotness", "learned"):
        t0 = time.time()
        eng = dg.Engine(algo, weight_mode="stored" if algo == "sssp" else "hash128",
                        hbm_graph_budget_bytes=0 if policy == "none" else budget,
                        cache_policy="none" if policy == "none" else "hotness", epsilon=1e-4,
                        device=local, mutation_ctas=args.mutation_ctas)
        eng.load_rmat(args.scale, args.edge_factor, seed=args.seed, wlo=1, whi=64)
        t_load = time.time() - t0
        t0 = time.time()
        eng.start()
        t_init = time.time() - t0
        first = snaps is None
        if first:
            # the first engine draws each phase's snapshots from its graph at
            # that point; the other engines replay the same records
            rng = np.random.default_rng(args.seed + 77)
            perm = rng.permutation(eng.n)
            snaps = zipf_snapshots(eng, T, args.batch, rng, perm)
        eng.reserve_batch(args.batch)
        if policy == "learned":
            eng.policy_trace(T)
        for d, a in snaps[:T]:
            eng.apply_batch(d, a)
        if policy == "learned":
            report = eng.policy_train(epochs=args.train_epochs, lr=args.train_lr,
                                      batch=args.train_batch, seed=args.seed)
            eng.set_cache_policy("learned")
        if first:
            snaps += zipf_snapshots(eng, W, args.batch, rng, perm)
        for d, a in snaps[T:T + W]:
            eng.apply_batch(d, a)
        if first:
            snaps += zipf_snapshots(eng, K, args.batch, rng, perm)
        dev = [(torch.from_numpy(d.astype(np.int32)).cuda(), torch.from_numpy(a.astype(np.int32)).cuda())
               for d, a in snaps[T + W:T + W + K]]
        stream = torch.cuda.ExternalStream(eng.stream())
        st = dg.BatchStats()
        per = []
        clocks = Clocks(local) if policy == "learned" else None
        torch.cuda.synchronize()
        if clocks:
            clocks.start()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        t_begin = time.time()
        ev0.record(stream)
        for d, a in dev:
            eng.apply_batch_device(d.data_ptr(), d.shape[0], a.data_ptr(), a.shape[0], st)
            per.append(st.as_dict())
        eng.stream()
        ev1.record(stream)
        torch.cuda.synchronize()
        clk = None
        if clocks:
            clocks.mark(t_begin, time.time())
            clk = clocks.stop()
        ms = ev0.elapsed_time(ev1)
        e2e_ms, e2e_upd = 0.0, 0
        if first and E:
            snaps += zipf_snapshots(eng, E, args.batch, rng, perm)
        if E:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for d, a in snaps[T + W + K:]:
                eng.apply_batch(d, a)
            eng.stream()
            e1.record(stream)
            torch.cuda.synchronize()
            e2e_ms = e0.elapsed_time(e1)
            e2e_upd = int(sum(len(d) + len(a) for d, a in snaps[T + W + K:]))
        upd = int(sum(len(d) + len(a) for d, a in snaps[T + W:T + W + K]))
        link = int(sum(p["link_bytes"] for p in per))
        hbm = int(sum(p["hbm_adj_bytes"] for p in per))
        vals = eng.gather()[0] if algo != "pr" else eng.gather_ranks()[0]
        info = eng.info()
        res[policy] = {
            "value": round(upd / (ms / 1e3), 1), "ms_per_step": round(ms / K, 3),
            "e2e": round(e2e_upd / (e2e_ms / 1e3), 1) if e2e_ms > 0 else None,
            "median_ms_per_step": round(float(np.median([p["ms_total"] for p in per])), 3),
            "link_bytes_per_step": link // K, "hbm_adj_bytes_per_step": hbm // K,
            "hit_rate": round(hbm / max(1, hbm + link), 4),
            "per_step": {k: round(float(np.mean([p[k] for p in per])), 4) for k in
                         ("ms_ingest", "ms_mutate", "ms_repair", "ms_cache", "ms_total",
                          "affected", "edges_scanned", "cache_pages_loaded", "missing_deletes",
                          "mutate_link_bytes", "mutate_hbm_bytes")},
            "cached_pages": info["cached_pages"], "cache_slots": info["cache_slots"],
            "load_s": round(t_load, 1), "static_solve_s": round(t_init, 1),
            "gpu_launches": int(sum(p["kernel_launches"] for p in per)),
            # per snapshot, so slow snapshots can be matched across policies
            "steps_ms_total": [round(p["ms_total"], 2) for p in per],
            "steps_ms_mutate": [round(p["ms_mutate"], 2) for p in per],
            "steps_link_mb": [round(p["link_bytes"] / 1e6, 1) for p in per],
            "steps_relocated_rows": [int(p["relocated_rows"]) for p in per],
            "_vals": vals, "_clk": clk, "_per": per, "_info": info,
        }
        eng.close()
        del eng, dev
    L = res["learned"]
    if algo == "pr":
        # FP32 ranks: accumulation order differs between runs, so the policies
        # are compared by their largest rank difference, absolute and on the
        # normalised scale (ranks / their sum)
        ref = L["_vals"].astype(np.float64)
        tot = float(np.sum(ref))
        parity = {}
        for p in res:
            d = float(np.max(np.abs(res[p]["_vals"].astype(np.float64) - ref)))
            parity[p] = {"max_abs": d, "max_abs_normalized": d / tot,
                         "max_rel": float(np.max(np.abs(res[p]["_vals"].astype(np.float64) - ref) /
                                                 np.maximum(np.abs(ref), 1.0)))}
    else:
        parity = {p: bool((res[p]["_vals"] == L["_vals"]).all()) for p in res}
    per = L["_per"]
    info = L["_info"]
    page_bytes = (4 << 12) * (2 if algo == "sssp" else 1)
    rep_ms = float(np.sum([p["ms_repair"] for p in per]))
    rep_link = float(np.sum([p["link_bytes"] - p["mutate_link_bytes"] - p["cache_pages_loaded"] * page_bytes
                             for p in per]))
    rep_hbm = float(np.sum([p["hbm_adj_bytes"] - p["mutate_hbm_bytes"] - p["cache_pages_loaded"] * page_bytes
                            + p["state_bytes"] for p in per]))
    hbm_peak, peak_kind = peaks()
    link_h2d, link_zc = dg.measure_host_link(local, 1 << 30)
    tx_ns = dg.measure_host_random(local, 8 << 30, 128, False, 1 << 22)
    roofline = {
        "kernel": f"repair_kernel<{algo}>" if algo != "pr" else "pr_kernel",
        "bound": "hbm", "achieved": round(rep_hbm / (rep_ms * 1e6), 2), "peak": hbm_peak,
        "unit": "GB/s", "frac": round(rep_hbm / (rep_ms * 1e6) / hbm_peak, 5), "traffic": None,
        "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                       else "fallback 6650 GB/s",
        "algorithmic_bytes_per_launch": {"hbm": int(rep_hbm / K), "host_link": int(rep_link / K)},
        "launch_ms": round(rep_ms / K, 4),
        "host_link": {"achieved": round(rep_link / (rep_ms * 1e6), 2),
                      "peak_zero_copy": round(link_zc, 2), "peak_h2d_copy": round(link_h2d, 2),
                      "unit": "GB/s", "frac": round(rep_link / (rep_ms * 1e6) / link_zc, 5),
                      "transactions": link_transactions(rep_link / K, rep_ms / K, tx_ns)},
    }
    policies = {p: {k: v for k, v in r.items() if not k.startswith("_")} for p, r in res.items()}
    H = res["hotness"]
    return {
        "metric": METRIC + ", learned admission vs hotness and no cache on the same snapshots",
        "value": L["value"], "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": W,
        "ms_per_step": L["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32" if algo != "pr" else "f32",
        "data": "synthetic (seeded R-MAT, Zipf(1.1) update endpoints; real graphs not available)",
        "config": {"workload": f"rmat{args.scale}-ef{args.edge_factor} {algo}, "
                               f"{args.batch // 1000}K Zipf(1.1) updates per snapshot, HBM graph "
                               f"budget {args.budget_gb:g} GB, learned admission trained on the "
                               f"first {T} snapshots",
                   "vertices": info["nodes"], "edges": info["live_edges"],
                   "graph_host_bytes": info["host_bytes"], "snapshots": T + W + K + E,
                   "l2": "inputs larger than L2 (graph in pinned host memory)",
                   "parallelism": "single GPU (replicas only)"},
        "clocks": L["_clk"],
        "e2e": {"value": L["e2e"], "unit": UNIT, "h2d_bytes_per_step": args.batch * 12,
                "d2h_bytes_per_step": 256, "steps": E},
        "gpu_launches": L["gpu_launches"],
        "roofline": roofline,
        "policies": policies,
        "gain_vs_hotness": {"updates_per_s": round(L["value"] / H["value"], 3),
                            "median_ms_per_step": round(H["median_ms_per_step"] /
                                                        L["median_ms_per_step"], 3),
                            "link_bytes": round(H["link_bytes_per_step"] /
                                                max(1, L["link_bytes_per_step"]), 3),
                            "hit_rate": [H["hit_rate"], L["hit_rate"]]},
        "training": report,
        "results_equal_across_policies": parity,
        "cpu_baseline": {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                         "sample": "not run for this configuration (the CPU oracle at scale 27 "
                                   "needs the whole graph in host memory twice); see the rmat26 "
                                   "and batched configurations"},
    }


def main():
    args = parse()
    if args.impl == "reference":
        out = run_reference(args)
    elif args.config == "batched":
        out = run_batched(args)
    elif args.config == "learned":
        out = run_learned(args)
    else:
        out = run_dycg(args)
    if out is not None:
        line = json.dumps(out)
        print(line, flush=True)
        if args.json_out:
            with open(args.json_out, "w") as f:
                f.write(line + "\n")


if __name__ == "__main__":
    main()
