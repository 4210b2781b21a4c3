"""C-ABI library checks that need no GPU: it loads, exports every symbol
include/dycg.h declares, and its host-side helpers behave."""
import ctypes
import os
import re

import numpy as np
import pytest

import dycgraph_b200 as dg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "dycg.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char \*|uint32_t)\s*\*?\s*(dycg_\w+)\s*\(",
                                 text, re.M)))


def test_library_exports_every_declared_symbol():
    L = dg.lib()
    names = header_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(L, name), name


def test_version_and_defaults():
    L = dg.lib()
    assert b"sm_100a" in L.dycg_version()
    opt = dg.engine.Options()
    assert L.dycg_options_default(ctypes.byref(opt)) == 0
    assert opt.algo == 0 and opt.max_rounds == 100 and abs(opt.alpha - 0.85) < 1e-6


def test_create_without_gpu_fails_cleanly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is visible")
    except ImportError:
        pass
    with pytest.raises(dg.DycgError) as ei:
        dg.Engine("sssp")
    assert ei.value.code == -8  # DYCG_ENOGPU


def test_null_arguments_rejected():
    L = dg.lib()
    assert L.dycg_create(None, None) == -1
    assert L.dycg_gather(None, None, None) == -1
    assert L.dycg_last_error(None, None, 0) == -1


def test_rmat_draws_deterministic_and_skewed():
    a = dg.gen_rmat_edges(16, 20000, seed=7)
    b = dg.gen_rmat_edges(16, 20000, seed=7)
    c = dg.gen_rmat_edges(16, 10000, seed=7, first=10000)
    assert (a == b).all()
    assert (a[10000:] == c).all()
    assert a[:, :2].max() < (1 << 16)
    assert ((a[:, 2] >= 1) & (a[:, 2] <= 64)).all()
    # a=0.57: the top bit of u is 0 with probability a+b = 0.76
    frac = np.mean(a[:, 0] < (1 << 15))
    assert 0.73 < frac < 0.79
    # weights are a function of (u, v)
    for u, v, w in a[:50]:
        assert dg.hash_weight(7, int(u), int(v)) == w


def test_binary_formats_round_trip(tmp_path):
    from dycgraph_b200 import formats
    off = np.array([0, 2, 2, 5], np.uint64)
    dst = np.array([1, 2, 0, 1, 1], np.uint32)
    w = np.array([3, 4, 5, 6, 7], np.uint32)
    formats.write_graph(tmp_path / "g.bin", off, dst, w)
    n, o2, d2, w2 = formats.read_graph(tmp_path / "g.bin")
    assert n == 3 and (o2 == off).all() and (d2 == dst).all() and (w2 == w).all()
    batches = [(np.array([[0, 1, 3]]), np.array([[2, 0, 9], [1, 2, 1]])), (np.zeros((0, 3)), np.array([[0, 2, 2]]))]
    formats.write_updates(tmp_path / "u.bin", batches)
    back = formats.read_updates(tmp_path / "u.bin")
    assert len(back) == 2
    for (d, a), (d2_, a2) in zip(batches, back):
        assert (np.asarray(d, np.uint32).reshape(-1, 3) == d2_).all()
        assert (np.asarray(a, np.uint32).reshape(-1, 3) == a2).all()


def test_cli_usage_and_loud_failure_without_a_gpu(tmp_path):
    import subprocess
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is visible")
    except ImportError:
        pass
    for name in ("hybrid_sssp", "hybrid_bfs", "hybrid_cc", "hybrid_pr"):
        exe = os.path.join(ROOT, "dycgraph_b200", name)
        p = subprocess.run([exe], capture_output=True, text=True, timeout=60)
        assert p.returncode == 2 and "usage: " + name in p.stderr
        g = tmp_path / "g.txt"
        g.write_text("0 1\n1 2\n")
        # the reference's flag spellings are accepted; no device means a clear error, no fallback
        p = subprocess.run([exe, f"-graphfile={g}", "-format", "market_big", "--source_node=0",
                            "-check"], capture_output=True, text=True, timeout=60)
        assert p.returncode == 1 and "no CUDA device" in p.stderr


def test_text_graph_converts_to_the_binary_format(tmp_path):
    """dycg_convert_graph_text reads a text edge list the way the text loader
    does (comment, blank and malformed lines skipped, a missing weight is 1,
    rows in file order, duplicates and self-loops kept for the loader's rules)
    and writes the binary graph file."""
    from dycgraph_b200 import formats
    lines = ["%%MatrixMarket matrix coordinate pattern general", "# comment", "3 1 7", "0 2 5",
             "3 1 2", "", "0 4", "4 4 9", "not an edge", "1 0 3"]
    txt = tmp_path / "g.txt"
    txt.write_text("\n".join(lines) + "\n")
    edges = [tuple(int(x) for x in ln.split()) for ln in lines
             if ln and ln[0] not in "#%" and ln.split()[0].isdigit()]
    for weighted, min_nodes in ((True, 0), (False, 9)):
        out = tmp_path / f"g{int(weighted)}.bin"
        dg.engine.convert_graph_text(txt, out, min_nodes, weighted)
        n, off, dst, w = formats.read_graph(out)
        assert n == max(5, min_nodes)
        want_rows = [[(e[1], e[2] if len(e) > 2 else 1) for e in edges if e[0] == u]
                     for u in range(n)]
        assert list(np.diff(off.astype(np.int64))) == [len(r) for r in want_rows]
        assert list(dst) == [v for r in want_rows for v, _ in r]
        assert (w is not None) == weighted
        if weighted:
            assert list(w) == [x for r in want_rows for _, x in r]
    with pytest.raises(dg.DycgError):
        dg.engine.convert_graph_text(tmp_path / "missing.txt", tmp_path / "x.bin")


def test_text_updates_convert_to_the_binary_stream(tmp_path):
    """The update converter splits a text stream per the reference's Loader
    (tests/cases.replay_batches restates it) and the binary stream reads back
    the same snapshots, weights included (default 1)."""
    from dycgraph_b200 import formats
    from tests import cases
    lines = ["# header", "a 1 2 5", "d 3 4", "a 5 6", "x 1 1", "d 7 8 9", "a 9 10 2",
             "d 11 12", "bad", "a 13 14 1"]
    (tmp_path / "u.txt").write_text("\n".join(lines) + "\n")
    (tmp_path / "s.txt").write_text("2 1\n\n1 2\n1 0\n")
    nb = formats.text_updates_to_binary(tmp_path / "u.txt", tmp_path / "s.txt", tmp_path / "u.bin")
    assert nb == 3
    back = formats.read_updates(tmp_path / "u.bin")
    recs = [ln.split() for ln in lines if ln[:1] in ("a", "d") and len(ln.split()) >= 3]
    weight = {(int(p[1]), int(p[2])): int(p[3]) if len(p) > 3 else 1 for p in recs}
    want = cases.replay_batches([(p[0], int(p[1]), int(p[2])) for p in recs],
                                [(2, 1), (1, 2), (1, 0)])
    assert len(back) == len(want)
    for (d, a), (wd, wa) in zip(back, want):
        assert [tuple(r) for r in d.tolist()] == [(u, v, weight[(u, v)]) for u, v in wd]
        assert [tuple(r) for r in a.tolist()] == [(u, v, weight[(u, v)]) for u, v in wa]


def test_reference_engine_names_and_update_files(tmp_path):
    """The mirror answers to every Engine method the reference's sample drivers
    call; the update-file ones work without a GPU (an engine object made
    without a device handle)."""
    from dycgraph_b200 import formats
    names = ["LoadGraph", "SetOptions", "InitGraph", "Start", "compute_hot_vertices_sssp",
             "confirm_candidate_batch", "TraceCacheCandidates", "LoadCache", "MarkCachePublished",
             "get_update_file", "GetUpdateBatchCount", "del_edge", "add_edge",
             "CacheRefreshRequired", "evication_cache", "compact_cache", "GatherValue",
             "GatherParent", "GatherBuffer", "GetGraphDatum", "ChunkStore", "StartPageRank",
             "UpdatePageRank"]
    assert [n for n in names if not hasattr(dg.Engine, n)] == []
    e = dg.Engine.__new__(dg.Engine)
    e._h = None
    e.options = dg.engine.Options()
    dg.lib().dycg_options_default(ctypes.byref(e.options))
    assert e.GetUpdateBatchCount() == 0
    with pytest.raises(dg.DycgError):
        e._snapshot(0)
    (tmp_path / "u.txt").write_text("a 1 2 3\nd 4 5\na 6 7\n")
    (tmp_path / "s.txt").write_text("1 1\n1 0\n")
    assert e.get_update_file(tmp_path / "u.txt", tmp_path / "s.txt") == 2
    d, a = e._snapshot(1)
    assert d.shape == (0, 3) and a.tolist() == [[6, 7, 1]]
    with pytest.raises(dg.DycgError):
        e._snapshot(2)
    with pytest.raises(dg.DycgError):
        e.get_update_file(tmp_path / "u.txt")  # text needs its sizes file
    formats.write_updates(tmp_path / "u.bin", [(np.array([[4, 5, 1]]), np.array([[1, 2, 3]]))])
    assert e.get_update_file(tmp_path / "u.bin") == 1 and e.GetUpdateBatchCount() == 1
    assert e._snapshot(0)[1].tolist() == [[1, 2, 3]]
    assert e.CacheRefreshRequired() is True and e.compact_cache() is None
    e.SetOptions(algo="sssp", alpha=0.85, max_rounds=100)
    with pytest.raises(dg.DycgError):
        e.SetOptions(algo="bfs")
    with pytest.raises(dg.DycgError):
        e.SetOptions(no_such_option=1)


def test_smoke_fails_loudly_without_a_gpu():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is visible")
    except ImportError:
        pass
    import __graft_entry__
    with pytest.raises(dg.DycgError) as ei:
        __graft_entry__.smoke()
    assert ei.value.code == -8  # DYCG_ENOGPU: no CPU fallback


def test_random_link_probe_checks_its_arguments_before_the_device():
    L = dg.lib()
    ns = ctypes.c_double(0)
    for op in (0, 3, 32, 256):
        assert L.dycg_measure_host_random(0, 1 << 26, op, 0, 1000, ctypes.byref(ns)) == -1
    assert L.dycg_measure_host_random(0, 1 << 10, 128, 0, 1000, ctypes.byref(ns)) == -1
    assert L.dycg_measure_host_random(0, 1 << 26, 128, 0, 0, ctypes.byref(ns)) == -1
    assert L.dycg_measure_host_random(0, 1 << 26, 128, 0, 1000, None) == -1
    try:
        import torch
        if torch.cuda.is_available():
            return
    except ImportError:
        pass
    assert L.dycg_measure_host_random(0, 1 << 26, 16, 1, 1000, ctypes.byref(ns)) == -8


def test_edge_records_reach_the_abi_as_12_byte_rows():
    from dycgraph_b200.engine import edges_array
    assert edges_array([]).shape == (0, 3)
    assert edges_array([(1, 2), (3, 4, 5)]).tolist() == [[1, 2, 1], [3, 4, 5]]
    assert edges_array(np.array([[1, 2], [3, 4]])).tolist() == [[1, 2, 1], [3, 4, 1]]
    assert edges_array(np.arange(6)).tolist() == [[0, 1, 2], [3, 4, 5]]
    a = edges_array(np.array([[7, 8, 9]], np.int64))
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"] and a.strides == (12, 4)
    with pytest.raises(ValueError):
        edges_array(np.zeros((2, 4)))
    with pytest.raises(ValueError):
        edges_array(np.zeros((2, 3, 1)))


def test_csr_arrays_are_length_checked_before_the_abi():
    from dycgraph_b200.engine import csr_arrays
    off, d, w = csr_arrays(3, [0, 2, 2, 3], [1, 2, 0], [5, 6, 7])
    assert off.dtype == np.uint64 and d.dtype == np.uint32 and w.dtype == np.uint32
    with pytest.raises(ValueError):
        csr_arrays(3, [0, 2, 3], [1, 2, 0])          # offsets too short
    with pytest.raises(ValueError):
        csr_arrays(3, [0, 2, 2, 3], [1, 2])          # dst too short
    with pytest.raises(ValueError):
        csr_arrays(3, [0, 2, 2, 3], [1, 2, 0], [5])  # weights too short
