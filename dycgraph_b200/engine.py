"""ctypes binding of libdycg.so and the reference-shaped Engine class.

Method names follow sepgraph::engine::Engine (include/framework/framework.cuh:
LoadGraph :1569, InitGraph :1803, Start :1963, del_edge :2595, add_edge :2419,
compute_hot_vertices_sssp :1264, confirm_candidate_batch :1364, LoadCache :1509,
evication_cache :3038, compact_cache :2978, GatherValue/GatherParent :4959-4984,
StartPageRank :2681, UpdatePageRank :2692). Errors raise DycgError with the
library's status code and message, where the reference would abort.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

ALGOS = {"sssp": 0, "bfs": 1, "cc": 2, "pr": 3}
WEIGHTS = {"hash128": 0, "stored": 1}
CACHE = {"none": 0, "hotness": 1, "learned": 2}
POLICY_F, POLICY_H, POLICY_PARAMS = 8, 64, 4801
STATUS = {0: "DYCG_OK", -1: "DYCG_EINVAL", -2: "DYCG_ECUDA", -3: "DYCG_ENOMEM",
          -4: "DYCG_ESTATE", -5: "DYCG_ECAPACITY", -6: "DYCG_ELIMIT", -7: "DYCG_EIO",
          -8: "DYCG_ENOGPU"}
INF = 0xFFFFFFFF


class DycgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Edge(ctypes.Structure):
    _fields_ = [("u", ctypes.c_uint32), ("v", ctypes.c_uint32), ("w", ctypes.c_uint32)]


class Options(ctypes.Structure):
    _fields_ = [("algo", ctypes.c_uint32), ("weight_mode", ctypes.c_uint32),
                ("source", ctypes.c_uint32), ("segments", ctypes.c_uint32),
                ("hbm_graph_budget_bytes", ctypes.c_uint64), ("cache_policy", ctypes.c_uint32),
                ("symmetric", ctypes.c_uint32), ("epsilon", ctypes.c_float),
                ("alpha", ctypes.c_float), ("max_rounds", ctypes.c_uint32),
                ("device", ctypes.c_int32), ("page_shift", ctypes.c_uint32),
                ("ordered_delta", ctypes.c_uint32), ("arena_headroom_permille", ctypes.c_uint32),
                ("frontier_queue", ctypes.c_uint32), ("mutation_ctas", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32 * 3)]


_STAT_U64 = ["deletions", "insertions", "missing_deletes", "invalid_updates", "touched_sources",
             "relocated_rows", "affected", "expanded", "edges_scanned", "improvements", "waves",
             "link_bytes", "hbm_adj_bytes", "state_bytes", "cache_pages_loaded",
             "cache_pages_evicted", "kernel_launches"]
_STAT_F64 = ["ms_ingest", "ms_mutate", "ms_repair", "ms_cache", "ms_total"]
_STAT_TAIL = ["mutate_link_bytes", "mutate_hbm_bytes"]
_STAT_PHASE = ["ms_phase_invalidate", "ms_phase_pull", "ms_phase_seed", "ms_phase_closure"]


# Bytes of the engine's per-snapshot device control block, which every
# snapshot call reads back to the host (static_assert in csrc/common.cuh).
CTL_BYTES = 2904


class BatchStats(ctypes.Structure):
    _fields_ = ([(k, ctypes.c_uint64) for k in _STAT_U64] + [(k, ctypes.c_double) for k in _STAT_F64]
                + [(k, ctypes.c_uint64) for k in _STAT_TAIL]
                + [(k, ctypes.c_double) for k in _STAT_PHASE] + [("reserved", ctypes.c_uint64 * 2)])

    def as_dict(self):
        return {k: getattr(self, k) for k in _STAT_U64 + _STAT_F64 + _STAT_TAIL + _STAT_PHASE}


class QueryMapping(ctypes.Structure):
    _fields_ = [("qratio", ctypes.c_uint32), ("heavy", ctypes.c_uint32), ("tile", ctypes.c_uint32),
                ("pull_qratio", ctypes.c_uint32), ("queue", ctypes.c_uint32),
                ("repair_ms", ctypes.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PolicyReport(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_uint64), ("steps", ctypes.c_uint64),
                ("loss_before", ctypes.c_float), ("loss_after", ctypes.c_float),
                ("ms", ctypes.c_float), ("reserved", ctypes.c_uint32 * 5)]

    def as_dict(self):
        return {k: getattr(self, k) for k in ("samples", "steps", "loss_before", "loss_after", "ms")}


class GraphInfo(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in (
        "nodes", "live_edges", "arena_slots", "arena_used", "pages", "cache_slots",
        "cached_pages", "host_bytes", "device_bytes")] + [
        ("page_shift", ctypes.c_uint32), ("has_incoming", ctypes.c_uint32),
        ("reserved", ctypes.c_uint64 * 6)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}
        d["index_bytes"] = self.reserved[0]  # fence index + deletion bitmaps (in the budget)
        return d


def library_path():
    return os.environ.get("DYCG_LIBRARY", os.path.join(_HERE, "libdycg.so"))


def lib():
    """Load libdycg.so (built in-tree by `make -C dycgraph_b200`)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        raise ImportError(f"libdycg.so not built at {path}: run `make -C dycgraph_b200` "
                          "(there is no CPU fallback)")
    L = ctypes.CDLL(path)
    P = ctypes.c_void_p
    I = ctypes.c_int
    u32, u64, sz = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t
    u32p, u64p = ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64)
    ep = ctypes.POINTER(Edge)
    sp = ctypes.POINTER(BatchStats)
    sig = {
        "dycg_options_default": (I, [ctypes.POINTER(Options)]),
        "dycg_create": (I, [ctypes.POINTER(Options), ctypes.POINTER(P)]),
        "dycg_destroy": (None, [P]),
        "dycg_load_graph_csr": (I, [P, u32, u64p, u32p, u32p]),
        "dycg_load_graph_file": (I, [P, ctypes.c_char_p, u32, I]),
        "dycg_load_graph_binary": (I, [P, ctypes.c_char_p]),
        "dycg_convert_graph_text": (I, [ctypes.c_char_p, ctypes.c_char_p, u32, I]),
        "dycg_load_graph_rmat": (I, [P, u32, u32, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, u64, u32, u32, I]),
        "dycg_load_graph_grid": (I, [P, u32, u32, u32, u64, u32, u32]),
        "dycg_init": (I, [P]),
        "dycg_delete_edges": (I, [P, ep, sz, sp]),
        "dycg_insert_edges": (I, [P, ep, sz, sp]),
        "dycg_cache_maintenance": (I, [P, sp]),
        "dycg_apply_batch": (I, [P, ep, sz, ep, sz, sp]),
        "dycg_reserve_batch": (I, [P, sz]),
        "dycg_tune_query_mapping": (I, [P, ep, sz, ep, sz, ctypes.POINTER(QueryMapping), u32,
                                        ctypes.POINTER(ctypes.c_uint32), sp]),
        "dycg_apply_batches": (I, [P, ep, u64p, ep, u64p, u32, sp]),
        "dycg_apply_batches_device": (I, [P, P, u64p, P, u64p, u32, sp]),
        "dycg_apply_batch_device": (I, [P, P, sz, P, sz, sp]),
        "dycg_gather": (I, [P, u32p, u32p]),
        "dycg_gather_ranks": (I, [P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
        "dycg_get_row": (I, [P, u32, I, u32p, u32p, u32, u32p]),
        "dycg_export_csr": (I, [P, u64p, u32p, u32p]),
        "dycg_graph_info_get": (I, [P, ctypes.POINTER(GraphInfo)]),
        "dycg_sample_edges": (I, [P, u64, u64, ep]),
        "dycg_gen_rmat_edges": (I, [u32, ctypes.c_double, ctypes.c_double, ctypes.c_double, u64,
                                    u64, u64, u32, u32, ep]),
        "dycg_hash_weight": (u32, [u64, u32, u32, u32, u32]),
        "dycg_stream": (I, [P, ctypes.POINTER(P)]),
        "dycg_measure_host_link": (I, [I, u64, ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_double)]),
        "dycg_measure_host_random": (I, [I, u64, u32, I, u64, ctypes.POINTER(ctypes.c_double)]),
        "dycg_measure_host_sweep": (I, [I, u64, u32, I, u64, u32, ctypes.POINTER(ctypes.c_double)]),
        "dycg_check_bounded_wait": (I, [I, u32, u32p, u32p]),
        "dycg_group_updates": (I, [P, sz, u32, P, u32, P, P, P, P, P]),
        "dycg_group_updates_noalloc": (I, [P, sz, u32, P, u32, P, P, P, P, P]),
        "dycg_set_queries": (I, [P, u32p, u32, u32]),
        "dycg_set_query_mapping": (I, [P, u32, u32, u32]),
        "dycg_set_query_queue": (I, [P, u32]),
        "dycg_gather_query": (I, [P, u32, u32p, u32p]),
        "dycg_set_cache_policy": (I, [P, u32]),
        "dycg_policy_trace": (I, [P, u32]),
        "dycg_policy_train": (I, [P, u32, ctypes.c_float, u32, u64, ctypes.POINTER(PolicyReport)]),
        "dycg_policy_params": (I, [P, ctypes.POINTER(ctypes.c_float)]),
        "dycg_policy_set_params": (I, [P, ctypes.POINTER(ctypes.c_float)]),
        "dycg_mlp_infer": (I, [P, u32, P, P, P]),
        "dycg_mlp_loss_grad": (I, [P, P, u32, P, P, P, P]),
        "dycg_sample_row_edges": (I, [P, u32p, u64, u64, ep]),
        "dycg_last_error": (I, [P, ctypes.c_char_p, sz]),
        "dycg_version": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def _ptr(a, t):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(t))


def edges_array(edges):
    """(k,3) uint32 array from a list of (u, v[, w]) or an array."""
    if isinstance(edges, np.ndarray):
        arr = np.ascontiguousarray(edges, dtype=np.uint32)
        if arr.ndim == 1:
            arr = arr.reshape(-1, 3)
        if arr.ndim != 2 or arr.shape[1] not in (2, 3):
            raise ValueError(f"edge records must be (k, 2) or (k, 3), not {edges.shape}")
        if arr.shape[1] == 2:
            arr = np.concatenate([arr, np.ones((arr.shape[0], 1), np.uint32)], axis=1)
        return np.ascontiguousarray(arr)
    rows = [(e[0], e[1], e[2] if len(e) > 2 else 1) for e in edges]
    return np.asarray(rows, dtype=np.uint32).reshape(-1, 3)


def csr_arrays(n, offsets, dst, w=None):
    """CSR arrays as the C ABI reads them (offsets u64 [n+1], dst/w u32 [m]),
    with the lengths the ABI cannot check itself."""
    off = np.ascontiguousarray(offsets, np.uint64)
    d = np.ascontiguousarray(dst, np.uint32)
    ww = None if w is None else np.ascontiguousarray(w, np.uint32)
    if off.ndim != 1 or off.shape[0] != n + 1:
        raise ValueError(f"offsets must have n + 1 = {n + 1} entries, not {off.shape}")
    m = int(off[-1]) if n >= 0 and off.shape[0] else 0
    if d.shape[0] < m or (ww is not None and ww.shape[0] < m):
        raise ValueError(f"dst/w hold fewer than offsets[n] = {m} entries")
    return off, d, ww


def gen_rmat_edges(scale, count, seed, first=0, a=0.57, b=0.19, c=0.19, wlo=1, whi=64):
    out = np.empty((count, 3), np.uint32)
    rc = lib().dycg_gen_rmat_edges(scale, a, b, c, seed, first, count, wlo, whi,
                                   out.ctypes.data_as(ctypes.POINTER(Edge)))
    if rc:
        raise DycgError(rc, "dycg_gen_rmat_edges")
    return out


def mlp_infer(d_x, n, d_params, d_out, stream=None):
    """Policy network on device buffers (raw addresses): n bf16 feature rows."""
    rc = lib().dycg_mlp_infer(ctypes.c_void_p(d_x), n, ctypes.c_void_p(d_params),
                              ctypes.c_void_p(d_out), ctypes.c_void_p(stream))
    if rc:
        raise DycgError(rc, "dycg_mlp_infer")


def mlp_loss_grad(d_x, d_y, n, d_params, d_grad, d_loss, stream=None):
    """Adds sum((mlp(x) - y)^2) into *d_loss and its parameter gradient into d_grad."""
    rc = lib().dycg_mlp_loss_grad(ctypes.c_void_p(d_x), ctypes.c_void_p(d_y), n,
                                  ctypes.c_void_p(d_params), ctypes.c_void_p(d_grad),
                                  ctypes.c_void_p(d_loss), ctypes.c_void_p(stream))
    if rc:
        raise DycgError(rc, "dycg_mlp_loss_grad")


def measure_host_link(device=0, nbytes=1 << 30):
    """(h2d copy GB/s, zero-copy read GB/s) over the host link of `device`."""
    a, b = ctypes.c_double(0), ctypes.c_double(0)
    rc = lib().dycg_measure_host_link(device, nbytes, ctypes.byref(a), ctypes.byref(b))
    if rc:
        raise DycgError(rc, "dycg_measure_host_link")
    return a.value, b.value


def measure_host_random(device=0, nbytes=8 << 30, op_bytes=128, write=False, ops=1 << 24):
    """Device time (ns) per random host-link access of op_bytes over an
    nbytes pinned buffer (reads, or writes with write=True)."""
    ns = ctypes.c_double(0)
    rc = lib().dycg_measure_host_random(device, nbytes, op_bytes, int(write), ops,
                                        ctypes.byref(ns))
    if rc:
        raise DycgError(rc, "dycg_measure_host_random")
    return ns.value


def measure_host_sweep(device=0, nbytes=32 << 30, op_bytes=128, write=False, ops=1 << 20,
                       ctas=148):
    """Device time (ns) per host-link access of op_bytes at random offsets of
    an nbytes pinned buffer, issued in ascending address order by `ctas` CTAs."""
    ns = ctypes.c_double(0)
    rc = lib().dycg_measure_host_sweep(device, nbytes, op_bytes, int(write), ops, ctas,
                                       ctypes.byref(ns))
    if rc:
        raise DycgError(rc, "dycg_measure_host_sweep")
    return ns.value


def hash_weight(seed, u, v, wlo=1, whi=64):
    return lib().dycg_hash_weight(seed, u, v, wlo, whi)


def convert_graph_text(text_path, binary_path, min_nodes=0, weighted=False):
    """Text edge list -> binary CSR file (as load_file reads the text; no GPU)."""
    rc = lib().dycg_convert_graph_text(str(text_path).encode(), str(binary_path).encode(),
                                       min_nodes, int(weighted))
    if rc:
        raise DycgError(rc, f"dycg_convert_graph_text({text_path})")


class Engine:
    """One graph + one algorithm on one GPU (reference: sepgraph::engine::Engine)."""

    def __init__(self, algo="sssp", weight_mode="hash128", source=0, segments=1,
                 hbm_graph_budget_bytes=0, cache_policy=None, symmetric=False, epsilon=1e-6,
                 alpha=0.85, max_rounds=100, device=0, page_shift=12, ordered_delta=0,
                 arena_headroom_permille=0, frontier_queue="static", mutation_ctas=0):
        L = lib()
        opt = Options()
        L.dycg_options_default(ctypes.byref(opt))
        opt.algo = ALGOS[algo] if isinstance(algo, str) else int(algo)
        opt.weight_mode = WEIGHTS[weight_mode] if isinstance(weight_mode, str) else int(weight_mode)
        opt.source = source
        opt.segments = segments
        opt.hbm_graph_budget_bytes = int(hbm_graph_budget_bytes)
        if cache_policy is None:
            cache_policy = "hotness" if hbm_graph_budget_bytes else "none"
        opt.cache_policy = CACHE[cache_policy] if isinstance(cache_policy, str) else int(cache_policy)
        opt.symmetric = int(bool(symmetric))
        opt.epsilon = epsilon
        opt.alpha = alpha
        opt.max_rounds = max_rounds
        opt.device = device
        opt.page_shift = page_shift
        opt.ordered_delta = ordered_delta
        opt.arena_headroom_permille = arena_headroom_permille
        opt.frontier_queue = (self.QUEUE_SCHEMES[frontier_queue] if isinstance(frontier_queue, str)
                              else int(frontier_queue))
        opt.mutation_ctas = int(mutation_ctas)
        self.algo = opt.algo
        self.options = opt
        self._h = ctypes.c_void_p()
        rc = L.dycg_create(ctypes.byref(opt), ctypes.byref(self._h))
        if rc:
            self._h = None
            raise DycgError(rc, "dycg_create failed (is a CUDA device visible?)")
        self.n = 0
        self.last_stats = None

    # -- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib().dycg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc, what):
        if rc:
            buf = ctypes.create_string_buffer(512)
            lib().dycg_last_error(self._h, buf, 512)
            raise DycgError(rc, f"{what}: {buf.value.decode(errors='replace')}")

    # -- loading (Engine::LoadGraph) ------------------------------------------
    def load_csr(self, n, offsets, dst, w=None):
        off, d, ww = csr_arrays(n, offsets, dst, w)
        self._check(lib().dycg_load_graph_csr(self._h, n, _ptr(off, ctypes.c_uint64),
                                              _ptr(d, ctypes.c_uint32), _ptr(ww, ctypes.c_uint32)),
                    "load_csr")
        self.n = n

    def load_file(self, path, min_nodes=0, weighted=False):
        self._check(lib().dycg_load_graph_file(self._h, path.encode(), min_nodes, int(weighted)),
                    "load_file")
        self.n = self.info()["nodes"]

    def load_binary(self, path):
        self._check(lib().dycg_load_graph_binary(self._h, path.encode()), "load_binary")
        self.n = self.info()["nodes"]

    def load_rmat(self, scale, edge_factor=16, seed=1, a=0.57, b=0.19, c=0.19, wlo=1, whi=64,
                  symmetrize=False):
        self._check(lib().dycg_load_graph_rmat(self._h, scale, edge_factor, a, b, c, seed, wlo,
                                               whi, int(symmetrize)), "load_rmat")
        self.n = 1 << scale

    def load_grid(self, side, shortcut_permille=10, radius=8, seed=1, wlo=1, whi=1000):
        self._check(lib().dycg_load_graph_grid(self._h, side, shortcut_permille, radius, seed,
                                               wlo, whi), "load_grid")
        self.n = side * side

    LoadGraph = load_csr

    # -- solve (InitGraph + Start / StartPageRank) ----------------------------
    def start(self):
        self._check(lib().dycg_init(self._h), "init")

    Start = start
    StartPageRank = start

    def InitGraph(self, source=None):
        """The source is fixed at construction (dycg_options.source)."""
        if source is not None and source != self.options.source:
            raise DycgError(-1, "source differs from the engine's configured source")

    # -- batches ---------------------------------------------------------------
    # -- the reference's update files (Engine::get_update_file / GetUpdateBatchCount,
    #    include/framework/framework.cuh:2387-2415) ----------------------------------
    def get_update_file(self, updates, sizes=None):
        """Read an update stream for del_edge(b) / add_edge(b): a binary
        DYCGUPD1 file, or a text stream with its sizes file (split as the
        reference's Loader splits it). Returns the number of snapshots."""
        from . import formats
        with open(updates, "rb") as f:
            binary = f.read(8) == formats.UPD_MAGIC
        if binary:
            self._updates = formats.read_updates(updates)
        elif sizes is None:
            raise DycgError(-1, "a text update stream needs its sizes file")
        else:
            self._updates = formats.read_text_updates(updates, sizes)
        return len(self._updates)

    def GetUpdateBatchCount(self):
        return len(getattr(self, "_updates", None) or [])

    def _snapshot(self, b):
        ups = getattr(self, "_updates", None)
        if ups is None:
            raise DycgError(-1, "no update stream read (get_update_file)")
        if not 0 <= int(b) < len(ups):
            raise DycgError(-1, f"snapshot {b} out of range (0..{len(ups) - 1})")
        return ups[int(b)]

    def delete_edges(self, dels):
        """Delete one live occurrence per record; dels is a list of (u, v[, w])
        or, after get_update_file, a snapshot index (the reference's
        del_edge(offsets, b))."""
        if isinstance(dels, (int, np.integer)):
            dels = self._snapshot(dels)[0]
        arr = edges_array(dels)
        st = BatchStats()
        self._check(lib().dycg_delete_edges(self._h, arr.ctypes.data_as(ctypes.POINTER(Edge)),
                                            arr.shape[0], ctypes.byref(st)), "delete_edges")
        self.last_stats = st.as_dict()
        return self.last_stats

    def insert_edges(self, adds):
        """Append one occurrence per record; adds is a list of (u, v[, w]) or,
        after get_update_file, a snapshot index (the reference's add_edge)."""
        if isinstance(adds, (int, np.integer)):
            adds = self._snapshot(adds)[1]
        arr = edges_array(adds)
        st = BatchStats()
        self._check(lib().dycg_insert_edges(self._h, arr.ctypes.data_as(ctypes.POINTER(Edge)),
                                            arr.shape[0], ctypes.byref(st)), "insert_edges")
        self.last_stats = st.as_dict()
        return self.last_stats

    del_edge = delete_edges
    add_edge = insert_edges

    def apply_batch(self, dels, adds):
        d = edges_array(dels)
        a = edges_array(adds)
        st = BatchStats()
        self._check(lib().dycg_apply_batch(self._h, d.ctypes.data_as(ctypes.POINTER(Edge)),
                                           d.shape[0], a.ctypes.data_as(ctypes.POINTER(Edge)),
                                           a.shape[0], ctypes.byref(st)), "apply_batch")
        self.last_stats = st.as_dict()
        return self.last_stats

    UpdatePageRank = apply_batch

    def reserve_batch(self, max_records):
        """Size the per-batch buffers for up to max_records deletions (and as
        many insertions) before timing or replay."""
        self._check(lib().dycg_reserve_batch(self._h, int(max_records)), "reserve_batch")

    def apply_batch_device(self, d_dels_ptr, nd, d_adds_ptr, na, stats=None):
        """Records already in device memory (raw device addresses)."""
        st = stats if stats is not None else BatchStats()
        self._check(lib().dycg_apply_batch_device(self._h, ctypes.c_void_p(d_dels_ptr), nd,
                                                  ctypes.c_void_p(d_adds_ptr), na,
                                                  ctypes.byref(st)), "apply_batch_device")
        return st

    # -- learned cache admission -------------------------------------------------
    def set_cache_policy(self, policy):
        self._check(lib().dycg_set_cache_policy(self._h, CACHE[policy] if isinstance(policy, str)
                                                else int(policy)), "set_cache_policy")

    def policy_trace(self, snapshots):
        """Record features and page reads of the next `snapshots` snapshot calls."""
        self._check(lib().dycg_policy_trace(self._h, snapshots), "policy_trace")

    def policy_train(self, epochs=2, lr=1e-3, batch=4096, seed=1):
        rep = PolicyReport()
        self._check(lib().dycg_policy_train(self._h, epochs, lr, batch, seed, ctypes.byref(rep)),
                    "policy_train")
        return rep.as_dict()

    def policy_params(self):
        p = np.empty(POLICY_PARAMS, np.float32)
        self._check(lib().dycg_policy_params(self._h, _ptr(p, ctypes.c_float)), "policy_params")
        return p

    def policy_set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.shape != (POLICY_PARAMS,):
            raise ValueError(f"expected {POLICY_PARAMS} parameters, got shape {p.shape}")
        self._check(lib().dycg_policy_set_params(self._h, _ptr(p, ctypes.c_float)),
                    "policy_set_params")

    def sample_row_edges(self, sources, seed):
        """One live out-edge per source; rows (INF, INF, 0) for empty rows."""
        src = np.ascontiguousarray(np.ravel(sources), dtype=np.uint32)
        out = np.empty((len(src), 3), np.uint32)
        self._check(lib().dycg_sample_row_edges(self._h, _ptr(src, ctypes.c_uint32), len(src), seed,
                                                out.ctypes.data_as(ctypes.POINTER(Edge))),
                    "sample_row_edges")
        return out

    def tune_query_mapping(self, dels, adds):
        """Apply one snapshot while timing the batched repair under each
        candidate work mapping; keeps the fastest. Returns the candidates."""
        d = edges_array(dels)
        a = edges_array(adds)
        tried = (QueryMapping * 64)()
        nt = ctypes.c_uint32(0)
        st = BatchStats()
        self._check(lib().dycg_tune_query_mapping(
            self._h, d.ctypes.data_as(ctypes.POINTER(Edge)), d.shape[0],
            a.ctypes.data_as(ctypes.POINTER(Edge)), a.shape[0], tried, 64, ctypes.byref(nt),
            ctypes.byref(st)), "tune_query_mapping")
        self.last_stats = st.as_dict()
        return [tried[i].as_dict() for i in range(nt.value)]

    def apply_batches(self, snapshots):
        """Many snapshots [(dels, adds), ...] in one call; one stats dict each."""
        ds = [edges_array(d) for d, _ in snapshots]
        as_ = [edges_array(a) for _, a in snapshots]
        nd = np.asarray([x.shape[0] for x in ds], np.uint64)
        na = np.asarray([x.shape[0] for x in as_], np.uint64)
        d = np.ascontiguousarray(np.concatenate(ds) if ds else np.zeros((0, 3), np.uint32))
        a = np.ascontiguousarray(np.concatenate(as_) if as_ else np.zeros((0, 3), np.uint32))
        st = (BatchStats * max(len(snapshots), 1))()
        self._check(lib().dycg_apply_batches(
            self._h, d.ctypes.data_as(ctypes.POINTER(Edge)), _ptr(nd, ctypes.c_uint64),
            a.ctypes.data_as(ctypes.POINTER(Edge)), _ptr(na, ctypes.c_uint64), len(snapshots), st),
            "apply_batches")
        return [st[i].as_dict() for i in range(len(snapshots))]

    def apply_batches_device(self, d_dels_ptr, nd, d_adds_ptr, na, stats=None):
        """Records already in device memory: nd/na per-snapshot counts."""
        nd = np.ascontiguousarray(nd, np.uint64)
        na = np.ascontiguousarray(na, np.uint64)
        st = stats if stats is not None else (BatchStats * max(len(nd), 1))()
        self._check(lib().dycg_apply_batches_device(
            self._h, ctypes.c_void_p(d_dels_ptr), _ptr(nd, ctypes.c_uint64),
            ctypes.c_void_p(d_adds_ptr), _ptr(na, ctypes.c_uint64), len(nd), st),
            "apply_batches_device")
        return st

    def cache_maintenance(self):
        st = BatchStats()
        self._check(lib().dycg_cache_maintenance(self._h, ctypes.byref(st)), "cache_maintenance")
        return st.as_dict()

    # The reference's separate hotness/candidate/eviction/compaction/load steps
    # are one call here: the page cache has no compaction step.
    compute_hot_vertices_sssp = cache_maintenance
    LoadCache = cache_maintenance

    def CacheRefreshRequired(self):
        """The refresh gate runs inside cache_maintenance; a driver that asks is
        told to go on to LoadCache."""
        return True

    def confirm_candidate_batch(self, *args, **kwargs):
        """Candidate confirmation, eviction, compaction and publication happen
        inside cache_maintenance (compute_hot_vertices_sssp / LoadCache); the
        reference's separate calls have nothing left to do."""
        return None

    TraceCacheCandidates = confirm_candidate_batch
    MarkCachePublished = confirm_candidate_batch
    evication_cache = confirm_candidate_batch
    compact_cache = confirm_candidate_batch

    # -- results ---------------------------------------------------------------
    def gather(self):
        v = np.empty(self.n, np.uint32)
        p = np.empty(self.n, np.uint32)
        self._check(lib().dycg_gather(self._h, _ptr(v, ctypes.c_uint32), _ptr(p, ctypes.c_uint32)),
                    "gather")
        return v, p

    def GatherValue(self):
        return self.gather()[0]

    def GatherParent(self):
        return self.gather()[1]

    def GatherBuffer(self):
        """The reference's per-vertex buffer: equal to the value once a repair
        has finished (SSSP/BFS/CC); the residuals for PageRank."""
        if self.algo == ALGOS["pr"]:
            return self.gather_ranks()[1]
        return self.gather()[0]

    def GetGraphDatum(self):
        """Sizes and memory layout of the graph (the reference returns its
        GraphDatum)."""
        return self.info()

    def ChunkStore(self):
        """The live outgoing adjacency as CSR (offsets, dst, w)."""
        return self.csr()

    def SetOptions(self, **options):
        """Options are fixed when the engine is created (dycg_create takes them):
        values equal to the engine's are accepted, any other is an error."""
        names = {"algo": ALGOS, "weight_mode": WEIGHTS, "cache_policy": CACHE}
        for k, v in options.items():
            if not hasattr(self.options, k) or k == "reserved":
                raise DycgError(-1, f"unknown option {k}")
            if isinstance(v, str) and k in names:
                v = names[k][v]
            cur = getattr(self.options, k)
            same = abs(cur - v) <= 1e-6 * max(1.0, abs(v)) if isinstance(cur, float) else cur == v
            if not same:
                raise DycgError(-1, f"option {k} is fixed at creation ({cur}), not {v}")

    # -- many-query forms --------------------------------------------------------
    QUERY_MODES = {"batched": 0, "per_query": 1}

    def set_queries(self, sources, mode="batched"):
        """Keep the results of every source in `sources` (SSSP/BFS, up to 256):
        "batched" repairs all of them in one launch per snapshot, "per_query"
        launches the single-source repair once per query. Call before start()."""
        src = np.ascontiguousarray(np.ravel(sources), dtype=np.uint32)
        self._check(lib().dycg_set_queries(self._h, _ptr(src, ctypes.c_uint32), len(src),
                                           self.QUERY_MODES[mode]), "set_queries")
        self.queries = len(src)

    def set_query_mapping(self, qratio=4, heavy=64, tile=4096):
        """Batched form's work mapping (speed only): rows with
        4*active >= qratio*min(len, 32) map lanes to queries, others lanes to
        slots; rows above `heavy` warp iterations are tiled (tile slots)."""
        self._check(lib().dycg_set_query_mapping(self._h, qratio, heavy, tile),
                    "set_query_mapping")

    QUEUE_SCHEMES = {"static": 0, "claimed": 1, "ranges": 2, "claimed+ranges": 3, "async": 4,
                     "async+claimed": 5}

    def set_query_queue(self, scheme="static"):
        """Batched form's frontier-queue scheme (speed only): "static" (warp w
        takes items w, w + warps, ...), "claimed" (warps claim items one at a
        time), with "+ranges" the wave queues read by vertex range; "async"
        runs the invalidation and the closure on a worklist without waves."""
        self._check(lib().dycg_set_query_queue(
            self._h, self.QUEUE_SCHEMES[scheme] if isinstance(scheme, str) else int(scheme)),
            "set_query_queue")

    def gather_query(self, q):
        v = np.empty(self.n, np.uint32)
        p = np.empty(self.n, np.uint32)
        self._check(lib().dycg_gather_query(self._h, q, _ptr(v, ctypes.c_uint32),
                                            _ptr(p, ctypes.c_uint32)), "gather_query")
        return v, p

    def gather_ranks(self):
        x = np.empty(self.n, np.float32)
        r = np.empty(self.n, np.float32)
        self._check(lib().dycg_gather_ranks(self._h, _ptr(x, ctypes.c_float),
                                            _ptr(r, ctypes.c_float)), "gather_ranks")
        return x, r

    def row(self, v, incoming=False, cap=None):
        deg = ctypes.c_uint32(0)
        self._check(lib().dycg_get_row(self._h, v, int(incoming), None, None, 0, ctypes.byref(deg)),
                    "get_row")
        n = deg.value
        d = np.empty(max(n, 1), np.uint32)
        w = np.empty(max(n, 1), np.uint32)
        self._check(lib().dycg_get_row(self._h, v, int(incoming), _ptr(d, ctypes.c_uint32),
                                       _ptr(w, ctypes.c_uint32), n, ctypes.byref(deg)), "get_row")
        return d[:n], w[:n]

    def csr(self):
        m = self.info()["live_edges"]
        off = np.empty(self.n + 1, np.uint64)
        dst = np.empty(max(m, 1), np.uint32)
        w = np.empty(max(m, 1), np.uint32)
        self._check(lib().dycg_export_csr(self._h, _ptr(off, ctypes.c_uint64),
                                          _ptr(dst, ctypes.c_uint32), _ptr(w, ctypes.c_uint32)),
                    "export_csr")
        return off, dst[:m], w[:m]

    def info(self):
        gi = GraphInfo()
        self._check(lib().dycg_graph_info_get(self._h, ctypes.byref(gi)), "graph_info")
        return gi.as_dict()

    def sample_edges(self, count, seed):
        out = np.empty((count, 3), np.uint32)
        self._check(lib().dycg_sample_edges(self._h, count, seed,
                                            out.ctypes.data_as(ctypes.POINTER(Edge))),
                    "sample_edges")
        return out

    def stream(self):
        s = ctypes.c_void_p()
        self._check(lib().dycg_stream(self._h, ctypes.byref(s)), "stream")
        return s.value
