"""ctypes binding of the CPU oracle (oracle/oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline and reference legs, always as the checker or the CPU
reference, never by the product package.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

SSSP, BFS, CC, PR = 0, 1, 2, 3
WEIGHT_HASH128, WEIGHT_STORED = 0, 1
INF = 0xFFFFFFFF


class Edge(ctypes.Structure):
    _fields_ = [("u", ctypes.c_uint32), ("v", ctypes.c_uint32), ("w", ctypes.c_uint32)]


class Stats(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint64) for name in (
        "missing_deletes", "invalid_updates", "touched_sources", "changed_sources",
        "affected", "pull_iterations", "expanded", "edges_scanned", "pr_rounds")]


def build():
    """Compile liboracle.so (and oracle/_ref when the reference is present)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        u32p = ctypes.POINTER(ctypes.c_uint32)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        f64p = ctypes.POINTER(ctypes.c_double)
        ep = ctypes.POINTER(Edge)
        L.orc_create.restype = P
        L.orc_create.argtypes = [ctypes.c_uint32] * 4 + [ctypes.c_double, ctypes.c_double,
                                                         ctypes.c_uint32, ctypes.c_int]
        L.orc_destroy.argtypes = [P]
        L.orc_load_csr.argtypes = [P, ctypes.c_uint32, u64p, u32p, u32p]
        L.orc_init.argtypes = [P]
        L.orc_set_state.argtypes = [P, u32p, u32p, f64p, f64p]
        for fn in (L.orc_delete_edges, L.orc_insert_edges):
            fn.argtypes = [P, ep, ctypes.c_size_t]
        L.orc_apply_batch.argtypes = [P, ep, ctypes.c_size_t, ep, ctypes.c_size_t]
        L.orc_mutate.argtypes = [P, ep, ctypes.c_size_t, ep, ctypes.c_size_t]
        L.orc_values.argtypes = [P, u32p, u32p]
        L.orc_ranks.argtypes = [P, f64p, f64p]
        L.orc_last_stats.argtypes = [P, ctypes.POINTER(Stats)]
        L.orc_nodes.restype = ctypes.c_uint64
        L.orc_nodes.argtypes = [P]
        L.orc_live_edges.restype = ctypes.c_uint64
        L.orc_live_edges.argtypes = [P]
        L.orc_export_csr.argtypes = [P, u64p, u32p, u32p]
        L.orc_row_degree.restype = ctypes.c_uint64
        L.orc_row_degree.argtypes = [P, ctypes.c_uint32]
        L.orc_row_multiset_hash.restype = ctypes.c_uint64
        L.orc_row_multiset_hash.argtypes = [P, ctypes.c_uint32]
        L.orc_static_sssp.argtypes = [ctypes.c_uint32, u64p, u32p, u32p, ctypes.c_uint32,
                                      ctypes.c_uint32, u32p]
        L.orc_static_bfs.argtypes = [ctypes.c_uint32, u64p, u32p, ctypes.c_uint32, u32p]
        L.orc_static_cc.argtypes = [ctypes.c_uint32, u64p, u32p, u32p]
        L.orc_static_pr.restype = ctypes.c_int
        L.orc_static_pr.argtypes = [ctypes.c_uint32, u64p, u32p, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_uint32, f64p]
        L.orc_bellman_check.restype = ctypes.c_uint64
        L.orc_bellman_check.argtypes = [ctypes.c_uint32, u64p, u32p, u32p, ctypes.c_uint32,
                                        ctypes.c_uint32, ctypes.c_uint32, u32p, u64p]
        L.orc_distance_checksum.restype = ctypes.c_uint64
        L.orc_distance_checksum.argtypes = [u32p, ctypes.c_uint32]
        L.orc_rule_weight.restype = ctypes.c_uint32
        L.orc_rule_weight.argtypes = [ctypes.c_uint32] * 3
        L.orc_gen_rmat_edges.argtypes = [ctypes.c_uint32, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_uint64, ctypes.c_uint64,
                                         ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ep]
        L.orc_rmat_csr.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_uint64,
                                   ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(u64p), ctypes.POINTER(u32p),
                                   ctypes.POINTER(u32p), u64p]
        L.orc_free.argtypes = [P]
        L.orc_parallel_sssp.argtypes = [ctypes.c_uint32, u64p, u32p, u32p, ctypes.c_uint32,
                                        ctypes.c_uint32, ctypes.c_uint32, u32p, u32p]
        _LIB = L
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t)) if a is not None else None


def edges_array(edges):
    """list of (u, v[, w]) or an (k,3) uint32 array -> ctypes Edge array."""
    arr = np.asarray(edges, dtype=np.uint32).reshape(-1, 3) if len(edges) else np.zeros((0, 3), np.uint32)
    arr = np.ascontiguousarray(arr)
    return arr, arr.ctypes.data_as(ctypes.POINTER(Edge)), arr.shape[0]


def with_w(edges):
    return [(e[0], e[1], e[2] if len(e) > 2 else 1) for e in edges]


class Oracle:
    """The reference's per-snapshot repair restated on the CPU."""

    def __init__(self, algo, n, offsets, dst, w=None, weight_mode=WEIGHT_HASH128, source=0,
                 symmetric=False, epsilon=1e-6, alpha=0.85, max_rounds=100, threads=0):
        L = lib()
        self.algo, self.n = algo, n
        self.h = L.orc_create(algo, weight_mode, source, int(symmetric), epsilon, alpha,
                              max_rounds, threads)
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        d = np.ascontiguousarray(dst, dtype=np.uint32)
        ww = None if w is None else np.ascontiguousarray(w, dtype=np.uint32)
        if L.orc_load_csr(self.h, n, _p(off, ctypes.c_uint64), _p(d, ctypes.c_uint32),
                          _p(ww, ctypes.c_uint32)):
            raise MemoryError("oracle load failed")

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def init(self):
        lib().orc_init(self.h)

    def set_state(self, values=None, parents=None, ranks=None, residuals=None):
        v = None if values is None else np.ascontiguousarray(values, np.uint32)
        p = None if parents is None else np.ascontiguousarray(parents, np.uint32)
        r = None if ranks is None else np.ascontiguousarray(ranks, np.float64)
        s = None if residuals is None else np.ascontiguousarray(residuals, np.float64)
        lib().orc_set_state(self.h, _p(v, ctypes.c_uint32), _p(p, ctypes.c_uint32),
                            _p(r, ctypes.c_double), _p(s, ctypes.c_double))

    def _call(self, fn, *lists):
        args = []
        keep = []
        for e in lists:
            arr, ptr, k = edges_array(e)
            keep.append(arr)
            args += [ptr, k]
        rc = fn(self.h, *args)
        if rc:
            raise RuntimeError(f"oracle call failed: {rc}")

    def delete_edges(self, dels):
        self._call(lib().orc_delete_edges, dels)

    def insert_edges(self, adds):
        self._call(lib().orc_insert_edges, adds)

    def apply_batch(self, dels, adds):
        self._call(lib().orc_apply_batch, dels, adds)

    def mutate(self, dels, adds):
        self._call(lib().orc_mutate, dels, adds)

    def values(self):
        v = np.empty(self.n, np.uint32)
        p = np.empty(self.n, np.uint32)
        lib().orc_values(self.h, _p(v, ctypes.c_uint32), _p(p, ctypes.c_uint32))
        return v, p

    def ranks(self):
        x = np.empty(self.n, np.float64)
        r = np.empty(self.n, np.float64)
        lib().orc_ranks(self.h, _p(x, ctypes.c_double), _p(r, ctypes.c_double))
        return x, r

    def stats(self):
        s = Stats()
        lib().orc_last_stats(self.h, ctypes.byref(s))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def live_edges(self):
        return lib().orc_live_edges(self.h)

    def csr(self):
        m = self.live_edges()
        off = np.empty(self.n + 1, np.uint64)
        dst = np.empty(max(m, 1), np.uint32)
        w = np.empty(max(m, 1), np.uint32)
        lib().orc_export_csr(self.h, _p(off, ctypes.c_uint64), _p(dst, ctypes.c_uint32),
                             _p(w, ctypes.c_uint32))
        return off, dst[:m], w[:m]

    def row_degree(self, v):
        return lib().orc_row_degree(self.h, v)

    def row_multiset_hash(self, v):
        return lib().orc_row_multiset_hash(self.h, v)


def static_sssp(n, off, dst, w=None, weight_mode=WEIGHT_HASH128, source=0):
    out = np.empty(n, np.uint32)
    off = np.ascontiguousarray(off, np.uint64)
    dst = np.ascontiguousarray(dst, np.uint32)
    w = None if w is None else np.ascontiguousarray(w, np.uint32)
    lib().orc_static_sssp(n, _p(off, ctypes.c_uint64), _p(dst, ctypes.c_uint32),
                          _p(w, ctypes.c_uint32), weight_mode, source, _p(out, ctypes.c_uint32))
    return out


def static_bfs(n, off, dst, source=0):
    out = np.empty(n, np.uint32)
    off = np.ascontiguousarray(off, np.uint64)
    dst = np.ascontiguousarray(dst, np.uint32)
    lib().orc_static_bfs(n, _p(off, ctypes.c_uint64), _p(dst, ctypes.c_uint32), source,
                         _p(out, ctypes.c_uint32))
    return out


def static_cc(n, off, dst):
    out = np.empty(n, np.uint32)
    off = np.ascontiguousarray(off, np.uint64)
    dst = np.ascontiguousarray(dst, np.uint32)
    lib().orc_static_cc(n, _p(off, ctypes.c_uint64), _p(dst, ctypes.c_uint32),
                        _p(out, ctypes.c_uint32))
    return out


def static_pr(n, off, dst, alpha=0.85, tol=1e-12, max_iter=1000):
    out = np.empty(n, np.float64)
    off = np.ascontiguousarray(off, np.uint64)
    dst = np.ascontiguousarray(dst, np.uint32)
    it = lib().orc_static_pr(n, _p(off, ctypes.c_uint64), _p(dst, ctypes.c_uint32), alpha,
                             tol, max_iter, _p(out, ctypes.c_double))
    if it < 0:
        raise RuntimeError("static PageRank did not converge")
    return out


def bellman_check(n, off, dst, w, algo, weight_mode, source, dist):
    missing = ctypes.c_uint64(0)
    off = np.ascontiguousarray(off, np.uint64)
    dst = np.ascontiguousarray(dst, np.uint32)
    w = None if w is None else np.ascontiguousarray(w, np.uint32)
    dist = np.ascontiguousarray(dist, np.uint32)
    relax = lib().orc_bellman_check(n, _p(off, ctypes.c_uint64), _p(dst, ctypes.c_uint32),
                                    _p(w, ctypes.c_uint32), algo, weight_mode, source,
                                    _p(dist, ctypes.c_uint32), ctypes.byref(missing))
    return relax, missing.value


def checksum(values):
    v = np.ascontiguousarray(values, np.uint32)
    return lib().orc_distance_checksum(_p(v, ctypes.c_uint32), v.shape[0])


def csr_from_edges(n, edges):
    """CSR in edge-list order per source (the market_big reader's order)."""
    e = np.asarray([(a, b) for a, b, *_ in edges], dtype=np.uint64).reshape(-1, 2)
    w = np.asarray([x[2] if len(x) > 2 else 1 for x in edges], dtype=np.uint32)
    order = np.argsort(e[:, 0], kind="stable") if len(e) else np.zeros(0, np.int64)
    src = e[order, 0] if len(e) else np.zeros(0, np.uint64)
    off = np.zeros(n + 1, np.uint64)
    np.add.at(off, (src + 1).astype(np.int64), 1)
    off = np.cumsum(off).astype(np.uint64)
    dst = e[order, 1].astype(np.uint32) if len(e) else np.zeros(0, np.uint32)
    return off, dst, w[order] if len(e) else np.zeros(0, np.uint32)


def gen_rmat_edges(scale, count, seed, first=0, a=0.57, b=0.19, c=0.19, wlo=1, whi=64):
    out = np.empty((count, 3), np.uint32)
    lib().orc_gen_rmat_edges(scale, a, b, c, seed, first, count, wlo, whi,
                             out.ctypes.data_as(ctypes.POINTER(Edge)))
    return out


def rmat_csr(scale, ef, seed, a=0.57, b=0.19, c=0.19, wlo=1, whi=64, with_w=True,
             symmetrize=False):
    """De-duplicated R-MAT CSR built on the host cores (numpy views over C arrays,
    copied so the C allocations can be released); symmetrize adds the reverse
    of every draw."""
    L = lib()
    po = ctypes.POINTER(ctypes.c_uint64)()
    pd = ctypes.POINTER(ctypes.c_uint32)()
    pw = ctypes.POINTER(ctypes.c_uint32)()
    m = ctypes.c_uint64(0)
    if L.orc_rmat_csr(scale, ef, a, b, c, seed, wlo, whi, int(with_w), int(symmetrize),
                      ctypes.byref(po),
                      ctypes.byref(pd), ctypes.byref(pw), ctypes.byref(m)):
        raise MemoryError("rmat_csr failed")
    n = 1 << scale
    off = np.ctypeslib.as_array(po, shape=(n + 1,)).copy()
    dst = np.ctypeslib.as_array(pd, shape=(max(m.value, 1),))[:m.value].copy()
    w = np.ctypeslib.as_array(pw, shape=(max(m.value, 1),))[:m.value].copy() if with_w else None
    for p in (po, pd, pw):
        if p:
            L.orc_free(ctypes.cast(p, ctypes.c_void_p))
    return n, off, dst, w


_U64 = np.uint64


def _mix64(z):
    """64-bit finaliser over uint64 arrays (wrapping arithmetic); the same
    mixing function the library's generators use."""
    z = (z + _U64(0x9E3779B97F4A7C15)) & _U64(0xFFFFFFFFFFFFFFFF)
    z = (z ^ (z >> _U64(30))) * _U64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> _U64(27))) * _U64(0x94D049BB133111EB)
    return z ^ (z >> _U64(31))


def hash_weights(seed, u, v, wlo, whi):
    """Stored weight of each directed edge (u, v) of a generated graph: the
    library's hash of (seed, u, v) folded into [wlo, whi]."""
    s = _U64(seed) ^ _U64(0x5745494748545321)
    k = (np.asarray(u, _U64) << _U64(32)) | np.asarray(v, _U64)
    r = _mix64(s ^ _mix64(k))
    return (_U64(wlo) + r % _U64(whi - wlo + 1)).astype(np.uint32)


def grid_csr(side, permille, radius, seed, wlo=1, whi=1000, with_w=True):
    """The road-like grid graph of the library's generator, built on the host
    cores: side x side vertices, 4-neighbour edges in both directions, plus
    side^2 * permille / 1000 shortcut draws (each a vertex and an offset within
    the Chebyshev radius, kept when the target is another vertex inside the
    grid) in both directions; duplicates removed, rows sorted by target
    (dycgraph_b200/csrc/build.cu grid_keys_kernel). Returns n, off, dst, w."""
    with np.errstate(over="ignore"):
        n = side * side
        u = np.arange(n, dtype=_U64)
        r, c = u // _U64(side), u % _U64(side)
        right, down = u[c + _U64(1) < _U64(side)], u[r + _U64(1) < _U64(side)]
        parts = [(right << _U64(32)) | (right + _U64(1)), ((right + _U64(1)) << _U64(32)) | right,
                 (down << _U64(32)) | (down + _U64(side)), ((down + _U64(side)) << _U64(32)) | down]
        j = np.arange(n * permille // 1000, dtype=_U64)
        h = _mix64(_U64(seed) ^ _mix64(j + _U64(0x51ED270B)))
        su = h % _U64(n)
        span = _U64(2 * radius + 1)
        dr = ((h >> _U64(32)) % span).astype(np.int64) - radius
        dc = ((h >> _U64(48)) % span).astype(np.int64) - radius
        rr = (su // _U64(side)).astype(np.int64) + dr
        cc = (su % _U64(side)).astype(np.int64) + dc
        ok = ((dr != 0) | (dc != 0)) & (rr >= 0) & (cc >= 0) & (rr < side) & (cc < side)
        sv = (rr * side + cc)[ok].astype(_U64)
        su = su[ok]
        parts += [(su << _U64(32)) | sv, (sv << _U64(32)) | su]
        keys = np.unique(np.concatenate(parts))
        src = (keys >> _U64(32)).astype(np.uint32)
        dst = (keys & _U64(0xFFFFFFFF)).astype(np.uint32)
        off = np.zeros(n + 1, np.uint64)
        off[1:] = np.cumsum(np.bincount(src, minlength=n)).astype(np.uint64)
        w = hash_weights(seed, src, dst, wlo, whi) if with_w else None
    return n, off, dst, w


def tight_parents(n, off, dst, w, algo, weight_mode, source, dist):
    """Parents for static distances: the smallest in-neighbour x with
    dist[x] + w(x, y) == dist[y] (the tie rule of the repair), INF for the
    source and for unreachable vertices."""
    deg = np.diff(np.asarray(off, np.int64))
    src = np.repeat(np.arange(n, dtype=np.uint32), deg)
    dst = np.asarray(dst, np.uint32)
    if algo == BFS:
        wt = np.ones(len(dst), np.uint64)
    elif weight_mode == WEIGHT_STORED:
        wt = np.asarray(w, np.uint64)
    else:
        wt = (src.astype(np.uint64) + dst) % np.uint64(128) + np.uint64(1)
    d = np.asarray(dist, np.uint64)
    ok = (d[src] != np.uint64(INF)) & (d[src] + wt == d[dst])
    par = np.full(n, INF, np.uint32)
    np.minimum.at(par, dst[ok], src[ok])
    par[source] = INF
    return par


def parallel_sssp(n, off, dst, w, algo, weight_mode, source=0):
    dist = np.empty(n, np.uint32)
    par = np.empty(n, np.uint32)
    off = np.ascontiguousarray(off, np.uint64)
    dst = np.ascontiguousarray(dst, np.uint32)
    w = None if w is None else np.ascontiguousarray(w, np.uint32)
    lib().orc_parallel_sssp(n, _p(off, ctypes.c_uint64), _p(dst, ctypes.c_uint32),
                            _p(w, ctypes.c_uint32), algo, weight_mode, source,
                            _p(dist, ctypes.c_uint32), _p(par, ctypes.c_uint32))
    return dist, par
