"""Loaders for the golden fixtures and small seeded workloads used by tests."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def csr(n, pairs, weights=None):
    """CSR keeping each row's occurrences in list order (file order)."""
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    order = np.argsort(pairs[:, 0], kind="stable")
    off = np.zeros(n + 1, np.uint64)
    if len(pairs):
        np.add.at(off, pairs[:, 0] + 1, 1)
    off = np.cumsum(off).astype(np.uint64)
    dst = pairs[order, 1].astype(np.uint32)
    w = None if weights is None else np.asarray(weights, np.uint32)[order]
    return off, dst, w


def rule_w(algo, u, v):
    if algo == 1:
        return 1
    if algo == 2:
        return 0
    return (u + v) % 128 + 1


def triples(pairs, algo=0):
    return [(int(u), int(v), rule_w(algo, int(u), int(v))) for u, v in pairs]


def replay_batches(updates, sizes):
    """Split an update list the way the reference's Loader does
    (include/framework/Loader.h:30-101): all 'a' records in file order feed
    the add counts, all 'd' records the delete counts, per sizes line
    (adds dels)."""
    adds = [(u, v) for t, u, v in updates if t == "a"]
    dels = [(u, v) for t, u, v in updates if t == "d"]
    out, ia, idl = [], 0, 0
    for na, nd in sizes:
        out.append((dels[idl:idl + nd], adds[ia:ia + na]))
        ia += na
        idl += nd
    return out


def rmat_edges(scale, m, seed, a=0.57, b=0.19, c=0.19):
    """Small seeded R-MAT draws in numpy (test-only helper)."""
    rng = np.random.default_rng(seed)
    u = np.zeros(m, np.int64)
    v = np.zeros(m, np.int64)
    for _ in range(scale):
        r = rng.random(m)
        bu = (r >= a + b).astype(np.int64)
        bv = (((r >= a) & (r < a + b)) | (r >= a + b + c)).astype(np.int64)
        u = (u << 1) | bu
        v = (v << 1) | bv
    return u, v


def hw(u, v, wlo=1, whi=64):
    """Deterministic weight of (u, v): parallel copies of an edge agree."""
    x = (np.asarray(u, np.uint64) * np.uint64(0x9E3779B1) + np.asarray(v, np.uint64) * np.uint64(0x85EBCA77)) % np.uint64(2**32)
    x = (x ^ (x >> np.uint64(15))) * np.uint64(0x2C1B3C6D) % np.uint64(2**32)
    x = x ^ (x >> np.uint64(12))
    return (np.uint64(wlo) + x % np.uint64(whi - wlo + 1)).astype(np.uint32)


def small_rmat(scale=10, ef=8, seed=1, wlo=1, whi=64):
    n = 1 << scale
    u, v = rmat_edges(scale, n * ef, seed)
    keep = u != v
    key = np.unique(u[keep] * n + v[keep])
    uu, vv = key // n, key % n
    w = hw(uu, vv, wlo, whi)
    off = np.zeros(n + 1, np.uint64)
    np.add.at(off, uu + 1, 1)
    off = np.cumsum(off).astype(np.uint64)
    return n, off, vv.astype(np.uint32), w


def random_batch(n, off, dst, w, nd, na, seed, wlo=1, whi=64, stored=True):
    """nd distinct live edges to delete and na R-MAT-ish random inserts."""
    rng = np.random.default_rng(seed)
    m = len(dst)
    src = np.repeat(np.arange(n), np.diff(off).astype(np.int64))
    pick = rng.choice(m, size=min(nd, m), replace=False) if m else np.zeros(0, np.int64)
    dels = [(int(src[i]), int(dst[i]), int(w[i]) if w is not None else 1) for i in pick]
    scale = max(1, int(np.log2(n)))
    au, av = rmat_edges(scale, na, seed + 1)
    au, av = au % n, av % n
    aw = hw(au, av, wlo, whi)
    adds = [(int(x), int(y), int(z)) for x, y, z in zip(au, av, aw)]
    return dels, adds


def zipf_vertices(n, count, rng, s=1.1, perm=None):
    """count vertex ids whose ranks follow Zipf(s) over n vertices (rank 1 most
    frequent), mapped through a permutation so the hot ids are scattered."""
    out = np.empty(0, np.int64)
    while len(out) < count:
        k = rng.zipf(s, size=2 * (count - len(out)) + 16)
        out = np.concatenate([out, k[k <= n] - 1])
    out = out[:count]
    return (perm[out] if perm is not None else out).astype(np.uint32)


def zipf_snapshot(eng, n, nd, na, rng, perm, s=1.1, wlo=1, whi=64):
    """nd deletions of live edges out of Zipf-chosen sources and na insertions
    with both endpoints Zipf-chosen (weights hashed from the endpoints)."""
    src = zipf_vertices(n, nd, rng, s, perm)
    d = eng.sample_row_edges(src, int(rng.integers(1 << 62)))
    d = d[d[:, 0] != 0xFFFFFFFF]
    u = zipf_vertices(n, na, rng, s, perm)
    v = zipf_vertices(n, na, rng, s, perm)
    keep = u != v
    u, v = u[keep], v[keep]
    a = np.stack([u, v, hw(u, v, wlo, whi)], 1).astype(np.uint32)
    return d, a
