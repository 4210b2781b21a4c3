"""GPU parity of deletions in rows with long unsorted suffixes (the sort-merge
path): hub rows receive thousands of appended occurrences, including
duplicates, then deletions hit the sorted prefix, the suffix (with
multiplicity) and absent edges. The live adjacency (per-row multiset), the
missing-delete count and the SSSP results must equal the oracle's."""
import numpy as np
import pytest

import dycgraph_b200 as dg
import oracle
from tests import cases

pytestmark = pytest.mark.gpu


def _rows(off, dst, w):
    out = {}
    for u in range(len(off) - 1):
        a, b = int(off[u]), int(off[u + 1])
        if b > a:
            out[u] = sorted(zip(dst[a:b].tolist(), w[a:b].tolist()))
    return out


@pytest.mark.parametrize("symmetric", [False, True])
def test_long_suffix_deletions_match_oracle(symmetric):
    n, off, dst, w = cases.small_rmat(11, 4, 61)

    def wt(u, v):  # symmetric weights: the symmetric mode reads in-rows as out-rows
        return cases.hw(np.minimum(u, v), np.maximum(u, v))

    if symmetric:
        src = np.repeat(np.arange(n), np.diff(off).astype(np.int64))
        pairs = np.unique(np.concatenate([np.stack([src, dst], 1), np.stack([dst, src], 1)]), axis=0)
        off, dst, _ = cases.csr(n, pairs)
        w = wt(np.repeat(np.arange(n), np.diff(off).astype(np.int64)), dst)
    e = dg.Engine("sssp", weight_mode="stored", page_shift=8, symmetric=symmetric)
    e.load_csr(n, off, dst, w)
    e.start()
    orc = oracle.Oracle(oracle.SSSP, n, off, dst, w, weight_mode=oracle.WEIGHT_STORED,
                        symmetric=symmetric)
    orc.init()
    rng = np.random.default_rng(5)
    hubs = [0, 7, 300]

    def sym(recs):
        return recs + [(v, u, x) for u, v, x in recs] if symmetric else recs

    # snapshot 1: 3000+ appends per hub, some targets two or three times
    adds = []
    for h in hubs:
        t = rng.integers(1, n, 2500)
        t = np.concatenate([t, t[:400], t[:150]])
        t = t[t != h]
        adds += [(h, int(v), int(wt(h, v))) for v in t]
    e.apply_batch([], sym(adds))
    orc.apply_batch([], sym(adds))
    # snapshot 2: deletions in the same rows -- suffix occurrences (with
    # multiplicity up to 4), prefix edges, edges that do not exist
    dels = []
    for h in hubs:
        app = [r for r in adds if r[0] == h]
        pick = rng.choice(len(app), 900, replace=False)
        dels += [app[i] for i in pick]
        dels += [app[i] for i in pick[:200]]   # second occurrence of the same edge
        dels += [app[i] for i in pick[:60]]    # third
        dels += [app[i] for i in pick[:30]]    # fourth: may exceed the copies
        a, b = int(off[h]), int(off[h + 1])
        dels += [(h, int(dst[j]), int(w[j])) for j in range(a, min(b, a + 5))]  # prefix
        dels += [(h, n - 1 - k, 1) for k in range(20)]                          # mostly absent
    more_adds = [(hubs[0], int(v), int(wt(hubs[0], v))) for v in rng.integers(1, n, 200)]
    st = e.apply_batch(sym(dels), sym(more_adds))
    orc.apply_batch(sym(dels), sym(more_adds))
    assert st["missing_deletes"] == orc.stats()["missing_deletes"]
    assert _rows(*e.csr()) == _rows(*orc.csr())
    assert (e.gather()[0] == orc.values()[0]).all()
    o, d, ww = orc.csr()
    assert (e.gather()[0] == oracle.static_sssp(n, o, d, ww, oracle.WEIGHT_STORED, 0)).all()
    # snapshot 3: delete everything left in one hub row through the long suffix
    o, d, ww = orc.csr()
    h = hubs[1]
    rest = [(h, int(d[j]), int(ww[j])) for j in range(int(o[h]), int(o[h + 1]))]
    e.apply_batch(sym(rest), [])
    orc.apply_batch(sym(rest), [])
    assert e.row(h)[0].size == 0
    assert _rows(*e.csr()) == _rows(*orc.csr())
    assert (e.gather()[0] == orc.values()[0]).all()
