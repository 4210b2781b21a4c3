"""dycg_group_updates (device grouping of an update batch) against numpy."""
import ctypes

import numpy as np
import pytest

import dycgraph_b200 as dg

pytestmark = pytest.mark.gpu


def group_ref(rec, nv, ends):
    ok = (rec[:, 0] < nv) & (rec[:, 1] < nv)
    keys = rec[ok, 0].astype(np.uint64) << np.uint64(32) | rec[ok, 1].astype(np.uint64)
    uk, cnt = np.unique(keys, return_counts=True)
    u = (uk >> np.uint64(32)).astype(np.uint32)
    seg = np.bincount(np.searchsorted(ends, u, side="right"), minlength=len(ends))[:len(ends)]
    return uk, cnt.astype(np.uint32), int((~ok).sum()), seg.astype(np.uint32)


def run_group(fn, rec, nv, ends):
    import torch
    n = rec.shape[0]
    d_rec = torch.from_numpy(rec.astype(np.int32).reshape(-1)).cuda()
    d_uv = torch.zeros(2 * max(n, 1), dtype=torch.int32, device="cuda")
    d_mult = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    d_ends = torch.from_numpy(ends.astype(np.int32)).cuda()
    d_seg = torch.zeros(max(len(ends), 1), dtype=torch.int32, device="cuda")
    d_cnt = torch.full((2,), 7, dtype=torch.int32, device="cuda")
    rc = fn(ctypes.c_void_p(d_rec.data_ptr()), n, nv, ctypes.c_void_p(d_ends.data_ptr()), len(ends),
            ctypes.c_void_p(d_uv.data_ptr()), ctypes.c_void_p(d_mult.data_ptr()),
            ctypes.c_void_p(d_seg.data_ptr()), ctypes.c_void_p(d_cnt.data_ptr()), None)
    torch.cuda.synchronize()
    cnt = d_cnt.cpu().numpy().astype(np.uint32)
    k = int(cnt[0])
    uv = d_uv.cpu().numpy().astype(np.uint32)[:2 * k].reshape(-1, 2)
    keys = uv[:, 0].astype(np.uint64) << np.uint64(32) | uv[:, 1].astype(np.uint64)
    return rc, keys, d_mult.cpu().numpy().astype(np.uint32)[:k], int(cnt[1]), d_seg.cpu().numpy().astype(np.uint32)[:len(ends)]


@pytest.mark.parametrize("n", [0, 1, 1000, 200_000])
def test_group_updates_matches_numpy(n):
    rng = np.random.default_rng(n + 3)
    nv = 5000
    rec = rng.integers(0, nv + 50, size=(n, 3)).astype(np.uint32)  # some endpoints invalid
    if n > 10:
        rec[n // 2:n // 2 + 10] = rec[0]  # duplicates
    ends = np.array([1000, 2500, 4000, nv], np.uint32)
    rc, keys, mult, bad, seg = run_group(dg.lib().dycg_group_updates, rec, nv, ends)
    assert rc == 0
    uk, cnt, rbad, rseg = group_ref(rec, nv, ends)
    assert (keys == uk).all() and (mult == cnt).all()
    assert bad == rbad and (seg == rseg).all()


def _hub_records(n, nv, seed):
    """One hub row: every record has the same source and one of three
    destinations (runs of ~n/3 copies), plus a few out-of-range records."""
    rng = np.random.default_rng(seed)
    rec = np.empty((n, 3), np.uint32)
    rec[:, 0] = 17
    rec[:, 1] = rng.choice(np.array([5, 6, nv - 1], np.uint32), size=n)
    rec[:, 2] = 1
    rec[rng.integers(0, n, size=8), 0] = nv + 3
    return rec


@pytest.mark.parametrize("fn", ["dycg_group_updates", "dycg_group_updates_noalloc"])
def test_group_updates_single_hub_batch(fn):
    """A batch of 262,144 records for one hub row: run lengths come from the
    run starts, so each run of ~87K copies costs one thread, not a walk."""
    nv = 5000
    rec = _hub_records(262_144, nv, 11)
    ends = np.array([16, 18, nv], np.uint32)
    rc, keys, mult, bad, seg = run_group(getattr(dg.lib(), fn), rec, nv, ends)
    assert rc == 0
    uk, cnt, rbad, rseg = group_ref(rec, nv, ends)
    assert (keys == uk).all() and (mult == cnt).all()
    assert bad == rbad and (seg == rseg).all()
    assert int(mult.sum()) == 262_144 - rbad
