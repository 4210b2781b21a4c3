"""dycg_group_updates_noalloc -- grouping an update batch without allocating.

Some callers of this library cannot call cudaMalloc at the point where they
need a batch grouped: code that must not synchronise the device, processes
whose device memory is held by another allocator, host components that may
not own GPU allocations. The no-allocation entry point keeps its scratch in a
fixed device array of the library; these tests check, through the C ABI, that
it returns exactly what the allocating dycg_group_updates returns, on calls in
a row, and that it refuses batches above its fixed capacity.
"""
import ctypes

import numpy as np
import pytest

import dycgraph_b200 as dg

pytestmark = pytest.mark.gpu
MAX_RECORDS = 262144  # DYCG_GROUP_NOALLOC_MAX_RECORDS
DYCG_ECAPACITY = -5


def _group(fn, rec, nv, ends):
    import torch
    n = rec.shape[0]
    d_rec = torch.from_numpy(rec.astype(np.int32).reshape(-1)).cuda()
    d_uv = torch.zeros(2 * max(n, 1), dtype=torch.int32, device="cuda")
    d_mult = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    d_ends = torch.from_numpy(ends.astype(np.int32)).cuda()
    d_seg = torch.zeros(len(ends), dtype=torch.int32, device="cuda")
    d_cnt = torch.full((2,), 9, dtype=torch.int32, device="cuda")
    rc = fn(ctypes.c_void_p(d_rec.data_ptr()), n, nv, ctypes.c_void_p(d_ends.data_ptr()),
            len(ends), ctypes.c_void_p(d_uv.data_ptr()), ctypes.c_void_p(d_mult.data_ptr()),
            ctypes.c_void_p(d_seg.data_ptr()), ctypes.c_void_p(d_cnt.data_ptr()), None)
    torch.cuda.synchronize()
    cnt = d_cnt.cpu().numpy()
    k = int(cnt[0])
    return (rc, d_uv.cpu().numpy()[:2 * k].copy(), d_mult.cpu().numpy()[:k].copy(), cnt.copy(),
            d_seg.cpu().numpy().copy())


def _records(n, seed, nv):
    rng = np.random.default_rng(seed)
    rec = rng.integers(0, nv + 40, size=(n, 3)).astype(np.uint32)  # some endpoints out of range
    rec[n // 3:n // 3 + 25] = rec[1]                              # repeated records
    return rec


def test_noalloc_matches_allocating_entry_point_on_calls_in_a_row():
    L = dg.lib()
    nv = 70_000
    ends = np.array([10_000, 30_000, 50_000, nv], np.uint32)
    inputs = [_records(60_000, 1, nv), _records(MAX_RECORDS, 2, nv), _records(60_000, 1, nv)]
    for rec in inputs:
        want = _group(L.dycg_group_updates, rec, nv, ends)
        got = _group(L.dycg_group_updates_noalloc, rec, nv, ends)
        assert want[0] == 0 and got[0] == 0
        for a, b in zip(want[1:], got[1:]):
            assert np.array_equal(a, b)


def _numpy_group(rec, nv, ends):
    ok = (rec[:, 0] < nv) & (rec[:, 1] < nv)
    keys = rec[ok, 0].astype(np.uint64) << np.uint64(32) | rec[ok, 1].astype(np.uint64)
    uk, cnt = np.unique(keys, return_counts=True)
    u = (uk >> np.uint64(32)).astype(np.uint32)
    seg = np.bincount(np.searchsorted(ends, u, side="right"), minlength=len(ends))[:len(ends)]
    uv = np.stack([u, (uk & np.uint64(0xFFFFFFFF)).astype(np.uint32)], 1).reshape(-1)
    return uv, cnt.astype(np.uint32), int((~ok).sum()), seg.astype(np.uint32)


def test_noalloc_full_capacity_single_hub_matches_numpy():
    """Every record of a full-capacity batch in one hub row (one source, three
    destinations, so three runs of ~87K copies), all in one segment: the
    multiplicities and segment counts must be numpy's, on two calls in a row."""
    L = dg.lib()
    nv = 70_000
    rng = np.random.default_rng(5)
    rec = np.empty((MAX_RECORDS, 3), np.uint32)
    rec[:, 0] = 40_000
    rec[:, 1] = rng.choice(np.array([3, 39_999, 69_999], np.uint32), size=MAX_RECORDS)
    rec[:, 2] = 7
    ends = np.array([10_000, 30_000, 50_000, nv], np.uint32)
    uv, mult, bad, seg = _numpy_group(rec, nv, ends)
    for _ in range(2):
        rc, guv, gmult, cnt, gseg = _group(L.dycg_group_updates_noalloc, rec, nv, ends)
        assert rc == 0
        assert int(cnt[0]) == len(mult) and int(cnt[1]) == bad
        assert np.array_equal(guv.astype(np.uint32), uv)
        assert np.array_equal(gmult.astype(np.uint32), mult)
        assert np.array_equal(gseg.astype(np.uint32), seg)


def test_noalloc_rejects_batches_above_capacity():
    import torch
    L = dg.lib()
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    rc = L.dycg_group_updates_noalloc(p, MAX_RECORDS + 1, 10, None, 0, p, p, None, p, None)
    assert rc == DYCG_ECAPACITY
