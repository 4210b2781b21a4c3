"""Failure detection of the persistent kernels without a GPU fault: a block
that never arrives at a grid barrier is reported through the bounded wait's
error status, within the time limit, and the context stays usable (a second
launch completes, and an engine on the same context repairs correctly)."""
import ctypes
import time

import numpy as np
import pytest

import dycgraph_b200 as dg
import oracle
from tests import cases

pytestmark = pytest.mark.gpu
ERR_BARRIER = 1


def test_absent_block_is_reported_and_the_context_stays_usable():
    absent, present = ctypes.c_uint32(99), ctypes.c_uint32(99)
    t0 = time.time()
    rc = dg.lib().dycg_check_bounded_wait(0, 200, ctypes.byref(absent), ctypes.byref(present))
    elapsed = time.time() - t0
    assert rc == 0
    assert absent.value == ERR_BARRIER  # the waiting blocks gave up and said so
    assert present.value == 0           # the same barrier completes when every block arrives
    assert elapsed < 10.0
    # an engine on the same context still repairs exactly
    n, off, dst, w = cases.small_rmat(10, 8, 3)
    e = dg.Engine("sssp", weight_mode="stored")
    e.load_csr(n, off, dst, w)
    e.start()
    orc = oracle.Oracle(oracle.SSSP, n, off, dst, w, weight_mode=oracle.WEIGHT_STORED)
    orc.init()
    dels, adds = cases.random_batch(n, off, dst, w, 100, 100, 5)
    e.apply_batch(dels, adds)
    orc.apply_batch(dels, adds)
    assert np.array_equal(e.gather()[0], orc.values()[0])
    e.close()


def test_bounded_wait_argument_checks():
    a, b = ctypes.c_uint32(0), ctypes.c_uint32(0)
    assert dg.lib().dycg_check_bounded_wait(0, 0, ctypes.byref(a), ctypes.byref(b)) == -1
    assert dg.lib().dycg_check_bounded_wait(0, 20000, ctypes.byref(a), ctypes.byref(b)) == -1
