"""The status path of the kernels' bounded waits, exercised without a GPU
fault: a warp waits on a copy that never arrives, gives up after a few
milliseconds and reports HNSWGPU_STATUS_TIMEOUT; the device stays usable and
the next search on it is exact."""
import ctypes as C
import os

import numpy as np
import pytest

import hnsw_rabitq_b200 as H
from hnsw_rabitq_b200 import _capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_bounded_wait_reports_timeout_and_device_stays_usable():
    bits = _capi.U32(0)
    _capi.check(_capi.lib().hnswgpu_selftest_wait_timeout(0, C.byref(bits)))
    assert bits.value == _capi.STATUS_TIMEOUT
    g = np.load(os.path.join(GOLDEN, "golden.npz"))
    q = g["hnsw_l2_d16/queries"]
    path = os.path.join(GOLDEN, "hnsw_l2_d16.bin")
    idx = H.Index("l2", 16)
    idx.load_index(path)
    idx.set_ef(32)
    idx.tie_order = "id"
    labels, dists = idx.knn_query(q, k=10)
    ol, od, _ = O.Hnsw(path, "l2", 16).search(q, 10, 32, mode=O.CANONICAL)
    assert np.array_equal(labels, ol) and np.array_equal(dists.view(np.uint32), od.view(np.uint32))
    assert idx.get_status() == 0
