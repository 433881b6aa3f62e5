"""hnswgpu_search_noalloc: the HNSW search for callers that must not allocate
device memory -- a process whose memory budget is owned by someone else (a
framework's caching allocator, a serving loop that reserves everything at
start-up) or that cannot afford the device-wide synchronisation a cudaMalloc or
cudaFree may trigger.  Its scratch lives in a fixed array inside the library,
so the caller brings only the loaded index, the queries and the outputs.

The test calls it through the C ABI, twice in a row, and checks each result
against hnswgpu_search on the same queries, bit for bit (the tolerance every
parity test here uses).  This file is collected last on purpose."""
import ctypes as C
import os

import numpy as np
import pytest

import hnsw_rabitq_b200 as H
from hnsw_rabitq_b200 import _capi

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _reference_call(idx, q, k, ef, flags):
    """The existing entry point with host buffers."""
    nq = q.shape[0]
    labels = np.empty((nq, k), np.uint64)
    dists = np.empty((nq, k), np.float32)
    counts = np.empty(nq, np.int32)
    opts = _capi.SearchOpts()
    opts.ef = ef
    opts.flags = flags
    _capi.check(_capi.lib().hnswgpu_search(idx._h, q.ctypes.data, nq, k, C.byref(opts), labels.ctypes.data,
                                           dists.ctypes.data, counts.ctypes.data))
    return labels, dists, counts


def test_noalloc_matches_search_two_calls():
    import torch

    g = np.load(os.path.join(GOLDEN, "golden.npz"))
    q_all = g["hnsw_l2_d16/queries"].astype(np.float32)
    idx = H.Index("l2", 16)
    idx.load_index(os.path.join(GOLDEN, "hnsw_l2_d16.bin"))
    lib = _capi.lib()
    k, ef = 10, 32
    stream = torch.cuda.Stream()
    for flags in (_capi.EXACT_TIES, 0):
        # two calls in a row, different batches: the second relies on the
        # shared scratch having been cleared for it
        for q in (q_all[:25], q_all[10:]):
            q = np.ascontiguousarray(q)
            nq = q.shape[0]
            dq = torch.from_numpy(q).cuda()
            dl = torch.empty((nq, k), dtype=torch.int64, device="cuda")
            dd = torch.empty((nq, k), dtype=torch.float32, device="cuda")
            dc = torch.empty((nq,), dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            _capi.check(lib.hnswgpu_search_noalloc(idx._h, dq.data_ptr(), nq, k, ef, flags, None, dl.data_ptr(),
                                                   dd.data_ptr(), dc.data_ptr(), stream.cuda_stream))
            stream.synchronize()
            rl, rd, rc = _reference_call(idx, q, k, ef, flags)
            assert np.array_equal(dc.cpu().numpy(), rc)
            assert np.array_equal(dl.cpu().numpy().view(np.uint64), rl)
            assert np.array_equal(dd.cpu().numpy().view(np.uint32), rd.view(np.uint32))


def test_noalloc_rejects_oversized_batches():
    idx = H.Index("l2", 16)
    idx.load_index(os.path.join(GOLDEN, "hnsw_l2_d16.bin"))
    lib = _capi.lib()
    rc = lib.hnswgpu_search_noalloc(idx._h, 16, 1 << 31, 10, 0, 0, None, 16, 16, 16, None)
    assert rc == _capi.ERR_ARG
    assert b"2^31" in lib.hnswgpu_last_error()
