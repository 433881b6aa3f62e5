"""hnswgpu_search_noalloc: the HNSW search for callers that must not allocate
device memory -- a process whose memory budget is owned by someone else (a
framework's caching allocator, a serving loop that reserves everything at
start-up) or that cannot afford the device-wide synchronisation a cudaMalloc or
cudaFree may trigger.  Its scratch lives in a fixed array inside the library,
so the caller brings only the loaded index, the queries and the outputs.

The tests call it through the C ABI, twice in a row, and check each result
against hnswgpu_search on the same queries, bit for bit (the tolerance every
parity test here uses), over the golden indexes of every space, with an allow
mask, with deleted elements and in both tie orders; and they read its status
word through hnswgpu_noalloc_get_status.  This file is collected last on
purpose."""
import ctypes as C
import os

import numpy as np
import pytest

import hnsw_rabitq_b200 as H
from hnsw_rabitq_b200 import _capi

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# golden index, space, dim (dim % 16 != 0 runs the one-lane-per-row distances)
INDEXES = [("hnsw_l2_d16", "l2", 16), ("hnsw_cos_d12", "cosine", 12), ("hnsw_ip_d20", "ip", 20),
           ("hnsw_l2_d7_int", "l2", 7)]


def _reference_call(idx, q, k, ef, flags, allow=None):
    """The existing entry point with host buffers."""
    nq = q.shape[0]
    labels = np.empty((nq, k), np.uint64)
    dists = np.empty((nq, k), np.float32)
    counts = np.empty(nq, np.int32)
    opts = _capi.SearchOpts()
    opts.ef = ef
    opts.flags = flags
    if allow is not None:
        opts.allow = allow.ctypes.data
    _capi.check(_capi.lib().hnswgpu_search(idx._h, q.ctypes.data, nq, k, C.byref(opts), labels.ctypes.data,
                                           dists.ctypes.data, counts.ctypes.data))
    return labels, dists, counts


def _noalloc_call(idx, q, k, ef, flags, stream, allow=None):
    import torch
    nq = q.shape[0]
    dq = torch.from_numpy(q).cuda()
    dl = torch.empty((nq, k), dtype=torch.int64, device="cuda")
    dd = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    dc = torch.empty((nq,), dtype=torch.int32, device="cuda")
    da = torch.from_numpy(allow).cuda() if allow is not None else None
    torch.cuda.synchronize()
    _capi.check(_capi.lib().hnswgpu_search_noalloc(idx._h, dq.data_ptr(), nq, k, ef, flags,
                                                   None if da is None else da.data_ptr(), dl.data_ptr(),
                                                   dd.data_ptr(), dc.data_ptr(), stream.cuda_stream))
    stream.synchronize()
    return dl.cpu().numpy().view(np.uint64), dd.cpu().numpy(), dc.cpu().numpy()


def _status(stream):
    bits = _capi.U32(0)
    _capi.check(_capi.lib().hnswgpu_noalloc_get_status(0, stream.cuda_stream, C.byref(bits)))
    return bits.value


def _same(a, b):
    al, ad, ac = a
    bl, bd, bc = b
    assert np.array_equal(ac, bc)
    assert np.array_equal(al, bl)
    assert np.array_equal(ad.view(np.uint32), bd.view(np.uint32))


@pytest.mark.parametrize("name,space,dim", INDEXES)
def test_noalloc_matches_search_two_calls(name, space, dim):
    import torch

    g = np.load(os.path.join(GOLDEN, "golden.npz"))
    q_all = g[f"{name}/queries"].astype(np.float32)
    idx = H.Index(space, dim)
    idx.load_index(os.path.join(GOLDEN, f"{name}.bin"))
    stream = torch.cuda.Stream()
    _status(stream)  # start from a clear status word
    k = 10
    for flags in (_capi.EXACT_TIES, 0):
        for ef in (32, 100):
            # two calls in a row, different batches: the second relies on the
            # shared scratch having been cleared for it
            for q in (q_all[:25], q_all[10:]):
                q = np.ascontiguousarray(q)
                _same(_noalloc_call(idx, q, k, ef, flags, stream), _reference_call(idx, q, k, ef, flags))
    assert _status(stream) == 0


@pytest.mark.parametrize("name,space,dim", INDEXES)
def test_noalloc_filter_and_deletes(name, space, dim):
    """The delete- and filter-aware beam: an allow mask over internal ids
    (labels divisible by 2), then the same after marking the golden fixture's
    deleted labels."""
    import torch

    g = np.load(os.path.join(GOLDEN, "golden.npz"))
    q = np.ascontiguousarray(g[f"{name}/queries"].astype(np.float32))
    idx = H.Index(space, dim)
    idx.load_index(os.path.join(GOLDEN, f"{name}.bin"))
    allow = np.ascontiguousarray((idx.labels_by_internal_id() % 2 == 0).astype(np.uint8))
    stream = torch.cuda.Stream()
    _status(stream)
    k = 10
    for phase in ("filter", "deleted"):
        if phase == "deleted":
            for lab in g[f"{name}/deleted"]:
                idx.mark_deleted(int(lab))
        for flags in (_capi.EXACT_TIES, 0):
            for ef in (10, 64):
                for a in (allow, None):
                    _same(_noalloc_call(idx, q, k, ef, flags, stream, a), _reference_call(idx, q, k, ef, flags, a))
    assert _status(stream) == 0


def test_noalloc_status_reports_overflow():
    """A filter that rejects every label: the beam accepts every node it
    reaches as a candidate, more than the 512-entry shared-memory candidate
    heap of the tie-exact form holds and more than the list of disallowed
    candidates holds, so the call raises HNSWGPU_STATUS_OVERFLOW.  The word
    keeps it through a later clean call until it is read, and reads clear it."""
    import torch

    g = np.load(os.path.join(GOLDEN, "golden.npz"))
    q = np.ascontiguousarray(g["hnsw_l2_d16/queries"].astype(np.float32))
    idx = H.Index("l2", 16)
    idx.load_index(os.path.join(GOLDEN, "hnsw_l2_d16.bin"))
    assert idx.get_current_count() > 512
    stream = torch.cuda.Stream()
    _status(stream)
    none = np.zeros(idx.get_current_count(), np.uint8)
    lab, dist, cnt = _noalloc_call(idx, q, 10, 32, _capi.EXACT_TIES, stream, none)
    assert np.all(cnt == 0) and np.all(lab == np.iinfo(np.uint64).max)
    _noalloc_call(idx, q, 10, 32, 0, stream)  # a clean call does not clear the bit
    assert _status(stream) & _capi.STATUS_OVERFLOW
    assert _status(stream) == 0


def test_noalloc_rejects_oversized_batches():
    idx = H.Index("l2", 16)
    idx.load_index(os.path.join(GOLDEN, "hnsw_l2_d16.bin"))
    lib = _capi.lib()
    rc = lib.hnswgpu_search_noalloc(idx._h, 16, 1 << 31, 10, 0, 0, None, 16, 16, 16, None)
    assert rc == _capi.ERR_ARG
    assert b"nq must be < 2^31" in lib.hnswgpu_last_error()
    rc = lib.hnswgpu_search_noalloc(idx._h, 16, 4, 1 << 32, 0, 0, None, 16, 16, 16, None)
    assert rc == _capi.ERR_ARG
    assert b"k must be < 2^32" in lib.hnswgpu_last_error()
