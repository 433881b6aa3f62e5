"""Python surface of the serving loop (hnswgpu_server_* in include/hnswgpu.h).

A ``Server`` wraps one GPU ``Index``: requests with their own k, ef, filter,
tie order, precision and learned termination are queued, batched with others
of the same configuration and run while the GPU works on other batches
(continuous batching, admission by shared-memory footprint); see the C header
for the scheduling rules.

``replay`` drives the server natively with an open-loop arrival schedule
(e.g. Poisson) so that latencies at high request rates are not limited by
the Python interpreter.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Optional, Sequence

import numpy as np

from . import _capi
from .index import _PRECISIONS, _input_rows, _ptr


class Server:
    def __init__(self, index, max_inflight: int = 32, max_batch: int = 4096, smem_budget: int = 0):
        index._require()
        self.index = index
        o = _capi.ServerOpts(max_inflight=int(max_inflight), max_batch=int(max_batch), smem_budget=int(smem_budget))
        h = C.c_void_p()
        _capi.check(_capi.lib().hnswgpu_server_create(index._h, C.byref(o), C.byref(h)))
        self._h = h
        self._filters = {}

    def close(self) -> None:
        if self._h:
            _capi.check(_capi.lib().hnswgpu_server_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_filter(self, filter: Callable[[int], bool]) -> int:
        """Register a label filter (evaluated once over all labels); returns its id."""
        labels = self.index.labels_by_internal_id()
        mask = np.fromiter((1 if filter(int(l)) else 0 for l in labels), np.uint8, count=labels.shape[0])
        return self.add_filter_mask(mask)

    def add_filter_mask(self, mask: np.ndarray) -> int:
        mask = np.ascontiguousarray(mask, np.uint8)
        fid = C.c_int32()
        _capi.check(_capi.lib().hnswgpu_server_add_filter(self._h, _ptr(mask), C.byref(fid)))
        return fid.value

    @staticmethod
    def request(k: int = 10, ef: int = 0, filter: int = -1, tie_order: str = "id", learned: bool = False,
                precision: str = "fp32", rerank: int = 0) -> _capi.Request:
        flags = (_capi.EXACT_TIES if tie_order == "reference" else 0) | (_capi.LEARNED_STOP if learned else 0)
        return _capi.Request(k=int(k), ef=int(ef), filter=int(filter), flags=flags,
                             precision=_PRECISIONS[precision], rerank=int(rerank))

    def submit(self, query, **req) -> int:
        q = _input_rows(query)[0]
        t = C.c_uint64()
        r = self.request(**req)
        _capi.check(_capi.lib().hnswgpu_server_submit(self._h, _ptr(q), C.byref(r), C.byref(t)))
        return (t.value, r.k)

    def wait(self, ticket):
        tid, k = ticket
        lab = np.empty(k, np.uint64)
        dist = np.empty(k, np.float32)
        cnt = C.c_int32()
        lat = C.c_double()
        _capi.check(_capi.lib().hnswgpu_server_wait(self._h, tid, _ptr(lab), _ptr(dist), C.byref(cnt), C.byref(lat)))
        return lab[:cnt.value], dist[:cnt.value], lat.value

    def replay(self, queries, requests: Sequence[_capi.Request], arrival_us: np.ndarray):
        """Submit request i at arrival_us[i] (microseconds from the start),
        natively, and collect everything: (labels [n, kmax], dists, counts,
        latency_us)."""
        q = _input_rows(queries)
        n = q.shape[0]
        assert len(requests) == n and len(arrival_us) == n
        reqs = (_capi.Request * n)(*requests)
        kmax = max((r.k for r in requests), default=1)
        arr = np.ascontiguousarray(arrival_us, np.float64)
        lab = np.empty((n, kmax), np.uint64)
        dist = np.empty((n, kmax), np.float32)
        cnt = np.empty(n, np.int32)
        lat = np.empty(n, np.float64)
        _capi.check(_capi.lib().hnswgpu_server_replay(self._h, _ptr(q), n, reqs, _ptr(arr), kmax, _ptr(lab),
                                                      _ptr(dist), _ptr(cnt), _ptr(lat)))
        return lab, dist, cnt, lat

    def stats(self, reset: bool = False) -> dict:
        st = _capi.ServerStats()
        _capi.check(_capi.lib().hnswgpu_server_get_stats(self._h, C.byref(st), int(reset)))
        return {f: getattr(st, f) for f, _ in _capi.ServerStats._fields_}


def poisson_arrivals(n: int, rate_qps: float, seed: int = 0) -> np.ndarray:
    """Arrival times (microseconds) of a Poisson process of this rate."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1e6 / rate_qps, n))
