"""Float64 ground truth for recall and distance-error measurements.

``fp64_topk`` returns each query's exact top-k in float64 arithmetic, on the
GPU: the exact float32 scan (bit-identical to the reference's brute force)
proposes the top k + margin rows, ``hnswgpu_fp64_distances`` re-scores them in
float64, and the k smallest (distance, label) pairs are kept.  A query is
*certified* when no row outside the proposal can belong to the float64
top-k: its float64 k-th distance lies below the proposal's last float32
distance minus a rigorous bound on float32 summation error,
dim * 2^-24 * (|d| + 1) for distances of unit-scale terms.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi


def fp64_distances(index, queries: np.ndarray, labels: np.ndarray) -> np.ndarray:
    """Float64 distances [nq, m] between each query and its row of labels."""
    if hasattr(index, "_sync"):
        index._sync()  # a BFIndex uploads its rows on first use
    index._require()
    q = np.ascontiguousarray(queries, np.float32)
    lab = np.ascontiguousarray(labels, np.uint64)
    out = np.empty(lab.shape, np.float64)
    _capi.check(_capi.lib().hnswgpu_fp64_distances(index._h, q.ctypes.data_as(C.c_void_p), q.shape[0],
                                                   lab.ctypes.data_as(C.c_void_p), lab.shape[1],
                                                   out.ctypes.data_as(C.c_void_p)))
    return out


def fp64_topk(index, queries: np.ndarray, k: int, margin: int = 64):
    """(labels [nq, k], float64 distances [nq, k], certified [nq] bool)."""
    prec = getattr(index, "precision", "fp32")
    index.precision = "fp32"
    try:
        l32, d32 = index.knn_query(queries, k + margin)
    finally:
        index.precision = prec
    d64 = fp64_distances(index, queries, l32)
    order = np.lexsort((l32, d64), axis=1)
    lab = np.take_along_axis(l32, order, 1)[:, :k]
    dk = np.take_along_axis(d64, order, 1)[:, :k]
    dim = queries.shape[1]
    last = d32[:, -1].astype(np.float64)
    bound = dim * 2.0 ** -24 * (np.abs(last) + 1.0)
    certified = dk[:, -1] < last - bound
    return lab, dk, certified
