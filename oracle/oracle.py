"""ctypes wrapper of the CPU oracle (oracle/liboracle.so) -- test infrastructure.

Only tests, the smoke check and the benchmark's CPU-baseline leg use this
module, always as the checker.  The product package never imports it.

``Hnsw.search(mode=REFERENCE)`` reproduces hnswlib 0.9.0's ``searchKnn``
bit-for-bit (heap tie order included); ``mode=CANONICAL`` is the tie-broken
form the CUDA kernel implements.  ``ref_module()`` imports the reference's own
compiled extension from ``oracle/_ref`` when it has been built;
``ref_stopcond()``, ``ref_l2u8()`` and ``ref_multivec()`` load the harnesses
compiled from the reference's headers there (epsilon search, L2SpaceI
indexes, multi-vector search), which the Python bindings cannot reach.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

REFERENCE = 0
CANONICAL = 1
SPACES = {"l2": 0, "ip": 1, "cosine": 1, "l2_uint8": 3}

_lib = None


def build(force: bool = False, ref_dir: str | None = None) -> None:
    """Compile liboracle.so; with `ref_dir` (or the environment variable
    HNSW_REFERENCE_DIR), the hnswlib source tree, also the reference's own
    extension and harnesses into oracle/_ref."""
    ref_dir = ref_dir or os.environ.get("HNSW_REFERENCE_DIR")
    targets = ["oracle"]
    extra = []
    if ref_dir and os.path.isdir(ref_dir):
        targets.append("ref")
        extra = [f"REF={ref_dir}"]
    if force or not os.path.exists(LIB_PATH) or targets != ["oracle"]:
        subprocess.check_call(["make", "-s", "-C", HERE] + targets + extra)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P, U64, I32, F32 = C.c_void_p, C.c_uint64, C.c_int32, C.c_float
        L.orc_last_error.restype = C.c_char_p
        L.orc_distance.restype = F32
        L.orc_distance.argtypes = [C.c_int, P, P, U64]
        L.orc_distances.argtypes = [C.c_int, P, P, U64, U64, P]
        L.orc_normalize.argtypes = [P, P, U64, U64]
        L.orc_hnsw_load.restype = P
        L.orc_hnsw_load.argtypes = [C.c_char_p, C.c_int, U64]
        L.orc_hnsw_free.argtypes = [P]
        L.orc_hnsw_count.restype = U64
        L.orc_hnsw_count.argtypes = [P]
        L.orc_hnsw_num_deleted.restype = U64
        L.orc_hnsw_num_deleted.argtypes = [P]
        L.orc_hnsw_maxM0.restype = U64
        L.orc_hnsw_maxM0.argtypes = [P]
        L.orc_hnsw_maxlevel.restype = C.c_int
        L.orc_hnsw_maxlevel.argtypes = [P]
        L.orc_hnsw_labels.argtypes = [P, P]
        L.orc_hnsw_set_deleted.restype = C.c_int
        L.orc_hnsw_set_deleted.argtypes = [P, U64, C.c_int]
        L.orc_hnsw_search.restype = C.c_int
        L.orc_hnsw_search.argtypes = [P, P, U64, U64, U64, C.c_int, P, P, P, P, P, C.c_int]
        L.orc_hnsw_search_multivector.restype = C.c_int
        L.orc_hnsw_search_multivector.argtypes = [P, P, U64, U64, U64, U64, P, P, P, C.c_int]
        L.orc_hnsw_search_epsilon.restype = C.c_int
        L.orc_hnsw_search_epsilon.argtypes = [P, P, U64, F32, U64, U64, P, P, P, P, C.c_int]
        L.orc_bf_load.restype = P
        L.orc_bf_load.argtypes = [C.c_char_p, C.c_int, U64]
        L.orc_bf_free.argtypes = [P]
        L.orc_bf_count.restype = U64
        L.orc_bf_count.argtypes = [P]
        L.orc_bf_search.restype = C.c_int
        L.orc_bf_search.argtypes = [P, P, U64, U64, P, P, P, P, C.c_int]
        L.orc_bf_matrix.restype = C.c_int
        L.orc_bf_matrix.argtypes = [C.c_int, P, U64, U64, P, U64, U64, P, P, C.c_int]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def distances(space: str, q: np.ndarray, x: np.ndarray) -> np.ndarray:
    """Reference-order distances from one query to every row of ``x``."""
    q = np.ascontiguousarray(q, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty(x.shape[0], np.float32)
    lib().orc_distances(SPACES[space], _ptr(q), _ptr(x), x.shape[0], x.shape[1], _ptr(out))
    return out


def normalize(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(np.atleast_2d(x), np.float32)
    out = np.empty_like(x)
    lib().orc_normalize(_ptr(x), _ptr(out), x.shape[0], x.shape[1])
    return out


class Hnsw:
    """A reference-format HNSW index file loaded by the oracle."""

    def __init__(self, path: str, space: str, dim: int):
        self.space, self.dim = space, dim
        self._h = lib().orc_hnsw_load(path.encode(), SPACES[space], dim)
        if not self._h:
            raise RuntimeError(lib().orc_last_error().decode())

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_hnsw_free(self._h)
            self._h = None

    @property
    def count(self) -> int:
        return lib().orc_hnsw_count(self._h)

    @property
    def num_deleted(self) -> int:
        return lib().orc_hnsw_num_deleted(self._h)

    def labels(self) -> np.ndarray:
        out = np.empty(self.count, np.uint64)
        lib().orc_hnsw_labels(self._h, _ptr(out))
        return out

    def set_deleted(self, label: int, flag: bool) -> int:
        return lib().orc_hnsw_set_deleted(self._h, int(label), int(bool(flag)))

    def search(self, q, k, ef, mode=REFERENCE, allow=None, trace=False, nthreads=0):
        q = np.ascontiguousarray(np.atleast_2d(q), np.float32)
        if self.space == "cosine":
            q = normalize(q)
        nq = q.shape[0]
        labels = np.empty((nq, k), np.uint64)
        dists = np.empty((nq, k), np.float32)
        counts = np.empty(nq, np.int32)
        tr = np.zeros((nq, 7), np.int64) if trace else None
        if allow is not None:
            allow = np.ascontiguousarray(allow, np.uint8)
        rc = lib().orc_hnsw_search(self._h, _ptr(q), nq, k, ef, mode, _ptr(allow), _ptr(labels), _ptr(dists),
                                   _ptr(counts), _ptr(tr), nthreads)
        if rc != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return (labels, dists, counts, tr) if trace else (labels, dists, counts)

    def search_multivector(self, q, num_docs, ef_collection, cap, nthreads=0):
        """searchStopConditionClosest with MultiVectorSearchStopCondition on a
        multi-vector index (a uint32 document id after each vector): (ids,
        dists) of `cap` slots in the reference's result order (internal ids),
        counts (-1 where the result is longer than cap)."""
        q = np.ascontiguousarray(np.atleast_2d(q), np.float32)
        nq = q.shape[0]
        ids = np.empty((nq, cap), np.uint64)
        dists = np.empty((nq, cap), np.float32)
        counts = np.empty(nq, np.int32)
        rc = lib().orc_hnsw_search_multivector(self._h, _ptr(q), nq, int(num_docs), int(ef_collection), int(cap),
                                               _ptr(ids), _ptr(dists), _ptr(counts), nthreads)
        if rc != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return ids, dists, counts

    def search_epsilon(self, q, epsilon, min_candidates, max_candidates, allow=None, nthreads=0):
        """searchStopConditionClosest with EpsilonSearchStopCondition(epsilon,
        min_candidates, max_candidates) per query: (ids, dists) of
        max_candidates slots in the reference's result order, counts.  As in
        the reference, the ids are internal ids, not labels."""
        q = np.ascontiguousarray(np.atleast_2d(q), np.float32)
        nq, m = q.shape[0], int(max_candidates)
        labels = np.empty((nq, m), np.uint64)
        dists = np.empty((nq, m), np.float32)
        counts = np.empty(nq, np.int32)
        if allow is not None:
            allow = np.ascontiguousarray(allow, np.uint8)
        rc = lib().orc_hnsw_search_epsilon(self._h, _ptr(q), nq, float(epsilon), int(min_candidates), m, _ptr(allow),
                                           _ptr(labels), _ptr(dists), _ptr(counts), nthreads)
        if rc != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return labels, dists, counts


class Bf:
    """A reference-format brute-force index file loaded by the oracle."""

    def __init__(self, path: str, space: str, dim: int):
        self.space, self.dim = space, dim
        self._h = lib().orc_bf_load(path.encode(), SPACES[space], dim)
        if not self._h:
            raise RuntimeError(lib().orc_last_error().decode())

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_bf_free(self._h)
            self._h = None

    def search(self, q, k, allow=None, nthreads=0):
        q = np.ascontiguousarray(np.atleast_2d(q), np.float32)
        if self.space == "cosine":
            q = normalize(q)
        nq = q.shape[0]
        labels = np.empty((nq, k), np.uint64)
        dists = np.empty((nq, k), np.float32)
        counts = np.empty(nq, np.int32)
        if allow is not None:
            allow = np.ascontiguousarray(allow, np.uint8)
        lib().orc_bf_search(self._h, _ptr(q), nq, k, _ptr(allow), _ptr(labels), _ptr(dists), _ptr(counts), nthreads)
        return labels, dists, counts


def bf_matrix(space: str, x: np.ndarray, q: np.ndarray, k: int, nthreads: int = 0):
    """Exact top-k rows of ``x`` for each query, in reference arithmetic."""
    x = np.ascontiguousarray(x, np.float32)
    q = np.ascontiguousarray(np.atleast_2d(q), np.float32)
    labels = np.empty((q.shape[0], k), np.uint64)
    dists = np.empty((q.shape[0], k), np.float32)
    lib().orc_bf_matrix(SPACES[space], _ptr(x), x.shape[0], x.shape[1], _ptr(q), q.shape[0], k, _ptr(labels),
                        _ptr(dists), nthreads)
    return labels, dists


def ref_stopcond():
    """ctypes handle of oracle/_ref/libref_stopcond.so (the reference's own
    searchStopConditionClosest), or None where it was not built."""
    path = os.path.join(HERE, "_ref", "libref_stopcond.so")
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    P, U64 = C.c_void_p, C.c_uint64
    L.ref_epsilon_search.restype = C.c_int
    L.ref_epsilon_search.argtypes = [C.c_char_p, C.c_int, U64, P, U64, P, U64, P, U64, C.c_float, U64, U64, P, P, P]
    return L


def ref_epsilon_search(path, space, q, epsilon, min_candidates, max_candidates, deleted=(), allow_by_label=None):
    """Run the reference's epsilon search (needs ref_stopcond())."""
    L = ref_stopcond()
    q = np.ascontiguousarray(np.atleast_2d(q), np.float32)
    nq, dim, m = q.shape[0], q.shape[1], int(max_candidates)
    dele = np.ascontiguousarray(np.asarray(deleted, np.uint64))
    labels = np.empty((nq, m), np.uint64)
    dists = np.empty((nq, m), np.float32)
    counts = np.empty(nq, np.int32)
    allow = None if allow_by_label is None else np.ascontiguousarray(allow_by_label, np.uint8)
    rc = L.ref_epsilon_search(str(path).encode(), SPACES[space], dim, _ptr(dele), dele.size, _ptr(allow),
                              0 if allow is None else allow.size, _ptr(q), nq, float(epsilon), int(min_candidates), m,
                              _ptr(labels), _ptr(dists), _ptr(counts))
    if rc != 0:
        raise RuntimeError("reference epsilon search failed")
    return labels, dists, counts


def ref_multivec():
    """ctypes handle of oracle/_ref/libref_multivec.so (the reference's
    multi-vector search), or None where it was not built."""
    path = os.path.join(HERE, "_ref", "libref_multivec.so")
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    P, U64 = C.c_void_p, C.c_uint64
    L.ref_mv_build.restype = C.c_int
    L.ref_mv_build.argtypes = [C.c_char_p, C.c_int, P, P, P, U64, U64, U64, U64, U64]
    L.ref_mv_search.restype = C.c_int
    L.ref_mv_search.argtypes = [C.c_char_p, C.c_int, U64, P, U64, U64, U64, U64, P, P, P]
    return L


def ref_mv_build(path, space, x, docs, labels, M=16, efc=100, seed=100):
    x = np.ascontiguousarray(x, np.float32)
    d = np.ascontiguousarray(docs, np.uint32)
    lab = np.ascontiguousarray(labels, np.uint64)
    if ref_multivec().ref_mv_build(str(path).encode(), SPACES[space], _ptr(x), _ptr(d), _ptr(lab), x.shape[0],
                                   x.shape[1], M, efc, seed) != 0:
        raise RuntimeError("reference multi-vector build failed")


def ref_mv_search(path, space, q, num_docs, ef_collection, cap):
    q = np.ascontiguousarray(np.atleast_2d(q), np.float32)
    nq, dim = q.shape
    ids = np.empty((nq, cap), np.uint64)
    dists = np.empty((nq, cap), np.float32)
    counts = np.empty(nq, np.int32)
    if ref_multivec().ref_mv_search(str(path).encode(), SPACES[space], dim, _ptr(q), nq, int(num_docs),
                                    int(ef_collection), int(cap), _ptr(ids), _ptr(dists), _ptr(counts)) != 0:
        raise RuntimeError("reference multi-vector search failed")
    return ids, dists, counts


def ref_l2u8():
    """ctypes handle of oracle/_ref/libref_l2u8.so (the reference's
    HierarchicalNSW<int> over L2SpaceI), or None where it was not built."""
    path = os.path.join(HERE, "_ref", "libref_l2u8.so")
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    P, U64 = C.c_void_p, C.c_uint64
    L.ref_l2u8_build.restype = C.c_int
    L.ref_l2u8_build.argtypes = [C.c_char_p, P, P, U64, U64, U64, U64, U64]
    L.ref_l2u8_search.restype = C.c_int
    L.ref_l2u8_search.argtypes = [C.c_char_p, U64, P, U64, U64, U64, P, U64, P, U64, P, P, P]
    return L


def ref_l2u8_build(path, x_u8, labels, M=16, efc=100, seed=100):
    """Build and save a uint8 L2SpaceI index with the reference's addPoint."""
    x = np.ascontiguousarray(x_u8, np.uint8)
    lab = np.ascontiguousarray(labels, np.uint64)
    if ref_l2u8().ref_l2u8_build(str(path).encode(), _ptr(x), _ptr(lab), x.shape[0], x.shape[1], M, efc, seed) != 0:
        raise RuntimeError("reference L2SpaceI build failed")


def ref_l2u8_search(path, q_u8, k, ef, deleted=(), allow_by_label=None):
    """The reference's searchKnn on a uint8 index: (labels, int32 dists, counts)."""
    q = np.ascontiguousarray(np.atleast_2d(q_u8), np.uint8)
    nq, dim = q.shape
    dele = np.ascontiguousarray(np.asarray(deleted, np.uint64))
    allow = None if allow_by_label is None else np.ascontiguousarray(allow_by_label, np.uint8)
    labels = np.empty((nq, k), np.uint64)
    dists = np.empty((nq, k), np.int32)
    counts = np.empty(nq, np.int32)
    rc = ref_l2u8().ref_l2u8_search(str(path).encode(), dim, _ptr(q), nq, k, ef, _ptr(dele), dele.size, _ptr(allow),
                                    0 if allow is None else allow.size, _ptr(labels), _ptr(dists), _ptr(counts))
    if rc != 0:
        raise RuntimeError("reference L2SpaceI search failed")
    return labels, dists, counts


def ref_module():
    """The reference's compiled ``hnswlib`` extension from oracle/_ref, or None."""
    if not os.path.isdir(REF_DIR):
        return None
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    try:
        import hnswlib  # noqa: F401  (the reference build, not this project)
    except ImportError:
        return None
    return sys.modules["hnswlib"]
