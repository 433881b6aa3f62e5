"""Python surface of the GPU query path, shaped like hnswlib's own module.

``Index`` and ``BFIndex`` keep the names, arguments, return types and error
messages of the reference's pybind11 classes (python_bindings/bindings.cpp:
``Index`` :145-723 / module table :933-999, ``BFIndex`` :725-930 / :1011-1033)
for the query path: ``load_index``, ``knn_query``, ``set_ef`` / ``ef``,
``mark_deleted`` / ``unmark_deleted`` and the metadata accessors.  Searches run
on the GPU through libhnswgpu.so; ``num_threads`` is accepted for signature
compatibility and has no effect.

Index construction (``init_index`` / ``add_items`` / ``save_index`` on an HNSW
``Index``) stays with the reference library: build and save there, load here.
``BFIndex`` has no graph, so ``init_index`` / ``add_items`` work directly.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Callable, Optional

import numpy as np

from . import _capi

_SPACES = {"l2": _capi.SPACE_L2, "ip": _capi.SPACE_IP, "cosine": _capi.SPACE_COSINE}
# An extension for the C++ API's HierarchicalNSW<int> over L2SpaceI: an index
# of uint8 vectors (built with hnswlib's C++ API), queried with rows holding
# uint8 values; distances are the reference's integers, as float32.
_HNSW_ONLY_SPACES = {"l2_uint8": _capi.SPACE_L2_UINT8}
_PRECISIONS = {"fp32": _capi.PREC_FP32, "bf16": _capi.PREC_BF16, "fp8": _capi.PREC_FP8}


def _input_rows(data) -> np.ndarray:
    """The binding's forcecast + shape rules (bindings.cpp:97-112, 617)."""
    a = np.ascontiguousarray(np.asarray(data), dtype=np.float32)
    if a.ndim == 1:
        return a.reshape(1, -1)
    if a.ndim != 2:
        raise RuntimeError(
            f"Input vector data wrong shape. Number of dimensions {a.ndim}. Data must be a 1D or 2D array.")
    return a


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class RegisteredFilter:
    """A filter evaluated once and kept on the GPU (Index.register_filter);
    ``release()`` frees it."""

    def __init__(self, index, fid: int):
        self.index, self.id = index, fid

    def release(self) -> None:
        if self.id and self.index._h:
            _capi.check(_capi.lib().hnswgpu_filter_destroy(self.index._h, self.id))
        self.id = 0


class _GpuIndex:
    _extra_spaces: dict = {}

    def __init__(self, space: str, dim: int):
        if space not in _SPACES and space not in self._extra_spaces:
            raise RuntimeError("Space name must be one of l2, ip, or cosine.")
        self.space = space
        self.dim = int(dim)
        self.num_threads = -1
        self.device = 0
        self._h = None
        self._labels = None

    # -- lifecycle
    def _free(self):
        if self._h:
            _capi.lib().hnswgpu_free(self._h)
            self._h = None
        self._labels = None

    def __del__(self):
        try:
            self._free()
        except Exception:
            pass

    def set_num_threads(self, num_threads: int) -> None:
        self.num_threads = num_threads

    def _info(self) -> _capi.Info:
        info = _capi.Info()
        _capi.check(_capi.lib().hnswgpu_get_info(self._h, C.byref(info)))
        return info

    def _require(self):
        if not self._h:
            raise RuntimeError("Index not loaded: call load_index first")

    def labels_by_internal_id(self) -> np.ndarray:
        """External labels in internal-id order (positions used by filters)."""
        self._require()
        if self._labels is None:
            n = self._info().count
            out = np.empty(n, np.uint64)
            _capi.check(_capi.lib().hnswgpu_get_labels(self._h, _ptr(out)))
            self._labels = out
        return self._labels

    def _allow_mask(self, filter: Optional[Callable[[int], bool]]) -> Optional[np.ndarray]:
        """Evaluate the filter functor for every label, at every call (the
        reference calls it per candidate during the search,
        bindings.cpp:83-94, so a callable whose answers change is honoured);
        a filter registered with ``register_filter`` is not re-evaluated."""
        if filter is None or isinstance(filter, RegisteredFilter):
            return None
        labels = self.labels_by_internal_id()
        return np.fromiter((1 if filter(int(l)) else 0 for l in labels), dtype=np.uint8, count=labels.shape[0])

    def register_filter(self, filter: Callable[[int], bool]) -> "RegisteredFilter":
        """Evaluate `filter` once over the index's labels and keep the answers
        on the GPU: pass the returned object as ``filter=`` to search without
        re-evaluating the callable or copying a mask (an extension; the
        reference has no such form)."""
        self._require()
        labels = self.labels_by_internal_id()
        mask = np.fromiter((1 if filter(int(l)) else 0 for l in labels), dtype=np.uint8, count=labels.shape[0])
        fid = _capi.U32(0)
        _capi.check(_capi.lib().hnswgpu_filter_create(self._h, _ptr(mask), C.byref(fid)))
        return RegisteredFilter(self, fid.value)

    def _filter_id(self, filter) -> int:
        if not isinstance(filter, RegisteredFilter):
            return 0
        if filter.index is not self or not filter.id:
            raise RuntimeError("the registered filter belongs to another index or was released")
        return filter.id

    def _queries(self, data, k: int):
        self._require()
        q = _input_rows(data)
        if q.shape[1] != self.dim:
            raise RuntimeError("Wrong dimensionality of the vectors")
        k = int(k)
        if k <= 0:
            raise RuntimeError("k must be positive")
        return q, k

    def _search(self, data, k: int, filter, ef: int = 0, trace: bool = False, exact_ties: bool = False,
                precision: str = "fp32", rerank: int = 0, flags: int = 0):
        q, k = self._queries(data, k)
        nq = q.shape[0]
        labels = np.empty((nq, k), np.uint64)
        dists = np.empty((nq, k), np.float32)
        counts = np.empty(nq, np.int32)
        opts = _capi.SearchOpts()
        opts.ef = int(ef)
        opts.precision = _PRECISIONS[precision]
        opts.rerank = int(rerank)
        opts.flags = int(flags)
        if exact_ties and opts.precision == _capi.PREC_FP32 and not flags & _capi.LEARNED_STOP:
            opts.flags |= _capi.EXACT_TIES
            if exact_ties == "replay":
                opts.flags |= _capi.REPLAY_ALL
        mask = self._allow_mask(filter)
        opts.allow = mask.ctypes.data if mask is not None else None
        opts.filter = self._filter_id(filter)
        tr = None
        if trace:
            tr = np.zeros((nq, 4), np.uint32)
            opts.flags |= _capi.TRACE
            opts.trace = tr.ctypes.data
        _capi.check(_capi.lib().hnswgpu_search(self._h, _ptr(q), nq, k, C.byref(opts), _ptr(labels), _ptr(dists),
                                               _ptr(counts)))
        return labels, dists, counts, tr

    def get_current_count(self) -> int:
        return self._info().count if self._h else 0

    def get_max_elements(self) -> int:
        if getattr(self, "_max_elements", None) is not None:
            return self._max_elements
        return self._info().max_elements if self._h else 0

    def get_ids_list(self):
        return [int(x) for x in self.labels_by_internal_id()]

    @property
    def element_count(self) -> int:
        return self.get_current_count()

    @property
    def max_elements(self) -> int:
        return self.get_max_elements()

    def get_status(self) -> int:
        """OR of kernel status bits since the last call (STATUS_OVERFLOW:
        a filtered search overflowed its candidate list; STATUS_TIMEOUT)."""
        self._require()
        v = C.c_uint32()
        _capi.check(_capi.lib().hnswgpu_get_status(self._h, C.byref(v)))
        return int(v.value)

    def device_bytes(self) -> int:
        return self._info().device_bytes if self._h else 0


class Index(_GpuIndex):
    """GPU-backed ``hnswlib.Index`` (query path)."""

    _extra_spaces = _HNSW_ONLY_SPACES

    def __init__(self, space=None, dim=None, params: Optional[dict] = None, index: Optional["Index"] = None):
        """Index(space, dim), or, as the reference's other constructors
        (bindings.cpp:937-939), Index(params) from a getIndexParams dict and
        Index(index) as a copy of another Index."""
        if isinstance(space, dict) or params is not None:
            self.__setstate__((params if params is not None else space,))
            return
        if isinstance(space, Index) or index is not None:
            self.__setstate__((index if index is not None else space).__getstate__())
            return
        super().__init__(space, dim)
        self._default_ef = 10
        self._source = None       # file the index was loaded from
        self._state_bytes = None  # or its bytes (an index made from a pickled state)
        self._marks = {}          # label -> deleted, for marks changed since the load
        self._max_elements = None  # set by resize_index
        # "reference": equal distances resolve exactly as hnswlib's heaps do
        # (results identical to searchKnn); "id": ties break by internal id
        # (identical except where distances tie exactly; faster).
        self.tie_order = "reference"
        # traversal copy: "fp32" (the reference's search), or "bf16" / "fp8"
        # (approximate beam over a low-precision copy, then the best `rerank`
        # candidates, default ef, re-ranked with exact float32 distances)
        self.precision = "fp32"
        self.rerank = 0
        # learned early termination: when True (and a model is set with
        # set_termination_model), knn_query ends each query's beam as soon as
        # the network judges its top-k final; ef is the cap (id tie order)
        self.learned_stop = False
        self._term_model = None

    def __repr__(self):
        return f"<hnsw_rabitq_b200.Index(space='{self.space}', dim={self.dim})>"

    def load_index(self, path_to_index: str, max_elements: int = 0, allow_replace_deleted: bool = False) -> None:
        """Load a file written by hnswlib's ``save_index`` onto the GPU
        (bindings.cpp:230-238 -> HierarchicalNSW::loadIndex).  ef is reset to
        10 as the reference does (hnswalg.h:794)."""
        self._free()
        h = C.c_void_p()
        space_id = _SPACES.get(self.space, self._extra_spaces.get(self.space))
        _capi.check(_capi.lib().hnswgpu_load_hnsw(str(path_to_index).encode(), space_id, self.dim,
                                                  int(max_elements), self.device, C.byref(h)))
        self._h = h
        self._default_ef = 10
        # the file the index came from, and the delete marks changed since:
        # pickling and save_index rebuild the reference's state from them
        self._source = os.path.abspath(str(path_to_index))
        self._marks = {}
        self._max_elements = None

    # -- the reference's pickled state and saved file (bindings.cpp:465-529, 1001-1008)
    def _file_bytes(self) -> bytes:
        from . import pickling
        self._require()
        if self._source is None:
            buf = self._state_bytes
        else:
            with open(self._source, "rb") as f:
                buf = f.read()
        dele = {lab for lab, m in self._marks.items() if m}
        keep = {lab for lab, m in self._marks.items() if not m}
        buf = pickling.set_delete_marks(buf, dele, keep)
        if self._max_elements is not None:
            buf = pickling.with_max_elements(buf, self._max_elements)
        return buf

    def get_items(self, ids=None, return_type: str = "numpy"):
        """Stored vectors by label (bindings.cpp:307-338 -> getDataByLabel):
        a numpy array or a list of lists; no ids gives none.  Read from the
        index's saved form (for the cosine space these are the normalised
        vectors the reference stores)."""
        from . import pickling
        if return_type not in ("numpy", "list"):
            raise ValueError('return_type should be "numpy" or "list"')
        ids = [] if ids is None else np.asarray(ids)
        if isinstance(ids, np.ndarray) and ids.ndim == 0:
            raise ValueError("get_items accepts a list of indices and returns a list of vectors")
        self._require()
        elem = np.uint8 if self.space == "l2_uint8" else np.float32
        where = {int(v): i for i, v in enumerate(self.labels_by_internal_id().tolist())}
        rows = np.empty((len(ids), self.dim), np.float32)
        with pickling.RecordReader(self._source if self._source is not None else self._state_bytes) as rd:
            for r, lab in enumerate(np.asarray(ids).reshape(-1).tolist()):
                i = where.get(int(lab))
                if i is None:
                    raise RuntimeError("Label not found")
                # a mark changed in this session overrides the file's
                dead = self._marks[int(lab)] if int(lab) in self._marks else rd.deleted(i)
                if dead:
                    raise RuntimeError("Label not found")
                rows[r] = rd.vector(i, self.dim, elem)
        return rows.tolist() if return_type == "list" else rows

    def index_file_size(self) -> int:
        """HierarchicalNSW::indexFileSize (hnswalg.h:658-683): bytes save_index writes."""
        self._require()
        if self._source is not None:
            return os.path.getsize(self._source)
        return len(self._state_bytes)

    def resize_index(self, new_size: int) -> None:
        """resizeIndex (hnswalg.h:633-656): the capacity recorded with the
        index (max_elements); the GPU index itself holds exactly its elements."""
        self._require()
        if int(new_size) < self.get_current_count():
            raise RuntimeError("Cannot resize, max element is less than the current number of elements")
        self._max_elements = int(new_size)

    def save_index(self, path: str) -> None:
        """HierarchicalNSW::saveIndex (hnswalg.h:685-712): the loaded index,
        with the delete marks made since, in the reference's file layout."""
        buf = self._file_bytes()
        with open(path, "wb") as f:
            f.write(buf)

    def __getstate__(self):
        """The reference's pickled state: (getIndexParams() dict,)."""
        from . import pickling
        if not self._h:
            return ({"ser_version": pickling.SER_VERSION, "space": self.space, "dim": self.dim,
                     "index_inited": False, "ep_added": False, "normalize": self.space == "cosine",
                     "num_threads": self.num_threads, "seed": 100, "ef": self._default_ef},)
        return (pickling.file_bytes_to_state(self._file_bytes(), self.space, self.dim, self.ef, self.num_threads),)

    def __setstate__(self, state):
        """createFromParams (bindings.cpp:485-519): also accepts the state of
        a reference hnswlib.Index (``ref_index.__getstate__()``)."""
        from . import pickling
        if not isinstance(state, tuple) or len(state) != 1:
            raise RuntimeError("Invalid state!")
        d = state[0]
        if int(d["ser_version"]) > pickling.SER_VERSION:
            raise RuntimeError("Invalid serialization version!")
        Index.__init__(self, d["space"], int(d["dim"]))
        self.num_threads = int(d.get("num_threads", -1))
        if not d.get("index_inited", False):
            self._default_ef = int(d.get("ef", 10))
            return
        # the state's index image goes to the GPU loader straight from memory;
        # a later pickle or save_index rebuilds from the same bytes
        buf = pickling.state_to_file_bytes(d)
        self._free()
        h = C.c_void_p()
        space_id = _SPACES.get(self.space, self._extra_spaces.get(self.space))
        cbuf = C.c_char_p(buf)
        _capi.check(_capi.lib().hnswgpu_load_hnsw_buffer(C.cast(cbuf, C.c_void_p), len(buf), space_id, self.dim, 0,
                                                         self.device, C.byref(h)))
        self._h = h
        self._state_bytes = buf
        self._source = None
        self._marks = {}
        self._max_elements = None
        self.set_ef(int(d["ef"]))

    @classmethod
    def from_params(cls, d: dict) -> "Index":
        """Index from a getIndexParams dict (e.g. a reference hnswlib.Index's
        ``__getstate__()[0]``): its index goes straight to the GPU."""
        obj = cls.__new__(cls)
        obj.__setstate__((d,))
        return obj

    def init_index(self, *args, **kwargs):
        raise NotImplementedError(
            "graph construction is not part of the GPU query path: build the index with hnswlib "
            "(init_index/add_items/save_index) and load the saved file with load_index")

    def add_items(self, *args, **kwargs):
        self.init_index()

    # -- ef
    def set_ef(self, ef: int) -> None:
        self._default_ef = int(ef)
        if self._h:
            _capi.check(_capi.lib().hnswgpu_set_ef(self._h, int(ef)))

    @property
    def ef(self) -> int:
        return self._info().ef if self._h else self._default_ef

    @ef.setter
    def ef(self, value: int) -> None:
        self.set_ef(value)

    @property
    def M(self) -> int:
        return self._info().M if self._h else 0

    @property
    def ef_construction(self) -> int:
        return self._info().ef_construction if self._h else 0

    # -- deletes
    def mark_deleted(self, label: int) -> None:
        self._require()
        _capi.check(_capi.lib().hnswgpu_mark_deleted(self._h, int(label)))
        self._marks[int(label)] = True

    def unmark_deleted(self, label: int) -> None:
        self._require()
        _capi.check(_capi.lib().hnswgpu_unmark_deleted(self._h, int(label)))
        self._marks[int(label)] = False

    # -- learned early termination
    def set_termination_model(self, model) -> None:
        """Install a trained ``learned.TerminationModel`` (or None to remove
        it) on the GPU index."""
        self._require()
        if model is None:
            _capi.check(_capi.lib().hnswgpu_set_termination_model(self._h, None, 0, 0.0))
            self._term_model = None
            return
        p = np.ascontiguousarray(model.params, dtype=np.float32)
        if p.shape != (_capi.TERM_PARAMS,):
            raise ValueError(f"termination parameters must have shape ({_capi.TERM_PARAMS},)")
        _capi.check(_capi.lib().hnswgpu_set_termination_model(self._h, _ptr(p), int(model.period),
                                                              float(model.threshold)))
        self._term_model = model

    def _flags(self, learned: Optional[bool]) -> int:
        use = self.learned_stop if learned is None else learned
        return _capi.LEARNED_STOP if use else 0

    def search_checkpoints(self, data, k: int, ef: int = 0, period: int = 4, max_ckpt: int = 128,
                           precision: Optional[str] = None, rerank: Optional[int] = None,
                           ids_width: int = 0, dists: bool = False):
        """The id-tie-order search, recording at every checkpoint (every
        `period` level-0 expansions, at the first state where no waiting
        candidate is closer than the k-th result) the termination features
        and the internal ids of the first `ids_width` (default k) beam
        entries.  Returns a dict with feat [nq, max_ckpt, TERM_FEATURES], ids
        [nq, max_ckpt, W] (uint32, 0xffffffff = none), nckpt [nq], labels,
        dists, counts; with dists=True also ckpt_dists [nq, max_ckpt, W],
        the float32 distances of those entries (+inf = none)."""
        q, k = self._queries(data, k)
        nq = q.shape[0]
        w = int(ids_width) or k
        out = dict(feat=np.zeros((nq, max_ckpt, _capi.TERM_FEATURES), np.float32),
                   ids=np.full((nq, max_ckpt, w), 0xffffffff, np.uint32), nckpt=np.zeros(nq, np.uint32),
                   labels=np.empty((nq, k), np.uint64), dists=np.empty((nq, k), np.float32),
                   counts=np.empty(nq, np.int32))
        if dists:
            out["ckpt_dists"] = np.full((nq, max_ckpt, w), np.inf, np.float32)
        opts = _capi.SearchOpts()
        opts.ef = int(ef)
        opts.precision = _PRECISIONS[precision or self.precision]
        opts.rerank = int(self.rerank if rerank is None else rerank)
        _capi.check(_capi.lib().hnswgpu_search_checkpoints(
            self._h, _ptr(q), nq, k, C.byref(opts), int(period), int(max_ckpt), int(ids_width), _ptr(out["feat"]),
            _ptr(out["ids"]), _ptr(out["ckpt_dists"]) if dists else None, _ptr(out["nckpt"]), _ptr(out["labels"]),
            _ptr(out["dists"]), _ptr(out["counts"])))
        return out

    def search_epsilon(self, data, epsilon: float, min_candidates: int, max_candidates: int,
                       filter: Optional[Callable[[int], bool]] = None):
        """The C++ API's searchStopConditionClosest with an
        EpsilonSearchStopCondition(epsilon, min_candidates, max_candidates)
        (hnswalg.h:1326-1377), per query: (ids uint64 [N, max_candidates],
        distances float32 [N, max_candidates], counts int32 [N]), closest
        first in the reference's result order.  As in the reference, the ids
        are internal ids (labels_by_internal_id() maps them to labels)."""
        q, _ = self._queries(data, 1)
        nq, m = q.shape[0], int(max_candidates)
        if m <= 0 or int(min_candidates) < 0 or int(min_candidates) > m:
            raise RuntimeError("need 0 < max_candidates and 0 <= min_candidates <= max_candidates")
        ids = np.empty((nq, m), np.uint64)
        dists = np.empty((nq, m), np.float32)
        counts = np.empty(nq, np.int32)
        opts = _capi.SearchOpts()
        mask = self._allow_mask(filter)
        opts.allow = mask.ctypes.data if mask is not None else None
        _capi.check(_capi.lib().hnswgpu_search_epsilon(self._h, _ptr(q), nq, float(epsilon), int(min_candidates), m,
                                                       C.byref(opts), _ptr(ids), _ptr(dists), _ptr(counts)))
        return ids, dists, counts

    def load_multivector_index(self, path_to_index: str, max_elements: int = 0) -> None:
        """Load a multi-vector index: a HierarchicalNSW that the C++ API built
        over a MultiVectorL2Space (hnswlib/stop_condition.h:7-76), whose
        elements carry a 32-bit document id after the vector (L2 only)."""
        if self.space != "l2":
            raise RuntimeError("multi-vector indexes use the l2 space")
        self._free()
        h = C.c_void_p()
        _capi.check(_capi.lib().hnswgpu_load_hnsw_multivector(str(path_to_index).encode(), self.dim,
                                                              int(max_elements), self.device, C.byref(h)))
        self._h = h
        self._default_ef = 10
        self._source = os.path.abspath(str(path_to_index))
        self._marks = {}
        self._max_elements = None

    def search_multivector(self, data, num_docs: int, ef_collection: int, cap: int = 1024):
        """The C++ API's searchStopConditionClosest with a
        MultiVectorSearchStopCondition(space, num_docs, ef_collection)
        (hnswalg.h:1326-1377, stop_condition.h:146-216) on an index loaded by
        load_multivector_index: per query, the elements of the num_docs
        nearest documents in the reference's result order, (ids uint64 [N,
        cap], distances float32 [N, cap], counts int32 [N]); as in the
        reference the ids are internal ids; a count of -1 means the result
        has more than `cap` elements (or outgrew the kernel's heaps)."""
        q, _ = self._queries(data, 1)
        nq, cap = q.shape[0], int(cap)
        ids = np.empty((nq, cap), np.uint64)
        dists = np.empty((nq, cap), np.float32)
        counts = np.empty(nq, np.int32)
        _capi.check(_capi.lib().hnswgpu_search_multivector(self._h, _ptr(q), nq, int(num_docs), int(ef_collection),
                                                           cap, _ptr(ids), _ptr(dists), _ptr(counts)))
        return ids, dists, counts

    def knn_query_exact(self, data, k: int = 1, filter: Optional[Callable[[int], bool]] = None):
        """Exact k-NN by an exhaustive GPU scan of the index's vectors (the
        ground truth of recall measurements): (labels, distances)."""
        labels, dists, counts, _ = self._search(data, k, filter, flags=_capi.EXACT_SCAN)
        return labels, dists

    # -- search
    def knn_query(self, data, k: int = 1, num_threads: int = -1, filter: Optional[Callable[[int], bool]] = None):
        """(labels uint64 [N, k], distances float32 [N, k]), closest first
        (bindings.cpp:612-697).  Raises RuntimeError when a query has fewer
        than k results, with the reference's message."""
        labels, dists, counts, _ = self._search(data, k, filter, exact_ties=self.tie_order == "reference",
                                                precision=self.precision, rerank=self.rerank,
                                                flags=self._flags(None))
        if counts.size and counts.min() < k:
            raise RuntimeError(
                "Cannot return the results in a contiguous 2D array. Probably ef or M is too small")
        return labels, dists

    def knn_query_traced(self, data, k: int = 1, filter=None, ef: int = 0, tie_order: Optional[str] = None,
                         precision: Optional[str] = None, rerank: Optional[int] = None,
                         learned: Optional[bool] = None):
        """knn_query plus per-query work counters [upper link lists read,
        upper distances, level-0 expansions, level-0 distances] and counts;
        no exception for short results.  tie_order "replay" gives the
        "reference" results by replaying the reference's heaps for every query
        in one pass (the default reference order replays only the queries whose
        id-order run met a steering tie)."""
        order = tie_order or self.tie_order
        if order not in ("reference", "id", "replay"):
            raise ValueError("tie_order must be 'reference', 'id' or 'replay'")
        prec = precision or self.precision
        rr = self.rerank if rerank is None else rerank
        exact = "replay" if order == "replay" else order == "reference"
        return self._search(data, k, filter, ef=ef, trace=True, exact_ties=exact, precision=prec,
                            rerank=rr, flags=self._flags(learned))


class BFIndex(_GpuIndex):
    """GPU-backed ``hnswlib.BFIndex``."""

    def __init__(self, space: str, dim: int):
        super().__init__(space, dim)
        self._rows = None
        self._row_labels = None
        self._maxel = 0
        self._dirty = False
        self._source = None  # the file a loaded index came from
        self.cur_l = 0
        # "fp32": the reference's exact scan; "bf16" / "fp8": tensor-core scores
        # over a low-precision copy, the best `rerank` candidates (default
        # 4 k, at most 1024) re-ranked with exact float32 distances
        self.precision = "fp32"
        self.rerank = 0

    def __repr__(self):
        return f"<hnsw_rabitq_b200.BFIndex(space='{self.space}', dim={self.dim})>"

    def init_index(self, max_elements: int) -> None:
        if self._rows is not None or self._h:
            raise RuntimeError("The index is already initiated.")
        self._maxel = int(max_elements)
        self._rows = np.empty((0, self.dim), np.float32)
        self._row_labels = np.empty(0, np.uint64)
        self._dirty = True
        self.cur_l = 0

    def add_items(self, data, ids=None) -> None:
        """BruteforceSearch::addPoint per row (bruteforce.h:64-83): a known
        label overwrites its row in place, a new label is appended."""
        if self._rows is None:
            if self._h:
                self._pull_rows()
            else:
                raise RuntimeError("Index not initialised: call init_index first")
        x = _input_rows(data)
        if x.shape[1] != self.dim:
            raise RuntimeError("Wrong dimensionality of the vectors")
        n = x.shape[0]
        if ids is None:
            ids = np.arange(self.cur_l, self.cur_l + n, dtype=np.uint64)
        else:
            ids = np.atleast_1d(np.asarray(ids, dtype=np.uint64))
            if ids.shape[0] != n:
                raise RuntimeError(
                    f"The input label shape {ids.ndim} does not match the input data vector shape {x.ndim}")
        if self._rows.shape[0] == 0 and np.unique(ids).shape[0] == n:
            # fast path: a fresh index and distinct labels
            if n > self._maxel:
                raise RuntimeError("The number of elements exceeds the specified limit\n")
            self._rows = x.copy()
            self._row_labels = ids.astype(np.uint64).copy()
            self.cur_l += n
            self._dirty = True
            return
        pos = {int(l): i for i, l in enumerate(self._row_labels)}
        rows, labs = list(self._rows), list(self._row_labels)
        for i in range(n):
            lab = int(ids[i])
            if lab in pos:
                rows[pos[lab]] = x[i]
            else:
                if len(rows) >= self._maxel:
                    raise RuntimeError("The number of elements exceeds the specified limit\n")
                pos[lab] = len(rows)
                rows.append(x[i])
                labs.append(lab)
        self._rows = np.asarray(rows, np.float32).reshape(-1, self.dim)
        self._row_labels = np.asarray(labs, np.uint64)
        self.cur_l += n
        self._dirty = True

    def delete_vector(self, label: int) -> None:
        """BruteforceSearch::removePoint (bruteforce.h:86-103): the last row
        moves into the freed slot; unknown labels are ignored."""
        if self._rows is None:
            self._pull_rows()
        idx = np.nonzero(self._row_labels == np.uint64(label))[0]
        if idx.size == 0:
            return
        i, last = int(idx[0]), self._rows.shape[0] - 1
        self._rows[i] = self._rows[last]
        self._row_labels[i] = self._row_labels[last]
        self._rows = self._rows[:last].copy()
        self._row_labels = self._row_labels[:last].copy()
        self._dirty = True

    def _pull_rows(self):
        """The rows of a file-loaded index, from its file, so that add_items /
        delete_vector can change them (the index is rebuilt on the GPU at the
        next query).  Cosine files hold normalised rows that a rebuild would
        normalise again, so the cosine space keeps them read-only."""
        from . import pickling
        if self.space == "cosine" or getattr(self, "_source", None) is None:
            raise NotImplementedError("add_items / delete_vector after load_index: not supported for the cosine "
                                      "space (its file holds normalised rows)")
        with open(self._source, "rb") as f:
            self._maxel, self._rows, self._row_labels = pickling.bf_file_to_rows(f.read(), self.dim)

    def _sync(self):
        if self._rows is not None and (self._dirty or not self._h):
            if self._h:
                _capi.lib().hnswgpu_free(self._h)
                self._h = None
            self._labels = None
            h = C.c_void_p()
            r = np.ascontiguousarray(self._rows, np.float32)
            lab = np.ascontiguousarray(self._row_labels, np.uint64)
            _capi.check(_capi.lib().hnswgpu_create_bf(_SPACES[self.space], self.dim, _ptr(r), _ptr(lab), r.shape[0],
                                                      self._maxel, self.device, C.byref(h)))
            self._h = h
            self._dirty = False

    def load_index(self, path_to_index: str, max_elements: int = 0) -> None:
        """Load a file written by ``BFIndex.save_index`` (bruteforce.h:142-161)."""
        self._free()
        self._rows = None
        h = C.c_void_p()
        _capi.check(_capi.lib().hnswgpu_load_bf(str(path_to_index).encode(), _SPACES[self.space], self.dim,
                                                self.device, C.byref(h)))
        self._h = h
        self.cur_l = self._info().count
        self._source = os.path.abspath(str(path_to_index))

    def save_index(self, path_to_index: str) -> None:
        """BruteforceSearch::saveIndex (bruteforce.h:128-139).  A loaded,
        unchanged index is written back as loaded; rows added here are written
        as the reference stores them (cosine: normalised with the reference's
        arithmetic)."""
        from . import pickling
        if self._rows is None:
            if getattr(self, "_source", None) is None:
                raise RuntimeError("nothing to save: call init_index / add_items or load_index first")
            with open(self._source, "rb") as f:
                buf = f.read()
        else:
            rows = pickling.normalize_rows(self._rows) if self.space == "cosine" else self._rows
            buf = pickling.bf_rows_to_file(rows, self._row_labels, max(self._maxel, self._rows.shape[0]), self.dim)
        with open(path_to_index, "wb") as f:
            f.write(buf)

    def get_current_count(self) -> int:
        if self._rows is not None:
            return int(self._rows.shape[0])
        return super().get_current_count()

    def get_max_elements(self) -> int:
        if self._rows is not None:
            return self._maxel
        return super().get_max_elements()

    def knn_query(self, data, k: int = 1, num_threads: int = -1, filter: Optional[Callable[[int], bool]] = None):
        """(labels, distances), closest first (bindings.cpp:850-929); raises
        when fewer than k elements pass."""
        data = _input_rows(data)
        if data.shape[1] != self.dim:
            raise RuntimeError("Wrong dimensionality of the vectors")
        self._sync()
        labels, dists, counts, _ = self._search(data, k, filter, precision=self.precision, rerank=self.rerank)
        if counts.size and counts.min() < k:
            raise RuntimeError("Cannot return the results in a contiguous 2D array. There are not enough elements.")
        return labels, dists

    def knn_query_traced(self, data, k: int = 1, filter=None, precision: Optional[str] = None,
                         rerank: Optional[int] = None):
        """knn_query plus, for the tensor-core forms, per-query counters
        [candidates below the threshold, 0, 1 if answered by the exact
        kernel, 0]; no exception for short results."""
        data = _input_rows(data)
        self._sync()
        return self._search(data, k, filter, trace=True, precision=precision or self.precision,
                            rerank=self.rerank if rerank is None else rerank)
