"""The Python surface keeps every name the reference's bindings define
(python_bindings/bindings.cpp:930-1040), so hnswlib code finds them.  Graph
construction (Index.init_index / add_items) is present but raises: it is not
part of the GPU query path (indexes are built with hnswlib and loaded)."""
import pickle

import pytest

import hnsw_rabitq_b200 as H

INDEX_METHODS = ["init_index", "knn_query", "add_items", "get_items", "get_ids_list", "set_ef", "set_num_threads",
                 "index_file_size", "save_index", "load_index", "mark_deleted", "unmark_deleted", "resize_index",
                 "get_max_elements", "get_current_count", "__getstate__", "__setstate__"]
INDEX_PROPERTIES = ["space", "dim", "num_threads", "ef", "max_elements", "element_count", "ef_construction", "M"]
BF_METHODS = ["init_index", "knn_query", "add_items", "delete_vector", "set_num_threads", "save_index", "load_index",
              "get_max_elements", "get_current_count"]


def test_index_names():
    i = H.Index("l2", 8)
    for name in INDEX_METHODS:
        assert callable(getattr(i, name)), name
    for name in INDEX_PROPERTIES:
        assert hasattr(type(i), name) or name in vars(i), name
    assert repr(i).endswith("Index(space='l2', dim=8)>")
    assert pickle.loads(pickle.dumps(i)).dim == 8
    with pytest.raises(NotImplementedError):
        i.init_index(10)


def test_bfindex_names():
    b = H.BFIndex("ip", 4)
    for name in BF_METHODS:
        assert callable(getattr(b, name)), name
    assert b.num_threads == -1
    assert repr(b).endswith("BFIndex(space='ip', dim=4)>")
