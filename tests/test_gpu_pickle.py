"""Pickling, from_params and save_index of the GPU Index against the
reference's recorded outputs (needs a B200)."""
import pickle

import numpy as np
import pytest

import hnsw_rabitq_b200 as H
from hnsw_rabitq_b200 import pickling as PK
from tests.helpers import GOLDEN, golden

pytestmark = pytest.mark.gpu


def _check(idx, g, key, k=10):
    l, d = idx.knn_query(g["hnsw_l2_d16/queries"], k=k)
    assert np.array_equal(l, g[f"hnsw_l2_d16/{key}/labels"]), key
    assert np.array_equal(d.view(np.uint32), g[f"hnsw_l2_d16/{key}/dists"].view(np.uint32)), key


def test_pickle_from_params_and_save_index(tmp_path):
    g = golden()
    idx = H.Index("l2", 16)
    idx.load_index(f"{GOLDEN}/hnsw_l2_d16.bin")
    idx.set_ef(32)
    # pickle round trip: same results, ef kept
    j = pickle.loads(pickle.dumps(idx))
    assert j.ef == 32
    _check(j, g, "ef32_k10")
    # a state dict (as a reference hnswlib.Index pickles it) goes to the GPU
    buf = open(f"{GOLDEN}/hnsw_l2_d16.bin", "rb").read()
    f = H.Index.from_params(PK.file_bytes_to_state(buf, "l2", 16, ef=32))
    _check(f, g, "ef32_k10")
    # delete marks travel through pickling and save_index
    for lab in g["hnsw_l2_d16/deleted"]:
        idx.mark_deleted(int(lab))
    _check(idx, g, "ef32_k10_del")
    _check(pickle.loads(pickle.dumps(idx)), g, "ef32_k10_del")
    idx.save_index(str(tmp_path / "s.bin"))
    s = H.Index("l2", 16)
    s.load_index(str(tmp_path / "s.bin"))
    s.set_ef(32)
    _check(s, g, "ef32_k10_del")
    assert s.get_current_count() == idx.get_current_count()
    # get_items: the stored rows of the returned labels give back their distances
    from oracle import oracle as O
    q = g["hnsw_l2_d16/queries"]
    l, d = s.knn_query(q[:3], k=4)
    for i in range(3):
        rows = s.get_items(l[i])
        assert np.array_equal(O.distances("l2", q[i], rows).view(np.uint32), d[i].view(np.uint32))
    with pytest.raises(RuntimeError, match="Label not found"):
        s.get_items([int(g["hnsw_l2_d16/deleted"][0])])
    s.resize_index(5000)
    assert s.get_max_elements() == 5000 and s.index_file_size() == len(open(tmp_path / "s.bin", "rb").read())
    c = H.Index(s)  # the copy constructor
    c.set_ef(32)
    _check(c, g, "ef32_k10_del")
    assert c.get_max_elements() == 5000


def test_load_from_memory_image():
    """hnswgpu_load_hnsw_buffer (the unpickling path) reads the file image in
    place: the same results as the file, bit for bit; a truncated or
    corrupted image is rejected with the loader's format error."""
    import ctypes as C
    from hnsw_rabitq_b200 import _capi
    g = golden()
    buf = open(f"{GOLDEN}/hnsw_l2_d16.bin", "rb").read()
    a = H.Index("l2", 16)
    a.load_index(f"{GOLDEN}/hnsw_l2_d16.bin")
    a.set_ef(32)
    b = H.Index.from_params(PK.file_bytes_to_state(buf, "l2", 16, ef=32))
    la, da = a.knn_query(g["hnsw_l2_d16/queries"], k=10)
    lb, db = b.knn_query(g["hnsw_l2_d16/queries"], k=10)
    assert np.array_equal(la, lb) and np.array_equal(da.view(np.uint32), db.view(np.uint32))
    lib = _capi.lib()
    for bad in (buf[: len(buf) // 2], buf[:40], buf + b"\0" * 8):
        h = C.c_void_p()
        cb = C.c_char_p(bad)
        rc = lib.hnswgpu_load_hnsw_buffer(C.cast(cb, C.c_void_p), len(bad), 0, 16, 0, 0, C.byref(h))
        assert rc == _capi.ERR_FORMAT and not h.value, (len(bad), rc)
