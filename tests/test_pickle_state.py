"""The reference's pickled state of hnswlib.Index (getIndexParams) and its
saveIndex file, each built from the other (hnsw_rabitq_b200/pickling.py),
checked against the reference itself (oracle/_ref) on the CPU: byte-equal
files, equal states, and reference indexes rebuilt from our states that
answer queries exactly as the originals."""
import pickle

import numpy as np
import pytest

import hnsw_rabitq_b200 as H
from hnsw_rabitq_b200 import pickling as PK
from tests.helpers import ref_or_skip

SCALARS = ["offset_level0", "max_elements", "cur_element_count", "size_data_per_element", "label_offset",
           "offset_data", "max_level", "enterpoint_node", "max_M", "max_M0", "M", "mult", "ef_construction", "ef",
           "has_deletions", "size_links_per_element", "space", "dim", "index_inited", "normalize"]


def _ref_index(hnswlib, space, dim, n, extra, M, seed, deleted=()):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, dim)).astype(np.float32)
    p = hnswlib.Index(space, dim)
    p.init_index(n + extra, M=M, ef_construction=60, random_seed=seed)
    p.add_items(x, np.arange(n) * 5 + 1, num_threads=1)
    p.set_ef(37)
    for lab in deleted:
        p.mark_deleted(int(lab))
    return p, x


CASES = [("l2", 16, 700, 0, 8, ()), ("cosine", 12, 500, 300, 6, ()), ("ip", 20, 600, 50, 10, (1, 6, 101, 2996))]


@pytest.mark.parametrize("space,dim,n,extra,M,deleted", CASES)
def test_state_and_file_round_trip(tmp_path, space, dim, n, extra, M, deleted):
    hnswlib = ref_or_skip()
    p, x = _ref_index(hnswlib, space, dim, n, extra, M, seed=dim, deleted=deleted)
    path = tmp_path / "i.bin"
    p.save_index(str(path))
    buf = path.read_bytes()
    st = p.__getstate__()[0]
    # reference state -> the reference's own file, byte for byte
    assert PK.state_to_file_bytes(st) == buf
    # the reference's file -> a state equal to the reference's
    ours = PK.file_bytes_to_state(buf, space, dim, ef=37)
    for key in SCALARS:
        assert ours[key] == st[key], key
    for key in ("data_level0", "link_lists", "element_levels"):
        assert np.array_equal(np.asarray(ours[key]).view(np.uint8), np.asarray(st[key]).view(np.uint8)), key
    ref_map = dict(zip(np.asarray(st["label_lookup_external"]).tolist(), np.asarray(st["label_lookup_internal"]).tolist()))
    our_map = dict(zip(ours["label_lookup_external"].tolist(), ours["label_lookup_internal"].tolist()))
    assert our_map == ref_map
    assert PK.state_to_file_bytes(ours) == buf
    # the reference accepts our state (createFromParams) and answers as before
    r2 = hnswlib.Index.__new__(hnswlib.Index)
    r2.__setstate__((ours,))
    q = np.random.default_rng(1).standard_normal((50, dim)).astype(np.float32)
    a = p.knn_query(q, k=5, num_threads=1)
    b = r2.knn_query(q, k=5, num_threads=1)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_delete_marks_match_the_reference(tmp_path):
    hnswlib = ref_or_skip()
    p, _ = _ref_index(hnswlib, "l2", 16, 400, 0, 8, seed=3)
    before = tmp_path / "a.bin"
    p.save_index(str(before))
    p.mark_deleted(6)
    p.mark_deleted(11)
    p.unmark_deleted(6)
    after = tmp_path / "b.bin"
    p.save_index(str(after))
    assert PK.set_delete_marks(before.read_bytes(), {11}, {6}) == after.read_bytes()


def test_unloaded_index_pickles():
    i = H.Index("cosine", 7)
    i.set_ef(55)
    j = pickle.loads(pickle.dumps(i))
    assert (j.space, j.dim, j.ef, j._h) == ("cosine", 7, 55, None)
    with pytest.raises(RuntimeError, match="Invalid serialization version"):
        H.Index.from_params({"ser_version": 2, "space": "l2", "dim": 4})


def test_get_items_file_size_and_resize_match_the_reference(tmp_path):
    hnswlib = ref_or_skip()
    for space in ("l2", "cosine"):
        p, x = _ref_index(hnswlib, space, 16, 300, 20, 8, seed=9)
        p.mark_deleted(11)
        path = tmp_path / f"{space}.bin"
        p.save_index(str(path))
        buf = path.read_bytes()
        ids = [1, 6, 1496, 51]
        assert np.array_equal(PK.items_from_file(buf, ids, 16), np.asarray(p.get_items(ids)))
        for bad in (11, 2):  # deleted, absent
            with pytest.raises(RuntimeError, match="Label not found"):
                PK.items_from_file(buf, [bad], 16)
            with pytest.raises(RuntimeError, match="Label not found"):
                p.get_items([bad])
        assert p.index_file_size() == len(buf)
        p.resize_index(777)
        p.save_index(str(path))
        assert PK.with_max_elements(buf, 777) == path.read_bytes()


def test_constructor_overloads_unloaded():
    i = H.Index(params={"ser_version": 1, "space": "ip", "dim": 9, "index_inited": False, "ef": 21})
    assert (i.space, i.dim, i.ef) == ("ip", 9, 21)
    j = H.Index(i)
    assert (j.space, j.dim, j.ef) == ("ip", 9, 21)
    with pytest.raises(ValueError, match="return_type"):
        H.Index("l2", 4).get_items([1], return_type="tuple")


@pytest.mark.parametrize("space", ["l2", "ip", "cosine"])
def test_bf_save_index_matches_the_reference(tmp_path, space):
    """BFIndex built in memory (init_index / add_items / delete_vector, no GPU
    needed) saves the reference's file: header and every current record
    byte-equal (slots past the count hold leftovers in the reference)."""
    hnswlib = ref_or_skip()
    rng = np.random.default_rng(5)
    x = rng.standard_normal((330, 12)).astype(np.float32)
    ops = [("add", x[:300], np.arange(300) * 2 + 3), ("del", 5), ("del", 17), ("del", 12345),
           ("add", x[300:330], np.arange(30) * 2 + 1000), ("add", x[:2], [3, 5])]
    ref = hnswlib.BFIndex(space, 12)
    ref.init_index(400)
    ours = H.BFIndex(space, 12)
    ours.init_index(400)
    for op in ops:
        for idx in (ref, ours):
            if op[0] == "add":
                idx.add_items(op[1], op[2])
            else:
                idx.delete_vector(op[1])
    ref.save_index(str(tmp_path / "r.bin"))
    ours.save_index(str(tmp_path / "o.bin"))
    a, b = (tmp_path / "r.bin").read_bytes(), (tmp_path / "o.bin").read_bytes()
    cur = int(np.frombuffer(a[16:24], np.uint64)[0])
    assert len(a) == len(b) and a[:24] == b[:24]
    assert a[24:24 + cur * (12 * 4 + 8)] == b[24:24 + cur * (12 * 4 + 8)]
    maxel, rows, labels = PK.bf_file_to_rows(a, 12)
    want = PK.normalize_rows(ours._rows) if space == "cosine" else ours._rows
    assert maxel == 400 and np.array_equal(rows, want) and np.array_equal(labels, ours._row_labels)


def test_normalize_rows_is_the_references(tmp_path):
    """normalize_rows against the rows the reference's cosine BFIndex
    stores, bit for bit, for dims with and without a remainder mod 4."""
    hnswlib = ref_or_skip()
    rng = np.random.default_rng(8)
    for dim in (1, 3, 7, 16, 33, 100, 768):
        x = (rng.standard_normal((300, dim)) * rng.uniform(0.01, 100, (300, 1))).astype(np.float32)
        b = hnswlib.BFIndex("cosine", dim)
        b.init_index(300)
        b.add_items(x)
        b.save_index(str(tmp_path / "n.bin"))
        _, rows, _ = PK.bf_file_to_rows((tmp_path / "n.bin").read_bytes(), dim)
        assert np.array_equal(PK.normalize_rows(x).view(np.uint32), rows.view(np.uint32)), dim


def test_record_reader_matches_whole_file_reads(tmp_path):
    hnswlib = ref_or_skip()
    p, _ = _ref_index(hnswlib, "l2", 16, 300, 0, 8, seed=4)
    p.mark_deleted(21)
    path = tmp_path / "r.bin"
    p.save_index(str(path))
    buf = path.read_bytes()
    st = PK.file_bytes_to_state(buf, "l2", 16, ef=10)
    for src in (str(path), buf):
        with PK.RecordReader(src) as rd:
            assert rd.cur == 300
            for i, lab in enumerate(st["label_lookup_external"].tolist()):
                assert rd.deleted(i) == (lab == 21)
                if lab != 21:
                    assert np.array_equal(rd.vector(i, 16), PK.items_from_file(buf, [lab], 16)[0])


def test_get_items_uses_labels_and_marks_without_gpu(tmp_path, monkeypatch):
    """Index.get_items over a recorder in place of the GPU handle: labels
    from the index, delete marks from the file and from this session."""
    hnswlib = ref_or_skip()
    p, _ = _ref_index(hnswlib, "l2", 16, 200, 0, 8, seed=6)
    p.mark_deleted(11)
    path = tmp_path / "g.bin"
    p.save_index(str(path))
    buf = path.read_bytes()
    idx = H.Index("l2", 16)
    idx._h = object()  # never passed to the library here
    idx._source = str(path)
    idx._labels = PK.file_bytes_to_state(buf, "l2", 16, ef=10)["label_lookup_external"]
    try:
        assert np.array_equal(idx.get_items([1, 6, 16]), np.asarray(p.get_items([1, 6, 16])))
        assert idx.get_items([1], return_type="list") == np.asarray(p.get_items([1])).tolist()
        with pytest.raises(RuntimeError, match="Label not found"):
            idx.get_items([11])
        idx._marks[11] = False  # unmarked in this session
        assert np.array_equal(idx.get_items([11]), PK.items_from_file(PK.set_delete_marks(buf, set(), {11}), [11], 16))
        idx._marks[6] = True
        with pytest.raises(RuntimeError, match="Label not found"):
            idx.get_items([6])
        assert idx.index_file_size() == len(buf)
    finally:
        idx._h = None
