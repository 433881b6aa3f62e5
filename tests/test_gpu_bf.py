"""GPU brute force parity (needs a B200): bit-identical to the reference's
BruteforceSearch::searchKnn (labels and distances)."""
import numpy as np
import pytest

import hnsw_rabitq_b200 as H
from oracle import oracle as O
from tests.helpers import GOLDEN, build_bf, golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("space,dim", [("l2", 128), ("ip", 96), ("cosine", 48), ("l2", 7), ("ip", 20), ("l2", 33)])
def test_bf_matches_oracle(tmp_path, space, dim):
    rng = np.random.default_rng(dim)
    x = rng.standard_normal((3000, dim)).astype(np.float32)
    q = rng.standard_normal((130, dim)).astype(np.float32)
    build_bf(tmp_path / "bf.bin", x, space, extra=10)
    g = H.BFIndex(space, dim)
    g.load_index(str(tmp_path / "bf.bin"))
    o = O.Bf(str(tmp_path / "bf.bin"), space, dim)
    for k in (1, 10, 100):
        gl, gd = g.knn_query(q, k=k)
        ol, od, _ = o.search(q, k)
        assert np.array_equal(gl, ol)
        assert np.array_equal(gd.view(np.uint32), od.view(np.uint32))
    filt = lambda l: l % 3 == 1  # noqa: E731
    gl, gd = g.knn_query(q, k=10, filter=filt)
    allow = np.array([filt(i) for i in range(3000)], np.uint8)
    ol, od, _ = o.search(q, 10, allow=allow)
    assert np.array_equal(gl, ol) and np.array_equal(gd.view(np.uint32), od.view(np.uint32))


def test_bf_golden():
    g = golden()
    for name, space in (("bf_l2_d7", "l2"), ("bf_ip_d16", "ip"), ("bf_cos_d9", "cosine")):
        q = g[f"{name}/queries"]
        idx = H.BFIndex(space, q.shape[1])
        idx.load_index(f"{GOLDEN}/{name}.bin")
        for k in (1, 10, 25):
            for suffix, filt in (("", None), ("_even", lambda l: l % 2 == 0)):
                l, d = idx.knn_query(q, k=k, filter=filt)
                assert np.array_equal(l, g[f"{name}/k{k}{suffix}/labels"])
                assert np.array_equal(d.view(np.uint32), g[f"{name}/k{k}{suffix}/dists"].view(np.uint32))


def test_bf_add_items_and_ties():
    """In-memory BFIndex (init_index/add_items) with integer data: exact ties
    at the k-th distance are resolved by label as the reference heap does."""
    rng = np.random.default_rng(4)
    x = rng.integers(0, 3, (2000, 16)).astype(np.float32)
    q = rng.integers(0, 3, (64, 16)).astype(np.float32)
    labels = rng.permutation(2000).astype(np.uint64) + 10
    g = H.BFIndex("l2", 16)
    g.init_index(2000)
    g.add_items(x, labels)
    hnswlib = O.ref_module()
    if hnswlib is not None:
        p = hnswlib.BFIndex("l2", 16)
        p.init_index(2000)
        p.add_items(x, labels)
        rl, rd = p.knn_query(q, k=30)
        gl, gd = g.knn_query(q, k=30)
        assert np.array_equal(gl, rl) and np.array_equal(gd, rd)
    with pytest.raises(RuntimeError, match="not enough elements"):
        g.knn_query(q, k=3000)
    g.delete_vector(int(labels[0]))
    assert g.get_current_count() == 1999


def test_bf_loaded_then_changed_and_saved(tmp_path):
    """A file-loaded BFIndex: delete_vector pulls its rows from the file, the
    next query runs on the changed set (the recorded top-25 minus the deleted
    label), and save_index / load_index keep it."""
    g = golden()
    b = H.BFIndex("l2", 7)
    b.load_index(f"{GOLDEN}/bf_l2_d7.bin")
    q = g["bf_l2_d7/queries"]
    top = g["bf_l2_d7/k25/labels"]
    gone = int(top[0, 0])
    b.delete_vector(gone)
    want = np.stack([row[row != gone][:10] for row in top])
    l, _ = b.knn_query(q, k=10)
    assert np.array_equal(l, want)
    b.save_index(str(tmp_path / "c.bin"))
    c = H.BFIndex("l2", 7)
    c.load_index(str(tmp_path / "c.bin"))
    l2, _ = c.knn_query(q, k=10)
    assert np.array_equal(l2, want)
    assert c.get_current_count() == b.get_current_count()
