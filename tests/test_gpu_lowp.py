"""Low-precision traversal (bf16 / per-row-scaled fp8 copies, fp32
accumulation) followed by the exact float32 re-rank (needs a B200)."""
import numpy as np
import pytest

import hnsw_rabitq_b200 as H
from oracle import oracle as O
from tests.helpers import build_hnsw

pytestmark = pytest.mark.gpu


def _recall(found, gt):
    return np.mean([len(np.intersect1d(found[i], gt[i])) / gt.shape[1] for i in range(gt.shape[0])])


def test_bf16_is_exact_on_8bit_data(tmp_path):
    """Integer vectors in [0, 255] are exact in bf16 and their squared
    distances are exact in fp32, so the bf16 beam takes the float32 beam's
    decisions: results identical to the float32 search (id tie order)."""
    from hnsw_rabitq_b200.datasets import gmm_1m_128
    x, q = gmm_1m_128(n=20000, nq=800)
    path = tmp_path / "gmm.bin"
    build_hnsw(path, x, "l2", M=16, efc=100, num_threads=8)
    g = H.Index("l2", 128)
    g.load_index(str(path))
    for ef in (16, 48, 128):
        g.set_ef(ef)
        fl, fd, fc, ft = g.knn_query_traced(q, 10, tie_order="id", precision="fp32")
        bl, bd, bc, bt = g.knn_query_traced(q, 10, tie_order="id", precision="bf16", rerank=10)
        assert np.array_equal(fl, bl) and np.array_equal(fd.view(np.uint32), bd.view(np.uint32))
        assert np.array_equal(ft[:, 2], bt[:, 2])  # same expansions


@pytest.mark.parametrize("space", ["l2", "ip", "cosine"])
def test_fp8_rerank_exact_distances_and_recall(tmp_path, space):
    rng = np.random.default_rng(7)
    x = rng.standard_normal((20000, 64)).astype(np.float32)
    q = rng.standard_normal((500, 64)).astype(np.float32)
    path = tmp_path / "f.bin"
    build_hnsw(path, x, space, M=16, efc=100, num_threads=8)
    g = H.Index(space, 64)
    g.load_index(str(path))
    gt, _ = O.bf_matrix("ip" if space != "l2" else "l2", O.normalize(x) if space == "cosine" else x,
                        O.normalize(q) if space == "cosine" else q, 10)
    g.set_ef(64)
    fl, fd, _, _ = g.knn_query_traced(q, 10, tie_order="id", precision="fp32")
    for prec in ("fp8", "bf16"):
        l, d, c, _ = g.knn_query_traced(q, 10, tie_order="id", precision=prec)
        assert (c == 10).all()
        # every returned distance is the exact reference distance of its label
        xs = O.normalize(x) if space == "cosine" else x
        qs = O.normalize(q) if space == "cosine" else q
        for i in range(0, 500, 25):
            ref = O.distances("ip" if space != "l2" else "l2", qs[i], xs[l[i].astype(np.int64)])
            assert np.array_equal(ref.view(np.uint32), d[i].view(np.uint32))
            assert np.all(np.diff(d[i]) >= 0)
        assert _recall(l, gt) >= _recall(fl, gt) - 0.03, (prec, _recall(l, gt), _recall(fl, gt))


def test_lowp_rejects_unsupported(tmp_path):
    rng = np.random.default_rng(1)
    x = rng.standard_normal((500, 20)).astype(np.float32)
    build_hnsw(tmp_path / "d20.bin", x, "l2", M=8)
    g = H.Index("l2", 20)
    g.load_index(str(tmp_path / "d20.bin"))
    with pytest.raises(RuntimeError, match="dim % 16"):
        g.knn_query_traced(x[:3], 5, tie_order="id", precision="fp8")
    x = rng.standard_normal((500, 32)).astype(np.float32)
    build_hnsw(tmp_path / "d32.bin", x, "l2", M=8)
    g = H.Index("l2", 32)
    g.load_index(str(tmp_path / "d32.bin"))
    with pytest.raises(RuntimeError, match="id tie order"):
        _exact_lowp(g, x[:3])


def _exact_lowp(g, q):
    """The low-precision beam with the reference tie order, straight through
    the C ABI (the Python surface quietly uses the id order for it)."""
    import ctypes as C

    from hnsw_rabitq_b200 import _capi
    n, k = q.shape[0], 5
    lab = np.empty((n, k), np.uint64)
    dist = np.empty((n, k), np.float32)
    cnt = np.empty(n, np.int32)
    o = _capi.SearchOpts()
    o.flags, o.precision = _capi.EXACT_TIES, _capi.PREC_FP8
    q = np.ascontiguousarray(q, np.float32)
    _capi.check(_capi.lib().hnswgpu_search(g._h, q.ctypes.data, n, k, C.byref(o), lab.ctypes.data,
                                           dist.ctypes.data, cnt.ctypes.data))


def test_lowp_with_filter_and_deletes(tmp_path):
    """Deletes and a filter in the low-precision beam: bf16 on 8-bit data
    still takes the float32 beam's decisions (identical results and
    expansions); fp8 returns allowed labels only, with exact distances."""
    from hnsw_rabitq_b200.datasets import gmm_1m_128
    x, q = gmm_1m_128(n=20000, nq=500)
    path = tmp_path / "gmm.bin"
    build_hnsw(path, x, "l2", M=16, efc=100, num_threads=8)
    g = H.Index("l2", 128)
    g.load_index(str(path))
    dead = set(range(0, 20000, 23))
    for lab in dead:
        g.mark_deleted(lab)
    flt = lambda l: l % 2 == 0
    for ef in (32, 96):
        g.set_ef(ef)
        fl, fd, fc, ft = g.knn_query_traced(q, 10, filter=flt, tie_order="id", precision="fp32")
        bl, bd, bc, bt = g.knn_query_traced(q, 10, filter=flt, tie_order="id", precision="bf16", rerank=10)
        assert np.array_equal(fl, bl) and np.array_equal(fd.view(np.uint32), bd.view(np.uint32))
        assert np.array_equal(fc, bc) and np.array_equal(ft[:, 2], bt[:, 2])
        l, d, c, _ = g.knn_query_traced(q, 10, filter=flt, tie_order="id", precision="fp8")
        assert (c == 10).all()
        assert all(int(v) % 2 == 0 and int(v) not in dead for v in l.ravel())
        for i in range(0, 500, 50):
            ref = O.distances("l2", q[i], x[l[i].astype(np.int64)])
            assert np.array_equal(ref.view(np.uint32), d[i].view(np.uint32))
        assert _recall(l, fl) >= 0.97
