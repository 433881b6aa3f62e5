"""Tensor-core brute force (bf16 / fp8 copies, tcgen05 scores, fused candidate
filter, exact float32 re-rank) against the exact scan (needs a B200).

Tolerances: the k returned distances are bit-identical to the reference's
distance function on the returned labels (the re-rank recomputes them in its
summation order); recall@k against the exact scan >= 0.99 (bf16) / 0.97 (fp8)
at the default over-fetch of 4 k."""
import numpy as np
import pytest

import hnsw_rabitq_b200 as H
from hnsw_rabitq_b200 import learned
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _bf(x, space):
    g = H.BFIndex(space, x.shape[1])
    g.init_index(x.shape[0])
    g.add_items(x)
    return g


def _check(g, x, q, space, k, prec, min_recall, rerank=0, filt=None):
    g.precision = "fp32"
    el, ed = g.knn_query(q, k, filter=filt)
    l, d, c, tr = g.knn_query_traced(q, k, filter=filt, precision=prec, rerank=rerank)
    assert np.all(c == k)
    r = learned.recall(l, el)
    assert r >= min_recall, (prec, space, r)
    xs = O.normalize(x) if space == "cosine" else x
    qs = O.normalize(q) if space == "cosine" else q
    sp = "l2" if space == "l2" else "ip"
    for i in range(0, q.shape[0], max(1, q.shape[0] // 25)):
        ref = O.distances(sp, qs[i], xs[l[i].astype(np.int64)])
        assert np.array_equal(ref.view(np.uint32), d[i].view(np.uint32)), i
        assert np.all(np.diff(d[i]) >= 0)
    if filt is not None:
        assert all(filt(int(v)) for row in l for v in row)
    return r, tr


@pytest.mark.parametrize("space", ["l2", "ip"])
@pytest.mark.parametrize("prec", ["bf16", "fp8"])
def test_sampled_threshold_path(space, prec):
    rng = np.random.default_rng(3)
    x = rng.standard_normal((50000, 128)).astype(np.float32)
    q = rng.standard_normal((300, 128)).astype(np.float32)
    g = _bf(x, space)
    r, tr = _check(g, x, q, space, 10, prec, 0.99 if prec == "bf16" else 0.97)
    assert np.all(tr[:, 0] >= 40)  # every query kept at least the over-fetch
    assert tr[:, 2].sum() == 0     # no exact fallback needed


@pytest.mark.parametrize("prec", ["bf16", "fp8"])
def test_unit_768_cosine(prec):
    from hnsw_rabitq_b200.datasets import gmm_unit_ip
    x, q = gmm_unit_ip(n=40000, nq=200, dim=768)
    g = _bf(x, "cosine")
    _check(g, x, q, "cosine", 100, prec, 0.99 if prec == "bf16" else 0.97, rerank=400)


def test_small_set_takes_every_row():
    rng = np.random.default_rng(4)
    x = rng.standard_normal((5000, 96)).astype(np.float32)
    q = rng.standard_normal((150, 96)).astype(np.float32)
    g = _bf(x, "l2")
    r, tr = _check(g, x, q, "l2", 10, "bf16", 0.99)
    assert np.all(tr[:, 0] == 5000)


def test_filter_and_exact_fallback():
    """Few admissible rows: queries whose threshold lets fewer than R rows
    through are answered by the exact kernel, identically."""
    rng = np.random.default_rng(5)
    x = rng.standard_normal((60000, 64)).astype(np.float32)
    q = rng.standard_normal((120, 64)).astype(np.float32)
    g = _bf(x, "l2")
    filt = lambda l: l % 500 == 0  # 120 admissible rows
    g.precision = "fp32"
    el, ed = g.knn_query(q, 10, filter=filt)
    l, d, c, tr = g.knn_query_traced(q, 10, filter=filt, precision="fp8", rerank=200)
    assert np.all(tr[:, 2] == 1)
    assert np.array_equal(l, el) and np.array_equal(d.view(np.uint32), ed.view(np.uint32))
    _check(g, x, q, "l2", 10, "bf16", 0.99, filt=lambda l: l % 2 == 0)


def test_rejects_large_overfetch():
    rng = np.random.default_rng(6)
    x = rng.standard_normal((1000, 32)).astype(np.float32)
    g = _bf(x, "l2")
    with pytest.raises(RuntimeError, match="over-fetch"):
        g.knn_query_traced(x[:2], 10, precision="bf16", rerank=2000)


def test_fp64_oracle():
    """The float64 oracle against numpy float64; its top-k certified."""
    from hnsw_rabitq_b200.groundtruth import fp64_distances, fp64_topk
    rng = np.random.default_rng(8)
    x = rng.standard_normal((20000, 48)).astype(np.float32)
    q = rng.standard_normal((50, 48)).astype(np.float32)
    for space in ("l2", "ip", "cosine"):
        g = _bf(x, space)
        lab = rng.integers(0, 20000, (50, 7)).astype(np.uint64)
        d = fp64_distances(g, q, lab)
        xs = x.astype(np.float64)
        if space == "cosine":
            xs = O.normalize(x).astype(np.float64)  # stored rows are the binding's normalised float32
            qs = q.astype(np.float64) / np.linalg.norm(q.astype(np.float64), axis=1, keepdims=True)
        else:
            qs = q.astype(np.float64)
        rows = xs[lab.astype(np.int64)]
        ref = ((qs[:, None, :] - rows) ** 2).sum(-1) if space == "l2" else 1.0 - (qs[:, None, :] * rows).sum(-1)
        assert np.allclose(d, ref, rtol=1e-12, atol=1e-12)
        tl, td, cert = fp64_topk(g, q, 10)
        assert cert.all()
        full = ((qs[:, None, :] - xs[None]) ** 2).sum(-1) if space == "l2" else 1.0 - qs @ xs.T
        want = np.argsort(full, axis=1, kind="stable")[:, :10]
        assert np.array_equal(tl.astype(np.int64), want)
