"""The lean fp8 beam (hnsw_lean.cu): unfiltered id-order searches over the
per-row-scaled e4m3 copy with tensor-core distances, several link rows per
iteration, and the exact float32 re-rank (needs a B200).

Its beam is approximate by design, so the checks are the contract of the
low-precision forms: every returned distance is the reference's float32
distance of the returned label, rows are sorted, and recall@k against the
exact top-k stays within a small margin of the float32 beam at the same ef.
It covers M = 16 graphs (two link rows per iteration) and M = 32 graphs
(maxM0 = 64, one row of 64 links per iteration), row sizes of one to four
32-byte steps and the multi-block form (dim 256), and the learned stop."""
import numpy as np
import pytest

import hnsw_rabitq_b200 as H
from hnsw_rabitq_b200 import learned
from oracle import oracle as O
from tests.helpers import build_hnsw

pytestmark = pytest.mark.gpu


def _recall(found, gt):
    return float(np.mean([len(np.intersect1d(found[i], gt[i])) / gt.shape[1] for i in range(gt.shape[0])]))


def _check_exact_distances(space, x, q, lab, dist, every=20):
    xs = O.normalize(x) if space == "cosine" else x
    qs = O.normalize(q) if space == "cosine" else q
    for i in range(0, q.shape[0], every):
        ref = O.distances("ip" if space != "l2" else "l2", qs[i], xs[lab[i].astype(np.int64)])
        assert np.array_equal(ref.view(np.uint32), dist[i].view(np.uint32)), i
        assert np.all(np.diff(dist[i]) >= 0)


@pytest.mark.parametrize("dim,M,space", [(128, 16, "l2"), (128, 32, "l2"), (96, 32, "l2"), (64, 8, "ip"),
                                         (32, 12, "cosine"), (256, 16, "l2")])
def test_lean_fp8_recall_and_exact_distances(tmp_path, dim, M, space):
    rng = np.random.default_rng(dim + M)
    centres = rng.standard_normal((64, dim)).astype(np.float32) * 3
    x = (centres[rng.integers(0, 64, 12000)] + rng.standard_normal((12000, dim))).astype(np.float32)
    q = (centres[rng.integers(0, 64, 400)] + rng.standard_normal((400, dim))).astype(np.float32)
    path = tmp_path / "g.bin"
    build_hnsw(path, x, space, M=M, efc=100, num_threads=8)
    g = H.Index(space, dim)
    g.load_index(str(path))
    xs = O.normalize(x) if space == "cosine" else x
    qs = O.normalize(q) if space == "cosine" else q
    gt, _ = O.bf_matrix("l2" if space == "l2" else "ip", xs, qs, 10)
    # at small ef the beam has little room to absorb the fp8 rounding of the
    # distances (most on low-dimensional normalised rows, where near distances
    # differ least): within 0.05 there, 0.01 from ef 64
    for ef, margin in ((24, 0.05), (64, 0.01)):
        fl, fd, fc, ft = g.knn_query_traced(q, 10, ef=ef, tie_order="id", precision="fp32")
        ll, ld, lc, lt = g.knn_query_traced(q, 10, ef=ef, tie_order="id", precision="fp8")
        assert (lc == 10).all()
        assert g.get_status() == 0
        _check_exact_distances(space, x, q, ll, ld)
        assert _recall(ll, gt) >= _recall(fl, gt) - margin, (ef, _recall(ll, gt), _recall(fl, gt))
        # work counters: expansions and distance evaluations were made
        assert (lt[:, 2] > 0).all() and (lt[:, 3] >= lt[:, 2]).all()


def test_lean_gmm_8bit_matches_fp32_recall(tmp_path):
    """The 1M x 128 workload's distribution at 20k rows (integer values,
    reference-built M = 16 graph): fp8 lean recall within 0.01 of the float32
    beam at every ef of a sweep from 32 (at ef = k the beam has no room to
    absorb the fp8 rounding of the distances)."""
    from hnsw_rabitq_b200.datasets import gmm_1m_128
    x, q = gmm_1m_128(n=20000, nq=1000)
    path = tmp_path / "gmm.bin"
    build_hnsw(path, x, "l2", M=16, efc=100, num_threads=8)
    g = H.Index("l2", 128)
    g.load_index(str(path))
    gt = g.knn_query_exact(q, 10)[0]
    for ef in (32, 48, 96):
        fl, _, _, _ = g.knn_query_traced(q, 10, ef=ef, tie_order="id", precision="fp32")
        ll, ld, _, _ = g.knn_query_traced(q, 10, ef=ef, tie_order="id", precision="fp8")
        assert _recall(ll, gt) >= _recall(fl, gt) - 0.01, (ef, _recall(ll, gt), _recall(fl, gt))
        _check_exact_distances("l2", x, q, ll, ld, every=50)


def test_lean_learned_stop_bounds(tmp_path):
    """Threshold +inf (and 1e30, which evaluates the network) gives the plain
    lean beam; -inf stops at the first checkpoint taken; recording
    checkpoints does not change the search."""
    rng = np.random.default_rng(3)
    x = rng.standard_normal((10000, 64)).astype(np.float32)
    q = rng.standard_normal((300, 64)).astype(np.float32)
    path = tmp_path / "g.bin"
    build_hnsw(path, x, "l2", M=16, efc=100, num_threads=8)
    g = H.Index("l2", 64)
    g.load_index(str(path))
    k, ef, period = 10, 64, 4
    pl, pd, _, pt = g.knn_query_traced(q, k, ef=ef, tie_order="id", precision="fp8")
    f = rng.normal(size=(64, learned.F)).astype(np.float32)
    p = learned.init_params(f, 0)
    for never in (float("inf"), 1e30):
        g.set_termination_model(learned.TerminationModel(p, period, never, ef, "fp8"))
        ll, ld, _, lt = g.knn_query_traced(q, k, ef=ef, tie_order="id", precision="fp8", learned=True)
        assert np.array_equal(ll, pl) and np.array_equal(lt[:, 2], pt[:, 2])
    # -inf stops at the first checkpoint taken: the first one due (every
    # `period` expansions) at which the top-k has been stable for a period
    # and no unexpanded candidate is closer than the current k-th result
    g.set_termination_model(learned.TerminationModel(p, period, -float("inf"), ef, "fp8"))
    ll, ld, lc, lt = g.knn_query_traced(q, k, ef=ef, tie_order="id", precision="fp8", learned=True)
    assert np.all(lt[:, 2] <= pt[:, 2]) and lt[:, 2].mean() < 0.8 * pt[:, 2].mean() and np.all(lc == k)
    assert np.all(lt[:, 2] >= period)
    assert np.all(np.diff(ld, axis=1) >= 0)
    ck = g.search_checkpoints(q, k, ef=ef, period=period, max_ckpt=64, precision="fp8")
    assert np.array_equal(ck["labels"], pl)
    n = ck["nckpt"].astype(np.int64)
    assert np.all(n >= 1) and np.all(n - 1 <= pt[:, 2] // period)


@pytest.mark.parametrize("space", ["l2", "ip"])
def test_lean_traces_record_rerank_inputs(tmp_path, space):
    """Trace mode of the fp8 beam records the first R beam entries with their
    float32 distances (R = the re-rank count, the whole pool by default): the
    distances are the float32 distances of those ids (within summation-order
    rounding), and the final row's answer -- the k closest of its recorded
    entries -- is what the search itself returns after its re-rank."""
    rng = np.random.default_rng(11)
    x = rng.standard_normal((8000, 64)).astype(np.float32)
    q = rng.standard_normal((200, 64)).astype(np.float32)
    if space == "ip":
        x /= np.linalg.norm(x, axis=1, keepdims=True)
        q /= np.linalg.norm(q, axis=1, keepdims=True)
    path = tmp_path / "g.bin"
    build_hnsw(path, x, space, M=16, efc=100, num_threads=8)
    g = H.Index(space, 64)
    g.load_index(str(path))
    k, ef, period = 10, 48, 4
    ck = learned.traces(g, q, k, ef, period, 64, "fp8", 0)
    assert ck["ids"].shape[2] == ef and ck["ckpt_dists"].shape == ck["ids"].shape
    lab_of = g.labels_by_internal_id()
    n = ck["nckpt"].astype(np.int64)
    rows = np.arange(len(q))
    # recorded distances against numpy float32 (the stored rows are the inputs)
    for i in range(0, len(q), 7):
        for r in range(n[i]):
            ids = ck["ids"][i, r]
            ok = ids != 0xffffffff
            d = ck["ckpt_dists"][i, r]
            assert np.all(np.isinf(d[~ok]))
            xi = x[lab_of[ids[ok]].astype(np.int64)]
            ref = ((xi - q[i]) ** 2).sum(1) if space == "l2" else 1.0 - xi @ q[i]
            assert np.allclose(d[ok], ref, rtol=1e-4, atol=1e-4), (i, r)
    # the final row's re-rank answer is the search's own result
    final = learned.checkpoint_answers({"ids": ck["ids"][rows, n - 1][:, None, :],
                                        "ckpt_dists": ck["ckpt_dists"][rows, n - 1][:, None, :]}, k)[:, 0, :]
    assert np.all(final != 0xffffffff)  # full pools: 8,000 rows, ef 48
    got = lab_of[final.astype(np.int64)]
    same = np.mean([set(got[i]) == set(ck["labels"][i]) for i in rows])
    assert same >= 0.99, same


def test_lean_large_ef_budget(tmp_path):
    """The fixed-ef fp8 beam is budgeted at its own two warps per CTA: ef 3000
    runs (and finds nearly all true neighbours); the learned-stop form, four
    warps beside the network copy, reports that this ef does not fit."""
    rng = np.random.default_rng(17)
    x = rng.standard_normal((20000, 64)).astype(np.float32)
    q = rng.standard_normal((64, 64)).astype(np.float32)
    path = tmp_path / "g.bin"
    build_hnsw(path, x, "l2", M=16, efc=100, num_threads=8)
    g = H.Index("l2", 64)
    g.load_index(str(path))
    ll, ld, _, _ = g.knn_query_traced(q, 10, ef=3000, tie_order="id", precision="fp8")
    gt = g.knn_query_exact(q, 10)[0]
    assert learned.recall(ll, gt) >= 0.99
    g.set_termination_model(learned.TerminationModel(learned.init_params(rng.normal(size=(64, learned.F)), 0), 4,
                                                     0.5, 3000, "fp8"))
    with pytest.raises(RuntimeError, match="too large"):
        g.knn_query_traced(q, 10, ef=3000, tie_order="id", precision="fp8", learned=True)
