"""Serving loop (continuous batching) on the GPU: every request's result is
the same whether it runs alone or inside a mixed, overlapping load of other
k / ef / filter / tie-order / precision / learned-stop requests; admission by
footprint bounds what is in flight (needs a B200)."""
import numpy as np
import pytest

import hnsw_rabitq_b200 as H
from hnsw_rabitq_b200 import learned
from oracle import oracle as O
from hnsw_rabitq_b200.serving import Server, poisson_arrivals
from tests.helpers import build_hnsw

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def served(tmp_path_factory):
    rng = np.random.default_rng(5)
    x = (rng.standard_normal((20000, 64)) * 3).astype(np.float32)
    q = (rng.standard_normal((1200, 64)) * 3).astype(np.float32)
    path = tmp_path_factory.mktemp("srv") / "s.bin"
    build_hnsw(path, x, "l2", M=16, efc=100, num_threads=8)
    g = H.Index("l2", 64)
    g.load_index(str(path))
    for lab in range(0, 20000, 20):  # 5 % deleted
        g.mark_deleted(lab)
    # a termination network (random weights, finite threshold): what matters
    # here is that the learned stop is deterministic per query
    f = rng.normal(size=(100, learned.F)).astype(np.float32)
    g.set_termination_model(learned.TerminationModel(learned.init_params(f, 1), 4, 0.5))
    return g, x, q, path


def _mix(n, rng, parity_id):
    """The serving mix of the 1M x 768 workload in miniature: k over {1, 10,
    100}, ef over {32 .. 512}, 30 % filtered, 20 % tie-exact, 25 % fp8
    traversal (id order), ~30 % of the id-order requests with the learned
    stop."""
    reqs = []
    for i in range(n):
        exact = rng.random() < 0.2
        fp8 = not exact and rng.random() < 0.3
        reqs.append(Server.request(k=int(rng.choice([1, 10, 100])), ef=int(rng.choice([32, 64, 128, 256, 512])),
                                   filter=parity_id if rng.random() < 0.3 else -1,
                                   tie_order="reference" if exact else "id",
                                   learned=False, precision="fp8" if fp8 else "fp32"))
        if reqs[-1].flags == 0 and rng.random() < 0.3:
            reqs[-1].flags = H._capi.LEARNED_STOP
    return reqs


def test_same_alone_and_in_mix(served):
    g, x, q, _ = served
    rng = np.random.default_rng(9)
    with Server(g, max_inflight=6, max_batch=256) as srv:
        parity = srv.add_filter(lambda l: l % 2 == 0)
        reqs = _mix(len(q), rng, parity)
        # in the mix: Poisson arrivals at 100k requests/s
        ml, md, mc, lat = srv.replay(q, reqs, poisson_arrivals(len(q), 100_000, seed=2))
        st = srv.stats()
        assert st["completed"] == len(q) and st["batches"] > 1
        assert np.all(lat > 0) and st["p99_us"] >= st["p50_us"] > 0
        # alone: one request at a time through the same server
        for i in range(0, len(q), 7):
            r = reqs[i]
            t = srv.submit(q[i], k=r.k, ef=r.ef, filter=r.filter,
                           tie_order="reference" if r.flags & H._capi.EXACT_TIES else "id",
                           learned=bool(r.flags & H._capi.LEARNED_STOP),
                           precision="fp8" if r.precision == H._capi.PREC_FP8 else "fp32")
            al, ad, _ = srv.wait(t)
            assert mc[i] == len(al)
            assert np.array_equal(al, ml[i, :mc[i]]), i
            assert np.array_equal(ad.view(np.uint32), md[i, :mc[i]].view(np.uint32)), i


@pytest.mark.parametrize("precision", ["fp32", "fp8"])
def test_matches_batch_search(served, precision):
    """A served request equals the batched C-ABI search with the same settings."""
    g, x, q, _ = served
    with Server(g) as srv:
        parity = srv.add_filter(lambda l: l % 2 == 0)
        n = 300
        reqs = [Server.request(k=10, ef=64, filter=parity if i % 2 else -1, precision=precision) for i in range(n)]
        ml, md, mc, _ = srv.replay(q[:n], reqs, np.zeros(n))
    fl, fd, fc, _ = g.knn_query_traced(q[:n], 10, filter=lambda l: l % 2 == 0, ef=64, tie_order="id",
                                       precision=precision)
    ul, ud, uc, _ = g.knn_query_traced(q[:n], 10, ef=64, tie_order="id", precision=precision)
    for i in range(n):
        want = (fl, fc) if i % 2 else (ul, uc)
        assert mc[i] == want[1][i] and np.array_equal(ml[i, :mc[i]], want[0][i, :mc[i]])


def test_admission_budget_serialises(served):
    """A budget of one query's footprint forces batches of one."""
    g, x, q, _ = served
    with Server(g, smem_budget=1) as srv:
        with pytest.raises(RuntimeError, match="exceeds the admission budget"):
            srv.replay(q[:3], [Server.request(k=10, ef=64)] * 3, np.zeros(3))
    with Server(g, max_batch=1) as srv:
        ml, _, mc, _ = srv.replay(q[:20], [Server.request(k=10, ef=64)] * 20, np.zeros(20))
        st = srv.stats()
        assert st["batches"] == 20 and st["mean_batch"] == 1
    ul, _, _, _ = g.knn_query_traced(q[:20], 10, ef=64, tie_order="id")
    assert np.array_equal(ml, ul)


def test_rejects_bad_requests(served):
    g, x, q, _ = served
    with Server(g) as srv:
        with pytest.raises(RuntimeError, match="unknown filter"):
            srv.submit(q[0], k=10, filter=3)
        with pytest.raises(RuntimeError, match="id tie order"):
            srv.submit(q[0], k=10, tie_order="reference", learned=True)
        with pytest.raises(RuntimeError, match="k must be positive"):
            srv.submit(q[0], k=0)


def test_mix_matches_the_reference(served):
    """Float32 requests served inside the mix (5 % deleted, label-parity
    filter on 30 %, mixed k and ef, fp8 / learned-stop / tie-exact neighbours
    in flight) return the reference's own results: tie-exact requests
    hnswlib's searchKnn (the oracle's reference mode), plain id-order ones
    the oracle's canonical mode, labels and distance bits."""
    g, x, q, path = served
    o = O.Hnsw(str(path), "l2", 64)
    for lab in range(0, 20000, 20):
        assert o.set_deleted(lab, True) == 0
    allow = np.array([1 if int(l) % 2 == 0 else 0 for l in o.labels()], np.uint8)
    rng = np.random.default_rng(21)
    with Server(g, max_inflight=6, max_batch=256) as srv:
        parity = srv.add_filter(lambda l: l % 2 == 0)
        reqs = _mix(len(q), rng, parity)
        ml, md, mc, _ = srv.replay(q, reqs, poisson_arrivals(len(q), 100_000, seed=4))
    groups = {}
    for i, r in enumerate(reqs):
        if r.precision != H._capi.PREC_FP32 or r.flags & H._capi.LEARNED_STOP:
            continue
        mode = O.REFERENCE if r.flags & H._capi.EXACT_TIES else O.CANONICAL
        groups.setdefault((r.k, r.ef, r.filter >= 0, mode), []).append(i)
    checked = 0
    for (k, ef, filtered, mode), idx in groups.items():
        rl, rd, rc = o.search(q[idx], k, ef, mode=mode, allow=allow if filtered else None)
        for j, i in enumerate(idx):
            assert mc[i] == rc[j], (i, k, ef, filtered, mode)
            assert np.array_equal(ml[i, :mc[i]], rl[j, :rc[j]]), (i, k, ef, filtered, mode)
            assert np.array_equal(md[i, :mc[i]].view(np.uint32), rd[j, :rc[j]].view(np.uint32)), i
        checked += len(idx)
    assert checked > 300
