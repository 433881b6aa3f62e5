"""Multi-vector search on the GPU (searchStopConditionClosest with a
MultiVectorSearchStopCondition): ids, order, distances and counts identical
to the reference's recorded results, and to the oracle's restatement on
freshly built indexes (needs a B200)."""
import numpy as np
import pytest

import hnsw_rabitq_b200 as H
from oracle import oracle as O
from tests.helpers import GOLDEN

pytestmark = pytest.mark.gpu


def test_multivector_matches_reference_golden():
    e = np.load(f"{GOLDEN}/multivec.npz")
    g = H.Index("l2", 16)
    g.load_multivector_index(f"{GOLDEN}/hnsw_mv_l2_d16.bin")
    for nd, efc in ((10, 15), (5, 5), (3, 20), (20, 10)):
        key = f"docs{nd}_efc{efc}"
        ids, d, c = g.search_multivector(e["queries"], nd, efc, 400)
        assert np.array_equal(c, e[key + "/counts"]), key
        assert np.array_equal(ids, e[key + "/ids"]), key
        assert np.array_equal(d.view(np.uint32), e[key + "/dists"].view(np.uint32)), key
    assert g.get_status() == 0


def test_multivector_matches_oracle_fresh(tmp_path):
    if O.ref_multivec() is None:
        pytest.skip("oracle/_ref/libref_multivec.so not built")
    rng = np.random.default_rng(78)
    for n_docs_total, dim, M in ((30, 8, 12), (400, 24, 16), (60, 48, 32)):
        x = rng.standard_normal((3000, dim)).astype(np.float32)
        docs = rng.integers(0, n_docs_total, 3000)
        q = rng.standard_normal((50, dim)).astype(np.float32)
        path = tmp_path / f"mv{dim}.bin"
        O.ref_mv_build(path, "l2", x, docs, np.arange(3000), M=M, efc=80)
        o = O.Hnsw(str(path), "l2", dim)
        g = H.Index("l2", dim)
        g.load_multivector_index(str(path))
        # ef_collection below the number of documents: with every document
        # inside ef_collection the reference never evicts, and its
        # top_candidates grows past the kernel's fixed heaps
        for nd, efc in ((4, 8), (12, 12), (2, 20)):
            ol, od, oc = o.search_multivector(q, nd, efc, 800)
            gl, gd, gc = g.search_multivector(q, nd, efc, 800)
            assert np.array_equal(gc, oc) and np.array_equal(gl, ol), (dim, nd, efc)
            assert np.array_equal(gd.view(np.uint32), od.view(np.uint32))
        assert g.get_status() == 0
