"""hnswlib::L2SpaceI (uint8 vectors, integer squared L2) on the GPU: the
uint8 rows are widened exactly to float32 at load, so the beam computes the
reference's integer distances exactly (dim <= 258).  Checked against the
reference's HierarchicalNSW<int> searchKnn outputs recorded in
tests/golden/l2u8.npz, in both tie orders (needs a B200)."""
import numpy as np
import pytest

import hnsw_rabitq_b200 as H
from oracle import oracle as O
from tests.helpers import GOLDEN

pytestmark = pytest.mark.gpu


def test_l2_uint8_matches_reference_golden():
    e = np.load(f"{GOLDEN}/l2u8.npz")
    q = e["queries"]  # uint8 rows; knn_query takes them as float32 values
    keys = sorted({k.rsplit("/", 1)[0] for k in e.keys() if "/" in k})
    for key in keys:
        ef, k, variant = key.split("_")
        ef, k = int(ef[2:]), int(k[1:])
        g = H.Index("l2_uint8", 32)
        g.load_index(f"{GOLDEN}/hnsw_l2u8_d32.bin")
        o = O.Hnsw(f"{GOLDEN}/hnsw_l2u8_d32.bin", "l2_uint8", 32)
        flt, allow = None, None
        if variant == "even":
            flt = lambda lab: lab % 2 == 0  # noqa: E731
            allow = (o.labels() % 2 == 0).astype(np.uint8)
        if variant == "del":
            for lab in e["deleted"]:
                g.mark_deleted(int(lab))
                assert o.set_deleted(int(lab), True) == 0
        g.set_ef(ef)
        rl, rd, rc = e[key + "/labels"], e[key + "/dists"], e[key + "/counts"]
        l, d, c, _ = g.knn_query_traced(q, k, filter=flt, tie_order="reference")
        assert g.get_status() == 0, key
        assert np.array_equal(c, rc), key
        for i in range(q.shape[0]):
            assert np.array_equal(l[i, :c[i]], rl[i, :c[i]]), (key, i)
            assert np.array_equal(d[i, :c[i]], rd[i, :c[i]].astype(np.float32)), (key, i)
        # id order: the oracle's canonical form
        l2, d2, c2, _ = g.knn_query_traced(q, k, filter=flt, tie_order="id")
        cl, cd, cc = o.search(q.astype(np.float32), k, ef, mode=O.CANONICAL, allow=allow)
        assert np.array_equal(c2, cc) and np.array_equal(l2, cl) and np.array_equal(d2, cd), key


def test_l2_uint8_dim_limit(tmp_path):
    if O.ref_l2u8() is None:
        pytest.skip("oracle/_ref/libref_l2u8.so not built")
    rng = np.random.default_rng(3)
    x = rng.integers(0, 256, (50, 300)).astype(np.uint8)
    O.ref_l2u8_build(tmp_path / "big.bin", x, np.arange(50, dtype=np.uint64), M=4, efc=20)
    g = H.Index("l2_uint8", 300)
    with pytest.raises(RuntimeError, match="dim <= 258"):
        g.load_index(str(tmp_path / "big.bin"))
