"""Epsilon search (searchStopConditionClosest with EpsilonSearchStopCondition)
on the GPU against the reference's recorded outputs and the oracle: ids,
distances, result order (equal distances in the reference's heap pop order)
and counts, bit-exact (needs a B200)."""
import numpy as np
import pytest

import hnsw_rabitq_b200 as H
from oracle import oracle as O
from tests.helpers import GOLDEN, build_hnsw, golden

pytestmark = pytest.mark.gpu

SPACES = {"hnsw_l2_d16": ("l2", 16), "hnsw_ip_d20": ("ip", 20), "hnsw_l2_d7_int": ("l2", 7)}


def test_epsilon_matches_reference_golden():
    g = golden()
    e = np.load(f"{GOLDEN}/epsilon.npz")
    keys = sorted({k.rsplit("/", 1)[0] for k in e.keys()})
    assert len(keys) == 36
    for key in keys:
        name, _, variant = key.split("/")
        space, dim = SPACES[name]
        idx = H.Index(space, dim)
        idx.load_index(f"{GOLDEN}/{name}.bin")
        flt = None
        if variant == "even":
            flt = lambda lab: lab % 2 == 0  # noqa: E731
        if variant == "del":
            for lab in g[f"{name}/deleted"]:
                idx.mark_deleted(int(lab))
        eps, mn, mx = e[key + "/params"]
        ids, d, c = idx.search_epsilon(g[f"{name}/queries"], np.float32(eps), int(mn), int(mx), filter=flt)
        assert idx.get_status() == 0, key
        assert np.array_equal(c, e[key + "/counts"]), key
        assert np.array_equal(ids, e[key + "/labels"]), key
        assert np.array_equal(d.view(np.uint32), e[key + "/dists"].view(np.uint32)), key


@pytest.mark.parametrize("kind", ["uniform", "int"])
def test_epsilon_matches_oracle_fresh(tmp_path, kind):
    """Larger indexes, dim % 16 == 0 (the general tie-exact loop even where
    the plain search pipelines), up to 512 candidates, against the oracle."""
    rng = np.random.default_rng(31)
    if kind == "uniform":
        x = rng.random((20000, 32), dtype=np.float32)
        q = rng.random((300, 32), dtype=np.float32)
    else:
        x = rng.integers(0, 8, (20000, 32)).astype(np.float32)
        q = rng.integers(0, 8, (300, 32)).astype(np.float32)
    path = tmp_path / "e.bin"
    build_hnsw(path, x, "l2", M=16, efc=100, num_threads=8)
    idx = H.Index("l2", 32)
    idx.load_index(str(path))
    o = O.Hnsw(str(path), "l2", 32)
    ex = np.stack([O.distances("l2", q[i], x[:4000]) for i in range(20)])
    for quant, mn, mx in ((0.002, 10, 64), (0.01, 100, 512), (0.05, 0, 256)):
        eps = np.float32(np.quantile(ex, quant))
        ol, od, oc = o.search_epsilon(q, eps, mn, mx)
        ids, d, c = idx.search_epsilon(q, eps, mn, mx)
        assert idx.get_status() == 0
        assert np.array_equal(c, oc) and np.array_equal(ids, ol)
        assert np.array_equal(d.view(np.uint32), od.view(np.uint32))
        assert c.max() > 0


def test_epsilon_argument_errors(tmp_path):
    g = H.Index("l2", 16)
    g.load_index(f"{GOLDEN}/hnsw_l2_d16.bin")
    q = golden()["hnsw_l2_d16/queries"][:2]
    with pytest.raises(RuntimeError, match="min_candidates"):
        g.search_epsilon(q, 0.5, 10, 5)
    ids, d, c = g.search_epsilon(q, -1.0, 0, 8)  # an empty epsilon region
    assert (c == 0).all() and (ids == np.iinfo(np.uint64).max).all()
