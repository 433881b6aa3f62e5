"""Pin the CPU oracle to the reference (CPU only).

* against the committed fixtures the reference produced (always);
* against the reference's own compiled extension (oracle/_ref) on fresh
  random data, when it is built here.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import GOLDEN, build_bf, build_hnsw, golden, ref_or_skip

DIMS = list(range(1, 41)) + [48, 63, 64, 96, 100, 127, 128, 130, 768]


@pytest.mark.parametrize("space", ["l2", "ip"])
def test_distances_bit_exact_vs_reference(space):
    hnswlib = ref_or_skip()
    rng = np.random.default_rng(5)
    for dim in DIMS:
        x = rng.standard_normal((64, dim)).astype(np.float32)
        q = rng.standard_normal((2, dim)).astype(np.float32)
        p = hnswlib.BFIndex(space, dim)
        p.init_index(64)
        p.add_items(x)
        lab, dist = p.knn_query(q, k=64)
        for i in range(2):
            ref = np.empty(64, np.float32)
            ref[lab[i].astype(np.int64)] = dist[i]
            ours = O.distances(space, q[i], x)
            assert np.array_equal(ours.view(np.uint32), ref.view(np.uint32)), (space, dim)


def test_known_answer_distances_golden():
    g = golden()
    for key in g.files:
        if not key.startswith("spaces/") or not key.endswith("/dists"):
            continue
        _, space, lr, _ = key.split("/")
        left, right = map(int, lr.split("_"))
        base = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1]], np.float32)
        x = np.concatenate([np.zeros((5, left), np.float32), base, np.zeros((5, right), np.float32)], 1)
        xs = O.normalize(x) if space == "cosine" else x
        lab = g[key.replace("/dists", "/labels")].astype(np.int64)[0]
        ours = O.distances("ip" if space == "cosine" else space, xs[-1], xs)[lab]
        assert np.array_equal(ours.view(np.uint32), g[key][0].view(np.uint32)), key
    # the reference test's expected values (tests/python/bindings_test_spaces.py)
    exp = {"l2": [0, 1, 2, 2, 2], "ip": [-2, -1, 0, 0, 0], "cosine": [0, 0.1835, 0.423, 0.423, 0.423]}
    for space, e in exp.items():
        d = g[f"spaces/{space}/0_0/dists"][0]
        assert np.allclose(d, e, atol=1e-3), space


def _golden_hnsw_cases():
    return ["hnsw_l2_d16", "hnsw_ip_d20", "hnsw_cos_d12", "hnsw_l2_d7_int"]


@pytest.mark.parametrize("name", _golden_hnsw_cases())
def test_oracle_reference_mode_matches_golden(name):
    g = golden()
    space = {"hnsw_l2_d16": "l2", "hnsw_ip_d20": "ip", "hnsw_cos_d12": "cosine", "hnsw_l2_d7_int": "l2"}[name]
    q = g[f"{name}/queries"]
    dim = q.shape[1]
    idx = O.Hnsw(f"{GOLDEN}/{name}.bin", space, dim)
    labels = idx.labels()
    even = (labels % 2 == 0).astype(np.uint8)
    for ef in (10, 32, 100):
        for k in (1, 10):
            for suffix, allow in (("", None), ("_even", even)):
                l, d, c = idx.search(q, k, ef, mode=O.REFERENCE, allow=allow)
                assert np.array_equal(l, g[f"{name}/ef{ef}_k{k}{suffix}/labels"]), (name, ef, k, suffix)
                assert np.array_equal(d.view(np.uint32), g[f"{name}/ef{ef}_k{k}{suffix}/dists"].view(np.uint32))
    for lab in g[f"{name}/deleted"]:
        assert idx.set_deleted(int(lab), True) == 0
    for ef in (10, 32, 100):
        l, d, c = idx.search(q, 10, ef, mode=O.REFERENCE)
        assert np.array_equal(l, g[f"{name}/ef{ef}_k10_del/labels"])
        assert np.array_equal(d.view(np.uint32), g[f"{name}/ef{ef}_k10_del/dists"].view(np.uint32))


@pytest.mark.parametrize("name,space", [("bf_l2_d7", "l2"), ("bf_ip_d16", "ip"), ("bf_cos_d9", "cosine")])
def test_oracle_bruteforce_matches_golden(name, space):
    g = golden()
    q = g[f"{name}/queries"]
    bf = O.Bf(f"{GOLDEN}/{name}.bin", space, q.shape[1])
    for k in (1, 10, 25):
        l, d, c = bf.search(q, k)
        assert np.array_equal(l, g[f"{name}/k{k}/labels"])
        assert np.array_equal(d.view(np.uint32), g[f"{name}/k{k}/dists"].view(np.uint32))


def test_oracle_search_vs_reference_fresh(tmp_path):
    """Reference mode == reference knn_query; canonical mode agrees on almost all rows."""
    hnswlib = ref_or_skip()
    rng = np.random.default_rng(11)
    for space, dim, M in (("l2", 32, 8), ("ip", 24, 12), ("cosine", 40, 16)):
        x = rng.standard_normal((3000, dim)).astype(np.float32)
        q = rng.standard_normal((300, dim)).astype(np.float32)
        path = tmp_path / f"{space}.bin"
        p = build_hnsw(path, x, space, M=M, efc=80)
        idx = O.Hnsw(str(path), space, dim)
        for ef in (10, 64):
            p.set_ef(ef)
            rl, rd = p.knn_query(q, k=10, num_threads=1)
            ol, od, _ = idx.search(q, 10, ef, mode=O.REFERENCE)
            assert np.array_equal(ol, rl)
            assert np.array_equal(od.view(np.uint32), rd.view(np.uint32))
            _, _, _, rt = idx.search(q, 10, ef, mode=O.REFERENCE, trace=True)
            cl, cd, _ = idx.search(q, 10, ef, mode=O.CANONICAL)
            differ = ~np.all(cl == rl, axis=1)
            assert not (differ & (rt[:, 4] == 0)).any()   # every difference has a tie event
            assert differ.mean() <= 0.001


def test_oracle_bruteforce_vs_reference_fresh(tmp_path):
    ref_or_skip()
    rng = np.random.default_rng(12)
    for space, dim in (("l2", 21), ("ip", 36), ("cosine", 13)):
        x = rng.standard_normal((700, dim)).astype(np.float32)
        q = rng.standard_normal((50, dim)).astype(np.float32)
        p = build_bf(tmp_path / "bf.bin", x, space)
        bf = O.Bf(str(tmp_path / "bf.bin"), space, dim)
        rl, rd = p.knn_query(q, k=15)
        ol, od, _ = bf.search(q, 15)
        assert np.array_equal(ol, rl) and np.array_equal(od.view(np.uint32), rd.view(np.uint32))


def test_oracle_load_errors(tmp_path):
    with pytest.raises(RuntimeError, match="Cannot open file"):
        O.Hnsw(str(tmp_path / "missing.bin"), "l2", 4)
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"\x00" * 40)
    with pytest.raises(RuntimeError, match="corrupted"):
        O.Hnsw(str(bad), "l2", 4)


def test_tie_witness_on_integer_fixture():
    """On the tie-heavy fixture the two oracle modes differ, and only on
    queries whose reference run made a tie decision."""
    g = golden()
    q = g["hnsw_l2_d7_int/queries"]
    o = O.Hnsw(f"{GOLDEN}/hnsw_l2_d7_int.bin", "l2", 7)
    total = 0
    for ef in (10, 32, 100):
        rl, _, _, rt = o.search(q, 10, ef, mode=O.REFERENCE, trace=True)
        cl, _, _ = o.search(q, 10, ef, mode=O.CANONICAL)
        differ = ~np.all(rl == cl, axis=1)
        total += differ.sum()
        assert not (differ & (rt[:, 4] == 0)).any()
    assert total > 0


def test_listing_rule_covers_every_divergence(tmp_path):
    """The two-pass tie-exact search runs the id order for every query and
    replays the reference's heaps only for the queries its run lists: the
    entry popped next ties another unexpanded entry, an expansion drops an
    entry that ties the pool's new worst, or the k-th and (k+1)-th entries tie.
    On tie-heavy data every unlisted query must have the reference's labels,
    distances, counts and expansion count, and the rule must not list all."""
    from hnsw_rabitq_b200.datasets import gmm_1m_128
    ref_or_skip()
    g = golden()
    cases = [(O.Hnsw(f"{GOLDEN}/hnsw_l2_d7_int.bin", "l2", 7), g["hnsw_l2_d7_int/queries"])]
    rng = np.random.default_rng(5)
    # small-integer vectors: distances tie often (about a third to a half of
    # the queries listed at ef 10, a few percent of them steered)
    for hi, dim in ((16, 16), (32, 8)):
        x = rng.integers(0, hi, size=(4000, dim)).astype(np.float32)
        q = rng.integers(0, hi, size=(300, dim)).astype(np.float32)
        build_hnsw(tmp_path / f"i{hi}.bin", x, "l2", M=8, efc=60)
        cases.append((O.Hnsw(str(tmp_path / f"i{hi}.bin"), "l2", dim), q))
    x, q = gmm_1m_128(n=5000, nq=300)  # the 1M workload's distribution, few ties
    build_hnsw(tmp_path / "gmm.bin", x, "l2", M=8, efc=60)
    cases.append((O.Hnsw(str(tmp_path / "gmm.bin"), "l2", 128), q))
    listed = total = differ_total = 0
    for o, qs in cases:
        for ef, k in ((10, 1), (10, 10), (32, 10), (100, 10)):
            rl, rd, rc, rt = o.search(qs, k, ef, mode=O.REFERENCE, trace=True)
            cl, cd, cc, ct = o.search(qs, k, ef, mode=O.CANONICAL, trace=True)
            unl = ct[:, 6] == 0
            assert np.array_equal(cl[unl], rl[unl]) and np.array_equal(cc[unl], rc[unl])
            assert np.array_equal(cd[unl].view(np.uint32), rd[unl].view(np.uint32))
            assert np.array_equal(ct[unl, 2], rt[unl, 2])
            differ = ~np.all(cl == rl, axis=1)
            differ_total += int(differ.sum())
            listed += int((~unl).sum())
            total += len(qs)
    assert differ_total > 0  # the data does steer the heaps
    assert listed < total


def _epsilon_cases():
    e = np.load(f"{GOLDEN}/epsilon.npz")
    names = sorted({k.rsplit("/", 1)[0] for k in e.keys()})
    return e, names


def test_oracle_epsilon_search_matches_golden():
    """The oracle's searchStopConditionClosest (EpsilonSearchStopCondition)
    against the reference's own outputs recorded in tests/golden/epsilon.npz:
    labels, distances, result order (equal distances in the reference's heap
    pop order) and counts, bit-exact; with a filter and with deletions."""
    g = golden()
    e, names = _epsilon_cases()
    spaces = {"hnsw_l2_d16": ("l2", 16), "hnsw_ip_d20": ("ip", 20), "hnsw_l2_d7_int": ("l2", 7)}
    for key in names:
        name, _, variant = key.split("/")
        space, dim = spaces[name]
        o = O.Hnsw(f"{GOLDEN}/{name}.bin", space, dim)
        labels = o.labels()
        allow = None
        if variant == "even":
            allow = (labels % 2 == 0).astype(np.uint8)
        if variant == "del":
            for lab in g[f"{name}/deleted"]:
                assert o.set_deleted(int(lab), True) == 0
        eps, mn, mx = e[key + "/params"]
        ol, od, oc = o.search_epsilon(g[f"{name}/queries"], np.float32(eps), int(mn), int(mx), allow=allow)
        assert np.array_equal(oc, e[key + "/counts"]), key
        assert np.array_equal(ol, e[key + "/labels"]), key
        assert np.array_equal(od.view(np.uint32), e[key + "/dists"].view(np.uint32)), key


def test_oracle_epsilon_search_vs_reference_fresh(tmp_path):
    """Fresh indexes against the live reference harness (skipped where it was
    not built): uniform L2, inner product and small-integer L2 with ties."""
    if O.ref_stopcond() is None:
        pytest.skip("oracle/_ref/libref_stopcond.so not built")
    rng = np.random.default_rng(21)
    for space, dim, kind in (("l2", 24, "u"), ("ip", 32, "n"), ("l2", 8, "i")):
        if kind == "u":
            x = rng.random((2500, dim), dtype=np.float32)
            q = rng.random((60, dim), dtype=np.float32)
        elif kind == "n":
            x = rng.standard_normal((2500, dim), dtype=np.float32)
            q = rng.standard_normal((60, dim), dtype=np.float32)
        else:
            x = rng.integers(0, 5, (2500, dim)).astype(np.float32)
            q = rng.integers(0, 5, (60, dim)).astype(np.float32)
        path = tmp_path / f"{space}{dim}.bin"
        build_hnsw(path, x, space, M=12, efc=80)
        o = O.Hnsw(str(path), space, dim)
        ex = np.stack([O.distances(space, q[i], x) for i in range(q.shape[0])])
        for quant, mn, mx in ((0.01, 10, 48), (0.05, 40, 200), (0.2, 0, 150)):
            eps = np.float32(np.quantile(ex, quant))
            rl, rd, rc = O.ref_epsilon_search(path, space, q, eps, mn, mx)
            ol, od, oc = o.search_epsilon(q, eps, mn, mx)
            assert np.array_equal(oc, rc) and np.array_equal(ol, rl)
            assert np.array_equal(od.view(np.uint32), rd.view(np.uint32))
            assert all(np.all(od[i, :oc[i]] <= eps) for i in range(q.shape[0]))


def test_oracle_l2_uint8_matches_reference_golden():
    """hnswlib::L2SpaceI (uint8 vectors, integer squared L2): the oracle's
    restatement against the reference's HierarchicalNSW<int> searchKnn
    outputs recorded in tests/golden/l2u8.npz (plain, filtered, with
    deletions; clustered integers, so many exact ties)."""
    e = np.load(f"{GOLDEN}/l2u8.npz")
    q = e["queries"].astype(np.float32)
    keys = sorted({k.rsplit("/", 1)[0] for k in e.keys() if "/" in k})
    assert len(keys) == 18
    for key in keys:
        ef, k, variant = key.split("_")
        ef, k = int(ef[2:]), int(k[1:])
        o = O.Hnsw(f"{GOLDEN}/hnsw_l2u8_d32.bin", "l2_uint8", 32)
        allow = None
        if variant == "even":
            allow = (o.labels() % 2 == 0).astype(np.uint8)
        if variant == "del":
            for lab in e["deleted"]:
                assert o.set_deleted(int(lab), True) == 0
        ol, od, oc = o.search(q, k, ef, mode=O.REFERENCE, allow=allow)
        rc = e[key + "/counts"]
        assert np.array_equal(oc, rc), key
        for i in range(q.shape[0]):
            assert np.array_equal(ol[i, :rc[i]], e[key + "/labels"][i, :rc[i]]), (key, i)
            assert np.array_equal(od[i, :rc[i]], e[key + "/dists"][i, :rc[i]].astype(np.float32)), (key, i)


def test_oracle_l2_uint8_vs_reference_fresh(tmp_path):
    if O.ref_l2u8() is None:
        pytest.skip("oracle/_ref/libref_l2u8.so not built")
    rng = np.random.default_rng(41)
    for dim in (16, 20, 64):
        x = rng.integers(0, 256, (2000, dim)).astype(np.uint8)
        q = rng.integers(0, 256, (50, dim)).astype(np.uint8)
        path = tmp_path / f"u{dim}.bin"
        O.ref_l2u8_build(path, x, np.arange(2000, dtype=np.uint64), M=12, efc=80)
        o = O.Hnsw(str(path), "l2_uint8", dim)
        for ef, k in ((10, 10), (64, 5)):
            rl, rd, rc = O.ref_l2u8_search(path, q, k, ef)
            ol, od, oc = o.search(q.astype(np.float32), k, ef, mode=O.REFERENCE)
            assert np.array_equal(oc, rc) and np.array_equal(ol, rl)
            assert np.array_equal(od, rd.astype(np.float32))


def test_oracle_multivector_matches_reference_golden():
    """searchStopConditionClosest with MultiVectorSearchStopCondition over a
    multi-vector L2 index (a document id after each vector): the oracle's
    restatement against the reference's recorded results (ids in result
    order, distances, counts) for four (num_docs, ef_collection) pairs."""
    e = np.load(f"{GOLDEN}/multivec.npz")
    o = O.Hnsw(f"{GOLDEN}/hnsw_mv_l2_d16.bin", "l2", 16)
    for nd, efc in ((10, 15), (5, 5), (3, 20), (20, 10)):
        key = f"docs{nd}_efc{efc}"
        ids, d, c = o.search_multivector(e["queries"], nd, efc, 400)
        assert np.array_equal(c, e[key + "/counts"]), key
        assert np.array_equal(ids, e[key + "/ids"]), key
        assert np.array_equal(d.view(np.uint32), e[key + "/dists"].view(np.uint32)), key
        # every result row holds exactly num_docs documents
        for i in range(e["queries"].shape[0]):
            assert len(set(e["docs"][ids[i, :c[i]].astype(np.int64)].tolist())) == nd


def test_oracle_multivector_vs_reference_fresh(tmp_path):
    if O.ref_multivec() is None:
        pytest.skip("oracle/_ref/libref_multivec.so not built")
    rng = np.random.default_rng(77)
    for n_docs_total, dim in ((30, 8), (200, 24)):
        x = rng.standard_normal((1500, dim)).astype(np.float32)
        docs = rng.integers(0, n_docs_total, 1500)
        q = rng.standard_normal((40, dim)).astype(np.float32)
        path = tmp_path / f"mv{dim}.bin"
        O.ref_mv_build(path, "l2", x, docs, np.arange(1500), M=12, efc=80)
        o = O.Hnsw(str(path), "l2", dim)
        for nd, efc in ((4, 8), (12, 12), (2, 30)):
            rl, rd, rc = O.ref_mv_search(path, "l2", q, nd, efc, 600)
            ol, od, oc = o.search_multivector(q, nd, efc, 600)
            assert np.array_equal(oc, rc) and np.array_equal(ol, rl)
            assert np.array_equal(od.view(np.uint32), rd.view(np.uint32))


def test_config1_uniform_10k_oracle_vs_reference(tmp_path):
    """The CPU-runnable configuration: 10,000 x 128 U[0,1) vectors
    (default_rng(0)), M=16, ef_construction=200, random_seed=100, 1,000 queries
    from the same stream, k=10, ef=50, with BFIndex exact top-10 as ground
    truth.  The oracle's reference mode returns the reference's knn_query
    results for every query, and its brute force the reference's BFIndex."""
    from hnsw_rabitq_b200.datasets import uniform_10k
    hnswlib = ref_or_skip()
    x, q = uniform_10k()
    p = build_hnsw(tmp_path / "c1.bin", x, "l2", M=16, efc=200, seed=100, num_threads=8)
    p.set_ef(50)
    rl, rd = p.knn_query(q, k=10, num_threads=8)
    o = O.Hnsw(str(tmp_path / "c1.bin"), "l2", 128)
    ol, od, _ = o.search(q, 10, 50, mode=O.REFERENCE)
    assert np.array_equal(ol, rl) and np.array_equal(od.view(np.uint32), rd.view(np.uint32))
    bf = hnswlib.BFIndex("l2", 128)
    bf.init_index(x.shape[0])
    bf.add_items(x)
    gl, gd = bf.knn_query(q, k=10)
    ml, md = O.bf_matrix("l2", x, q, 10)
    assert np.array_equal(ml, gl) and np.array_equal(md.view(np.uint32), gd.view(np.uint32))
    # i.i.d. uniform 128-d data is hard for a graph: recall@10 at ef 50 is ~0.65
    recall = np.mean([len(np.intersect1d(rl[i], gl[i])) / 10 for i in range(q.shape[0])])
    assert 0.5 < recall < 0.8
