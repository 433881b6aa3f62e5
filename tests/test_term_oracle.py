"""CPU checks of the early-termination pieces that need no GPU: the float64
oracle's gradient against central finite differences, the parameter layout
shared with the C ABI, and the checkpoint labelling of the training set."""
import numpy as np

from hnsw_rabitq_b200 import _capi, learned
from oracle import term_mlp as T


def _problem(seed=0, n=40):
    rng = np.random.default_rng(seed)
    f = rng.normal(size=(n, T.F)) * 2 + 1
    y = (rng.random(n) < 0.4).astype(np.float64)
    p = learned.init_params(f, seed).astype(np.float64)
    p[T.OFF_B1:T.OFF_W2] = rng.normal(0, 0.1, T.H)
    p[T.OFF_B2:T.OFF_W3] = rng.normal(0, 0.1, T.H)
    p[T.OFF_B3] = 0.3
    return p, f, y


def test_layout_matches_c_abi():
    assert T.N_PARAMS == _capi.TERM_PARAMS == learned.N_PARAMS
    assert (T.OFF_W1, T.OFF_B1, T.OFF_W2, T.OFF_B2, T.OFF_W3, T.OFF_B3) == \
        (learned.OFF_W1, learned.OFF_B1, learned.OFF_W2, learned.OFF_B2, learned.OFF_W3, learned.OFF_B3)


def test_oracle_gradient_matches_finite_differences():
    p, f, y = _problem()
    for pw in (1.0, 3.0):
        loss, g = T.loss_grad(p, f, y, pw)
        assert np.all(g[:T.OFF_W1] == 0)
        rng = np.random.default_rng(1)
        idx = np.concatenate([rng.choice(np.arange(T.OFF_W1, T.N_PARAMS), 120, replace=False), [T.OFF_B3]])
        h = 1e-6
        for i in idx:
            a, b = p.copy(), p.copy()
            a[i] += h
            b[i] -= h
            num = (T.loss_grad(a, f, y, pw)[0] - T.loss_grad(b, f, y, pw)[0]) / (2 * h)
            assert abs(num - g[i]) <= 1e-6 + 1e-5 * abs(num), (i, num, g[i])


def test_forward_matches_loss_definition():
    p, f, y = _problem(2)
    z = T.forward(p, f)
    sp = lambda v: np.logaddexp(0, v)
    want = np.mean(2.0 * y * sp(-z) + (1 - y) * sp(z))
    assert abs(T.loss_grad(p, f, y, 2.0)[0] - want) < 1e-12


class _FakeIndex:
    def __init__(self, labels):
        self._l = np.asarray(labels, np.uint64)

    def labels_by_internal_id(self):
        return self._l


def test_checkpoint_labels():
    # internal id i has label 100 + i; k = 3; the last row of each query is
    # the beam's final state
    idx = _FakeIndex(100 + np.arange(10))
    N = 0xffffffff
    ck = dict(
        ids=np.array([[[0, 1, N], [0, 1, 2], [0, 1, 3], [9, 9, 9]],
                      [[5, 6, 7], [5, 6, 8], [0, 0, 0], [0, 0, 0]]], np.uint32),
        nckpt=np.array([3, 2], np.uint32),
        feat=np.arange(2 * 4 * learned.F, dtype=np.float32).reshape(2, 4, learned.F))
    gt = np.array([[100, 101, 102], [105, 106, 107]], np.uint64)
    X, y = learned.checkpoint_dataset(idx, ck, gt)
    # query 0: final row [0,1,3] hits 2; rows hit 2, 3 -> 1, 1
    # query 1: final row [5,6,8] hits 2; row 0 hits 3 -> 1
    assert X.shape == (3, learned.F) and np.array_equal(y, [1, 1, 1])
    assert np.array_equal(X[2], ck["feat"][1, 0])
    ck["ids"][0, 2] = [0, 1, 2]  # final hits 3: only row 1 reaches it
    X, y = learned.checkpoint_dataset(idx, ck, gt)
    assert np.array_equal(y, [0, 1, 1])


def test_checkpoint_answers_rerank_order():
    """With recorded float32 distances a row's answer is its k closest
    recorded entries (equal distances by beam position), as a re-rank
    returns them; without, the first k entries."""
    N = 0xffffffff
    ids = np.array([[[7, 3, 5, 9, N]]], np.uint32)
    d = np.array([[[0.5, 0.1, 0.3, 0.1, np.inf]]], np.float32)
    assert np.array_equal(learned.checkpoint_answers({"ids": ids}, 2), [[[7, 3]]])
    assert np.array_equal(learned.checkpoint_answers({"ids": ids, "ckpt_dists": d}, 3), [[[3, 9, 5]]])
    # labels then follow the re-ranked answer
    idx = _FakeIndex(100 + np.arange(10))
    ck = dict(ids=np.concatenate([ids, ids], axis=1), ckpt_dists=np.concatenate([d, d], axis=1),
              nckpt=np.array([2], np.uint32), feat=np.zeros((1, 2, learned.F), np.float32))
    X, y = learned.checkpoint_dataset(idx, ck, np.array([[103, 109]], np.uint64))
    assert X.shape == (1, learned.F) and np.array_equal(y, [1])


class _RecordingIndex:
    def __init__(self):
        self.calls = []

    def search_checkpoints(self, queries, k, **kw):
        self.calls.append(dict(k=k, **kw))
        return {}


def test_traces_record_what_the_rerank_sees():
    """fp32 traces record the top k; a low-precision beam records its first R
    entries (R = the re-rank count, the whole beam when 0, at most the cap)
    with their float32 distances."""
    q = np.zeros((2, 4), np.float32)
    idx = _RecordingIndex()
    learned.traces(idx, q, 10, 96, 4, 32, "fp32", 0)
    learned.traces(idx, q, 10, 96, 4, 32, "fp8", 0)
    learned.traces(idx, q, 10, 96, 4, 32, "fp8", 40)
    learned.traces(idx, q, 10, 96, 4, 32, "bf16", 500)
    learned.traces(idx, q, 10, 96, 4, 32, "fp8", 4)
    c = idx.calls
    assert "ids_width" not in c[0] and not c[0].get("dists", False)
    assert [x["ids_width"] for x in c[1:]] == [96, 40, 96, 10]
    assert all(x["dists"] for x in c[1:]) and all(x["ef"] == 96 and x["period"] == 4 for x in c)
