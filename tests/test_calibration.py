"""Host logic of the learned stop's calibration (learned.calibrate): over a
grid of caps and logit thresholds it returns the cheapest search whose
recall meets the target, with threshold +inf (the plain fixed-ef beam of
that cap) as the fallback and (largest cap, +inf) when nothing meets it.
The index is a stand-in whose recall and expansions are set functions of
the cap and threshold, so the choice can be checked against a brute-force
search over the same grid."""
import numpy as np
import pytest

from hnsw_rabitq_b200 import learned

NQ, K = 200, 10


class FakeIndex:
    """Answers knn_query_traced with a prescribed recall@K and mean
    expansion count for the termination model last set."""

    def __init__(self, gt, recall_fn, expansions_fn):
        self.gt = gt
        self.recall_fn, self.expansions_fn = recall_fn, expansions_fn
        self.model = None
        self.calls = []

    def set_termination_model(self, model):
        self.model = model

    def knn_query_traced(self, queries, k, ef, tie_order, precision, rerank, learned):
        t = self.model.threshold
        assert learned == np.isfinite(t)  # +inf runs the plain beam, no network
        self.calls.append((ef, t))
        r = self.recall_fn(ef, t)
        labels = self.gt.copy()
        misses = int(round((1.0 - r) * NQ * K))
        flat = labels.reshape(-1)
        flat[:misses] = 10**9 + np.arange(misses)  # labels outside the ground truth
        trace = np.zeros((NQ, 6), np.float32)
        trace[:, 2] = self.expansions_fn(ef, t)
        return labels, np.zeros((NQ, K), np.float32), np.full(NQ, K, np.int32), trace


def _model():
    return learned.TerminationModel(np.zeros(learned.N_PARAMS, np.float32), 4, float("inf"), 64, "fp8", 0)


def _gt():
    return np.arange(NQ * K, dtype=np.uint64).reshape(NQ, K)


# recall rises with the cap and falls as the threshold drops (the network
# stops earlier); expansions follow the same way
def _recall(cap, t):
    base = min(1.0, 0.80 + cap / 400.0)
    return base if not np.isfinite(t) else base - 0.01 * (6.0 - t)


def _expansions(cap, t):
    base = 1.1 * cap
    return base if not np.isfinite(t) else base - 3.0 * (6.0 - t) + 2.0  # a checkpoint costs 2


def _brute(caps, ths, target):
    best = (float("inf"), caps[-1], float("inf"))
    for cap in caps:
        for t in [float("inf")] + sorted(ths, reverse=True):
            if _recall(cap, t) >= target and _expansions(cap, t) < best[0]:
                best = (_expansions(cap, t), cap, t)
    return best[1], best[2]


@pytest.mark.parametrize("target", [0.90, 0.93, 0.95])
def test_calibration_picks_the_cheapest_point_meeting_the_target(target):
    caps, ths = [16, 32, 48, 64], list(np.linspace(6.0, -4.0, 21))
    idx = FakeIndex(_gt(), _recall, _expansions)
    cap, thr, curve = learned.calibrate(idx, np.zeros((NQ, 4), np.float32), _gt(), K, _model(), target,
                                        caps=caps, candidates=np.array(ths), cost="expansions")
    assert (cap, thr) == _brute(caps, ths, target)
    assert _recall(cap, thr) >= target
    # the curve records every point it evaluated, with its recall and cost
    for c, t, r, e, secs in curve:
        assert abs(r - _recall(c, t)) < 1e-9 and abs(e - _expansions(c, t)) < 1e-4 and secs is None


def test_calibration_falls_back_to_fixed_ef_when_the_network_costs_more():
    # a checkpoint that costs more than every stop saves: only +inf pays
    idx = FakeIndex(_gt(), _recall, lambda cap, t: 1.1 * cap + (0.0 if not np.isfinite(t) else 50.0))
    cap, thr, _ = learned.calibrate(idx, np.zeros((NQ, 4), np.float32), _gt(), K, _model(), 0.90,
                                    caps=[16, 32, 48, 64], cost="expansions")
    assert thr == float("inf") and cap == 48  # the smallest cap whose plain beam meets 0.90


def test_calibration_without_a_feasible_point_returns_the_largest_cap():
    idx = FakeIndex(_gt(), lambda cap, t: 0.5, _expansions)
    cap, thr, curve = learned.calibrate(idx, np.zeros((NQ, 4), np.float32), _gt(), K, _model(), 0.95,
                                        caps=[64, 16, 32], cost="expansions")
    assert (cap, thr) == (64, float("inf"))
    # a cap whose plain beam is far below the target tries no finite
    # threshold (each stops earlier still): one point per cap, caps in order
    assert [(c, t) for c, t, *_ in curve] == [(16, float("inf")), (32, float("inf")), (64, float("inf"))]


def test_calibration_leaves_the_model_threshold_to_the_caller():
    model = _model()
    idx = FakeIndex(_gt(), _recall, _expansions)
    learned.calibrate(idx, np.zeros((NQ, 4), np.float32), _gt(), K, model, 0.9, caps=[32], cost="expansions")
    assert model.threshold == float("inf") and model.ef_cap == 64
