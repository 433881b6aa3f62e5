"""Learned early termination of the HNSW level-0 beam.

The reference's beam (hnswlib/hnswalg.h:368-440) runs until its candidate
queue is exhausted, so every query pays for the hardest query's ef.  Here a
small network decides per query when the top-k has stopped changing:

1. ``Index.search_checkpoints`` runs the search (ef = the cap) and records,
   every `period` level-0 expansions, a 16-feature description of the beam
   and its first entries (GPU kernel, the same feature code the search uses);
2. each checkpoint is labelled 1 when stopping there loses nothing: the
   answer it would return (its top-k; for a low-precision beam, the top-k of
   the float32 re-rank of its first `rerank` entries) already holds as many
   true neighbours (exact GPU scan) as the beam's final answer;
3. the 16 -> 64 -> 64 -> 1 network is trained on the GPU (forward / backward /
   Adam kernels of libhnswgpu, float32 master weights);
4. the stop threshold on the logit is calibrated on held-out queries by
   running the learned search itself (fp16 weights, in-warp inference) and
   keeping the earliest stop whose recall@k meets the target.

With the model installed (``Index.set_termination_model``) and
``Index.learned_stop = True``, ``knn_query`` stops each query at the first
checkpoint whose logit exceeds the threshold; ef is the fallback cap.
"""
from __future__ import annotations

import ctypes as C
import json
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _capi

N_PARAMS = _capi.TERM_PARAMS
F, H = _capi.TERM_FEATURES, _capi.TERM_HIDDEN
OFF_MU, OFF_INV_SIGMA = 0, F
OFF_W1 = 2 * F
OFF_B1 = OFF_W1 + H * F
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
_NONE = 0xffffffff


@dataclass
class TerminationModel:
    """A trained network plus how it is applied."""
    params: np.ndarray            # float32 [HNSWGPU_TERM_PARAMS]
    period: int = 4               # expansions between checkpoints
    threshold: float = 0.0        # stop when logit > threshold
    ef_cap: int = 128             # ef of the learned search (the fallback cap)
    precision: str = "fp32"       # traversal precision it was trained with
    rerank: int = 0
    info: dict = field(default_factory=dict)

    def save(self, path: str) -> None:
        meta = dict(period=self.period, threshold=self.threshold, ef_cap=self.ef_cap, precision=self.precision,
                    rerank=self.rerank, info=self.info)
        np.savez(path, params=self.params, meta=json.dumps(meta))

    @staticmethod
    def load(path: str) -> "TerminationModel":
        z = np.load(path)
        meta = json.loads(str(z["meta"]))
        return TerminationModel(params=z["params"].astype(np.float32), **meta)


def init_params(feats: np.ndarray, seed: int = 0) -> np.ndarray:
    """He-initialised parameters; mu / inv_sigma standardise `feats`."""
    feats = np.asarray(feats, np.float64)
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    p[OFF_MU:OFF_MU + F] = feats.mean(0)
    p[OFF_INV_SIGMA:OFF_INV_SIGMA + F] = 1.0 / np.maximum(feats.std(0), 1e-6)
    p[OFF_W1:OFF_B1] = rng.normal(0, np.sqrt(2.0 / F), H * F)
    p[OFF_W2:OFF_B2] = rng.normal(0, np.sqrt(2.0 / H), H * H)
    p[OFF_W3:OFF_B3] = rng.normal(0, np.sqrt(1.0 / H), H)
    return p


def _hits(labels: np.ndarray, gt: np.ndarray) -> np.ndarray:
    """Number of ground-truth labels in each row: labels [..., k] against
    gt rows broadcast over the leading axes."""
    return (labels[..., :, None] == gt[..., None, :]).any(-1).sum(-1)


def recall(labels: np.ndarray, gt: np.ndarray) -> float:
    k = gt.shape[1]
    return float(_hits(labels[:, :k].astype(np.uint64), gt.astype(np.uint64)).mean() / k)


def traces(index, queries: np.ndarray, k: int, ef_cap: int, period: int, max_ckpt: int, precision: str,
           rerank: int = 0) -> dict:
    """Checkpoint traces of the search at ef = ef_cap.  A low-precision beam
    records its first R entries (R = the re-rank count the search uses: the
    whole beam when rerank is 0) with their float32 distances, so that
    checkpoint_answers sees what its re-rank would return."""
    if precision == "fp32":
        return index.search_checkpoints(queries, k, ef=ef_cap, period=period, max_ckpt=max_ckpt,
                                        precision=precision, rerank=rerank)
    width = max(k, min(int(rerank), ef_cap) if rerank else ef_cap)
    return index.search_checkpoints(queries, k, ef=ef_cap, period=period, max_ckpt=max_ckpt, precision=precision,
                                    rerank=rerank, ids_width=width, dists=True)


def checkpoint_answers(ck: dict, k: int) -> np.ndarray:
    """Internal ids [nq, R, k] each checkpoint row would return: the first k
    beam entries, or with recorded float32 distances (a low-precision beam)
    the k closest of the recorded entries (equal distances by beam position,
    as the re-rank orders them)."""
    ids = ck["ids"]
    if "ckpt_dists" not in ck or ids.shape[2] == k:
        return ids[:, :, :k]
    order = np.argsort(ck["ckpt_dists"], axis=2, kind="stable")[:, :, :k]
    return np.take_along_axis(ids, order, axis=2)


def checkpoint_dataset(index, ck: dict, gt: np.ndarray):
    """(features [n, TERM_FEATURES], labels [n]) of every recorded
    checkpoint: label 1 when the answer the checkpoint would return
    (checkpoint_answers) holds at least as many true neighbours as the beam's
    final answer (the last row of each query, itself not a sample)."""
    nq, R, _ = ck["ids"].shape
    k = gt.shape[1]
    lab_of = index.labels_by_internal_id()
    gt = gt.astype(np.uint64)
    n = ck["nckpt"].astype(np.int64)
    X, Y = [], []
    for a in range(0, nq, 512):
        b = min(nq, a + 512)
        ids = checkpoint_answers({key: v[a:b] for key, v in ck.items() if key in ("ids", "ckpt_dists")}, k)
        lab = np.where(ids == _NONE, np.uint64(2**64 - 1), lab_of[np.minimum(ids, len(lab_of) - 1)])
        hits = _hits(lab, gt[a:b, None, :])                         # [q, R]
        last = np.maximum(n[a:b] - 1, 0)
        final = hits[np.arange(b - a), last]                        # [q]
        valid = np.arange(R)[None, :] < last[:, None]               # rows before the final one
        y = (hits >= final[:, None]).astype(np.float32)
        X.append(ck["feat"][a:b][valid])
        Y.append(y[valid])
    return np.concatenate(X).astype(np.float32), np.concatenate(Y).astype(np.float32)


def train(feats: np.ndarray, labels: np.ndarray, params: Optional[np.ndarray] = None, epochs: int = 20,
          batch: int = 1024, lr: float = 2e-3, pos_weight: float = 1.0, weight_decay: float = 1e-4, seed: int = 0,
          device: int = 0):
    """Train on the GPU; returns (params float32 [N_PARAMS], per-epoch loss)."""
    feats = np.ascontiguousarray(feats, np.float32)
    labels = np.ascontiguousarray(labels, np.float32)
    p = np.array(init_params(feats, seed) if params is None else params, np.float32, copy=True)
    o = _capi.TermTrainOpts(epochs=int(epochs), batch=int(batch), lr=float(lr), pos_weight=float(pos_weight),
                            weight_decay=float(weight_decay), reserved=0, seed=int(seed))
    losses = np.zeros(max(1, int(epochs)), np.float32)
    _capi.check(_capi.lib().hnswgpu_term_train(int(device), feats.ctypes.data_as(C.c_void_p),
                                               labels.ctypes.data_as(C.c_void_p), feats.shape[0], C.byref(o),
                                               p.ctypes.data_as(C.c_void_p), losses.ctypes.data_as(C.c_void_p)))
    return p, losses[:epochs]


def loss_grad(params: np.ndarray, feats: np.ndarray, labels: np.ndarray, pos_weight: float = 1.0,
              device: int = 0):
    """Mean loss and gradient by the GPU training kernels."""
    p = np.ascontiguousarray(params, np.float32)
    f = np.ascontiguousarray(feats, np.float32)
    y = np.ascontiguousarray(labels, np.float32)
    loss = np.zeros(1, np.float32)
    g = np.zeros(N_PARAMS, np.float32)
    _capi.check(_capi.lib().hnswgpu_term_loss_grad(int(device), p.ctypes.data_as(C.c_void_p),
                                                   f.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p),
                                                   f.shape[0], float(pos_weight), loss.ctypes.data_as(C.c_void_p),
                                                   g.ctypes.data_as(C.c_void_p)))
    return float(loss[0]), g


def logits(params: np.ndarray, feats: np.ndarray, device: int = 0) -> np.ndarray:
    """Logits by the search's own in-warp inference (fp16 weights)."""
    p = np.ascontiguousarray(params, np.float32)
    f = np.ascontiguousarray(feats, np.float32)
    out = np.zeros(f.shape[0], np.float32)
    _capi.check(_capi.lib().hnswgpu_term_logits(int(device), p.ctypes.data_as(C.c_void_p),
                                                f.ctypes.data_as(C.c_void_p), f.shape[0],
                                                out.ctypes.data_as(C.c_void_p)))
    return out


def evaluate(index, queries: np.ndarray, gt: np.ndarray, k: int, model: TerminationModel, threshold: float,
             ef_cap: Optional[int] = None, timed: bool = False):
    """(recall@k, mean level-0 expansions, seconds per batch or None) of the
    learned search at this threshold and cap; `timed`: the best of 3 runs."""
    cap = int(ef_cap or model.ef_cap)
    m = TerminationModel(model.params, model.period, float(threshold), cap, model.precision, model.rerank)
    index.set_termination_model(m)
    run = lambda: index.knn_query_traced(queries, k, ef=cap, tie_order="id", precision=model.precision,
                                         rerank=model.rerank, learned=np.isfinite(threshold))
    lab, _, cnt, tr = run()
    secs = None
    if timed:
        secs = float("inf")
        for _ in range(3):
            t0 = time.perf_counter()
            run()
            secs = min(secs, time.perf_counter() - t0)
    return recall(lab, gt), float(tr[:, 2].mean()), secs


def calibrate(index, queries: np.ndarray, gt: np.ndarray, k: int, model: TerminationModel, target_recall: float,
              caps=None, candidates: Optional[np.ndarray] = None, cost: str = "time"):
    """Cap and logit threshold of the cheapest search whose recall@k on
    these queries meets the target.  A threshold of +inf is the plain
    fixed-ef search of that cap (no network evaluated), so the calibrated
    search is never slower than the best plain one it tried.  cost="time":
    measured batch time (best of 3); "expansions": mean level-0 expansions.
    Returns (cap, threshold, curve [(cap, threshold, recall, mean
    expansions, seconds)]); (max cap, +inf) when nothing meets the target."""
    caps = sorted(caps or [model.ef_cap])
    if candidates is None:
        candidates = np.linspace(6.0, -4.0, 21)
    ths = [float("inf")] + sorted((float(t) for t in candidates), reverse=True)
    curve = []
    best = (float("inf"), caps[-1], float("inf"))
    for cap in caps:
        for t in ths:
            r, e, _ = evaluate(index, queries, gt, k, model, t, cap)
            secs = None
            if r >= target_recall:
                if cost == "time":
                    secs = evaluate(index, queries, gt, k, model, t, cap, timed=True)[2]
                c = secs if cost == "time" else e
                if c < best[0]:
                    best = (c, int(cap), t)
            curve.append((int(cap), t, r, e, secs))
            if r < target_recall - 0.03:
                break  # lower thresholds stop earlier still
    return best[1], best[2], curve


def fit(index, queries: np.ndarray, k: int = 10, ef_cap: int = 64, period: int = 4, target_recall: float = 0.95,
        precision: Optional[str] = None, rerank: Optional[int] = None, holdout: float = 0.3,
        max_ckpt: Optional[int] = None, epochs: int = 20, seed: int = 0, gt: Optional[np.ndarray] = None,
        caps=None, device: int = 0, cost: str = "time"):
    """Trace (at ef = ef_cap), label, train and calibrate on `queries` (drawn
    from the query distribution; a `holdout` share is kept for the
    calibration of the cap, at most ef_cap, and threshold).  Returns
    (TerminationModel, report)."""
    precision = precision or index.precision
    rerank = index.rerank if rerank is None else rerank
    queries = np.ascontiguousarray(queries, np.float32)
    if gt is None:
        gt = index.knn_query_exact(queries, k)[0]
    n = queries.shape[0]
    perm = np.random.default_rng(seed).permutation(n)
    nh = max(1, int(round(n * holdout)))
    hold, tr = perm[:nh], perm[nh:]
    if max_ckpt is None:
        # checkpoints fall at most once per period; a beam of ef_cap rarely
        # exceeds twice ef_cap expansions
        max_ckpt = max(16, (2 * ef_cap) // period + 8)
    ck = traces(index, queries[tr], k, ef_cap, period, max_ckpt, precision, rerank)
    X, y = checkpoint_dataset(index, ck, gt[tr])
    params, losses = train(X, y, epochs=epochs, seed=seed, device=device)
    model = TerminationModel(params, period, float("inf"), ef_cap, precision, int(rerank))
    if caps is None:
        caps = [c for c in (k, 16, 24, 32, 40, 44, 48, 50, 52, 54, 56, 60, 64, 80, 96, 128, 192, 256, 384, 512)
                if k <= c <= ef_cap]
    cap, thr, curve = calibrate(index, queries[hold], gt[hold], k, model, target_recall, caps=caps, cost=cost)
    model.ef_cap, model.threshold = cap, thr
    model.info = dict(samples=int(X.shape[0]), positive=float(y.mean()), loss=[float(v) for v in losses],
                      curve=curve, trained_cap=ef_cap, target_recall=target_recall)
    index.set_termination_model(model)
    return model, model.info
