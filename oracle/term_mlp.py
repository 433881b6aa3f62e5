"""CPU oracle of the early-termination network (test infrastructure only).

Float64 numpy restatement of the network the GPU trains and evaluates
(hnsw_rabitq_b200/csrc/term_train.cu, term_mlp.cuh): the forward pass, the
class-weighted binary cross-entropy and its gradient by hand-written
backpropagation, and the inference form with fp16-rounded weights.  Only the
tests import this module, to check the GPU's gradients and logits.  The
reference (hnswlib) has no such network, so there is nothing in it to pin
against; the gradient itself is pinned by a finite-difference test.

Parameter vector (float32 on the GPU, HNSWGPU_TERM_PARAMS = 5345 entries):
mu[16], inv_sigma[16], W1[64][16], b1[64], W2[64][64], b2[64], w3[64], b3.
"""
from __future__ import annotations

import numpy as np

F, H = 16, 64
OFF_MU = 0
OFF_INV_SIGMA = OFF_MU + F
OFF_W1 = OFF_INV_SIGMA + F
OFF_B1 = OFF_W1 + H * F
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
N_PARAMS = OFF_B3 + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    assert p.shape == (N_PARAMS,)
    return dict(mu=p[OFF_MU:OFF_MU + F], inv_sigma=p[OFF_INV_SIGMA:OFF_INV_SIGMA + F],
                W1=p[OFF_W1:OFF_B1].reshape(H, F), b1=p[OFF_B1:OFF_W2], W2=p[OFF_W2:OFF_B2].reshape(H, H),
                b2=p[OFF_B2:OFF_W3], w3=p[OFF_W3:OFF_B3], b3=p[OFF_B3])


def _softplus(x):
    return np.maximum(x, 0.0) + np.log1p(np.exp(-np.abs(x)))


def _f16(a):
    return np.asarray(a, np.float64).astype(np.float16).astype(np.float64)


def forward(params, feats, fp16_weights: bool = False, fp16_activations: bool = False):
    """Logits (float64) of feature rows [n, 16].  fp16_weights: round W1, W2,
    w3 to fp16 first; fp16_activations: also round the standardised features
    (in float32 arithmetic) and the first hidden layer to fp16 -- the
    operands of the search's tensor-core inference form."""
    q = unpack(params)
    W1, W2, w3 = q["W1"], q["W2"], q["w3"]
    if fp16_weights:
        W1, W2, w3 = (_f16(a) for a in (W1, W2, w3))
    if fp16_activations:
        f32 = np.asarray(feats, np.float32)
        x = _f16((f32 - q["mu"].astype(np.float32)) * q["inv_sigma"].astype(np.float32))
    else:
        x = (np.asarray(feats, np.float64) - q["mu"]) * q["inv_sigma"]
    h1 = np.maximum(x @ W1.T + q["b1"], 0.0)
    if fp16_activations:
        h1 = _f16(h1)
    h2 = np.maximum(h1 @ W2.T + q["b2"], 0.0)
    return h2 @ w3 + q["b3"]


def loss_grad(params, feats, labels, pos_weight: float = 1.0):
    """(mean loss, gradient [N_PARAMS]) of
    pos_weight * y * softplus(-logit) + (1 - y) * softplus(logit);
    mu / inv_sigma get zero gradient (they are fixed by the caller)."""
    q = unpack(params)
    x = (np.asarray(feats, np.float64) - q["mu"]) * q["inv_sigma"]
    y = np.asarray(labels, np.float64)
    n = x.shape[0]
    z1 = x @ q["W1"].T + q["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ q["W2"].T + q["b2"]
    h2 = np.maximum(z2, 0.0)
    logit = h2 @ q["w3"] + q["b3"]
    loss = np.mean(pos_weight * y * _softplus(-logit) + (1.0 - y) * _softplus(logit))
    prob = 1.0 / (1.0 + np.exp(-logit))
    dl = (pos_weight * y * (prob - 1.0) + (1.0 - y) * prob) / n
    dz2 = (dl[:, None] * q["w3"][None, :]) * (z2 > 0)
    dz1 = (dz2 @ q["W2"]) * (z1 > 0)
    g = np.zeros(N_PARAMS)
    g[OFF_W1:OFF_B1] = (dz1.T @ x).ravel()
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    g[OFF_W2:OFF_B2] = (dz2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    g[OFF_W3:OFF_B3] = h2.T @ dl
    g[OFF_B3] = dl.sum()
    return float(loss), g

