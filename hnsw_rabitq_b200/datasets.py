"""Seeded synthetic stand-ins for the reference's benchmark workloads.

The reference publishes no datasets for this path (its SIFT/BigANN harnesses,
``tests/cpp/sift_1b.cpp:258-262``, read files that are not shipped), so every
workload here is generated from fixed seeds with the shapes, sizes and value
distributions of the five workload definitions:

* ``uniform_10k``      10,000 x 128 i.i.d. U[0,1) base vectors (numpy
                       ``default_rng(0)``), 1,000 queries from the same stream.
* ``gmm_1m_128``       1,000,000 x 128 vectors from 1,024 isotropic Gaussian
                       components (centres U[0,255]^128, sigma 20), rounded and
                       clipped to [0,255], stored as float32; 10,000 queries.
* ``gmm_1m_768_ip``    1,000,000 x 768 unit vectors around 256 random unit
                       centres (noise of norm ~0.3); 10,000 queries.
* ``gmm_10m_96``       10,000,000 x 96 vectors from 4,096 N(0,1) centres with
                       per-component sigma log-uniform in [0.05, 0.5].

Every generator is deterministic in its arguments; ``n``/``nq`` may be reduced
for parity tests, in which case the first rows of the full-size stream are
*not* guaranteed to coincide with the full-size data (each size is its own
seeded draw).
"""
from __future__ import annotations

import numpy as np


def uniform_10k(n: int = 10_000, nq: int = 1_000, dim: int = 128, seed: int = 0):
    """U[0,1) base and query vectors drawn from one ``default_rng(seed)``."""
    rng = np.random.default_rng(seed)
    x = rng.random((n, dim), dtype=np.float32)
    q = rng.random((nq, dim), dtype=np.float32)
    return x, q


def _gmm_centres_u255(n_comp: int, dim: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).uniform(0.0, 255.0, (n_comp, dim)).astype(np.float32)


def _draw_gmm_u255(rng, centres, n, sigma, chunk=1 << 17):
    out = np.empty((n, centres.shape[1]), np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        comp = rng.integers(0, centres.shape[0], e - s)
        v = centres[comp] + rng.standard_normal((e - s, centres.shape[1]), dtype=np.float32) * sigma
        np.clip(np.rint(v, out=v), 0.0, 255.0, out=v)
        out[s:e] = v
    return out


def gmm_1m_128(n: int = 1_000_000, nq: int = 10_000, dim: int = 128, n_comp: int = 1024,
               sigma: float = 20.0, seed: int = 0):
    """Integer-valued (0..255) float32 Gaussian-mixture data and queries.

    Centres come from ``default_rng(seed + 7)``, base rows from
    ``default_rng(seed)`` and queries from ``default_rng(seed + 1)``; the
    centres are shared by both.
    """
    centres = _gmm_centres_u255(n_comp, dim, seed + 7)
    x = _draw_gmm_u255(np.random.default_rng(seed), centres, n, sigma)
    q = _draw_gmm_u255(np.random.default_rng(seed + 1), centres, nq, sigma)
    return x, q


def gmm_1m_128_queries(nq: int, stream_seed: int, dim: int = 128, n_comp: int = 1024, sigma: float = 20.0,
                       seed: int = 0) -> np.ndarray:
    """More queries from the mixture of ``gmm_1m_128(seed=seed)`` (same
    centres), drawn from ``default_rng(stream_seed)``: the training queries
    of the learned termination, disjoint from the evaluation queries when
    ``stream_seed`` differs from ``seed + 1``."""
    centres = _gmm_centres_u255(n_comp, dim, seed + 7)
    return _draw_gmm_u255(np.random.default_rng(stream_seed), centres, nq, sigma)


def _unit_rows(a: np.ndarray) -> np.ndarray:
    a /= np.linalg.norm(a, axis=1, keepdims=True).astype(np.float32)
    return a


def gmm_unit_ip(n: int = 1_000_000, nq: int = 10_000, dim: int = 768, n_comp: int = 256,
                noise: float = 0.3, seed: int = 0, chunk: int = 1 << 16, query_seed=None):
    """Unit vectors ``normalize(c + noise * g / sqrt(dim))`` around unit centres.

    ``noise`` is the expected norm of the perturbation (per-coordinate scale
    ``noise / sqrt(dim)``), so the components stay distinguishable.  Queries
    come from ``default_rng(seed + 1)``, or from ``default_rng(query_seed)``
    (another stream of the same mixture, e.g. training queries).
    """
    crng = np.random.default_rng(seed + 7)
    centres = _unit_rows(crng.standard_normal((n_comp, dim), dtype=np.float32))
    scale = np.float32(noise / np.sqrt(dim))

    def draw(rng, m):
        out = np.empty((m, dim), np.float32)
        for s in range(0, m, chunk):
            e = min(m, s + chunk)
            comp = rng.integers(0, n_comp, e - s)
            v = centres[comp] + rng.standard_normal((e - s, dim), dtype=np.float32) * scale
            out[s:e] = _unit_rows(v)
        return out

    qs = seed + 1 if query_seed is None else query_seed
    return draw(np.random.default_rng(seed), n), draw(np.random.default_rng(qs), nq)


def gmm_lognormal_sigma(n: int = 10_000_000, nq: int = 10_000, dim: int = 96, n_comp: int = 4096,
                        seed: int = 0, chunk: int = 1 << 18, query_seed=None, sigma_range=(0.05, 0.5)):
    """N(0,1) centres with per-component sigma log-uniform in `sigma_range`
    (default [0.05, 0.5]; queries: ``default_rng(seed + 1)`` or
    ``default_rng(query_seed)``)."""
    crng = np.random.default_rng(seed + 7)
    centres = crng.standard_normal((n_comp, dim), dtype=np.float32)
    lo, hi = sigma_range
    sig = np.exp(crng.uniform(np.log(lo), np.log(hi), n_comp)).astype(np.float32)

    def draw(rng, m):
        out = np.empty((m, dim), np.float32)
        for s in range(0, m, chunk):
            e = min(m, s + chunk)
            comp = rng.integers(0, n_comp, e - s)
            out[s:e] = centres[comp] + rng.standard_normal((e - s, dim), dtype=np.float32) * sig[comp, None]
        return out

    qs = seed + 1 if query_seed is None else query_seed
    return draw(np.random.default_rng(seed), n), draw(np.random.default_rng(qs), nq)
