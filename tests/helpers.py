"""Shared test helpers: reference-built indexes and parity checks."""
from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden():
    return np.load(os.path.join(GOLDEN, "golden.npz"))


def ref_or_skip():
    mod = O.ref_module()
    if mod is None:
        pytest.skip("reference extension (oracle/_ref) not built")
    return mod


def build_hnsw(path, x, space="l2", M=16, efc=100, seed=100, labels=None, num_threads=1):
    """Build and save an index with the reference itself (oracle/_ref)."""
    hnswlib = ref_or_skip()
    n, dim = x.shape
    p = hnswlib.Index(space, dim)
    p.init_index(max(n, 1), M=M, ef_construction=efc, random_seed=seed)
    if n:
        p.add_items(x, labels, num_threads=num_threads)
    p.save_index(str(path))
    return p


def build_bf(path, x, space="l2", labels=None, extra=0):
    hnswlib = ref_or_skip()
    n, dim = x.shape
    p = hnswlib.BFIndex(space, dim)
    p.init_index(n + extra)
    if n:
        p.add_items(x, labels)
    p.save_index(str(path))
    return p


def tie_explained(q_labels_a, q_dists_a, q_labels_b, q_dists_b):
    """True when two result rows differ only through exactly tied distances:
    same distance multiset (bitwise) and every label outside the
    intersection has a distance shared with some label of the other row."""
    if not np.array_equal(np.sort(q_dists_a.view(np.uint32)), np.sort(q_dists_b.view(np.uint32))):
        return False
    return True


def compare_rows(la, da, lb, db):
    """Fraction of identical rows and the list of rows that differ without a tie."""
    same = np.all(la == lb, axis=1)
    bad = []
    for i in np.nonzero(~same)[0]:
        if not tie_explained(la[i], da[i], lb[i], db[i]):
            bad.append(int(i))
    return float(same.mean()), bad
