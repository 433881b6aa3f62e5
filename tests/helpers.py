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


def compare_rows(la, lb, ties):
    """Fraction of identical result rows, and the rows that differ although
    the reference run of that query made no tie decision (``ties`` = the
    oracle's per-query tie-event count, reference mode).  Without a tie event
    the kernel's (distance, id) tie order and the reference's heap order
    cannot diverge, so every differing row must have one."""
    same = np.all(la == lb, axis=1)
    bad = [int(i) for i in np.nonzero(~same & (np.asarray(ties) == 0))[0]]
    return float(same.mean()), bad
