"""Generate the golden fixtures in this directory from the reference itself.

Run in a container where the reference's own extension has been built into
oracle/_ref (``make -C oracle ref REF=<hnswlib source tree>``):

    python tests/golden/make_golden.py

It builds small indexes with hnswlib 0.9.0 (single-threaded, fixed seeds, so
the graphs are deterministic), saves them with the reference's ``save_index``
and records the reference's ``knn_query`` outputs for fixed query sets, with
and without a filter, before and after ``mark_deleted``.  Everything written
here is an output of the reference; the tests compare the CUDA path (and the
oracle) against it.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

# name, kind, space, dim, n, M, efc, data
CASES = [
    ("hnsw_l2_d16", "hnsw", "l2", 16, 800, 8, 60, "uniform"),
    ("hnsw_ip_d20", "hnsw", "ip", 20, 600, 6, 50, "normal"),
    ("hnsw_cos_d12", "hnsw", "cosine", 12, 600, 5, 40, "normal"),
    ("hnsw_l2_d7_int", "hnsw", "l2", 7, 700, 6, 40, "int"),
    ("bf_l2_d7", "bf", "l2", 7, 500, 0, 0, "normal"),
    ("bf_ip_d16", "bf", "ip", 16, 400, 0, 0, "normal"),
    ("bf_cos_d9", "bf", "cosine", 9, 300, 0, 0, "normal"),
]
EFS = [10, 32, 100]
KS = [1, 10]


def data_for(kind, n, dim, seed):
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        return rng.random((n, dim), dtype=np.float32)
    if kind == "normal":
        return rng.standard_normal((n, dim), dtype=np.float32)
    # integer-valued: many exact distance ties
    return rng.integers(0, 6, (n, dim)).astype(np.float32)


def main():
    hnswlib = O.ref_module()
    if hnswlib is None:
        raise SystemExit("oracle/_ref not built: run `make -C oracle ref REF=<hnswlib source tree>` first")
    out = {}
    for ci, (name, kind, space, dim, n, M, efc, dk) in enumerate(CASES):
        x = data_for(dk, n, dim, 100 + ci)
        q = data_for(dk, 40, dim, 200 + ci)
        path = os.path.join(HERE, name + ".bin")
        labels = (np.arange(n, dtype=np.uint64) * 3 + 7)  # non-trivial external labels
        out[f"{name}/queries"] = q
        filt = lambda l: l % 2 == 0  # noqa: E731
        if kind == "hnsw":
            p = hnswlib.Index(space, dim)
            p.init_index(n, M=M, ef_construction=efc, random_seed=100)
            p.add_items(x, labels, num_threads=1)
            p.save_index(path)
            for ef in EFS:
                p.set_ef(ef)
                for k in KS:
                    l, d = p.knn_query(q, k=k, num_threads=1)
                    out[f"{name}/ef{ef}_k{k}/labels"] = l
                    out[f"{name}/ef{ef}_k{k}/dists"] = d
                    l, d = p.knn_query(q, k=k, num_threads=1, filter=filt)
                    out[f"{name}/ef{ef}_k{k}_even/labels"] = l
                    out[f"{name}/ef{ef}_k{k}_even/dists"] = d
            dele = labels[np.random.default_rng(300 + ci).choice(n, n // 10, replace=False)]
            out[f"{name}/deleted"] = dele
            for lab in dele:
                p.mark_deleted(int(lab))
            for ef in EFS:
                p.set_ef(ef)
                l, d = p.knn_query(q, k=10, num_threads=1)
                out[f"{name}/ef{ef}_k10_del/labels"] = l
                out[f"{name}/ef{ef}_k10_del/dists"] = d
        else:
            p = hnswlib.BFIndex(space, dim)
            p.init_index(n + 50)
            p.add_items(x, labels)
            p.save_index(path)
            for k in (1, 10, 25):
                l, d = p.knn_query(q, k=k)
                out[f"{name}/k{k}/labels"] = l
                out[f"{name}/k{k}/dists"] = d
                l, d = p.knn_query(q, k=k, filter=filt)
                out[f"{name}/k{k}_even/labels"] = l
                out[f"{name}/k{k}_even/dists"] = d
    # known-answer distances: the reference's space test pattern (axis-aligned
    # rows padded with zeros on both sides, every SIMD dispatch branch)
    for space in ("l2", "ip", "cosine"):
        for left in range(0, 33, 3):
            for right in range(0, 33, 5):
                base = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1]], np.float32)
                x = np.concatenate([np.zeros((5, left), np.float32), base, np.zeros((5, right), np.float32)], 1)
                dim = x.shape[1]
                p = hnswlib.BFIndex(space, dim)
                p.init_index(5)
                p.add_items(x)
                l, d = p.knn_query(x[-1:], k=5)
                out[f"spaces/{space}/{left}_{right}/labels"] = l
                out[f"spaces/{space}/{left}_{right}/dists"] = d
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
