"""Generate the uint8 L2SpaceI fixtures from the reference itself.

Run where oracle/_ref/libref_l2u8.so has been built (``make -C oracle ref REF=<hnswlib source tree>``):

    python tests/golden/make_l2u8_golden.py

It builds an index of 1,500 uint8 vectors (dim 32, M=8, ef_construction=60,
seed 100, single-threaded addPoint with labels 3 i + 7) with the reference's
HierarchicalNSW<int> over L2SpaceI, saves it as hnsw_l2u8_d32.bin, and records
the reference's searchKnn on 40 uint8 queries for ef in {10, 32, 100} and k in
{1, 10}: plain, with the even-label filter, and with every 13th element's
label marked deleted.  The vectors are clustered integers, so exact distance
ties are common.  Everything recorded is an output of the reference.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

N, DIM, NQ = 1500, 32, 40


def data(n, seed):
    rng = np.random.default_rng(seed)
    centres = rng.integers(0, 256, (12, DIM))
    x = centres[rng.integers(0, 12, n)] + rng.integers(-12, 13, (n, DIM))
    return np.clip(x, 0, 255).astype(np.uint8)


def main():
    if O.ref_l2u8() is None:
        raise SystemExit("oracle/_ref/libref_l2u8.so not built: run `make -C oracle ref REF=<hnswlib source tree>` first")
    x = data(N, 300)
    q = data(NQ, 301)
    labels = np.arange(N, dtype=np.uint64) * 3 + 7
    path = os.path.join(HERE, "hnsw_l2u8_d32.bin")
    O.ref_l2u8_build(path, x, labels, M=8, efc=60, seed=100)
    mask = np.zeros(int(labels.max()) + 1, np.uint8)
    mask[labels[labels % 2 == 0].astype(np.int64)] = 1
    deleted = labels[::13]
    out = {"queries": q, "deleted": deleted}
    for ef in (10, 32, 100):
        for k in (1, 10):
            for variant, dele, allow in (("plain", (), None), ("even", (), mask), ("del", deleted, None)):
                rl, rd, rc = O.ref_l2u8_search(path, q, k, ef, deleted=dele, allow_by_label=allow)
                key = f"ef{ef}_k{k}_{variant}"
                out[key + "/labels"], out[key + "/dists"], out[key + "/counts"] = rl, rd, rc
    np.savez_compressed(os.path.join(HERE, "l2u8.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
