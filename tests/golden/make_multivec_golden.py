"""Generate the multi-vector fixtures from the reference itself.

Run where oracle/_ref/libref_multivec.so has been built (``make -C oracle ref REF=<hnswlib source tree>``):

    python tests/golden/make_multivec_golden.py

It builds an index of 1,000 vectors (dim 16, U[0,1), M=16,
ef_construction=100, seed 100), each carrying one of 50 document ids after
its vector, with the reference's HierarchicalNSW<float> over
MultiVectorL2Space<unsigned int> (single-threaded addPoint, labels 3 i + 7),
saves it as hnsw_mv_l2_d16.bin, and records the reference's
searchStopConditionClosest with MultiVectorSearchStopCondition(space,
num_docs, ef_collection) on 60 queries for four (num_docs, ef_collection)
pairs.  The results hold internal ids, as the reference returns them.  Only
the L2 space: the reference's MultiVectorInnerProductSpace never sets the
dimension its distance reads (dim_, stop_condition.h:78-141), so its results are
undefined.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

SETTINGS = [(10, 15), (5, 5), (3, 20), (20, 10)]
CAP = 400


def main():
    if O.ref_multivec() is None:
        raise SystemExit("oracle/_ref/libref_multivec.so not built: run `make -C oracle ref REF=<hnswlib source tree>` first")
    rng = np.random.default_rng(500)
    x = rng.random((1000, 16), dtype=np.float32)
    docs = rng.integers(0, 50, 1000).astype(np.uint32)
    q = rng.random((60, 16), dtype=np.float32)
    path = os.path.join(HERE, "hnsw_mv_l2_d16.bin")
    O.ref_mv_build(path, "l2", x, docs, np.arange(1000, dtype=np.uint64) * 3 + 7, M=16, efc=100)
    out = {"queries": q, "docs": docs}
    for nd, efc in SETTINGS:
        ids, d, c = O.ref_mv_search(path, "l2", q, nd, efc, CAP)
        assert (c >= 0).all()
        key = f"docs{nd}_efc{efc}"
        out[key + "/ids"], out[key + "/dists"], out[key + "/counts"] = ids, d, c
    np.savez_compressed(os.path.join(HERE, "multivec.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
