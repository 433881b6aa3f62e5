"""Generate tests/golden/epsilon.npz from the reference itself.

Run where the reference's stop-condition harness has been built into
oracle/_ref (``make -C oracle ref REF=<hnswlib source tree>``):

    python tests/golden/make_epsilon_golden.py

For three of the committed golden indexes (L2 uniform, inner product, and
integer-valued L2 with many exact ties) it records the reference's
``searchStopConditionClosest`` with ``EpsilonSearchStopCondition(epsilon,
min_num_candidates, max_num_candidates)`` on the fixture's queries: plain,
with the even-label filter, and with the fixture's deleted labels marked.
Epsilon is taken from quantiles of the exact query distances, so that the
regions hold from a few to a few hundred points.  Everything written here is
an output of the reference.  The recorded "labels" are what the reference
returns: internal ids, because searchStopConditionClosest copies
top_candidates' internal ids into its result unchanged.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from tests.golden import make_golden as MG  # noqa: E402

CASES = [("hnsw_l2_d16", "l2", 16), ("hnsw_ip_d20", "ip", 20), ("hnsw_l2_d7_int", "l2", 7)]
# (name, quantile of the exact distances giving epsilon, min, max)
SETTINGS = [("q02_min20_max64", 0.02, 20, 64), ("q10_min50_max128", 0.10, 50, 128), ("q005_min0_max32", 0.005, 0, 32),
            ("q30_min100_max100", 0.30, 100, 100)]


def main():
    if O.ref_stopcond() is None:
        raise SystemExit("oracle/_ref/libref_stopcond.so not built: run `make -C oracle ref REF=<hnswlib source tree>` first")
    g = np.load(os.path.join(HERE, "golden.npz"))
    out = {}
    for name, space, dim in CASES:
        path = os.path.join(HERE, name + ".bin")
        q = g[f"{name}/queries"]
        o = O.Hnsw(path, space, dim)
        labels = o.labels()
        # the fixture's vectors, regenerated as make_golden.py made them, give
        # the exact query distances that epsilon is drawn from
        ci = [c[0] for c in MG.CASES].index(name)
        _, _, _, _, n, _, _, dk = MG.CASES[ci]
        x = MG.data_for(dk, n, dim, 100 + ci)
        ex = np.stack([O.distances(space, q[i], x) for i in range(q.shape[0])])
        deleted = g[f"{name}/deleted"] if f"{name}/deleted" in g else np.zeros(0, np.uint64)
        mask = np.zeros(int(labels.max()) + 1, np.uint8)
        mask[labels[labels % 2 == 0].astype(np.int64)] = 1
        for sname, quant, mn, mx in SETTINGS:
            eps = float(np.quantile(ex, quant))
            for variant, dele, allow in (("plain", (), None), ("even", (), mask), ("del", deleted, None)):
                key = f"{name}/{sname}/{variant}"
                rl, rd, rc = O.ref_epsilon_search(path, space, q, eps, mn, mx, deleted=dele, allow_by_label=allow)
                out[key + "/labels"] = rl
                out[key + "/dists"] = rd
                out[key + "/counts"] = rc
                out[key + "/params"] = np.array([eps, mn, mx], np.float64)
    np.savez_compressed(os.path.join(HERE, "epsilon.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
