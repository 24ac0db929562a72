"""Generates the golden fixtures of the aggregation setup from the
reference's own host oracle (test/support/NativeAggregationOracle.cu and
src/IO/MatrixMarket.cu of the reference, compiled from its sources by
oracle/Makefile into oracle/_ref/libref_oracle.so).

    python tests/golden/make_golden.py

Inputs are the reference sweep's sample(n) matrices (test/amg_native_test.cpp:
28-52; n in {1, 2, 4, 17, 61, 128}), the 4-point Galerkin case
(test/multigrid_operations_test.cpp:28-44) and a 1-D Poisson matrix.  For each
matrix the fixture stores the canonical form, the strength graph for
theta in {0, 0.25, 1}, the transfer for rounds in {1, 8} x absorb in
{False, True} and the Galerkin operator, exactly as the reference oracle
produced them.  A second fixture stores the reference reader's output on the
Matrix Market cases of test/matrix_market_test.cpp and test/matrix-market/
poisson.mtx (the accepted inputs), written out here as strings.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

SIZES = [1, 2, 4, 17, 61, 128]
THETAS = [0.0, 0.25, 1.0]
ROUNDS = [1, 8]

# Matrix Market inputs accepted by the reference reader (matrix_market_test.cpp:8-25)
MM_ACCEPTED = {
    "unsorted_duplicates": "%%MatrixMarket matrix coordinate real general\n% comment\n3 3 4\n3 1 2\n1 2 4\n1 2 -1\n3 3 5\n",
    "symmetric_integer": "%%MatrixMarket matrix coordinate integer symmetric\n2 2 3\n1 1 2\n2 1 -1\n2 2 3\n",
    "empty": "%%MatrixMarket matrix coordinate real general\n0 0 0\n",
    "poisson_fixture": ("%%MatrixMarket matrix coordinate real symmetric\n% Small integration fixture\n4 4 7\n"
                        "1 1 2\n2 1 -1\n2 2 2\n3 2 -1\n3 3 2\n4 3 -1\n4 4 2\n"),
}
# Inputs the reference reader rejects (matrix_market_test.cpp:27-45)
MM_REJECTED = [
    "",
    "%%MatrixMarket matrix array real general\n2 2\n",
    "%%MatrixMarket matrix coordinate complex general\n2 2 0\n",
    "%%MatrixMarket matrix coordinate real symmetric\n2 3 0\n",
    "%%MatrixMarket matrix coordinate real general\n-1 2 0\n",
    "%%MatrixMarket matrix coordinate real general\n2147483648 2 0\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n0 1 2\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 3 2\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 nan\n",
    "%%MatrixMarket matrix coordinate integer general\n2 2 1\n1 1 1.5\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 2 extra\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 0\n1 1 2\n",
    "%%MatrixMarket matrix coordinate real symmetric\n2 2 2\n1 2 1\n2 1 1\n",
]


def put(store, key, a: O.Csr):
    store[key + "/offsets"] = a.offsets.astype(np.int32)
    store[key + "/indices"] = a.indices.astype(np.int32)
    store[key + "/values"] = a.values.astype(np.float64)


def cases():
    out = {}
    for n in SIZES:
        out[f"sample{n}"] = O.sample_matrix(n)
    out["galerkin4"] = O.Csr(4, np.array([0, 2, 5, 8, 10], np.int32),
                             np.array([0, 1, 0, 1, 2, 1, 2, 3, 2, 3], np.int32),
                             np.array([2, -1, -1, 2, -1, -1, 2, -1, -1, 2], np.float64))
    o = np.concatenate([[0], np.cumsum([2] + [3] * 125 + [2])]).astype(np.int32)
    idx, val = [], []
    for i in range(127):
        for j in (i - 1, i, i + 1):
            if 0 <= j < 127:
                idx.append(j)
                val.append(2.0 if i == j else -1.0)
    out["poisson127"] = O.Csr(127, o, np.array(idx, np.int32), np.array(val, np.float64))
    return out


def main():
    if not O.ref_available():
        O.build()
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libref_oracle.so is missing: the reference sources are needed")
    store = {}
    for name, a in cases().items():
        put(store, f"{name}/input", a)
        ca = O.ref_canonical(a)
        put(store, f"{name}/canonical", ca)
        for th in THETAS:
            g = O.ref_strength(a, th)
            put(store, f"{name}/strength{th}", g)
            for rounds in ROUNDS:
                for absorb in (False, True):
                    key = f"{name}/agg_t{th}_r{rounds}_a{int(absorb)}"
                    t = O.ref_aggregate(g, rounds, absorb)
                    store[key + "/map"] = t.map
                    store[key + "/offsets"] = t.offsets
                    store[key + "/members"] = t.members
                    store[key + "/histogram"] = t.histogram
                    put(store, key + "/galerkin", O.ref_galerkin(a, t))
    np.savez_compressed(os.path.join(HERE, "aggregation_golden.npz"), **store)
    mm = {}
    for name, text in MM_ACCEPTED.items():
        m = O.ref_read_matrix_market(text)
        mm[name] = {"text": text, "rows": m.rows, "offsets": m.offsets.tolist(), "indices": m.indices.tolist(),
                    "values": m.values.tolist()}
    rejected = []
    for text in MM_REJECTED:
        try:
            O.ref_read_matrix_market(text)
            raise SystemExit(f"reference reader accepted {text!r}")
        except O.OracleError:
            rejected.append(text)
    with open(os.path.join(HERE, "matrix_market_golden.json"), "w") as f:
        json.dump({"accepted": mm, "rejected": rejected}, f, indent=1)
    print("wrote", len(store), "arrays")


if __name__ == "__main__":
    main()
