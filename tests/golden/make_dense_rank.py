"""Exact rank of the dense rank / null-space configuration, from the oracle.

A = L*R mod 2 with L 16384 x 12000 and R 12000 x 32768 (seed 2, streams 0
and 1 of the shared generator), then 164 rows (1%) replaced in order by the
XOR of two other rows (triples from mex_linear_algebra_b200.gen.
replacement_triples).  The oracle's product and Four-Russians rank run on the
CPU (about a minute on 8 cores); the result goes to dense_rank.json.

    python tests/golden/make_dense_rank.py
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import numpy as np  # noqa: E402
import oracle as O  # noqa: E402
from mex_linear_algebra_b200 import gen  # noqa: E402

M, R0, N = 16384, 12000, 32768
REPLACED = 164


def build():
    L = O.rand_dense(2, 0, M, R0)
    Rm = O.rand_dense(2, 1, R0, N)
    A = O.matmul(L, Rm, M, R0, N)
    for (i, a, b) in gen.replacement_triples(M, REPLACED):
        A[i] = A[a] ^ A[b]
    return A


def main():
    t0 = time.time()
    A = build()
    t1 = time.time()
    r = O.rank(A, M, N, 10)
    t2 = time.time()
    digest = int(np.bitwise_xor.reduce(A.ravel()))
    out = {"m": M, "n": N, "inner": R0, "replaced": REPLACED, "rank": int(r),
           "xor_of_all_words": str(digest), "seconds": {"build": t1 - t0, "rank": t2 - t1}}
    with open(os.path.join(HERE, "dense_rank.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(out)


if __name__ == "__main__":
    main()
