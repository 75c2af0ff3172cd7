"""Generate the golden fixtures from the reference library itself.

Runs the reference's six MEX gateways -- compiled unmodified from the
reference sources by oracle/Makefile into oracle/_ref -- through the
non-MATLAB MEX host on:

* the known-answer inputs of the reference's own tests (run_ci_tests.m:42-106,
  compile_mex.m:127-366, gf2null/gf2null.m:9-28, gf2null/gf2rref.m:13-34);
* seeded random logical / double inputs at the random shapes those tests
  use (their MATLAB RNG stream is not reproducible here, so the shapes are
  kept and the bits come from the repository's splitmix64 generator);
* error cases (argument counts, classes, sparse input, dimension mismatch,
  empty input),

and stores inputs with the reference's outputs or error texts in
golden.npz.  Needs the reference tree (only to build oracle/_ref); the
fixtures are committed so the tests need neither.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402


def logical(seed, stream, m, n):
    return O.unpack(O.rand_dense(seed, stream, m, n), m, n)


def double_vals(seed, stream, m, n):
    """Integers in [-7, 8] plus a few non-integers, from the seeded words."""
    w = O.rand_dense(seed, stream, m, max(n, 1) * 8)  # plenty of bits
    bytes_ = w.view(np.uint8).reshape(m, -1)[:, :n].astype(np.int64)
    vals = (bytes_ % 16) - 7
    a = vals.astype(np.float64)
    frac = (bytes_ % 7) == 3
    a[frac] += 0.5
    return np.asfortranarray(a)


def cases():
    out = []  # (name, function, args, sparse_idx, nlhs)
    A = np.array([[1, 0, 1, 1], [0, 1, 1, 0], [1, 1, 0, 1], [0, 0, 0, 0]], dtype=bool)
    # run_ci_tests.m test_rank (:58-74)
    for nm, X in [("zeros8", np.zeros((8, 8), bool)), ("eye12", np.eye(12, dtype=bool)),
                  ("fixed4", A), ("rand17x29", logical(42, 1, 17, 29)),
                  ("rand64", logical(42, 2, 64, 64))]:
        out.append((f"rank_{nm}", "rank", (X,), (), 1))
    # run_ci_tests.m test_nullspace (:76-90)
    H = np.array([[1, 0, 1, 1], [0, 1, 1, 0]], dtype=bool)
    for nm, X in [("fixed2x4", H), ("rand16x32", logical(42, 3, 16, 32)),
                  ("rand31x47", logical(42, 4, 31, 47))]:
        out.append((f"null_{nm}", "null", (X,), (), 1))
    # run_ci_tests.m test_matmul (:42-56) and test_double_inputs (:92-106)
    out.append(("matmul_rand37x23x31", "matmul", (logical(42, 5, 37, 23), logical(42, 6, 23, 31)), (), 1))
    out.append(("matmul_zeroA", "matmul", (np.zeros((5, 7), bool), logical(42, 7, 7, 3)), (), 1))
    Ad = np.array([[2, 3, 4], [5, 6, 7], [8, 9, 10]], dtype=np.float64)
    Bd = np.array([[1, 2], [3, 4], [5, 6]], dtype=np.float64)
    out.append(("matmul_double3x3x2", "matmul", (Ad, Bd), (), 1))
    R = np.array([[2, 3], [4, 5]], dtype=np.float64)
    out.append(("rank_double2x2", "rank", (R,), (), 1))
    out.append(("null_double2x2", "null", (R,), (), 1))
    # compile_mex.m smoke tests (:127-366)
    out.append(("matmul_rand100x50x30", "matmul", (logical(43, 1, 100, 50), logical(43, 2, 50, 30)), (), 1))
    out.append(("matmul_rand256x128x64", "matmul", (logical(43, 3, 256, 128), logical(43, 4, 128, 64)), (), 1))
    out.append(("null_rand50x100", "null", (logical(43, 5, 50, 100),), (), 1))
    X = logical(43, 6, 50, 50)
    out.append(("rank_rand50", "rank", (X,), (), 1))
    out.append(("rank_rand50_T", "rank", (np.asfortranarray(X.T),), (), 1))
    out.append(("rank_zeros10", "rank", (np.zeros((10, 10), bool),), (), 1))
    out.append(("rank_eye20", "rank", (np.eye(20, dtype=bool),), (), 1))
    out.append(("matmul_double10", "matmul", (logical(43, 7, 10, 10).astype(np.float64),
                                                logical(43, 8, 10, 10).astype(np.float64)), (), 1))
    # gf2null/gf2null.m:9-28 and gf2rref.m:13-34 examples
    out.append(("null_gf2null_example", "null", (np.array([[0, 0, 1], [1, 1, 1], [1, 1, 0]], bool),), (), 1))
    out.append(("rank_gf2rref_example", "rank",
                (np.array([[0, 0, 1, 1], [0, 1, 0, 0], [0, 1, 1, 1], [0, 1, 0, 0]], bool),), (), 1))
    out.append(("null_gf2rref_example", "null",
                (np.array([[0, 0, 1, 1], [0, 1, 0, 0], [0, 1, 1, 1], [0, 1, 0, 0]], bool),), (), 1))
    # seeded random shapes around word boundaries, logical and double
    shapes = [(1, 1), (1, 64), (64, 1), (63, 65), (65, 63), (100, 130), (130, 100),
              (128, 128), (200, 300), (257, 129)]
    for i, (m, n) in enumerate(shapes):
        out.append((f"rank_rand{m}x{n}", "rank", (logical(44, i, m, n),), (), 1))
        out.append((f"null_rand{m}x{n}", "null", (logical(45, i, m, n),), (), 1))
        out.append((f"rank_dbl{m}x{n}", "rank", (double_vals(46, i, m, n),), (), 1))
        out.append((f"null_dbl{m}x{n}", "null", (double_vals(47, i, m, n),), (), 1))
    for i, (m, k, n) in enumerate([(1, 1, 1), (3, 70, 5), (64, 64, 64), (65, 127, 129),
                                   (300, 200, 100), (17, 500, 33)]):
        out.append((f"matmul_rand{m}x{k}x{n}", "matmul", (logical(48, 2 * i, m, k), logical(48, 2 * i + 1, k, n)), (), 1))
        out.append((f"matmul_dbl{m}x{k}x{n}", "matmul", (double_vals(49, 2 * i, m, k), double_vals(49, 2 * i + 1, k, n)), (), 1))
    # low-rank and structured inputs
    L = logical(50, 1, 120, 20).astype(np.uint8)
    Rr = logical(50, 2, 20, 90).astype(np.uint8)
    low = ((L.astype(np.int64) @ Rr.astype(np.int64)) % 2).astype(bool)
    out.append(("rank_lowrank120x90", "rank", (np.asfortranarray(low),), (), 1))
    out.append(("null_lowrank120x90", "null", (np.asfortranarray(low),), (), 1))
    dup = logical(50, 3, 40, 70)
    dup[20:] = dup[:20]
    out.append(("null_duprows40x70", "null", (np.asfortranarray(dup),), (), 1))
    out.append(("null_ones30x40", "null", (np.ones((30, 40), bool),), (), 1))
    # error cases
    X = logical(51, 1, 6, 7)
    out.append(("err_matmul_nargin", "matmul", (X,), (), 1))
    out.append(("err_matmul_nlhs", "matmul", (X, logical(51, 2, 7, 3)), (), 2))
    out.append(("err_matmul_sparse", "matmul", (X, logical(51, 2, 7, 3)), (1,), 1))
    out.append(("err_matmul_dims", "matmul", (X, logical(51, 2, 6, 3)), (), 1))
    out.append(("err_matmul_type", "matmul", (X.astype(np.float32), logical(51, 2, 7, 3)), (), 1))
    out.append(("err_rank_nargin", "rank", (X, X), (), 1))
    out.append(("err_rank_type", "rank", (X.astype(np.int32),), (), 1))
    out.append(("err_null_nargin", "null", (X, X), (), 1))
    out.append(("err_null_nlhs", "null", (X,), (), 2))
    out.append(("err_null_sparse", "null", (X,), (0,), 1))
    out.append(("err_null_type", "null", (X.astype(np.float32),), (), 1))
    out.append(("empty_null_m0", "null", (np.zeros((0, 5), bool),), (), 1))
    out.append(("empty_null_n0", "null", (np.zeros((5, 0), bool),), (), 1))
    out.append(("empty_rank_m0", "rank", (np.zeros((0, 5), bool),), (), 1))
    out.append(("empty_matmul_m0", "matmul", (np.zeros((0, 5), bool), logical(51, 3, 5, 4)), (), 1))
    out.append(("empty_matmul_k0", "matmul", (np.zeros((3, 0), bool), np.zeros((0, 4), bool)), (), 1))
    return out


VARIANTS = {"matmul": ("mela_matmul_gf2", "mela_matmul_m4ri"),
            "rank": ("mela_rank_gf2", "mela_rank_m4ri"),
            "null": ("mela_null_gf2", "mela_null_m4ri")}


def main():
    store = {}
    names = []
    for (name, kind, args, sparse, nlhs) in cases():
        names.append(name)
        for i, a in enumerate(args):
            store[f"{name}/in{i}"] = np.asfortranarray(a)
        store[f"{name}/meta"] = np.array([kind, str(len(args)), ",".join(map(str, sparse)), str(nlhs)])
        for fn in VARIANTS[kind]:
            try:
                outs = O.ref_call(fn, *args, nlhs=nlhs, sparse=sparse)
                o = outs[0]
                store[f"{name}/{fn}"] = np.asfortranarray(o)
            except O.MexError as e:
                store[f"{name}/{fn}/err"] = np.array([e.ident, e.msg])
    store["_names"] = np.array(names)
    path = os.path.join(HERE, "golden.npz")
    np.savez_compressed(path, **store)
    print(f"{len(names)} cases -> {path} ({os.path.getsize(path)} bytes)")


if __name__ == "__main__":
    main()
