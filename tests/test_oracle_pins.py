"""Pin the oracle (CPU restatement) to the reference.

1. Known answers stated by the reference's own tests.
2. Every golden fixture (outputs of the reference gateways, tests/golden/).
3. When the compiled reference is present (oracle/_ref), live comparisons on
   more seeded inputs.
"""
import os

import numpy as np
from hypothesis import given, settings, strategies as st
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "golden.npz"))
NAMES = [str(x) for x in G["_names"]]


def meta(name):
    kind, nargs, sparse, nlhs = [str(x) for x in G[f"{name}/meta"]]
    args = [G[f"{name}/in{i}"] for i in range(int(nargs))]
    return kind, args, sparse, int(nlhs)


def mod2(a):
    a = np.asarray(a)
    if a.dtype == np.bool_:
        return a.astype(np.int64)
    return np.array([[O.lib().orc_parity_double(float(x)) for x in row] for row in a], dtype=np.int64)


# ---------------------------------------------------------------- 1. known answers
def test_kat_rank_fixed4():
    A = np.array([[1, 0, 1, 1], [0, 1, 1, 0], [1, 1, 0, 1], [0, 0, 0, 0]], dtype=bool)
    assert O.rank(O.pack(A), 4, 4) == 2          # run_ci_tests.m:62
    assert O.rank(O.pack(A), 4, 4, 10) == 2


def test_kat_rank_zero_identity():
    assert O.rank(O.pack(np.zeros((8, 8), bool)), 8, 8) == 0    # run_ci_tests.m:60
    assert O.rank(O.pack(np.eye(12, dtype=bool)), 12, 12) == 12  # run_ci_tests.m:61


def test_kat_null_fixed():
    H = np.array([[1, 0, 1, 1], [0, 1, 1, 0]], dtype=bool)      # run_ci_tests.m:78
    Z = O.null_logical(H)
    assert np.array_equal(Z.astype(int), [[1, 1], [1, 0], [1, 0], [0, 1]])


def test_kat_double_inputs():
    A = np.array([[2, 3, 4], [5, 6, 7], [8, 9, 10]], dtype=np.float64)  # run_ci_tests.m:93-97
    B = np.array([[1, 2], [3, 4], [5, 6]], dtype=np.float64)
    C = O.unpack(O.matmul(O.pack(A), O.pack(B), 3, 3, 2), 3, 2)
    assert np.array_equal(C.astype(int), [[1, 0], [0, 0], [1, 0]])
    R = np.array([[2, 3], [4, 5]], dtype=np.float64)                  # run_ci_tests.m:100-105
    assert O.rank(O.pack(R), 2, 2) == 1
    assert np.array_equal(O.null_logical(R).astype(int), [[1], [0]])


def test_kat_gf2null_examples():
    A = np.array([[0, 0, 1], [1, 1, 1], [1, 1, 0]], dtype=bool)      # gf2null/gf2null.m:9-28
    assert np.array_equal(O.null_logical(A).astype(int), [[1], [1], [0]])
    A = np.array([[0, 0, 1, 1], [0, 1, 0, 0], [0, 1, 1, 1], [0, 1, 0, 0]], dtype=bool)
    _, piv = O.rref(O.pack(A), 4, 4)                                  # gf2null/gf2rref.m:13-34
    assert list(piv + 1) == [2, 3]


def test_parity_rule():
    f = O.lib().orc_parity_double
    assert [f(x) for x in (0.0, 1.0, -1.0, 2.0, 3.5, -3.5, 2147483647.0)] == [0, 1, 1, 0, 1, 1, 1]
    assert [f(x) for x in (2147483648.0, float("nan"), float("inf"), -1e300)] == [0, 0, 0, 0]


# ---------------------------------------------------------------- 2. golden fixtures
def oracle_outputs(kind, args):
    """The oracle's answer for a golden case, in the gateway's output form."""
    if kind == "matmul":
        A, B = args
        m, k = A.shape
        n = B.shape[1]
        return O.unpack(O.matmul(O.pack(A), O.pack(B), m, k, n), m, n)
    if kind == "rank":
        (A,) = args
        m, n = A.shape
        return np.array([[float(O.rank(O.pack(A), m, n))]])
    (H,) = args
    return O.null_logical(H)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_golden(name):
    kind, args, sparse, nlhs = meta(name)
    fns = {"matmul": ("mela_matmul_gf2", "mela_matmul_m4ri"), "rank": ("mela_rank_gf2", "mela_rank_m4ri"),
           "null": ("mela_null_gf2", "mela_null_m4ri")}[kind]
    for fn in fns:
        key = f"{name}/{fn}"
        if key not in G:
            assert f"{key}/err" in G
            continue
        want = G[key]
        got = oracle_outputs(kind, args)
        assert got.shape == want.shape, (fn, got.shape, want.shape)
        assert np.array_equal(got, want), fn
        if kind == "null" and want.size:
            # A * Z = 0 and Z has full column rank (the reference's check_nullspace)
            H = mod2(args[0])
            assert not ((H @ want.astype(np.int64)) % 2).any()
            f = want.shape[1]
            assert O.rank(O.pack(want), want.shape[0], f) == f


def test_m4ri_restatements_agree_with_plain():
    for (m, n, seed) in [(300, 200, 1), (200, 300, 2), (129, 777, 3), (500, 64, 4)]:
        P = O.rand_dense(seed, 0, m, n)
        assert O.rank(P, m, n) == O.rank(P, m, n, 10) == O.rank(P, m, n, 6)
        assert np.array_equal(O.null_basis_packed(P, m, n, "gf2"), O.null_basis_packed(P, m, n, "m4ri"))
    A = O.rand_dense(5, 0, 200, 300)
    B = O.rand_dense(5, 1, 300, 150)
    assert np.array_equal(O.matmul(A, B, 200, 300, 150), O.matmul(A, B, 200, 300, 150, 8))


# ---------------------------------------------------------------- 3. live reference
ref = pytest.mark.skipif(not O.ref_available(), reason="compiled reference not present")


@ref
@pytest.mark.parametrize("shape", [(77, 150), (150, 77), (256, 256), (33, 400)])
def test_oracle_matches_reference_live(shape):
    m, n = shape
    X = O.unpack(O.rand_dense(99, m, m, n), m, n)
    for fn, k in (("mela_rank_gf2", 0), ("mela_rank_m4ri", 10)):
        assert O.ref_call(fn, X)[0][0, 0] == O.rank(O.pack(X), m, n, k)
    for fn, meth in (("mela_null_gf2", "gf2"), ("mela_null_m4ri", "m4ri")):
        assert np.array_equal(O.ref_call(fn, X)[0], O.null_logical(X, meth))
    Y = O.unpack(O.rand_dense(98, n, n, m), n, m)
    want = O.unpack(O.matmul(O.pack(X), O.pack(Y), m, n, m), m, m)
    for fn in ("mela_matmul_gf2", "mela_matmul_m4ri"):
        assert np.array_equal(O.ref_call(fn, X, Y)[0], want)


@ref
@settings(max_examples=40, deadline=None, derandomize=True)
@given(m=st.integers(1, 160), n=st.integers(1, 160), density=st.sampled_from([0.01, 0.1, 0.5, 0.9]),
       dup=st.booleans(), seed=st.integers(0, 2**31 - 1))
def test_oracle_matches_reference_random(m, n, density, dup, seed):
    """Sparse, dense and rank-deficient (duplicated rows and columns) inputs:
    the restatement and the compiled reference agree on all six functions."""
    rng = np.random.default_rng(seed)
    X = rng.random((m, n)) < density
    if dup and m > 1 and n > 1:
        X[rng.integers(m)] = X[rng.integers(m)]
        X[:, rng.integers(n)] = X[:, rng.integers(n)]
    for fn, k in (("mela_rank_gf2", 0), ("mela_rank_m4ri", 10)):
        assert O.ref_call(fn, X)[0][0, 0] == O.rank(O.pack(X), m, n, k)
    for fn, meth in (("mela_null_gf2", "gf2"), ("mela_null_m4ri", "m4ri")):
        assert np.array_equal(O.ref_call(fn, X)[0], O.null_logical(X, meth))
    p = int(rng.integers(1, 100))
    Y = rng.random((n, p)) < density
    want = O.unpack(O.matmul(O.pack(X), O.pack(Y), m, n, p), m, p)
    for fn in ("mela_matmul_gf2", "mela_matmul_m4ri"):
        assert np.array_equal(O.ref_call(fn, X, Y)[0], want)


@settings(max_examples=30, deadline=None, derandomize=True)
@given(m=st.integers(1, 200), n=st.integers(1, 300), density=st.sampled_from([0.05, 0.5]),
       seed=st.integers(0, 2**31 - 1))
def test_null_basis_read_off_the_rref(m, n, density, seed):
    """The identity the full-size null-space digest relies on
    (tests/golden/make_config_digests.py): the back-substituted basis equals
    the one read off the RREF -- vector i has bit f_i and, at pivot column
    c_p, the RREF's bit (p, f_i)."""
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location(
        "make_config_digests", os.path.join(os.path.dirname(__file__), "golden", "make_config_digests.py"))
    MD = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(MD)
    rng = np.random.default_rng(seed)
    X = rng.random((m, n)) < density
    if m > 2:
        X[rng.integers(m)] = X[rng.integers(m)]
    P = O.pack(X)
    R, piv = O.rref(P, m, n)
    want = O.null_basis_packed(P, m, n)
    got = MD.null_from_rref(R, piv, n)
    assert np.array_equal(got, want)
