"""The six gateways against the reference's own gateways.

Every golden case (outputs and error texts of the compiled reference,
tests/golden/) goes through (a) the Python front end
``mex_linear_algebra_b200.mela`` and (b) this library's MEX gateways
(mex/*.c) driven through the non-MATLAB MEX host exactly like the reference's.
Argument errors are decided before any device work, so those cases also run
without a GPU.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
G = np.load(os.path.join(HERE, "golden", "golden.npz"))
NAMES = [str(x) for x in G["_names"]]
FUNCS = {"matmul": ("mela_matmul_gf2", "mela_matmul_m4ri"), "rank": ("mela_rank_gf2", "mela_rank_m4ri"),
         "null": ("mela_null_gf2", "mela_null_m4ri")}
MEXDIR = os.path.join(ROOT, "mex_linear_algebra_b200", "mex", "_build")


def meta(name):
    kind, nargs, sparse, nlhs = [str(x) for x in G[f"{name}/meta"]]
    args = [G[f"{name}/in{i}"] for i in range(int(nargs))]
    sp = tuple(int(x) for x in sparse.split(",") if x != "")
    return kind, args, sp, int(nlhs)


_mex = {}


def our_gateway(fn):
    if fn not in _mex:
        path = os.path.join(MEXDIR, fn + ".so")
        if not os.path.exists(path):
            from mex_linear_algebra_b200 import build
            build.build_gateways()
        L = C.CDLL(path, mode=os.RTLD_LOCAL)
        L.mexhost_call.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.POINTER(O._MxArray)), C.c_int,
                                   C.POINTER(C.POINTER(O._MxArray)), C.c_char_p, C.c_size_t,
                                   C.c_char_p, C.c_size_t]
        L.mexhost_call.restype = C.c_int
        L.mexhost_wrap.argtypes = [C.c_int, C.c_size_t, C.c_size_t, C.c_void_p, C.c_int]
        L.mexhost_wrap.restype = C.POINTER(O._MxArray)
        L.mxDestroyArray.argtypes = [C.POINTER(O._MxArray)]
        _mex[fn] = L
    return _mex[fn]


def run_python(fn, args, sparse, nlhs):
    from mex_linear_algebra_b200 import mela
    if sparse:
        import scipy.sparse as sp
        args = [sp.csc_matrix(a) if i in sparse else a for i, a in enumerate(args)]
    return mela.call(fn, *args, nlhs=nlhs)


def check_case(name, front):
    from mex_linear_algebra_b200 import mela
    kind, args, sparse, nlhs = meta(name)
    for fn in FUNCS[kind]:
        key = f"{name}/{fn}"
        if front == "python":
            try:
                got = run_python(fn, args, sparse, nlhs)
                err = None
            except mela.MexError as e:
                got, err = None, (e.identifier, e.message)
        else:
            try:
                got = O.call_gateway(our_gateway(fn), args, nlhs=nlhs, sparse=sparse)[0]
                err = None
            except O.MexError as e:
                got, err = None, (e.ident, e.msg)
        if f"{key}/err" in G:
            want_id, want_msg = [str(x) for x in G[f"{key}/err"]]
            assert err == (want_id, want_msg), (fn, err)
        else:
            assert err is None, (fn, err)
            want = G[key]
            assert got.dtype == want.dtype and got.shape == want.shape, (fn, got.dtype, got.shape)
            assert np.array_equal(got, want), fn


ERROR_CASES = [n for n in NAMES if n.startswith("err_") or n in ("empty_null_m0", "empty_null_n0")]


@pytest.mark.parametrize("front", ["python", "mex"])
@pytest.mark.parametrize("name", ERROR_CASES)
def test_gateway_errors_match_reference(name, front):
    check_case(name, front)


@pytest.mark.gpu
@pytest.mark.parametrize("front", ["python", "mex"])
@pytest.mark.parametrize("name", [n for n in NAMES if n not in ERROR_CASES])
def test_gateway_outputs_match_reference(cuda, name, front):
    check_case(name, front)


@pytest.mark.gpu
def test_gateways_against_live_reference(cuda):
    """Fresh seeded inputs, our gateways vs the reference's (when built)."""
    if not O.ref_available():
        pytest.skip("compiled reference not present")
    from mex_linear_algebra_b200 import mela
    for (m, n, seed) in [(150, 230, 1), (230, 150, 2), (64, 640, 3), (700, 700, 4)]:
        X = O.unpack(O.rand_dense(seed, 7, m, n), m, n)
        assert mela.mela_rank_gf2(X) == O.ref_call("mela_rank_gf2", X)[0][0, 0]
        assert mela.mela_rank_m4ri(X) == O.ref_call("mela_rank_m4ri", X)[0][0, 0]
        assert np.array_equal(mela.mela_null_gf2(X), O.ref_call("mela_null_gf2", X)[0])
        assert np.array_equal(mela.mela_null_m4ri(X), O.ref_call("mela_null_m4ri", X)[0])
        Y = O.unpack(O.rand_dense(seed, 8, n, 90), n, 90).astype(np.float64) * 3 - 1
        assert np.array_equal(mela.mela_matmul_gf2(X, Y), O.ref_call("mela_matmul_gf2", X, Y)[0])
        assert np.array_equal(mela.mela_matmul_m4ri(X, Y), O.ref_call("mela_matmul_m4ri", X, Y)[0])
