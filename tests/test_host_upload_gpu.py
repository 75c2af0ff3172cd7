"""Host entry points on arrays large enough for the blocked upload: the
MATLAB array goes to the device in column blocks through page-locked
staging slots (host copy of one block overlapping the upload of the last),
each block packed as it lands.  Ragged last blocks, double and logical
input, products, ranks and null spaces -- all against the oracle."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _double(seed, m, n):
    # integers in [-3, 4] and a few fractions: read as ((int)x) & 1
    rng = np.random.default_rng(seed)
    a = rng.integers(-3, 5, size=(m, n)).astype(np.float64)
    a[rng.random((m, n)) < 0.01] += 0.5
    return np.asfortranarray(a)


def _bits(a):
    if a.dtype == np.bool_:
        return a
    return (np.trunc(a).astype(np.int64) & 1).astype(np.bool_)


@pytest.mark.parametrize("shape", [(3000, 1000, 700), (1100, 2500, 130)])
def test_product_blocked_upload(cuda, shape):
    from mex_linear_algebra_b200 import mela
    m, k, n = shape
    A = _double(1, m, k)
    B = O.unpack(O.rand_dense(2, 0, k, n), k, n)  # logical
    want = O.unpack(O.matmul(O.pack(_bits(A)), O.pack(B), m, k, n), m, n)
    for _ in range(2):  # the staging slots are reused by the second call
        assert np.array_equal(mela.mela_matmul_gf2(A, B), want)


@pytest.mark.parametrize("shape,kind", [((3000, 1000), "double"), ((40000, 3000), "logical"),
                                        ((5000, 2000), "logical")])
def test_rank_and_null_blocked_upload(cuda, shape, kind):
    from mex_linear_algebra_b200 import mela
    m, n = shape
    if kind == "double":
        H = _double(3, m, n)
    else:
        L = O.rand_dense(4, 0, m, 700)
        R = O.rand_dense(4, 1, 700, n)
        H = O.unpack(O.matmul(L, R, m, 700, n), m, n)  # rank <= 700
    P = O.pack(_bits(H))
    r = O.rank(P, m, n, 10)
    assert mela.mela_rank_gf2(H) == r
    if m * n <= 40_000_000:
        Z = mela.mela_null_gf2(H)
        assert np.array_equal(Z, O.null_logical(_bits(H)))


def test_large_arrays_take_the_blocked_upload(cuda):
    """A 32 MiB double array goes through the page-locked staging slots in
    column blocks (mela_upload_stats_get), a 1 MiB one is copied directly."""
    import ctypes as C
    from mex_linear_algebra_b200 import _lib, mela
    L = _lib.lib()
    st = _lib.UploadStats()
    L.mela_upload_stats_get(C.byref(st), 1)
    A = _double(5, 2048, 2048)            # 32 MiB
    B = _double(6, 2048, 64)              # 1 MiB
    C_ = mela.mela_matmul_gf2(A, B)
    L.mela_upload_stats_get(C.byref(st), 1)
    assert st.blocked_bytes == A.nbytes and st.blocks >= 4
    assert st.direct_bytes == B.nbytes
    want = O.unpack(O.matmul(O.pack(A), O.pack(B), 2048, 2048, 64), 2048, 64)
    assert np.array_equal(C_, want)
