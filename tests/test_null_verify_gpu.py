"""On-device null-space verifier (mela_dev_null_verify): it counts the rows of
A that some basis vector does not annihilate.  Correct bases come from the
oracle; wrong ones are made on the CPU by flipping one bit of an oracle basis,
and the count must equal the host's count of rows with A_i . z != 0."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (5, 3), (33, 64), (64, 130), (100, 90), (257, 1000), (300, 700), (0, 70), (70, 0)]


def _bad_rows_host(P, m, n, Zt, f):
    if m == 0 or n == 0 or f == 0:
        return 0
    A = O.unpack(P, m, n).astype(np.int64)
    Z = O.unpack(Zt, f, n).astype(np.int64)
    return int(((A @ Z.T) % 2).any(axis=1).sum())


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int64)).cuda()


@pytest.mark.parametrize("shape", SHAPES)
def test_verifier_accepts_the_oracle_basis(cuda, shape):
    from mex_linear_algebra_b200 import device as D
    m, n = shape
    P = O.rand_dense(61, 7 * m + n, m, n)
    Zt = O.null_basis_packed(P, m, n)
    f = Zt.shape[0]
    assert D.null_verify(_dev(P), m, n, _dev(Zt), f) == 0


@pytest.mark.parametrize("shape", [s for s in SHAPES if s[0] and s[1]])
def test_verifier_counts_rows_a_wrong_basis_misses(cuda, shape):
    from mex_linear_algebra_b200 import device as D
    m, n = shape
    P = O.rand_dense(62, 7 * m + n, m, n)
    Zt = O.null_basis_packed(P, m, n)
    f = Zt.shape[0]
    if f == 0:
        pytest.skip("full column rank: no basis vector to alter")
    rng = np.random.default_rng(m * 1000 + n)
    for _ in range(3):
        Zb = Zt.copy()
        i, j = int(rng.integers(f)), int(rng.integers(n))
        Zb[i, j >> 6] ^= np.uint64(1) << np.uint64(j & 63)
        want = _bad_rows_host(P, m, n, Zb, f)
        assert D.null_verify(_dev(P), m, n, _dev(Zb), f) == want
