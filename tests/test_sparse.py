"""Sparse (CSC) input: rank and null space of a sparse matrix packed on the
GPU from MATLAB's own sparse layout.  The reference has no such path (its
gateways reject sparse arrays or misread them), so the results are checked
against the oracle on the dense form of the same matrix: repeated entries
add mod 2, double values read as ((int)x) & 1.  Argument checks run on the
host before any device work and are tested without a GPU."""
import numpy as np
import pytest

import oracle as O


def random_csc(seed, m, n, per_col, doubles=False, dup=True):
    """CSC arrays with `per_col` entries per column (some repeated) and the
    dense 0/1 matrix they stand for."""
    rng = np.random.default_rng(seed)
    colptr = [0]
    rows, vals = [], []
    dense = np.zeros((m, n), dtype=np.uint8)
    for j in range(n):
        k = int(rng.integers(0, per_col + 1))
        r = rng.integers(0, m, size=k)
        if dup and k > 1 and rng.random() < 0.3:
            r = np.concatenate([r, r[:1]])  # a repeated entry
        for i in r:
            if doubles:
                v = float(rng.choice([1.0, 2.0, 3.0, -1.0, 0.5, 7.9, -3.2]))
                bit = int(v) & 1
            else:
                v, bit = 1, 1
            rows.append(int(i))
            vals.append(v)
            dense[i, j] ^= bit
        colptr.append(len(rows))
    values = np.array(vals, dtype=np.float64) if doubles else None
    return (np.array(colptr, np.int64), np.array(rows, np.int64), values, (m, n)), dense.astype(bool)


def test_bad_csc_rejected_on_host():
    from mex_linear_algebra_b200 import _lib, mela
    bad = [
        ((np.array([1, 1], np.int64), np.array([0], np.int64), None, (2, 1)), "start at 0"),
        ((np.array([0, 2, 1], np.int64), np.array([0, 1], np.int64), None, (2, 2)), "not decrease"),
        ((np.array([0, 1], np.int64), np.array([5], np.int64), None, (2, 1)), "outside"),
    ]
    for H, msg in bad:
        with pytest.raises(_lib.MelaError) as e:
            mela.rank_csc(H)
        assert e.value.status == _lib.ERR_INVALID and msg in str(e.value)
    # empty shapes need no device
    assert mela.rank_csc((np.zeros(1, np.int64), np.zeros(0, np.int64), None, (0, 0))) == 0
    assert mela.rank_csc((np.zeros(4, np.int64), np.zeros(0, np.int64), None, (0, 3))) == 0
    assert mela.rank_csc((np.zeros(1, np.int64), np.zeros(0, np.int64), None, (5, 0))) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("shape,per_col,doubles", [((70, 130), 3, False), ((300, 600), 3, True),
                                                   ((1000, 2100), 3, False), ((64, 64), 40, True),
                                                   ((500, 40), 60, False)])
def test_sparse_rank_and_null(cuda, shape, per_col, doubles):
    from mex_linear_algebra_b200 import mela
    m, n = shape
    H, dense = random_csc(m * 31 + n, m, n, per_col, doubles)
    P = O.pack(dense)
    assert mela.rank_csc(H) == O.rank(P, m, n)
    Z = mela.null_csc(H)
    want = O.null_basis_packed(P, m, n)
    got = O.pack(np.ascontiguousarray(Z.T)) if Z.shape[1] else np.zeros((0, want.shape[1]), np.uint64)
    assert np.array_equal(got[:, :want.shape[1]], want)


@pytest.mark.gpu
def test_sparse_matches_scipy_input(cuda):
    sp = pytest.importorskip("scipy.sparse")
    from mex_linear_algebra_b200 import mela
    rng = np.random.default_rng(5)
    D = rng.random((200, 450)) < 0.02
    S = sp.csc_matrix(D)
    P = O.pack(D)
    assert mela.rank_csc(S) == O.rank(P, 200, 450)
    assert np.array_equal(mela.null_csc(S), mela.mela_null_gf2(D))


@pytest.mark.gpu
def test_device_pack_csc(cuda):
    import torch
    from mex_linear_algebra_b200 import _lib
    from gpu_util import to_host
    m, n = 333, 517
    (colptr, rowidx, values, _), dense = random_csc(9, m, n, 5, doubles=True)
    wc = (n + 63) // 64
    out = torch.empty((m, wc), dtype=torch.int64, device="cuda")
    dc = torch.from_numpy(colptr).cuda()
    dr = torch.from_numpy(rowidx).cuda()
    dv = torch.from_numpy(values).cuda()
    s = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().mela_dev_pack_csc(dc.data_ptr(), dr.data_ptr(), dv.data_ptr(), _lib.KIND_DOUBLE,
                                            m, n, out.data_ptr(), wc, s))
    assert np.array_equal(to_host(out), O.pack(dense))
