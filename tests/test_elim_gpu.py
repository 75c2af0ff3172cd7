"""Rank, RREF and null space on the GPU against the oracle (bit-exact).

Every elimination form (plain per-pivot, blocked Four-Russians with 8- and
4-bit tables, single-CTA fused, tensor-core trailing update) must give the
reference's rank, its greedy pivot columns, its RREF rows and its null-space
basis.  Shapes cover word boundaries, tall and wide matrices, several
selection chunks (m > 1024), several update row tiles (m > 1024) and column
tiles, and degenerate inputs (zero, identity, all ones, duplicated rows,
low rank).
"""
import numpy as np
import pytest

import oracle as O
from gpu_util import to_dev, to_host, valid_words

pytestmark = pytest.mark.gpu

FORMS = ("plain", "m4ri", "m4ri_k4", "fused", "tc",
         # the blocked form's tuning: Four-Russians k and rows per update CTA
         "m4ri_k6", "m4ri_k7", "m4ri_k9_rt4096", "m4ri_k10_rt4096", "m4ri_k8_rt256", "m4ri_k10_rt256")


def variant_of(form):
    from mex_linear_algebra_b200 import _lib
    if form in _lib.ELIM_VARIANTS:
        return _lib.ELIM_VARIANTS[form]
    k, _, rt = form[len("m4ri_k"):].partition("_rt")
    tile = {"": 0, "256": 1, "1024": 2, "4096": 3}[rt]
    return _lib.tune(_lib.ELIM_M4RI, int(k), tile)


def dev_rref(P, m, n, form, rref=True):
    import torch
    from mex_linear_algebra_b200 import _lib
    L = _lib.lib()
    M = to_dev(P)
    mn = max(min(m, n), 1)
    rank = torch.zeros(1, dtype=torch.int64, device="cuda")
    piv = torch.full((mn,), -1, dtype=torch.int64, device="cuda")
    prow = torch.full((mn,), -1, dtype=torch.int64, device="cuda")
    wsb = L.mela_elim_workspace_size(m, n)
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
    fn = L.mela_dev_rref if rref else L.mela_dev_rank
    s = torch.cuda.current_stream().cuda_stream
    _lib.check(fn(variant_of(form), M.data_ptr(), M.shape[1], m, n, rank.data_ptr(),
                  piv.data_ptr(), prow.data_ptr(), ws.data_ptr(), wsb, s))
    r = int(rank.item())
    return M, r, to_host(piv)[:r].astype(np.int64), to_host(prow)[:r].astype(np.int64)


def dev_null(M, m, n, r, piv, prow):
    import torch
    from mex_linear_algebra_b200 import _lib
    L = _lib.lib()
    f = n - r
    ldz = (n + 63) // 64
    Zt = torch.zeros((max(f, 1), ldz), dtype=torch.int64, device="cuda")
    wsb = L.mela_null_workspace_size(n, r)
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
    dpiv = torch.from_numpy(np.ascontiguousarray(piv, dtype=np.int64)).cuda() if r else torch.zeros(1, dtype=torch.int64, device="cuda")
    dprow = torch.from_numpy(np.ascontiguousarray(prow, dtype=np.int64)).cuda() if r else torch.zeros(1, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    _lib.check(L.mela_dev_null_basis(M.data_ptr(), M.shape[1], m, n, r, dpiv.data_ptr(),
                                     dprow.data_ptr(), Zt.data_ptr(), ldz, ws.data_ptr(), wsb, s))
    return to_host(Zt)[:f]


def check_all(P, m, n, form):
    want_R, want_piv = O.rref(P, m, n)
    r = len(want_piv)
    # rank only (forward elimination)
    _, r_fwd, _, _ = dev_rref(P, m, n, form, rref=False)
    assert r_fwd == r
    # RREF
    M, rr, piv, prow = dev_rref(P, m, n, form, rref=True)
    assert rr == r
    assert np.array_equal(piv, want_piv)
    Mh = to_host(M)
    assert np.array_equal(valid_words(Mh[prow], n), valid_words(want_R[:r], n))
    # null basis
    Zt = dev_null(M, m, n, r, piv, prow)
    want_Z = O.null_basis_packed(P, m, n)
    assert np.array_equal(valid_words(Zt, n), want_Z)


SHAPES = [(1, 1), (1, 200), (200, 1), (3, 3), (64, 64), (63, 65), (65, 63), (100, 130),
          (130, 100), (256, 256), (300, 1000), (1000, 300), (1100, 700), (2100, 1500),
          (512, 4500), (40, 5000)]


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("shape", SHAPES)
def test_random(cuda, form, shape):
    m, n = shape
    check_all(O.rand_dense(31, m * 7 + n, m, n), m, n, form)


def structured():
    out = []
    out.append(("zeros", np.zeros((50, 90), bool)))
    out.append(("eye", np.eye(130, dtype=bool)))
    out.append(("ones", np.ones((70, 110), bool)))
    X = O.unpack(O.rand_dense(5, 1, 60, 200), 60, 200)
    X[30:] = X[:30]
    out.append(("duplicates", X))
    L = O.unpack(O.rand_dense(5, 2, 600, 40), 600, 40).astype(np.int64)
    R = O.unpack(O.rand_dense(5, 3, 40, 900), 40, 900).astype(np.int64)
    out.append(("lowrank", ((L @ R) % 2).astype(bool)))
    E = np.zeros((100, 300), bool)
    E[np.arange(100), 3 * np.arange(100)] = True  # pivots spread across words
    out.append(("spread", E))
    S = np.zeros((2000, 64 * 40), bool)
    rng = np.random.default_rng(3)
    for i in range(2000):  # 6 ones per row, like a parity-check matrix
        S[i, rng.choice(64 * 40, 6, replace=False)] = True
    out.append(("ldpc", S))
    return out


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("case", [c[0] for c in structured()])
def test_structured(cuda, form, case):
    X = dict(structured())[case]
    m, n = X.shape
    check_all(O.pack(X), m, n, form)


def test_forms_agree_large(cuda):
    """4096 x 8192 of rank 3000 (L*R) with 1% of rows replaced by sums of two others."""
    import torch
    from mex_linear_algebra_b200 import device as D
    m, n, r0 = 4096, 8192, 3000
    Ld = D.rand_dense(9, 0, m, r0)
    Rd = D.rand_dense(9, 1, r0, n)
    A = D.matmul(Ld, Rd, m, r0, n, variant="tc")
    Ah = to_host(A)
    rng = np.random.default_rng(9)
    for _ in range(m // 100):
        i, a, b = rng.choice(m, 3, replace=False)
        Ah[i] = Ah[a] ^ Ah[b]
    want = O.rank(Ah, m, n, 10)
    for form in FORMS:
        _, r, piv, _ = dev_rref(Ah, m, n, form, rref=False)
        assert r == want
    torch.cuda.synchronize()


def _rref_rows(M, m, n, r, prow):
    rows = to_host(M)[prow]
    return valid_words(rows, n)


@pytest.mark.parametrize("shape,rank", [((3000, 2600), None), ((2600, 3000), 1900), ((1500, 9000), None),
                                        ((5000, 700), 300)])
def test_tc_rref_matches_blocked(cuda, shape, rank):
    """The tensor-core form against the 8-bit blocked form: dense windows that
    fill after a few hundred rows, several scan chunks and update tiles, and
    low-rank inputs whose later windows hold no pivot."""
    from mex_linear_algebra_b200 import device as D
    m, n = shape
    if rank is None:
        P = O.rand_dense(41, m + n, m, n)
    else:
        L = D.rand_dense(43, 0, m, rank)
        R = D.rand_dense(43, 1, rank, n)
        P = to_host(D.matmul(L, R, m, rank, n, variant="plain"))
    for rref in (False, True):
        Ma, ra, pa, qa = dev_rref(P, m, n, "m4ri", rref=rref)
        Mb, rb, pb, qb = dev_rref(P, m, n, "tc", rref=rref)
        assert ra == rb
        assert np.array_equal(pa, pb)
        if rref:
            assert np.array_equal(_rref_rows(Ma, m, n, ra, qa), _rref_rows(Mb, m, n, rb, qb))


def test_tc_graph_replay_follows_the_data(cuda):
    """The tensor-core form replays its launch sequence as a CUDA graph from
    the second call with the same buffers on.  The sequence must not depend
    on the data: the same matrix buffer, workspace and outputs get inputs of
    full rank, lower rank and rank 0 in turn (rank and RREF), and every call
    matches the oracle."""
    import torch
    from mex_linear_algebra_b200 import _lib, device as D
    L = _lib.lib()
    m, n = 700, 1400  # six 256-column windows
    Lr = D.rand_dense(47, 0, m, 250)
    Rr = D.rand_dense(47, 1, 250, n)
    inputs = [O.rand_dense(47, 2, m, n),
              to_host(D.matmul(Lr, Rr, m, 250, n, variant="plain")),
              np.zeros((m, (n + 63) // 64), dtype=np.uint64),
              O.rand_dense(47, 3, m, n),
              to_host(D.matmul(Lr, Rr, m, 250, n, variant="plain"))]
    M = torch.empty((m, (n + 63) // 64), dtype=torch.int64, device="cuda")
    rank = torch.zeros(1, dtype=torch.int64, device="cuda")
    piv = torch.empty(m, dtype=torch.int64, device="cuda")
    prow = torch.empty(m, dtype=torch.int64, device="cuda")
    wsb = L.mela_elim_workspace_size(m, n)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    for rref in (False, True):
        fn = L.mela_dev_rref if rref else L.mela_dev_rank
        for P in inputs:
            want_R, want_piv = O.rref(P, m, n)
            M.copy_(to_dev(P))
            _lib.check(fn(_lib.ELIM_TC, M.data_ptr(), M.shape[1], m, n, rank.data_ptr(), piv.data_ptr(),
                          prow.data_ptr(), ws.data_ptr(), wsb, s))
            r = int(rank.item())
            assert r == len(want_piv)
            assert np.array_equal(to_host(piv)[:r].astype(np.int64), want_piv)
            if rref:
                rows = to_host(M)[to_host(prow)[:r].astype(np.int64)]
                assert np.array_equal(valid_words(rows, n), valid_words(want_R[:r], n))
