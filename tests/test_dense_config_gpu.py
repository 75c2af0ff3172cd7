"""The dense rank / null-space configuration at full size (16384 x 32768,
A = L*R of inner dimension 12000, 1% of rows replaced by XORs of two others).

Exact rank from the oracle (tests/golden/dense_rank.json, made by
make_dense_rank.py); at this size the null space is checked through
size-independent properties: A * Z = 0, nullity = n - rank, Z of full column
rank, Z equal to the identity on the free columns, and every elimination form
giving the same rank.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def build(torch):
    from mex_linear_algebra_b200 import device as D, gen
    m, r0, n = 16384, 12000, 32768
    L = D.rand_dense(2, 0, m, r0)
    R = D.rand_dense(2, 1, r0, n)
    A = D.matmul(L, R, m, r0, n, variant="tc")
    for (i, a, b) in gen.replacement_triples(m, 164):
        A[i] = A[a] ^ A[b]
    return A, m, n


def test_dense_rank_and_null_full_size(cuda):
    import torch
    from mex_linear_algebra_b200 import _lib, device as D
    golden = json.load(open(os.path.join(HERE, "golden", "dense_rank.json")))
    A, m, n = build(torch)
    # the same input bits as the oracle's
    x = int(np.bitwise_xor.reduce(A.cpu().numpy().view(np.uint64).ravel()))
    assert str(x) == golden["xor_of_all_words"]
    L = _lib.lib()
    s = torch.cuda.current_stream().cuda_stream
    wc = n // 64
    wsb = L.mela_elim_workspace_size(m, n)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    dr = torch.zeros(1, dtype=torch.int64, device="cuda")
    dpv = torch.empty(m, dtype=torch.int64, device="cuda")
    dpr = torch.empty(m, dtype=torch.int64, device="cuda")
    forms = {f: _lib.ELIM_VARIANTS[f] for f in ("m4ri", "m4ri_k4", "plain", "tc")}
    forms["m4ri_k10_rt4096"] = _lib.tune(_lib.ELIM_M4RI, 10, 3)  # the reference rank_m4ri's own k
    forms["m4ri_k6"] = _lib.tune(_lib.ELIM_M4RI, 6)
    for form, v in forms.items():
        Mx = A.clone()
        _lib.check(L.mela_dev_rank(v, Mx.data_ptr(), wc, m, n, dr.data_ptr(),
                                   dpv.data_ptr(), dpr.data_ptr(), ws.data_ptr(), wsb, s))
        assert int(dr.item()) == golden["rank"], form
    # RREF by the tensor-core form equals the blocked form's (pivots and rows)
    Mt = A.clone()
    _lib.check(L.mela_dev_rref(_lib.ELIM_TC, Mt.data_ptr(), wc, m, n, dr.data_ptr(), dpv.data_ptr(),
                               dpr.data_ptr(), ws.data_ptr(), wsb, s))
    rt = int(dr.item())
    piv_t = dpv[:rt].clone()
    rows_t = Mt[dpr[:rt]].clone()
    del Mt
    Mx = A.clone()
    _lib.check(L.mela_dev_rref(_lib.ELIM_M4RI, Mx.data_ptr(), wc, m, n, dr.data_ptr(), dpv.data_ptr(),
                               dpr.data_ptr(), ws.data_ptr(), wsb, s))
    r = int(dr.item())
    assert rt == r
    assert torch.equal(piv_t, dpv[:r])
    assert torch.equal(rows_t, Mx[dpr[:r]])
    del rows_t
    f = n - r
    Zt = torch.empty((f, wc), dtype=torch.int64, device="cuda")
    nwb = L.mela_null_workspace_size(n, r)
    nws = torch.empty(nwb, dtype=torch.uint8, device="cuda")
    _lib.check(L.mela_dev_null_basis(Mx.data_ptr(), wc, m, n, r, dpv.data_ptr(), dpr.data_ptr(),
                                     Zt.data_ptr(), wc, nws.data_ptr(), nwb, s))
    Z = D.transpose(Zt, f, n)
    prod = D.matmul(A, Z, m, n, f, variant="tc")
    assert int(prod.abs().max().item()) == 0          # A * Z = 0
    assert D.null_verify(A, m, n, Zt, f) == 0          # the same, by the on-device verifier
    # identity on the free columns: Z restricted to free rows is I
    piv = dpv[:r].cpu().numpy()
    free = np.setdiff1d(np.arange(n), piv)
    zt = Zt.cpu().numpy().view(np.uint64)
    rows = np.arange(f)
    bits = (zt[rows, free >> 6] >> (free & 63).astype(np.uint64)) & np.uint64(1)
    assert bits.all()
    # full column rank of Z (rank of Zt = f)
    Zc = Zt.clone()
    w2 = L.mela_elim_workspace_size(f, n)
    ws2 = torch.empty(w2, dtype=torch.uint8, device="cuda")
    d2 = torch.empty(f, dtype=torch.int64, device="cuda")
    d3 = torch.empty(f, dtype=torch.int64, device="cuda")
    _lib.check(L.mela_dev_rank(_lib.ELIM_M4RI, Zc.data_ptr(), wc, f, n, dr.data_ptr(), d2.data_ptr(),
                               d3.data_ptr(), ws2.data_ptr(), w2, s))
    assert int(dr.item()) == f
