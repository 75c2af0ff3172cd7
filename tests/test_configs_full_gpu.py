"""The benchmark configurations at full size against the checker's digests.

tests/golden/make_config_digests.py computed these results on the CPU with
the oracle (and, where it says so, with the reference's own compiled
gateways) and stored digests of them; every GPU path must reproduce them bit
for bit:

* all 20,000 parity-check matrices (seed 3): rank and null-space basis of
  each, from packed and from logical (MATLAB layout) input;
* the drop-in call mela_matmul_gf2 on the 2048 x 2048 * 2048 x 1024 double
  product (seed 0), through the gateway;
* the 16384 x 32768 rank-12000 matrix (seed 2): pivot columns, RREF rows
  and null-space basis from the tensor-core elimination.

The 32768^3 product (seed 1) is in test_gemm_gpu.py.
"""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def digest(words) -> str:
    return hashlib.blake2b(np.ascontiguousarray(words, dtype=np.uint64).tobytes(), digest_size=16).hexdigest()


def golden(name):
    return json.load(open(os.path.join(GOLDEN, "config_digests.json")))[name]


@pytest.mark.parametrize("logical", [False, True])
def test_ldpc_batch_all_20000(cuda, logical):
    import torch
    from mex_linear_algebra_b200 import device as D, gen
    g = np.load(os.path.join(GOLDEN, "ldpc_20000.npz"))
    shapes, offsets, buf = gen.ldpc_batch(20000, 3)
    plan = D.BatchPlan(shapes)
    d_in = torch.from_numpy(buf.view(np.int64)).cuda()
    if logical:
        d_in = plan.unpack_logical(d_in)
        ranks, zt = plan.run_logical(d_in)
    else:
        ranks, zt = plan.run(d_in)
    del d_in
    rk = ranks.cpu().numpy()
    z = zt.cpu().numpy().view(np.uint64)
    plan_classes = plan.stats()
    assert np.array_equal(rk, g["ranks"].astype(np.int64))
    want = g["null_digests"]
    bad = [i for i in range(len(shapes))
           if bytes.fromhex(digest(plan.basis(z, rk, i))) != want[i].tobytes()]
    plan.close()
    assert not bad, f"{len(bad)} of 20000 null-space bases differ (first {bad[:5]}); classes {plan_classes}"
    assert D.device_error_flags() == 0


def test_matmul_gateway_config(cuda):
    """mela_matmul_gf2(A, B) on double 0/1 input through the drop-in gateway."""
    import oracle as O
    from mex_linear_algebra_b200 import mela
    g = golden("matmul_gateway_2048")
    m, k, n = g["shape"]
    A = O.unpack(O.rand_dense(0, 0, m, k), m, k).astype(np.float64)
    B = O.unpack(O.rand_dense(0, 1, k, n), k, n).astype(np.float64)
    for fn in (mela.mela_matmul_gf2, mela.mela_matmul_m4ri):
        C = fn(A, B)
        assert C.dtype == np.bool_ and C.shape == (m, n)
        assert digest(O.pack(C)) == g["digest"], fn.__name__
        assert int(np.asfortranarray(C).sum()) == g["ones"]


def test_dense_config_pivots_rref_null(cuda):
    import torch
    from mex_linear_algebra_b200 import _lib
    from test_dense_config_gpu import build
    g = golden("dense_16384x32768")
    A, m, n = build(torch)
    L = _lib.lib()
    s = torch.cuda.current_stream().cuda_stream
    wc = n // 64
    wsb = L.mela_elim_workspace_size(m, n)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    dr = torch.zeros(1, dtype=torch.int64, device="cuda")
    dpv = torch.empty(m, dtype=torch.int64, device="cuda")
    dpr = torch.empty(m, dtype=torch.int64, device="cuda")
    _lib.check(L.mela_dev_rref(_lib.ELIM_TC, A.data_ptr(), wc, m, n, dr.data_ptr(), dpv.data_ptr(),
                               dpr.data_ptr(), ws.data_ptr(), wsb, s))
    r = int(dr.item())
    assert r == g["rank"]
    assert digest(dpv[:r].cpu().numpy().view(np.uint64)) == g["pivots_digest"]
    assert digest(A[dpr[:r]].cpu().numpy().view(np.uint64)) == g["rref_rows_digest"]
    f = n - r
    Zt = torch.empty((f, wc), dtype=torch.int64, device="cuda")
    nwb = L.mela_null_workspace_size(n, r)
    nws = torch.empty(nwb, dtype=torch.uint8, device="cuda")
    _lib.check(L.mela_dev_null_basis(A.data_ptr(), wc, m, n, r, dpv.data_ptr(), dpr.data_ptr(),
                                     Zt.data_ptr(), wc, nws.data_ptr(), nwb, s))
    assert f == g["nullity"]
    assert digest(Zt.cpu().numpy().view(np.uint64)) == g["null_digest"]
