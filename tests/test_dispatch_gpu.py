"""How a request is computed never changes what it computes.

* the tensor-core products on single CTAs and on CTA pairs (the tile field);
* the device popcount the dispatcher's density comes from;
* AUTO dispatch through an installed cost model, forced by the model's
  weights onto each configuration in turn, for products and eliminations;
* batched plans whose engine per matrix the cost model picks (with the
  densities counted on the device), against the oracle.
"""
import numpy as np
import pytest

import oracle as O
from gpu_util import to_dev, to_host, valid_words

pytestmark = pytest.mark.gpu


def _forcing_model(op_count, index):
    """Weights whose prediction is lowest for configuration `index` whatever
    the input: zero weights, output biases 10 except 0 at `index`."""
    from mex_linear_algebra_b200 import _lib
    p = np.zeros(_lib.MLP_PARAMS, dtype=np.float32)
    b3 = p[-_lib.MLP_OUT:]
    b3[:] = 10.0
    b3[index] = 0.0
    return p


@pytest.mark.parametrize("tile", [1, 2])
@pytest.mark.parametrize("base", ["tc", "tc_fp4"])
def test_tensor_core_tiles(cuda, base, tile):
    from mex_linear_algebra_b200 import _lib, device as D
    for (m, k, n) in [(300, 700, 500), (512, 1000, 256), (2048, 4096, 1024)]:
        A, B = O.rand_dense(91, m, m, k), O.rand_dense(91, k, k, n)
        v = _lib.tune(_lib.GEMM_VARIANTS[base], 0, tile)
        got = to_host(D.matmul(to_dev(A), to_dev(B), m, k, n, variant=v))
        assert np.array_equal(valid_words(got, n), O.matmul(A, B, m, k, n)), (m, k, n)


def test_popcount(cuda):
    import torch
    from mex_linear_algebra_b200 import _lib
    L = _lib.lib()
    for (m, n) in [(1, 1), (37, 65), (1000, 3000), (5, 64)]:
        P = O.rand_dense(92, m, m, n)
        d = to_dev(P)
        cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        _lib.check(L.mela_dev_popcount(d.data_ptr(), d.shape[1], m, n, cnt.data_ptr(),
                                       torch.cuda.current_stream().cuda_stream))
        want = int(np.unpackbits(P.view(np.uint8)).sum())
        assert int(cnt.item()) == want


def test_auto_through_every_product_configuration(cuda):
    from mex_linear_algebra_b200 import costmodel, device as D
    m, k, n = 1500, 1100, 1300
    A, B = O.rand_dense(93, 0, m, k), O.rand_dense(93, 1, k, n)
    want = O.matmul(A, B, m, k, n)
    try:
        for i, name in enumerate(costmodel.CONFIG_NAMES["matmul"]):
            costmodel.install(_forcing_model(6, i))
            assert costmodel.choose("matmul", m, k, n, 0.5) == name
            got = to_host(D.matmul(to_dev(A), to_dev(B), m, k, n, variant="auto"))
            assert np.array_equal(valid_words(got, n), want), name
    finally:
        costmodel.install_default()


@pytest.mark.parametrize("op", ["rank", "null"])
def test_auto_through_every_elimination_configuration(cuda, op):
    import torch
    from mex_linear_algebra_b200 import _lib, costmodel
    from test_elim_gpu import dev_null
    L = _lib.lib()
    m, n = 700, 1500
    Lr, Rr = O.rand_dense(94, 0, m, 300), O.rand_dense(94, 1, 300, n)
    P = O.matmul(Lr, Rr, m, 300, n)  # rank 300
    want_R, want_piv = O.rref(P, m, n)
    want_Z = O.null_basis_packed(P, m, n)
    s = torch.cuda.current_stream().cuda_stream
    try:
        for i, name in enumerate(costmodel.CONFIG_NAMES[op]):
            costmodel.install(_forcing_model(10, i))
            assert costmodel.choose(op, m, n, 0, 0.5) == name
            M = to_dev(P)
            rank = torch.zeros(1, dtype=torch.int64, device="cuda")
            piv = torch.empty(m, dtype=torch.int64, device="cuda")
            prow = torch.empty(m, dtype=torch.int64, device="cuda")
            wsb = L.mela_elim_workspace_size(m, n)
            ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
            fn = L.mela_dev_rref if op == "null" else L.mela_dev_rank
            _lib.check(fn(_lib.ELIM_AUTO, M.data_ptr(), M.shape[1], m, n, rank.data_ptr(), piv.data_ptr(),
                          prow.data_ptr(), ws.data_ptr(), wsb, s))
            r = int(rank.item())
            assert r == len(want_piv), name
            pv = to_host(piv)[:r].astype(np.int64)
            assert np.array_equal(pv, want_piv), name
            if op == "null":
                Zt = dev_null(M, m, n, r, pv, to_host(prow)[:r].astype(np.int64))
                assert np.array_equal(valid_words(Zt, n), want_Z), name
    finally:
        costmodel.install_default()


def test_learned_batch_engines(cuda):
    """Each engine forced through the model, and the densities counted on
    the device: bit-exact against the oracle, matrix by matrix."""
    import torch
    from mex_linear_algebra_b200 import costmodel, device as D, gen
    mats = [gen.ldpc_packed(3, b) for b in range(30)]
    mats += [(m, n, O.rand_dense(95, i, m, n)) for i, (m, n) in enumerate([(40, 90), (100, 230), (300, 700)])]
    shapes = [(m, n) for (m, n, _) in mats]
    plan0 = D.BatchPlan(shapes)
    buf = np.zeros(max(plan0.in_words, 1), dtype=np.uint64)
    for i, (m, n, P) in enumerate(mats):
        o = int(plan0.in_offsets[i])
        buf[o:o + P.size] = P.ravel()
    d_in = torch.from_numpy(buf.view(np.int64)).cuda()
    dens = plan0.densities(d_in)
    want_dens = [np.unpackbits(P.view(np.uint8)).sum() / (m * n) for (m, n, P) in mats]
    assert np.allclose(dens, want_dens, rtol=0, atol=1e-12)
    plan0.close()
    try:
        for c in range(3):
            costmodel.install(_forcing_model(3, c))
            plan = D.BatchPlan(shapes, force_class=-2, densities=dens)
            st = plan.stats()
            ranks, zt = plan.run(d_in)
            rk = to_host(ranks)
            z = to_host(zt)
            for i, (m, n, P) in enumerate(mats):
                assert rk[i] == O.rank(P, m, n), (c, i)
                assert np.array_equal(plan.basis(z, rk, i), O.null_basis_packed(P, m, n)), (c, i)
            # the forced engine took every matrix that fits it
            if c == 0:
                assert st["cta"] == len(mats)
            plan.close()
    finally:
        costmodel.install_default()


def test_trained_model_gains_live(cuda):
    """The library's compiled-in model against its fixed rule, timed live on
    held-out product requests of the mixed stream where the rule stays on
    the plain form because one dimension is under 1024 (the model sends them
    to the FP4 tensor cores on single CTAs): AUTO with the model, including
    its device density measurement, is faster in total, and bit-exact."""
    import torch
    from mex_linear_algebra_b200 import _lib, costmodel, device as D
    L = _lib.lib()
    assert L.mela_costmodel_choose(_lib.OP_MATMUL, 775, 6198, 6701, 0.1, 1, 22.2) >= 0, \
        "the library was built without its trained model"
    params = costmodel.load()
    reqs = [(775, 6198, 6701), (5695, 5715, 962), (6592, 824, 4978), (3020, 7212, 935)]

    def med(fn, reps=7):
        fn()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    t_model = t_rule = 0.0
    try:
        for (m, k, n) in reqs:
            A, B = D.rand_dense(96, 0, m, k), D.rand_dense(96, 1, k, n)
            out = {}
            for label, model in (("model", params), ("rule", None)):
                costmodel.install(model)
                C = D.empty_packed(m, n)
                wsb = D.matmul_workspace("auto", m, k, n)
                ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
                t = med(lambda: D.matmul(A, B, m, k, n, variant="auto", out=C, workspace=ws))
                out[label] = C.clone()
                if label == "model":
                    t_model += t
                else:
                    t_rule += t
            assert torch.equal(out["model"], out["rule"]), (m, k, n)
    finally:
        costmodel.install_default()
    assert t_model < 0.8 * t_rule, (t_model, t_rule)


def _density_model(op, dense_cfg, sparse_cfg):
    """Weights whose choice flips with the density feature x3 = log10(d)/3 + 1
    (predictions in log2 microseconds): y[dense_cfg] = 10 - 20 * x3,
    y[sparse_cfg] = 6, the others 10 -- dense_cfg above d = 10^-2.4 (about
    0.004), sparse_cfg below; either fixed choice loses 64 us or more at some
    density, so the dispatcher measures it."""
    from mex_linear_algebra_b200 import _lib
    IN, H1, H2, OUT = _lib.MLP_IN, _lib.MLP_H1, _lib.MLP_H2, _lib.MLP_OUT
    p = np.zeros(_lib.MLP_PARAMS, dtype=np.float32)
    oW1, ob1 = 0, IN * H1
    oW2, ob2 = ob1 + H1, ob1 + H1 + H1 * H2
    oW3 = ob2 + H2
    ob3 = oW3 + H2 * OUT
    p[oW1 + 3 * H1 + 0] = 1.0         # h1[0] = relu(x3)
    p[oW2 + 0 * H2 + 0] = 1.0         # h2[0] = relu(h1[0])
    p[oW3 + 0 * OUT + dense_cfg] = -20.0
    p[ob3:ob3 + OUT] = 10.0
    p[ob3 + sparse_cfg] = 6.0
    return p


def test_auto_measures_density_when_it_matters(cuda):
    """With a model whose choice depends on the density, the AUTO call
    counts the input's ones on the device and follows the count: dense
    input -> one configuration, sparse input -> the other (read back with
    mela_dispatch_last), with the oracle's results either way."""
    import ctypes as C
    import torch
    from mex_linear_algebra_b200 import _lib, costmodel
    L = _lib.lib()
    names = costmodel.CONFIG_NAMES["rank"]
    dense_i, sparse_i = names.index("m4ri_k8"), names.index("tc")
    m, n = 600, 1300
    s = torch.cuda.current_stream().cuda_stream
    try:
        costmodel.install(_density_model("rank", dense_i, sparse_i))
        for dens, want_i in ((0.5, dense_i), (0.002, sparse_i)):
            from mex_linear_algebra_b200 import gen
            P = gen.sparse_packed(97, 0, m, n, dens)
            M = to_dev(P)
            rank = torch.zeros(1, dtype=torch.int64, device="cuda")
            piv = torch.empty(m, dtype=torch.int64, device="cuda")
            prow = torch.empty(m, dtype=torch.int64, device="cuda")
            wsb = L.mela_elim_workspace_size(m, n)
            ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
            _lib.check(L.mela_dev_rank(_lib.ELIM_AUTO, M.data_ptr(), M.shape[1], m, n, rank.data_ptr(),
                                       piv.data_ptr(), prow.data_ptr(), ws.data_ptr(), wsb, s))
            d = C.c_double(0)
            v = L.mela_dispatch_last(C.byref(d))
            ones = int(np.unpackbits(P.view(np.uint8)).sum())
            assert abs(d.value - ones / (m * n)) < 1e-12           # measured on the device
            assert v == costmodel.config_codes("rank")[want_i], (dens, hex(v))
            assert int(rank.item()) == O.rank(P, m, n)
        # a model whose choice does not depend on the density: nothing is measured
        costmodel.install(_forcing_model(10, dense_i))
        M = to_dev(gen.sparse_packed(97, 1, m, n, 0.3))
        _lib.check(L.mela_dev_rank(_lib.ELIM_AUTO, M.data_ptr(), M.shape[1], m, n, rank.data_ptr(),
                                   piv.data_ptr(), prow.data_ptr(), ws.data_ptr(), wsb, s))
        d = C.c_double(0)
        assert L.mela_dispatch_last(C.byref(d)) == costmodel.config_codes("rank")[dense_i]
        assert d.value < 0
    finally:
        costmodel.install_default()
