"""The cost-model MLP: oracle self-check, GPU kernels against the oracle,
training, and what the trained model gains over the fixed rule."""
import json
import os

import numpy as np
import pytest

import mlp_oracle as MO

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DATA = os.path.join(ROOT, "mex_linear_algebra_b200", "data")


def _data(n=300, seed=1):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, MO.IN)).astype(np.float32)
    T = rng.normal(size=(n, MO.OUT)).astype(np.float32)
    M = (rng.random((n, MO.OUT)) < 0.8).astype(np.float32)
    return X, T, M


def test_oracle_gradient_matches_finite_differences():
    X, T, M = _data(40)
    p = MO.init(3)
    _, g = MO.loss_and_grad(p, X, T, M)
    gn = MO.numeric_grad(p, X, T, M)
    assert np.allclose(g, gn, rtol=1e-4, atol=1e-7)


def test_parameter_count_matches_library():
    from mex_linear_algebra_b200 import _lib
    assert MO.NPARAMS == _lib.MLP_PARAMS


def test_features_are_scaled_log_shapes():
    from mex_linear_algebra_b200 import costmodel
    x = costmodel.features("matmul", 1024, 2048, 4096, 0.01)
    assert np.allclose(x, [10 / 14, 11 / 14, 12 / 14, -2 / 3 + 1, 0, 0, 1, 0, 0, 21 / 28], atol=1e-6)
    x = costmodel.features("null", 32, 8192, 0, 0.5)
    assert x[2] == 0 and x[5] == 1 and x[6] == 0 and x[7] == 0 and x[8] == 0
    # batch mix: 4096 matrices of mean log2(m*n) 19.5
    x = costmodel.features("batch", 700, 1500, 0, 0.004, 4096, 19.5)
    assert x[7] == 1 and np.isclose(x[8], 12 / 16) and np.isclose(x[9], 19.5 / 28)


def test_configurations_match_the_library():
    """The Python names and the library's configuration table agree, and
    every configuration is a valid variant argument."""
    from mex_linear_algebra_b200 import _lib, costmodel
    L = _lib.lib()
    tune = _lib.tune
    assert costmodel.config_codes("rank") == (
        _lib.ELIM_PLAIN, _lib.ELIM_M4RI_K4, tune(_lib.ELIM_M4RI, 6), tune(_lib.ELIM_M4RI, 7),
        tune(_lib.ELIM_M4RI, 8), tune(_lib.ELIM_M4RI, 8, 1), tune(_lib.ELIM_M4RI, 9, 3),
        tune(_lib.ELIM_M4RI, 10, 3), _lib.ELIM_FUSED, _lib.ELIM_TC)
    assert costmodel.config_codes("null") == costmodel.config_codes("rank")
    assert costmodel.config_codes("matmul") == (
        _lib.GEMM_PLAIN, _lib.GEMM_M4RI, tune(_lib.GEMM_M4RI, 0, 1), tune(_lib.GEMM_TC, 0, 2),
        tune(_lib.GEMM_TC, 0, 1), tune(_lib.GEMM_TC_FP4, 0, 2), tune(_lib.GEMM_TC_FP4, 0, 1))
    assert costmodel.config_codes("batch") == (0, 1, 2)
    for op in ("rank", "matmul", "batch"):
        assert len(costmodel.CONFIG_NAMES[op]) == L.mela_costmodel_config_count(costmodel.OPS[op])
        assert L.mela_costmodel_config(costmodel.OPS[op], len(costmodel.CONFIG_NAMES[op])) == -1
    for v in costmodel.config_codes("matmul"):
        # the Four-Russians product needs no workspace; every other form does
        assert (L.mela_matmul_workspace_size(v, 2048, 2048, 2048) > 0) == (_lib.GEMM_M4RI != (v & 0xff))


def test_bad_tuning_fields_are_rejected_before_device_work():
    """Out-of-range tuning fields fail with MELA_ERR_INVALID up front (no
    device is touched: fake pointers are never dereferenced)."""
    import ctypes as C
    from mex_linear_algebra_b200 import _lib
    L = _lib.lib()
    tune = _lib.tune
    fake = C.c_void_p(64)
    bad_elim = [tune(_lib.ELIM_M4RI, 5), tune(_lib.ELIM_M4RI, 11), tune(_lib.ELIM_M4RI_K4, 8),
                tune(_lib.ELIM_M4RI, 8, 4), tune(_lib.ELIM_TC, 8), tune(_lib.ELIM_PLAIN, 0, 1), 1 << 16, 6]
    for v in bad_elim:
        for fn in (L.mela_dev_rank, L.mela_dev_rref):
            assert fn(v, fake, 2, 100, 100, fake, fake, fake, fake, 1 << 20, None) == _lib.ERR_INVALID, hex(v)
    bad_gemm = [tune(_lib.GEMM_TC, 0, 3), tune(_lib.GEMM_M4RI, 6), tune(_lib.GEMM_M4RI, 0, 3),
                tune(_lib.GEMM_PLAIN, 0, 1), 5]
    for v in bad_gemm:
        assert L.mela_dev_matmul(v, fake, 2, fake, 2, fake, 2, 100, 100, 100, fake, 1 << 30, None) \
            == _lib.ERR_INVALID, hex(v)
        assert L.mela_matmul_workspace_size(v, 100, 100, 100) == 0


@pytest.mark.gpu
def test_gpu_forward_matches_oracle(cuda):
    from mex_linear_algebra_b200 import costmodel
    X, _, _ = _data(1000)
    p = MO.init(5).astype(np.float32)
    y_gpu = costmodel.predict(p, X)
    y_cpu, _ = MO.forward(p, X)
    assert np.allclose(y_gpu, y_cpu, rtol=1e-4, atol=1e-4)


@pytest.mark.gpu
def test_gpu_gradient_matches_oracle(cuda):
    import torch
    from mex_linear_algebra_b200 import _lib
    X, T, M = _data(700)
    p = MO.init(7).astype(np.float32)
    loss_cpu, g_cpu = MO.loss_and_grad(p, X, T, M)
    L = _lib.lib()
    dP, dX, dT, dM = (torch.from_numpy(a).cuda() for a in (p, X, T, M))
    G = torch.zeros_like(dP)
    ls = torch.zeros(1, device="cuda")
    inv = 1.0 / float(M.sum())
    _lib.check(L.mela_mlp_gradient(dP.data_ptr(), dX.data_ptr(), dT.data_ptr(), dM.data_ptr(), len(X),
                                   inv, G.data_ptr(), ls.data_ptr(), torch.cuda.current_stream().cuda_stream))
    g_gpu = G.cpu().numpy()
    assert abs(ls.item() * inv - loss_cpu) < 1e-4 * max(1.0, loss_cpu)
    assert np.allclose(g_gpu, g_cpu, rtol=2e-3, atol=2e-5)


@pytest.mark.gpu
def test_training_fits_a_timing_surface(cuda):
    """Synthetic timings with a known crossover: the trained model must pick
    the faster variant almost everywhere."""
    from mex_linear_algebra_b200 import costmodel
    rng = np.random.default_rng(0)
    recs = []
    for i in range(600):
        m, n = (int(x) for x in np.exp(rng.uniform(np.log(32), np.log(8192), 2)))
        d = float(np.exp(rng.uniform(np.log(1e-3), np.log(0.5))))
        lg = np.log2(m) + np.log2(n)
        t = {"plain": 2 ** (0.9 * lg - 3), "m4ri_k8": 2 ** (0.6 * lg + 1), "m4ri_k4": 2 ** (0.7 * lg)}
        recs.append({"op": "rank", "m": m, "n": n, "p": 0, "density": d, "times_us": t})
    params, loss = costmodel.train(recs[:400], steps=2500)
    rep = costmodel.evaluate(params, recs[400:])
    assert loss < 0.05
    assert rep["regret"] < 0.05


@pytest.mark.skipif(not os.path.exists(os.path.join(DATA, "autotune_eval.json")),
                    reason="no timing database recorded yet")
def test_trained_model_beats_fixed_rule():
    """On held-out requests with every configuration timed (recorded on B200
    by the autotuner), the installed model's choices cost less in total than
    the fixed rule's, and its regret against the exhaustive best is smaller.
    Host-side inference through the library's dispatcher; no GPU needed."""
    from mex_linear_algebra_b200 import costmodel
    params = costmodel.load()
    ev = json.load(open(os.path.join(DATA, "autotune_eval.json")))
    assert all(r["agree"] for r in ev)  # every configuration returned the same bits
    costmodel.install(params)
    try:
        tot_model = tot_rule = tot_best = 0.0
        per_model, per_rule = [], []
        for r in ev:
            t = r["times_us"]
            best = min(t.values())
            # batch engines: among those the matrices fit (the ones timed), as the library does
            among = list(t) if r["op"] == "batch" else None
            tm = t[costmodel.choose(r["op"], r["m"], r["n"], r.get("p", 0), r["density"],
                                    r.get("batch_count", 1), r.get("batch_log2_cells"), among=among)]
            tr = t[costmodel.heuristic(r["op"], r["m"], r["n"], r.get("p", 0), r["density"], r.get("rule"))]
            tot_best += best
            tot_model += tm
            tot_rule += tr
            per_model.append(tm / best - 1)
            per_rule.append(tr / best - 1)
    finally:
        costmodel.install_default()
    assert tot_model < tot_rule
    assert tot_model / tot_best - 1 < tot_rule / tot_best - 1
    # per request, too: the mean slowdown against the exhaustive best shrinks
    assert np.mean(per_model) < np.mean(per_rule)


def test_dispatch_plan_before_the_data():
    """What AUTO decides before seeing the data, recomputed from the model's
    own predictions at the four probe densities: the configuration with the
    smallest worst-case predicted loss, and a density read-back only when
    that loss exceeds 15 microseconds.  Host-side, no GPU."""
    import ctypes as C
    from mex_linear_algebra_b200 import _lib, costmodel, gen
    L = _lib.lib()
    costmodel.install_default()
    if L.mela_costmodel_choose(_lib.OP_RANK, 100, 100, 0, 0.5, 1, 13.3) < 0:
        pytest.skip("the library was built without a trained model")
    probes = (0.001, 0.01, 0.1, 0.5)
    for r in gen.mixed_stream(400, 4)[::7]:
        op, m, n, p = r["op"], r["m"], r["n"], r.get("p", 0)
        ys = [costmodel.predict_host(op, m, n, p, d) for d in probes]
        names = costmodel.CONFIG_NAMES[op]
        best = [min(2.0 ** v for v in y.values()) for y in ys]
        loss = {c: max(2.0 ** y[c] - b for y, b in zip(ys, best)) for c in names}
        want = min(names, key=lambda c: loss[c])
        meas = C.c_int32(-1)
        got = L.mela_costmodel_plan(costmodel.OPS[op], m, n, p, C.byref(meas))
        assert names[got] == want or abs(loss[names[got]] - loss[want]) < 1e-3 * max(1.0, loss[want]), (r, want)
        assert meas.value == int(loss[names[got]] > 15.0)



def test_request_generators_and_stratified_sampling():
    """The timing database's request sources: the size-stratified pick keeps
    the largest requests, and the batch requests stay within their bounds."""
    from mex_linear_algebra_b200 import autotune, gen
    window = gen.mixed_stream(100000 + 5000, 4)[100000:]
    pick = autotune.stratified(window, 240, bins=12)
    size = lambda r: r["m"] * r["n"] + (r["n"] * r["p"] if r["op"] == "matmul" else 0)
    assert 200 <= len(pick) <= 240
    lw = np.log2([size(r) for r in window])
    top_edge = lw.max() - (lw.max() - lw.min()) / 12
    assert np.log2(max(size(r) for r in pick)) >= top_edge                # the largest bin is sampled
    lg = np.log2([size(r) for r in pick])
    # the largest quarter of the size range gets a larger share than in the stream itself
    q3 = lw.max() - (lw.max() - lw.min()) / 4
    assert np.mean(lg > q3) > 1.5 * np.mean(lw > q3)
    for r in gen.batch_requests_sparse(200, 4, 7):
        assert 48 <= r["m"] <= 600 and 1.5 * r["m"] - 1 <= r["n"] <= 2.5 * r["m"] + 1
        assert 0.003 <= r["density"] <= 0.1 and r["batch_count"] in (1024, 4096, 16384)
        assert r["batch_count"] == 1024 or r["batch_count"] * r["m"] * r["n"] <= (1 << 31)
    for r in gen.batch_requests(200, 4, 7):
        assert 32 <= r["m"] <= 1024 and r["batch_count"] in (64, 256, 1024, 4096)
