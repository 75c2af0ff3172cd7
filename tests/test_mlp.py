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
    assert np.allclose(x, [10 / 14, 11 / 14, 12 / 14, -2 / 3 + 1, 0, 0, 1, 1], atol=1e-6)
    x = costmodel.features("null", 32, 8192, 0, 0.5)
    assert x[2] == 0 and x[5] == 1 and x[6] == 0


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
        t = {"plain": 2 ** (0.9 * lg - 3), "m4ri": 2 ** (0.6 * lg + 1), "m4ri_k4": 2 ** (0.7 * lg)}
        recs.append({"op": "rank", "m": m, "n": n, "p": 0, "density": d, "times_us": t})
    params, loss = costmodel.train(recs[:400], steps=2500)
    rep = costmodel.evaluate(params, recs[400:])
    assert loss < 0.05
    assert rep["regret"] < 0.05


@pytest.mark.skipif(not os.path.exists(os.path.join(DATA, "autotune_eval.json")),
                    reason="no timing database recorded yet")
def test_trained_model_beats_fixed_rule():
    """On held-out requests with every variant timed (recorded on B200 by the
    autotuner), the installed model's choices cost less in total than the
    fixed rule's, and its regret against the exhaustive best is smaller.
    Host-side inference through the library's dispatcher; no GPU needed."""
    from mex_linear_algebra_b200 import costmodel
    params = costmodel.load()
    ev = json.load(open(os.path.join(DATA, "autotune_eval.json")))
    costmodel.install(params)
    try:
        tot_model = tot_rule = tot_best = 0.0
        for r in ev:
            names = costmodel.VARIANT_NAMES[r["op"]]
            t = r["times_us"]
            tot_best += min(t[x] for x in names)
            tot_model += t[costmodel.choose(r["op"], r["m"], r["n"], r.get("p", 0), r["density"])]
            tot_rule += t[costmodel.heuristic(r["op"], r["m"], r["n"], r.get("p", 0), r["density"])]
    finally:
        costmodel.install(None)
    assert all(r["agree"] for r in ev)  # every variant returned the same bits
    assert tot_model < tot_rule
    assert tot_model / tot_best - 1 < tot_rule / tot_best - 1
    # per request, too: the mean slowdown against the exhaustive best shrinks
    rep = {}
    costmodel.install(params)
    try:
        per_model = [r["times_us"][costmodel.choose(r["op"], r["m"], r["n"], r.get("p", 0), r["density"])]
                     / min(r["times_us"].values()) - 1 for r in ev]
    finally:
        costmodel.install(None)
    per_rule = [r["times_us"][costmodel.heuristic(r["op"], r["m"], r["n"], r.get("p", 0), r["density"])]
                / min(r["times_us"].values()) - 1 for r in ev]
    assert np.mean(per_model) < np.mean(per_rule)
