"""The learned cost model: training on the GPU, saving, loading, choosing.

Training runs entirely in the library's kernels (mela_mlp_gradient +
mela_mlp_adam_step, full-batch Adam); torch only holds the buffers.  The
model predicts log2(microseconds) for each configuration of a request -- a
variant with its tuning fields (Four-Russians k, tile), or for a matrix in a
batched launch the engine that runs it; ``choose`` returns the configuration
with the smallest prediction, and ``install`` hands the weights to the
library's dispatcher (the library also installs costmodel.json by itself
when it is built with one).  Without an installed model the library uses its
fixed rule.

Inputs per request: shape, density, the op, and the batch mix (how many
matrices share the launch and their mean log2(m*n); 1 and the request's own
size for single calls).  Timing databases come from
:mod:`mex_linear_algebra_b200.autotune`.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os

import numpy as np

from . import _lib
from ._lib import check, lib

PKG = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(PKG, "costmodel.json")
OPS = {"rank": _lib.OP_RANK, "null": _lib.OP_NULL, "matmul": _lib.OP_MATMUL, "batch": _lib.OP_BATCH}

# Configuration names in the model's output order (dispatch.cu lists the
# variant arguments; config_codes() reads them from the library).
ELIM_CONFIGS = ("plain", "m4ri_k4", "m4ri_k6", "m4ri_k7", "m4ri_k8", "m4ri_k8_rt256", "m4ri_k9_rt4096",
                "m4ri_k10_rt4096", "fused", "tc")
CONFIG_NAMES = {"rank": ELIM_CONFIGS, "null": ELIM_CONFIGS,
                "matmul": ("plain", "m4ri", "m4ri_w8", "tc_pair", "tc_single", "tc_fp4_pair", "tc_fp4_single"),
                "batch": ("cta", "group", "warp")}
# kept for callers of the earlier name
VARIANT_NAMES = CONFIG_NAMES


def config_codes(op: str) -> tuple:
    """Variant arguments of the op's configurations, from the library."""
    L = lib()
    n = L.mela_costmodel_config_count(OPS[op])
    return tuple(int(L.mela_costmodel_config(OPS[op], i)) for i in range(n))


def config_code(op: str, name: str) -> int:
    return config_codes(op)[CONFIG_NAMES[op].index(name)]


def _mix(m, n, batch_log2_cells):
    if batch_log2_cells is not None:
        return float(batch_log2_cells)
    return math.log2(max(float(m) * float(n), 1.0))


def features(op: str, m: int, n: int, p: int, density: float, batch_count: int = 1,
             batch_log2_cells: float | None = None) -> np.ndarray:
    x = (C.c_float * _lib.MLP_IN)()
    lib().mela_costmodel_features(OPS[op], int(m), int(n), int(p), float(density), int(batch_count),
                                  _mix(m, n, batch_log2_cells), x)
    return np.array(list(x), dtype=np.float32)


def record_features(r) -> np.ndarray:
    return features(r["op"], r["m"], r["n"], r.get("p", 0), r["density"], r.get("batch_count", 1),
                    r.get("batch_log2_cells"))


def dataset(records):
    """Records (autotune DB rows) -> X (N x IN), T (N x OUT log2 us), mask (N x OUT)."""
    X = np.stack([record_features(r) for r in records]) if records else np.zeros((0, _lib.MLP_IN), np.float32)
    T = np.zeros((len(records), _lib.MLP_OUT), dtype=np.float32)
    Mk = np.zeros_like(T)
    for i, r in enumerate(records):
        for v, name in enumerate(CONFIG_NAMES[r["op"]]):
            t = r["times_us"].get(name)
            if t is not None and t > 0:
                T[i, v] = np.log2(t)
                Mk[i, v] = 1.0
    return X, T, Mk


def init_params(seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((_lib.MLP_IN, _lib.MLP_H1), (_lib.MLP_H1, _lib.MLP_H2), (_lib.MLP_H2, _lib.MLP_OUT)):
        parts.append(rng.normal(0, np.sqrt(2.0 / fan_in), size=(fan_in, fan_out)).ravel())
        parts.append(np.zeros(fan_out))
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == _lib.MLP_PARAMS
    return p


def train(records, steps: int = 3000, lr: float = 3e-3, seed: int = 0, log_every: int = 0):
    """Full-batch Adam on the GPU.  Returns (params float32, final loss)."""
    import torch
    X, T, Mk = dataset(records)
    dev = torch.device("cuda")
    dX = torch.from_numpy(X).to(dev)
    dT = torch.from_numpy(T).to(dev)
    dM = torch.from_numpy(Mk).to(dev)
    P = torch.from_numpy(init_params(seed)).to(dev)
    G = torch.zeros_like(P)
    m1 = torch.zeros_like(P)
    m2 = torch.zeros_like(P)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    inv = 1.0 / max(float(Mk.sum()), 1.0)
    s = torch.cuda.current_stream().cuda_stream
    L = lib()
    for step in range(1, steps + 1):
        check(L.mela_mlp_gradient(P.data_ptr(), dX.data_ptr(), dT.data_ptr(), dM.data_ptr(), len(X),
                                  inv, G.data_ptr(), loss.data_ptr(), s))
        check(L.mela_mlp_adam_step(P.data_ptr(), G.data_ptr(), m1.data_ptr(), m2.data_ptr(), step, lr, s))
        if log_every and step % log_every == 0:
            print(f"step {step} loss {loss.item() * inv:.4f}")
    last = float(loss.item()) * inv
    return P.cpu().numpy(), last


def predict(params: np.ndarray, X: np.ndarray) -> np.ndarray:
    import torch
    dP = torch.from_numpy(np.ascontiguousarray(params, dtype=np.float32)).cuda()
    dX = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).cuda()
    dY = torch.empty((len(X), _lib.MLP_OUT), dtype=torch.float32, device="cuda")
    check(lib().mela_mlp_forward(dP.data_ptr(), dX.data_ptr(), len(X), dY.data_ptr(),
                                 torch.cuda.current_stream().cuda_stream))
    return dY.cpu().numpy()


def save(params: np.ndarray, path: str = DEFAULT_MODEL, meta: dict | None = None):
    with open(path, "w") as f:
        json.dump({"params": [float(x) for x in params], "meta": meta or {}}, f)


def load(path: str = DEFAULT_MODEL) -> np.ndarray:
    with open(path) as f:
        p = np.array(json.load(f)["params"], dtype=np.float32)
    if p.size != _lib.MLP_PARAMS:
        raise ValueError(f"{path}: {p.size} parameters, the library's network has {_lib.MLP_PARAMS}")
    return p


def install(params: np.ndarray | None):
    """Give the weights to the library's dispatcher (None removes them)."""
    if params is None:
        check(lib().mela_costmodel_load(None))
        return
    buf = np.ascontiguousarray(params, dtype=np.float32)
    if buf.size != _lib.MLP_PARAMS:
        raise ValueError(f"cost model has {buf.size} parameters, the library expects {_lib.MLP_PARAMS}")
    check(lib().mela_costmodel_load(buf.ctypes.data))


def predict_host(op: str, m: int, n: int, p: int, density: float, batch_count: int = 1,
                 batch_log2_cells: float | None = None):
    """The installed model's predicted log2 microseconds per configuration
    (dict by name), evaluated on the host by the library; None without a model."""
    y = (C.c_float * _lib.MLP_OUT)()
    cnt = lib().mela_costmodel_predict(OPS[op], int(m), int(n), int(p), float(density), int(batch_count),
                                       _mix(m, n, batch_log2_cells), y)
    if cnt < 0:
        return None
    return {CONFIG_NAMES[op][i]: float(y[i]) for i in range(cnt)}


def install_default():
    """Put back the model the library loads with (costmodel.json), if any."""
    install(load() if os.path.exists(DEFAULT_MODEL) else None)


def choose(op: str, m: int, n: int, p: int, density: float, batch_count: int = 1,
           batch_log2_cells: float | None = None, among=None) -> str:
    """Configuration the installed model picks (name) -- among the names in
    `among` when given (e.g. the batch engines a matrix fits); the fixed
    rule without a model."""
    if among is not None:
        y = predict_host(op, m, n, p, density, batch_count, batch_log2_cells)
        if y is None:
            return heuristic(op, m, n, p, density)
        return min(among, key=lambda name: y[name])
    v = lib().mela_costmodel_choose(OPS[op], int(m), int(n), int(p), float(density), int(batch_count),
                                    _mix(m, n, batch_log2_cells))
    if v < 0:
        return heuristic(op, m, n, p, density)
    return CONFIG_NAMES[op][v]


def heuristic(op: str, m: int, n: int, p: int, density: float, rule: str | None = None) -> str:
    """The library's fixed rule (what dispatch does without a model).  For
    batch records the rule's engine depends on shared-memory fit, which the
    autotuner records with each request (``rule``)."""
    if op == "batch":
        return rule or "cta"
    if op == "matmul":
        if m >= 1024 and n >= 1024 and p >= 1024:
            return "tc_fp4_pair" if n < (1 << 23) else "tc_pair"
        return "plain"
    return "fused" if m * n < 8192 else "tc"


def evaluate(params: np.ndarray, records):
    """Measured cost of the model's choices vs the exhaustive best and vs the
    fixed rule, on records with every feasible configuration timed: totals
    (dominated by the largest requests) and per-request means of
    time/best - 1."""
    X, T, Mk = dataset(records)
    Y = predict(params, X) if len(X) else np.zeros((0, _lib.MLP_OUT))
    tot_best = tot_model = tot_rule = 0.0
    reg_model, reg_rule = [], []
    agree = used = 0
    for i, r in enumerate(records):
        names = CONFIG_NAMES[r["op"]]
        times = [r["times_us"].get(nm) for nm in names]
        feasible = [j for j, t in enumerate(times) if t is not None]
        rule_name = heuristic(r["op"], r["m"], r["n"], r.get("p", 0), r["density"], r.get("rule"))
        if not feasible or rule_name not in r["times_us"]:
            continue
        used += 1
        best = min(times[j] for j in feasible)
        pred = feasible[int(np.argmin([Y[i, j] for j in feasible]))]
        t_rule = r["times_us"][rule_name]
        tot_best += best
        tot_model += times[pred]
        tot_rule += t_rule
        reg_model.append(times[pred] / best - 1.0)
        reg_rule.append(t_rule / best - 1.0)
        agree += int(times[pred] == best)
    return {"records": used, "total_best_us": tot_best, "total_model_us": tot_model,
            "total_rule_us": tot_rule,
            "regret": tot_model / tot_best - 1.0 if tot_best else 0.0,
            "rule_regret": tot_rule / tot_best - 1.0 if tot_best else 0.0,
            "speedup_vs_rule": tot_rule / tot_model if tot_model else 0.0,
            "mean_request_regret": float(np.mean(reg_model)) if reg_model else 0.0,
            "rule_mean_request_regret": float(np.mean(reg_rule)) if reg_rule else 0.0,
            "picked_best_frac": agree / max(used, 1)}
