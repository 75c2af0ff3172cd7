"""Exhaustive autotuner: time every configuration of a request on the GPU.

A configuration is a kernel variant with its tuning fields (Four-Russians k
and update row tile for the blocked elimination, single CTAs or CTA pairs
for the tensor-core products), or, for a matrix inside a batched launch, the
engine that runs it.  For each request the inputs are generated on the
device from the seeded Bernoulli generator, every configuration runs once to
warm up and ``reps`` times under CUDA events, and the median is recorded in
microseconds.  The results are compared with each other (they must be
bit-identical) and the record says so.  Records form the timing database
the cost model is trained on, and the exhaustive best time of each request
is the judge of the model's regret.

Requests: the mixed stream of rank, null-space and product requests (m, n,
p log-uniform in [32, 8192], density log-uniform in [0.001, 0.5],
``gen.mixed_stream``) and batch requests, half broad (``gen.batch_requests``)
and half shaped like parity-check batches (``gen.batch_requests_sparse``):
a batch of `count` m x n Bernoulli matrices; per-matrix time of each engine.

    python -m mex_linear_algebra_b200.autotune --count 600 --offset 100000 --out db.json
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import _lib, gen
from ._lib import check, lib
from .costmodel import CONFIG_NAMES, config_codes

SEED = 4
SLOW_US = 200_000.0  # a configuration slower than this is timed once, not `reps` times


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _bernoulli(torch, seed, stream_id, m, n, density):
    wc = (n + 63) // 64
    t = torch.empty((max(m, 1), max(wc, 1)), dtype=torch.int64, device="cuda")
    check(lib().mela_dev_rand_bernoulli(seed, stream_id, m, n, density, t.data_ptr(), t.shape[1],
                                        torch.cuda.current_stream().cuda_stream))
    return t


def _time(torch, fn, reps, setup=None):
    """Median of `reps` CUDA-event timings (us) after one untimed call; a
    call slower than SLOW_US is timed once."""
    if setup:
        setup()
    fn()
    ts = []
    for _ in range(reps):
        if setup:
            setup()
        e0, e1 = _events(torch)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1) * 1e3)
        if ts[-1] > SLOW_US:
            break
    return float(np.median(ts))


def time_matmul(torch, m, k, n, density, stream_id, reps=3, extra=None):
    """Every product configuration (and the `extra` variant arguments, e.g.
    AUTO) on one request: (times by name, all results identical)."""
    L = lib()
    s = torch.cuda.current_stream().cuda_stream
    A = _bernoulli(torch, SEED, 2 * stream_id, m, k, density)
    B = _bernoulli(torch, SEED, 2 * stream_id + 1, k, n, density)
    wn = (n + 63) // 64
    times, outs = {}, {}
    todo = list(zip(CONFIG_NAMES["matmul"], config_codes("matmul"))) + list((extra or {}).items())
    for name, v in todo:
        wsb = L.mela_matmul_workspace_size(v, m, k, n)
        ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
        C_ = torch.empty((m, wn), dtype=torch.int64, device="cuda")

        def run():
            check(L.mela_dev_matmul(v, A.data_ptr(), A.shape[1], B.data_ptr(), B.shape[1],
                                    C_.data_ptr(), wn, m, k, n, ws.data_ptr(), wsb, s))
        times[name] = _time(torch, run, reps)
        outs[name] = C_
        del ws
    agree = all(torch.equal(outs[x], outs["plain"]) for x in outs)
    return times, agree


def time_elim(torch, op, m, n, density, stream_id, reps=3, extra=None):
    """Every elimination configuration (rank, or RREF + null-space basis for
    op 'null'), plus the `extra` variant arguments."""
    L = lib()
    s = torch.cuda.current_stream().cuda_stream
    A0 = _bernoulli(torch, SEED, 2 * stream_id, m, n, density)
    wc = (n + 63) // 64
    mn = max(min(m, n), 1)
    wsb = L.mela_elim_workspace_size(m, n)
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
    rank = torch.zeros(1, dtype=torch.int64, device="cuda")
    piv = torch.empty(mn, dtype=torch.int64, device="cuda")
    prow = torch.empty(mn, dtype=torch.int64, device="cuda")
    M = A0.clone()
    Zt = torch.empty((max(n, 1), wc), dtype=torch.int64, device="cuda")
    nwb = L.mela_null_workspace_size(n, min(m, n))  # the largest null-space workspace (full rank)
    nws = torch.empty(max(nwb, 1), dtype=torch.uint8, device="cuda")
    fn = L.mela_dev_rref if op == "null" else L.mela_dev_rank
    times, results = {}, {}
    todo = list(zip(CONFIG_NAMES[op], config_codes(op))) + list((extra or {}).items())
    for name, v in todo:
        def setup():
            M.copy_(A0)

        def run():
            check(fn(v, M.data_ptr(), wc, m, n, rank.data_ptr(), piv.data_ptr(), prow.data_ptr(),
                     ws.data_ptr(), wsb, s))
            if op == "null":
                r = int(rank.item())
                check(L.mela_dev_null_basis(M.data_ptr(), wc, m, n, r, piv.data_ptr(), prow.data_ptr(),
                                            Zt.data_ptr(), wc, nws.data_ptr(), nwb, s))
        times[name] = _time(torch, run, reps, setup)
        r = int(rank.item())
        results[name] = (r, Zt[:n - r].clone() if op == "null" else None)
    base = results["plain"]
    agree = all(x[0] == base[0] and (op != "null" or torch.equal(x[1], base[1])) for x in results.values())
    return times, agree


def time_batch(torch, m, n, density, count, stream_id, reps=3):
    """A batch of `count` m x n Bernoulli(density) matrices (one device
    stream, stacked: the packed batch layout) run with each engine forced;
    per-matrix microseconds by engine name, the engine the size rule picks,
    and whether every engine gave the same ranks and bases."""
    from .device import BatchPlan
    s_ = [(m, n)] * count
    d_in = _bernoulli(torch, SEED, 100000 + stream_id, count * m, n, density).reshape(-1)
    times, outs, rule = {}, {}, None
    base = BatchPlan(s_)
    st = base.stats()
    rule = "cta" if st["cta"] == count else "group" if st["group128"] == count else "warp"
    base.close()
    for c, name in enumerate(CONFIG_NAMES["batch"]):
        plan = BatchPlan(s_, force_class=c)
        st = plan.stats()
        if st[("cta", "group128", "warp")[c]] != count:  # the matrices do not fit that engine
            plan.close()
            continue
        ranks, zt = plan.outputs()
        zt.zero_()  # words past each basis stay zero, so whole buffers compare

        def run():
            plan.run(d_in, ranks, zt)
        times[name] = _time(torch, run, reps) / count
        outs[name] = (ranks.clone(), zt.clone())
        plan.close()
        del ranks, zt
    first = next(iter(outs.values()))
    agree = all(torch.equal(o[0], first[0]) and torch.equal(o[1], first[1]) for o in outs.values())
    return times, rule, agree


def time_request(req, reps=3, extra=None):
    import torch
    op, m, n, p, d, sid = req["op"], req["m"], req["n"], req.get("p", 0), req["density"], req["stream"]
    out = dict(req)
    if op == "matmul":
        times, agree = time_matmul(torch, m, n, p, d, sid, reps, extra)
    elif op == "batch":
        times, rule, agree = time_batch(torch, m, n, d, req["batch_count"], sid, reps)
        out["rule"] = rule
        out["batch_log2_cells"] = float(np.log2(max(m * n, 1)))
    else:
        times, agree = time_elim(torch, op, m, n, d, sid, reps, extra)
    out["times_us"] = times
    out["agree"] = bool(agree)
    return out


def stratified(reqs, count: int, bins: int = 12):
    """About `count` requests of `reqs`, an equal share from each of `bins`
    log2-size bins (bits touched: m*n, plus n*p for products), evenly spaced
    within each bin."""
    cells = np.array([r["m"] * r["n"] + (r["n"] * r["p"] if r["op"] == "matmul" else 0) for r in reqs],
                     dtype=np.float64)
    lg = np.log2(cells)
    edges = np.linspace(lg.min(), lg.max() + 1e-9, bins + 1)
    per = max(1, count // bins)
    out = []
    for b in range(bins):
        idx = np.nonzero((lg >= edges[b]) & (lg < edges[b + 1]))[0]
        if len(idx):
            out.extend(int(i) for i in np.unique(idx[np.linspace(0, len(idx) - 1, min(per, len(idx))).astype(np.int64)]))
    return [reqs[i] for i in sorted(out)]


def build_db(count: int, offset: int, reps: int = 3, max_cells: float = 7e7, batch_count: int = 0,
             verbose: bool = False, out: str | None = None, budget_s: float = 0.0, window: int = 0):
    """Time `count` requests of the mixed stream from request `offset` on
    (requests above `max_cells` bits are skipped; the stream's largest,
    8192 x 8192, is 6.7e7), then `batch_count` batch requests.  With `out`
    the records so far are written there every 25 requests; with `budget_s`
    each part stops once it has used its share of that many seconds."""
    import torch
    if window > count:
        # `count` requests spread evenly over log2-size bins of a window of
        # `window` requests: the large requests, which dominate total time,
        # get as many records as the small ones
        reqs = stratified(gen.mixed_stream(offset + window, SEED)[offset:], count)
    else:
        reqs = gen.mixed_stream(offset + count, SEED)[offset:]
    db = []
    t0 = time.time()

    def save():
        if out:
            with open(out, "w") as f:
                json.dump(db, f)
    share = budget_s * (0.75 if batch_count else 1.0)
    for i, r in enumerate(reqs):
        cells = r["m"] * r["n"] + (r["n"] * r["p"] if r["op"] == "matmul" else 0)
        if cells > max_cells:
            continue
        db.append(time_request(r, reps))
        torch.cuda.empty_cache()
        if (i + 1) % 25 == 0:
            save()
            if verbose:
                print(f"{i + 1}/{len(reqs)} timed, {time.time() - t0:.1f}s", flush=True)
        if budget_s and time.time() - t0 > share:
            break
    t1 = time.time()
    breqs = gen.batch_requests(batch_count - batch_count // 2, SEED, offset) + \
        gen.batch_requests_sparse(batch_count // 2, SEED, offset)
    for j, r in enumerate(breqs):
        db.append(time_request(r, reps))
        torch.cuda.empty_cache()
        if (j + 1) % 25 == 0:
            save()
            if verbose:
                print(f"batch {j + 1}/{batch_count} timed, {time.time() - t0:.1f}s", flush=True)
        if budget_s and time.time() - t1 > budget_s - share:
            break
    save()
    return db


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=600)
    ap.add_argument("--offset", type=int, default=100000)
    ap.add_argument("--batches", type=int, default=0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--budget", type=float, default=0.0, help="seconds (0: no limit)")
    ap.add_argument("--window", type=int, default=0,
                    help="pick --count requests stratified by size from this many (0: consecutive)")
    ap.add_argument("--out", default="autotune_db.json")
    a = ap.parse_args()
    db = build_db(a.count, a.offset, a.reps, batch_count=a.batches, verbose=True, out=a.out,
                  budget_s=a.budget, window=a.window)
    print(f"{len(db)} records -> {a.out}; all configurations agree: {all(r['agree'] for r in db)}")


if __name__ == "__main__":
    main()
