#!/usr/bin/env python
"""Benchmark: GF(2) GEMM Tbitop/s at 32768^3; batched rank+null mats/s.

Headline (value): C = A*B over GF(2) with A, B 32768 x 32768, iid
Bernoulli(1/2) from seed 1, packed uint64 row-major, by the FP4 tensor-core
form (tcgen05 kind::mxf4 on CTA pairs; --variant tc for the INT8 form):
operand preparation -- expansion of A and transposing expansion of B into
K-major e2m1 values -- plus the tensor-core kernel.  Bit-ops are counted as
2*m*n*k (one AND and one XOR per term), the analogue of 2mnk FLOPs.

  value  -- device-timed (CUDA events, max over ranks) with packed inputs
            resident in HBM; inputs are 256 MiB packed + 1 GiB of expanded
            operands per step, all larger than L2 (126 MB).
  e2e    -- the same product through the C ABI host entry point
            mela_matmul_packed_host with pinned host buffers: host->device copy
            of A and B and device->host copy of C inside every timed step
            (host clock around the blocking call).
  roofline -- the tensor-core kernel alone, CUDA events on its stream, against
            dense INT8 measured in the same run (cuBLASLt int8 through
            torch._int_mm).
  cpu_baseline -- the reference's own mela_matmul_gf2 (compiled from its
            sources with its AVX512/OpenMP flags) on A * B[:, :4096]
            (32768 x 32768 * 32768 x 4096), 1/8 of the same product's terms.
  batched -- the second half of the metric: 20,000 parity-check matrices
            (m uniform [64,1024], n = 2m +/- [0, m/4], six ones per row, seed 3)
            ranked and null-spaced from their logical (MATLAB layout) form in
            one persistent launch replayed as a CUDA graph, versus the plain
            per-matrix path (one call sequence per matrix) on a sample.
  dense_rank_null -- 16384 x 32768 rank-12000 matrix (seed 2): rank and null
            space per elimination form, checked against the oracle's rank.
  learned_dispatch -- a bounded sample of the mixed request stream (seed 4):
            time of the installed cost model's choices vs the fixed rule vs the
            exhaustive best.

``--impl reference`` times only the reference's CPU code (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

M = K = N = 32768
SEED = 1
BITOPS = 2.0 * M * N * K
# rows of A, K and columns of B for the CPU legs: A times B's first 4096
# columns (1/8 of the full product's terms).  The reference's cost has three
# parts: its serial packing of B (K x N logical), its XOR of packed rows of B
# into row blocks of C (M*K row operations of N/64 words) and its unpacking
# of C (M x N logical, column-major); all three shrink by the same factor
# only when N is the dimension cut.  This sample runs at 1.45-1.5 T bit-ops/s
# on 8 cores against 1.77 for the full product (39.7 s).
CPU_SAMPLE = (32768, 32768, 4096)


def set_size(size: int) -> None:
    global M, K, N, BITOPS
    M = K = N = size
    BITOPS = 2.0 * M * N * K


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        return self.summarize(self.lines)

    @staticmethod
    def summarize(lines) -> dict:
        """Median SM clock, the max clock and the throttle reasons seen active
        in `nvidia-smi --format=csv,noheader,nounits` lines of FIELDS."""
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                cur, mx = float(parts[0]), float(parts[1])
            except ValueError:
                continue
            sm.append(cur)
            smax = mx
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ CPU legs
def cpu_reference_sample(steps: int = 1):
    """Time the reference gateway mela_matmul_gf2 (oracle/_ref) on the CPU
    sample; returns (Tbitop/s, seconds per call, threads, isa)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ms, ks, ns = CPU_SAMPLE
    # all of A, the first ns columns of B (whose rows are N bits long)
    A = O.unpack(O.rand_dense(SEED, 0, ms, ks), ms, ks)
    B = O.unpack(O.rand_dense(SEED, 1, ks, N)[:, :(ns + 63) // 64], ks, ns)
    O.ref_call("mela_matmul_gf2", A[:256], B)  # warm the code and pages
    times = []
    for _ in range(max(1, steps)):
        t0 = time.perf_counter()
        O.ref_call("mela_matmul_gf2", A, B)
        times.append(time.perf_counter() - t0)
    times.sort()
    dt = times[len(times) // 2]
    return 2.0 * ms * ks * ns / dt / 1e12, dt, O.num_threads(), O.host_isa()


def run_reference(args, ws, rank):
    if rank != 0:
        return 0
    os.environ.setdefault("OMP_DYNAMIC", "FALSE")
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference gateways not built (oracle/_ref missing)"}))
        return 0
    for _ in range(args.warmup):
        cpu_reference_sample(1)
    rate, dt, threads, isa = cpu_reference_sample(args.steps)
    ms, ks, ns = CPU_SAMPLE
    sample = (f"reference mela_matmul_gf2 ({isa} build, OpenMP) on A * B[:, :{ns}] "
              f"({ms}x{ks} * {ks}x{ns} logical), 1/8 of the 32768^3 product's terms; "
              f"median of {args.steps} calls")
    line = {
        "impl": "reference",
        "metric": "GF(2) GEMM Tbitop/s at 32k^3",
        "value": round(rate, 4),
        "unit": "Tbitop/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(dt * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u64",
        "data": "synthetic (seeded splitmix64 Bernoulli(1/2))",
        "config": {"workload": "gemm_gf2_32768^3", "m": 32768, "k": 32768, "n": 32768, "seed": SEED,
                   "sample_per_step": {"m": ms, "k": ks, "n": ns}},
        "cpu_baseline": {"value": round(rate, 4), "unit": "Tbitop/s", "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": round(rate, 4), "unit": "Tbitop/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ GPU pieces
def measure_int8_peak(torch):
    """Dense INT8 tensor throughput of cuBLASLt (torch._int_mm) at 8192^3."""
    n = 8192
    a = torch.randint(-2, 2, (n, n), dtype=torch.int8, device="cuda")
    b = torch.randint(-2, 2, (n, n), dtype=torch.int8, device="cuda")
    for _ in range(3):
        torch._int_mm(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch._int_mm(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def bench_batched(torch, count=20000, seed=3, baseline_sample=200):
    """Batched rank+null of the parity-check batch from logical input."""
    import numpy as np
    from mex_linear_algebra_b200 import device as D, gen, _lib
    from mex_linear_algebra_b200._lib import check, lib
    shapes, offsets, buf = gen.ldpc_batch(count, seed)
    plan = D.BatchPlan(shapes)
    d_packed = torch.from_numpy(buf.view(np.int64)).cuda()
    d_log = plan.unpack_logical(d_packed)
    ranks, zt = plan.outputs()
    for _ in range(3):
        plan.run_logical(d_log, ranks, zt)
    torch.cuda.synchronize()
    reps = 5
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        plan.run_logical(d_log, ranks, zt)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    # the packing step alone (logical bytes -> packed rows), same input
    d_pk = torch.zeros(max(plan.in_words, 1), dtype=torch.int64, device="cuda")
    plan.pack_logical(d_log, d_pk)
    e0.record()
    for _ in range(reps):
        plan.pack_logical(d_log, d_pk)
    e1.record()
    e1.synchronize()
    pack_ms = e0.elapsed_time(e1) / reps
    pack_ok = bool(torch.equal(d_pk, d_packed))
    del d_pk
    # plain per-matrix path: pack, RREF (plain form), null basis, one matrix at a time
    L = lib()
    s = torch.cuda.current_stream().cuda_stream
    idx = np.linspace(0, count - 1, baseline_sample).astype(np.int64)
    rk_host = ranks.cpu().numpy()
    ok = True
    t_base = 0.0
    for i in idx:
        m, n = int(shapes[i, 0]), int(shapes[i, 1])
        wc = (n + 63) // 64
        src = d_packed[offsets[i]:offsets[i] + m * wc].view(m, wc)
        Mx = src.clone()
        mn = min(m, n)
        dr = torch.zeros(1, dtype=torch.int64, device="cuda")
        dpv = torch.empty(mn, dtype=torch.int64, device="cuda")
        dpr = torch.empty(mn, dtype=torch.int64, device="cuda")
        wsb = L.mela_elim_workspace_size(m, n)
        wsp = torch.empty(wsb, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        check(L.mela_dev_rref(_lib.ELIM_PLAIN, Mx.data_ptr(), wc, m, n, dr.data_ptr(), dpv.data_ptr(),
                              dpr.data_ptr(), wsp.data_ptr(), wsb, s))
        r = int(dr.item())
        f = n - r
        Zt = torch.empty((max(f, 1), wc), dtype=torch.int64, device="cuda")
        nwb = L.mela_null_workspace_size(n, r)
        nws = torch.empty(max(nwb, 1), dtype=torch.uint8, device="cuda")
        check(L.mela_dev_null_basis(Mx.data_ptr(), wc, m, n, r, dpv.data_ptr(), dpr.data_ptr(),
                                    Zt.data_ptr(), wc, nws.data_ptr(), nwb, s))
        torch.cuda.synchronize()
        t_base += time.perf_counter() - t0
        ok = ok and r == int(rk_host[i])
        z0 = int(plan.z_offsets[i])
        ok = ok and bool(torch.equal(Zt[:f].reshape(-1), zt[z0:z0 + f * wc]))
    base_rate = baseline_sample / t_base
    # per matrix again, with the library's AUTO dispatch (the fused single-CTA
    # or tensor-core forms, chosen per matrix) and buffers allocated once
    mmax, nmax = int(shapes[:, 0].max()), int(shapes[:, 1].max())
    wcmax = (nmax + 63) // 64
    Mbuf = torch.empty(mmax * wcmax, dtype=torch.int64, device="cuda")
    Zbuf = torch.empty(nmax * wcmax, dtype=torch.int64, device="cuda")
    dr = torch.zeros(1, dtype=torch.int64, device="cuda")
    dpv = torch.empty(mmax, dtype=torch.int64, device="cuda")
    dpr = torch.empty(mmax, dtype=torch.int64, device="cuda")
    wsb = max(L.mela_elim_workspace_size(int(a), int(b)) for a, b in shapes[idx])
    wsp = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    nwb = max(L.mela_null_workspace_size(int(b), min(int(a), int(b))) for a, b in shapes[idx])
    nws = torch.empty(nwb, dtype=torch.uint8, device="cuda")
    ok_auto = True
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in idx:
        m, n = int(shapes[i, 0]), int(shapes[i, 1])
        wc = (n + 63) // 64
        Mx = Mbuf[:m * wc].view(m, wc)
        Mx.copy_(d_packed[offsets[i]:offsets[i] + m * wc].view(m, wc))
        check(L.mela_dev_rref(_lib.ELIM_AUTO, Mx.data_ptr(), wc, m, n, dr.data_ptr(), dpv.data_ptr(),
                              dpr.data_ptr(), wsp.data_ptr(), wsb, s))
        r = int(dr.item())
        check(L.mela_dev_null_basis(Mx.data_ptr(), wc, m, n, r, dpv.data_ptr(), dpr.data_ptr(),
                                    Zbuf.data_ptr(), wc, nws.data_ptr(), nwb, s))
        torch.cuda.synchronize()
        ok_auto = ok_auto and r == int(rk_host[i])
    t_auto = time.perf_counter() - t0
    auto_rate = baseline_sample / t_auto
    del Mbuf, Zbuf, wsp, nws
    # the same batch with each matrix's engine picked by the cost model from
    # its shape, its density (counted on the device) and the batch mix
    learned = {}
    try:
        dens = plan.densities(d_packed)
        lplan = D.BatchPlan(shapes, force_class=-2, densities=dens)
        r2, z2 = lplan.outputs()
        for _ in range(3):
            lplan.run_logical(d_log, r2, z2)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            lplan.run_logical(d_log, r2, z2)
        e1.record()
        e1.synchronize()
        lms = e0.elapsed_time(e1) / reps
        same = bool(torch.equal(r2, ranks))
        if same:  # the bases, matrix by matrix (words past each basis are not written)
            zh, z2h = zt.cpu().numpy(), z2.cpu().numpy()
            rkh = rk_host
            same = all(np.array_equal(plan.basis(zh, rkh, i), lplan.basis(z2h, rkh, i)) for i in range(count))
        learned = {"ms_per_batch": round(lms, 3), "speedup_vs_size_rule": round(ms / lms, 3),
                   "classes": lplan.stats(), "results_match": same,
                   "policy": "engine per matrix by the cost model (shape, device-counted density, batch mix)"}
        lplan.close()
        del r2, z2
    except Exception as e:  # reported, not fatal
        learned = {"error": f"{type(e).__name__}: {e}"}
    rate = count / (ms * 1e-3)
    in_bytes = plan.logical_bytes
    # forward-elimination work (rank m, pivots in the leading columns) and the bytes that must move
    ms_, ns_ = shapes[:, 0].astype(np.float64), shapes[:, 1].astype(np.float64)
    work = float(sum(2.0 * ((mm - 1 - np.arange(mm)) * (nn - np.arange(mm))).sum()
                     for mm, nn in zip(shapes[:, 0], shapes[:, 1])))
    z_bytes = float(((ns_ - ms_) * ((ns_ + 63) // 64) * 8).sum())
    classes = plan.stats()
    plan.close()
    return {"metric": "batched rank+null mats/s", "value": round(rate, 1), "unit": "matrices/s",
            "ms_per_batch": round(ms, 3), "matrices": count,
            "input": f"logical (MATLAB layout), {in_bytes / 1e9:.2f} GB resident in HBM",
            "engine": "one persistent launch replayed as a CUDA graph (warp / 128-thread group / CTA per matrix)",
            "classes": classes,
            "per_matrix_plain": {"value": round(base_rate, 1), "unit": "matrices/s",
                                 "sample": f"{baseline_sample} matrices spread over the batch, "
                                           "pack-free packed input, plain RREF + null basis per matrix, "
                                           "host clock per matrix"},
            "speedup_vs_per_matrix": round(rate / base_rate, 1), "results_match": ok,
            "per_matrix_auto": {"value": round(auto_rate, 1), "unit": "matrices/s", "ranks_match": ok_auto,
                                "sample": f"the same {baseline_sample} matrices, mela_dev_rref with AUTO "
                                          "(cost-model choice per matrix) + null basis, buffers allocated "
                                          "once, host clock"},
            "speedup_vs_per_matrix_auto": round(rate / auto_rate, 1),
            "learned_engines": learned,
            "pack": {"ms": round(pack_ms, 3), "exact": pack_ok,
                     "gbs": round((in_bytes + plan.in_words * 8) / (pack_ms * 1e-3) / 1e9, 1),
                     "note": "batch_pack_kernel alone: logical bytes read + packed words written"},
            "roofline": {"bound": "bit-op issue (shared memory / barrier chain), not HBM",
                         "work_tbitop": round(work / 1e12, 3),
                         "achieved_tbitops": round(work / (ms * 1e-3) / 1e12, 1),
                         "hbm_bytes": in_bytes + z_bytes,
                         "hbm_gbs": round((in_bytes + z_bytes) / (ms * 1e-3) / 1e9, 1),
                         "work_note": "sum over matrices of sum_p 2(m-p-1)(n-p): forward elimination "
                                      "with the pivots in the leading columns"}}


def bench_batched_sharded(torch, ws, rank, count=20000, seed=3, reps=5):
    """The parity-check batch split over the ranks by estimated cost
    (parallel.shard_batch; no data exchange): each rank runs its share from
    packed input in one persistent launch (graph replay), timed with CUDA
    events, the maximum over ranks; ranks gathered on the host and checked
    against the oracle's for all 20,000 matrices."""
    import numpy as np
    from mex_linear_algebra_b200 import device as D, gen, parallel
    shapes, offsets, buf = gen.ldpc_batch(count, seed)
    golden = np.load(os.path.join(ROOT, "tests", "golden", "ldpc_20000.npz"))["ranks"]
    state = {}

    def compute(idx):
        sub = shapes[idx]
        wcs = (sub[:, 1] + 63) // 64
        packed = np.concatenate([buf[offsets[i]:offsets[i] + shapes[i, 0] * w] for i, w in zip(idx, wcs)])
        plan = D.BatchPlan(sub)
        d = torch.from_numpy(packed.view(np.int64)).cuda()
        ranks, zt = plan.outputs()
        for _ in range(3):
            plan.run(d, ranks, zt)
        torch.cuda.synchronize()
        parallel.barrier(ws)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            plan.run(d, ranks, zt)
        e1.record()
        e1.synchronize()
        state["ms"] = e0.elapsed_time(e1) / reps
        state["mine"] = len(idx)
        rk = ranks.cpu().numpy()
        plan.close()
        return {int(i): int(rk[j]) for j, i in enumerate(idx)}

    merged, owners = parallel.run_sharded(shapes, ws, rank, compute)
    ms = parallel.max_over_ranks(ws, state["ms"])
    ok = all(merged[i] == int(golden[i]) for i in range(count))
    return {"metric": "batched rank+null mats/s, sharded over ranks", "value": round(count / (ms * 1e-3), 1),
            "unit": "matrices/s", "n_gpus": ws, "ms_per_batch_max_over_ranks": round(ms, 3),
            "matrices_per_rank": [len(o) for o in owners], "ranks_match_oracle": ok,
            "input": "packed, resident in HBM", "scaling": "strong (the 20,000 matrices split over the ranks)"}


def bench_dense_rank(torch):
    """Rank and null space of the 16384 x 32768 rank-12000 configuration."""
    import numpy as np
    from mex_linear_algebra_b200 import device as D, gen, _lib
    from mex_linear_algebra_b200._lib import check, lib
    m, r0, n = 16384, 12000, 32768
    golden = None
    gpath = os.path.join(ROOT, "tests", "golden", "dense_rank.json")
    if os.path.exists(gpath):
        golden = json.load(open(gpath))["rank"]
    Ld = D.rand_dense(2, 0, m, r0)
    Rd = D.rand_dense(2, 1, r0, n)
    A = D.matmul(Ld, Rd, m, r0, n, variant="tc")
    del Ld, Rd
    for (i, a, b) in gen.replacement_triples(m, 164):
        A[i] = A[a] ^ A[b]
    L = lib()
    s = torch.cuda.current_stream().cuda_stream
    wc = n // 64
    wsb = L.mela_elim_workspace_size(m, n)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    dr = torch.zeros(1, dtype=torch.int64, device="cuda")
    dpv = torch.empty(m, dtype=torch.int64, device="cuda")
    dpr = torch.empty(m, dtype=torch.int64, device="cuda")
    out = {"config": "A = L*R mod 2, L 16384x12000, R 12000x32768 (seed 2), 164 rows replaced by XORs "
                     "of two others", "golden_rank": golden, "rank_ms": {}, "null_ms": {}}
    ranks = set()
    for form in ("tc", "m4ri", "m4ri_k4", "plain"):
        v = _lib.ELIM_VARIANTS[form]
        # untimed calls first: one-time costs (the tensor-core form captures its
        # launch sequence into a CUDA graph on the second call with the same buffers)
        Mx = A.clone()
        for _ in range(2 if form == "tc" else 1):
            Mx.copy_(A)
            check(L.mela_dev_rank(v, Mx.data_ptr(), wc, m, n, dr.data_ptr(), dpv.data_ptr(), dpr.data_ptr(),
                                  ws.data_ptr(), wsb, s))
        Mx.copy_(A)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        check(L.mela_dev_rank(v, Mx.data_ptr(), wc, m, n, dr.data_ptr(), dpv.data_ptr(), dpr.data_ptr(),
                              ws.data_ptr(), wsb, s))
        e1.record()
        e1.synchronize()
        out["rank_ms"][form] = round(e0.elapsed_time(e1), 2)
        ranks.add(int(dr.item()))
    r = ranks.pop() if len(ranks) == 1 else None
    out["rank"] = r
    # work of forward elimination with these pivots: sum_t 2 (m - t - 1) (n - c_t) bit operations
    piv = dpv[:r].cpu().numpy().astype(np.float64) if r else np.zeros(0)
    t = np.arange(len(piv), dtype=np.float64)
    ge_ops = float(np.sum(2.0 * (m - t - 1) * (n - piv)))
    out["ge_bitops"] = ge_ops
    out["rank_tbitops"] = {k: round(ge_ops / (v * 1e-3) / 1e12, 1) for k, v in out["rank_ms"].items()}
    out["tc_over_m4ri_k4"] = round(out["rank_ms"]["m4ri_k4"] / out["rank_ms"]["tc"], 2)
    out["tc_over_plain"] = round(out["rank_ms"]["plain"] / out["rank_ms"]["tc"], 2)
    # RREF by the blocked form (for comparison), then by the tensor-core form + null basis,
    # then A * Z = 0 on the tensor cores
    Mx = A.clone()
    torch.cuda.synchronize()
    e0, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
    e0.record()
    check(L.mela_dev_rref(_lib.ELIM_M4RI, Mx.data_ptr(), wc, m, n, dr.data_ptr(), dpv.data_ptr(),
                          dpr.data_ptr(), ws.data_ptr(), wsb, s))
    e1.record()
    e1.synchronize()
    out["null_ms"]["m4ri_rref"] = round(e0.elapsed_time(e1), 2)
    rows_m4ri = Mx[dpr[:int(dr.item())]].clone()
    Mx = A.clone()
    for _ in range(2):  # untimed calls (the second captures the CUDA graph)
        Mx.copy_(A)
        check(L.mela_dev_rref(_lib.ELIM_TC, Mx.data_ptr(), wc, m, n, dr.data_ptr(), dpv.data_ptr(),
                              dpr.data_ptr(), ws.data_ptr(), wsb, s))
    Mx.copy_(A)
    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    check(L.mela_dev_rref(_lib.ELIM_TC, Mx.data_ptr(), wc, m, n, dr.data_ptr(), dpv.data_ptr(),
                          dpr.data_ptr(), ws.data_ptr(), wsb, s))
    e1.record()
    e1.synchronize()
    rr = int(dr.item())
    out["rref_rows_equal"] = bool(torch.equal(rows_m4ri, Mx[dpr[:rr]]))
    del rows_m4ri
    f = n - rr
    Zt = torch.empty((f, wc), dtype=torch.int64, device="cuda")
    nwb = L.mela_null_workspace_size(n, rr)
    nws = torch.empty(nwb, dtype=torch.uint8, device="cuda")
    e1.record()
    check(L.mela_dev_null_basis(Mx.data_ptr(), wc, m, n, rr, dpv.data_ptr(), dpr.data_ptr(),
                                Zt.data_ptr(), wc, nws.data_ptr(), nwb, s))
    e2.record()
    e2.synchronize()
    out["null_ms"]["tc_rref"] = round(e0.elapsed_time(e1), 2)
    out["null_ms"]["basis"] = round(e1.elapsed_time(e2), 2)
    Z = D.transpose(Zt, f, n)  # n x f
    prod = D.matmul(A, Z, m, n, f, variant="tc")
    out["nullity"] = f
    out["A_times_Z_is_zero"] = bool(int(prod.abs().max().item()) == 0)
    out["rank_matches_golden"] = (golden is None) or (r == golden and rr == golden)
    del Zt, Z, prod, Mx, A, ws
    torch.cuda.empty_cache()
    return out


def bench_gateway_config(torch, reps=5):
    """The drop-in call at its benchmark configuration: mela_matmul_gf2(A, B)
    with A 2048 x 2048 and B 2048 x 1024 double 0/1 (seed 0), host arrays
    in MATLAB layout, logical result -- through the library's gateway (the
    code the MEX file runs) and through the reference's own gateway on the
    host cores, on the same arrays; median of `reps` calls after two
    warm-ups each."""
    import hashlib
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from mex_linear_algebra_b200 import mela
    m, k, n = 2048, 2048, 1024
    A = O.unpack(O.rand_dense(0, 0, m, k), m, k).astype(np.float64)
    B = O.unpack(O.rand_dense(0, 1, k, n), k, n).astype(np.float64)
    golden = json.load(open(os.path.join(ROOT, "tests", "golden", "config_digests.json")))["matmul_gateway_2048"]

    def timed(fn):
        for _ in range(2):
            out = fn()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            out = fn()
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts)), out

    t_gpu, C = timed(lambda: mela.mela_matmul_gf2(A, B))
    ok = hashlib.blake2b(O.pack(C).tobytes(), digest_size=16).hexdigest() == golden["digest"]
    line = {"config": "mela_matmul_gf2(A 2048x2048 double, B 2048x1024 double), seed 0, logical out",
            "gpu_ms": round(t_gpu * 1e3, 3), "result_matches_reference_digest": ok,
            "h2d_bytes": int(A.nbytes + B.nbytes), "d2h_bytes": int(m * n),
            "timing": f"host clock around the call, median of {reps}"}
    if O.ref_available():
        os.environ.setdefault("OMP_DYNAMIC", "FALSE")
        t_ref, Cr = timed(lambda: O.ref_call("mela_matmul_gf2", A, B)[0])
        line.update({"reference_ms": round(t_ref * 1e3, 3), "reference_threads": O.num_threads(),
                     "reference_isa": O.host_isa(), "speedup_vs_reference": round(t_ref / t_gpu, 2),
                     "same_result_as_reference": bool(np.array_equal(Cr, C))})
    return line


def _stratified(reqs, per_bin, bins):
    """`per_bin` requests from each of `bins` log-size bins of the request
    list (bits touched: m*n, plus n*p for products), evenly spaced."""
    import numpy as np
    cells = np.array([r["m"] * r["n"] + (r["n"] * r["p"] if r["op"] == "matmul" else 0) for r in reqs],
                     dtype=np.float64)
    lg = np.log2(cells)
    edges = np.linspace(lg.min(), lg.max() + 1e-9, bins + 1)
    out = []
    for b in range(bins):
        idx = np.nonzero((lg >= edges[b]) & (lg < edges[b + 1]))[0]
        if len(idx):
            take = idx[np.linspace(0, len(idx) - 1, min(per_bin, len(idx))).astype(np.int64)]
            out.extend(int(i) for i in np.unique(take))
    return [reqs[i] for i in out]


def bench_dispatch(torch, per_bin=14, bins=8):
    """The learned dispatch on the mixed request stream (50,000 requests,
    seed 4: rank, null space and products, m, n, p log-uniform in [32, 8192],
    density log-uniform in [0.001, 0.5]): a sample stratified by request
    size, every size up to 8192 x 8192 kept.  Per request: every
    configuration timed (the exhaustive best), the library's own AUTO
    dispatch (the compiled-in cost model; the input's density measured on
    the device inside the call), and the fixed rule's configuration."""
    import numpy as np
    from mex_linear_algebra_b200 import _lib, autotune, costmodel, gen
    from mex_linear_algebra_b200._lib import lib
    if lib().mela_costmodel_choose(_lib.OP_RANK, 100, 100, 0, 0.5, 1, 13.3) < 0:
        return {"unavailable": "the library was built without a trained cost model"}
    import ctypes as C
    sample = _stratified(gen.mixed_stream(50000, 4), per_bin, bins)
    recs = []
    t0 = time.time()
    codes = {op: dict(zip(costmodel.config_codes(op), costmodel.CONFIG_NAMES[op])) for op in ("rank", "null", "matmul")}
    measured = 0
    for r in sample:
        rec = autotune.time_request(r, reps=2, extra={"auto": 0})
        # the configuration the last AUTO call (the timed ones above) resolved to
        d = C.c_double(0)
        rec["auto_choice"] = codes[r["op"]].get(int(lib().mela_dispatch_last(C.byref(d))))
        measured += int(d.value >= 0)
        recs.append(rec)
        torch.cuda.empty_cache()
    tot = {"best": 0.0, "auto": 0.0, "rule": 0.0, "auto_choice": 0.0}
    per = {"auto": [], "rule": []}
    by_op = {}
    for r in recs:
        t = r["times_us"]
        best = min(v for kname, v in t.items() if kname != "auto")
        rule = t[costmodel.heuristic(r["op"], r["m"], r["n"], r.get("p", 0), r["density"])]
        tot["best"] += best
        tot["auto"] += t["auto"]
        tot["rule"] += rule
        tot["auto_choice"] += t.get(r["auto_choice"], t["auto"])
        per["auto"].append(t["auto"] / best - 1)
        per["rule"].append(rule / best - 1)
        o = by_op.setdefault(r["op"], {"requests": 0, "best_us": 0.0, "auto_us": 0.0, "rule_us": 0.0})
        o["requests"] += 1
        o["best_us"] += best
        o["auto_us"] += t["auto"]
        o["rule_us"] += rule
    for o in by_op.values():
        o["auto_regret"] = round(o["auto_us"] / o["best_us"] - 1, 4)
        o["rule_regret"] = round(o["rule_us"] / o["best_us"] - 1, 4)
        for kname in ("best_us", "auto_us", "rule_us"):
            o[kname] = round(o[kname], 1)
    return {"requests": len(recs),
            "sample": f"{len(recs)} of the 50,000 requests (seed 4), {per_bin} per log2-size bin over {bins} "
                      "bins from the smallest to the 8192 x 8192 ones; every configuration timed "
                      "(median of 2 after a warm-up)",
            "library_auto_regret": round(tot["auto"] / tot["best"] - 1, 4),
            "auto_choice_regret": round(tot["auto_choice"] / tot["best"] - 1, 4),
            "density_measured": f"{measured} of {len(recs)} AUTO calls read the density back",
            "fixed_rule_regret": round(tot["rule"] / tot["best"] - 1, 4),
            "auto_speedup_vs_rule": round(tot["rule"] / tot["auto"], 4),
            "mean_request_regret": {"auto": round(float(np.mean(per["auto"])), 4),
                                    "rule": round(float(np.mean(per["rule"])), 4)},
            "total_us": {k_: round(v, 1) for k_, v in tot.items()},
            "by_op": by_op,
            "all_configurations_bit_identical": all(r["agree"] for r in recs),
            "seconds": round(time.time() - t0, 1),
            "note": "auto = mela_dev_rank / mela_dev_rref (+ null basis) / mela_dev_matmul with the AUTO "
                    "variant timed as a whole: the model on the host at four densities, a popcount of the "
                    "input and an 8-byte read-back when the choice depends on the density, then the "
                    "chosen configuration; auto_choice = the recorded time of the configuration AUTO "
                    "chose (the choice without the call's own overhead)"}


def run_mela(args, ws, rank, local):
    import torch
    from mex_linear_algebra_b200 import parallel
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from mex_linear_algebra_b200 import _lib, device as D
    from mex_linear_algebra_b200._lib import check, lib

    L = lib()
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    v = _lib.GEMM_VARIANTS[args.variant]
    wk = wn = N // 64
    A = D.rand_dense(SEED, 0, M, K)
    B = D.rand_dense(SEED, 1, K, N)
    C = torch.empty((M, wn), dtype=torch.int64, device="cuda")
    wsb = D.matmul_workspace(v, M, K, N)
    work = torch.empty(wsb, dtype=torch.uint8, device="cuda")

    def step(ev_mid=None):
        check(L.mela_dev_matmul_prepare(v, A.data_ptr(), wk, B.data_ptr(), wn, M, K, N,
                                        work.data_ptr(), wsb, sptr))
        if ev_mid is not None:
            ev_mid.record(stream)
        check(L.mela_dev_matmul_run(v, A.data_ptr(), wk, B.data_ptr(), wn, C.data_ptr(), wn,
                                    M, K, N, work.data_ptr(), wsb, sptr))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    parallel.barrier(ws)

    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
            torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    parallel.barrier(ws)
    torch.cuda.synchronize()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for (e0, e1, e2) in evs:
        e0.record(stream)
        step(e1)
        e2.record(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    parallel.barrier(ws)
    clk = clocks.stop()
    total_ms = parallel.max_over_ranks(ws, t_start.elapsed_time(t_end))
    kernel_ms = [e1.elapsed_time(e2) for (_, e1, e2) in evs]
    ms_step = total_ms / args.steps
    value = ws * BITOPS / (ms_step * 1e-3) / 1e12
    kern_avg = sum(kernel_ms) / len(kernel_ms)

    # correctness guard on the timed result: a block of rows against the plain form
    rows = 256
    Cp = D.matmul(A[:rows], B, rows, K, N, variant="plain")
    ok = bool(torch.equal(Cp, C[:rows]))
    flags = D.device_error_flags()

    forms = {args.variant + "_ms": round(ms_step, 3)}
    if not args.quick:
        other = "tc" if args.variant == "tc_fp4" else "tc_fp4"
        for name, var in (("plain", _lib.GEMM_PLAIN), ("m4ri", _lib.GEMM_M4RI),
                          (other, _lib.GEMM_VARIANTS[other])):
            wsv = D.matmul_workspace(var, M, K, N)
            wv = torch.empty(max(wsv, 1), dtype=torch.uint8, device="cuda")
            Cv = torch.empty_like(C)

            def run_form():
                check(L.mela_dev_matmul(var, A.data_ptr(), wk, B.data_ptr(), wn, Cv.data_ptr(), wn,
                                        M, K, N, wv.data_ptr(), wsv, sptr))
            run_form()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run_form()
            e1.record(stream)
            e1.synchronize()
            forms[name + "_ms"] = round(e0.elapsed_time(e1), 3)
            forms[name + "_equal"] = bool(torch.equal(Cv, C))
            del wv, Cv
        forms["headline_over_plain"] = round(forms["plain_ms"] / ms_step, 2)
        forms["headline_over_m4ri"] = round(forms["m4ri_ms"] / ms_step, 2)
        forms["tc_fp4_over_tc_int8"] = round(forms["tc_ms"] / forms["tc_fp4_ms"], 2)

    if args.quick:
        if rank == 0:
            print(json.dumps({"metric": "GF(2) GEMM Tbitop/s", "value": round(value, 3),
                              "unit": "Tbitop/s", "ms_per_step": round(ms_step, 4),
                              "kernel_ms": round(kern_avg, 4), "size": M, "result_check": ok}))
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 0 if ok else 1

    # e2e through the C ABI with pinned host buffers
    del work
    torch.cuda.empty_cache()
    hA = torch.empty((M, wk), dtype=torch.int64, pin_memory=True)
    hB = torch.empty((K, wn), dtype=torch.int64, pin_memory=True)
    hC = torch.empty((M, wn), dtype=torch.int64, pin_memory=True)
    hA.copy_(A)
    hB.copy_(B)
    del A, B, C, Cp
    torch.cuda.empty_cache()

    def e2e_step():
        check(L.mela_matmul_packed_host(hA.data_ptr(), wk, hB.data_ptr(), wn, hC.data_ptr(), wn,
                                        M, K, N, v))

    e2e_step()  # warm the stream-ordered pool
    parallel.barrier(ws)
    e2e_steps = max(1, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    dt_e2e = parallel.max_over_ranks(ws, (time.perf_counter() - t0) / e2e_steps)
    e2e = {"value": round(ws * BITOPS / dt_e2e / 1e12, 3), "unit": "Tbitop/s",
           "h2d_bytes_per_step": int(hA.numel() * 8 + hB.numel() * 8),
           "d2h_bytes_per_step": int(hC.numel() * 8), "ms_per_step": round(dt_e2e * 1e3, 3),
           "timing": "host clock around the blocking mela_matmul_packed_host call"}
    del hA, hB, hC

    extras = {}
    if ws > 1 and not args.no_extras:
        # every rank takes part (its share of the batch; the gather and the max are collectives)
        try:
            extras["batched_sharded"] = bench_batched_sharded(torch, ws, rank)
        except Exception as e:  # reported, never silently dropped
            extras["batched_sharded"] = {"error": f"{type(e).__name__}: {e}"}
        torch.cuda.empty_cache()
    if rank == 0 and not args.no_extras:
        for name, fn in (("drop_in_gateway", bench_gateway_config), ("batched", bench_batched),
                         ("dense_rank_null", bench_dense_rank), ("learned_dispatch", bench_dispatch)):
            try:
                extras[name] = fn(torch)
            except Exception as e:  # reported, never silently dropped
                extras[name] = {"error": f"{type(e).__name__}: {e}"}
            torch.cuda.empty_cache()
    if rank == 0:
        peak = measure_int8_peak(torch)
        if args.variant == "tc_fp4":
            # dense FP4 runs at twice the INT8 rate on this part (9 vs 4.5 P ops/s nominal)
            peak *= 2.0
        achieved = BITOPS / (kern_avg * 1e-3) / 1e12  # 2 ops per MAC
        cpu_rate, threads, isa = None, None, None
        try:
            os.environ.setdefault("OMP_DYNAMIC", "FALSE")
            cpu_rate, _, threads, isa = cpu_reference_sample(1)
        except Exception as e:  # reported, not fatal
            isa = f"unavailable: {e}"
        ms_, ks_, ns_ = CPU_SAMPLE
        line = {
            "metric": "GF(2) GEMM Tbitop/s at 32k^3",
            "value": round(value, 3),
            "unit": "Tbitop/s",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms_step, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": {"tc": "u8 (0/1 INT8 operands, INT32 sums)",
                      "tc_fp4": "fp4_e2m1 (0/1 operands, unit scales), f32 sums (exact below 2^24)"}[args.variant],
            "data": "synthetic (seeded splitmix64 Bernoulli(1/2), generated on device)",
            "config": {"workload": f"gemm_gf2_{M}^3" if M == K == N else f"gemm_gf2_{M}x{K}x{N}",
                       "m": M, "k": K, "n": N,
                       "variant": {"tc": "tc (tcgen05 kind::i8)",
                                   "tc_fp4": "tc_fp4 (tcgen05 kind::mxf4, e2m1 0/1, unit scales)"}[args.variant],
                       "seed": SEED,
                       "l2": "inputs larger than L2 (256 MiB packed + %s expanded operands)" % ("1 GiB" if args.variant == "tc_fp4" else "2 GiB"),
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                       "result_check": "ok" if ok else "MISMATCH"},
            "roofline": {"bound": "tensor", "achieved": round(achieved, 1), "peak": round(peak, 1),
                         "unit": "TFLOP/s", "frac": round(achieved / peak, 4),
                         # dram read + write bytes of one launch: an ncu capture of the FP4 kernel at
                         # 16384^3 (0.805 GB) scaled by m*n*k to the full launch
                         "traffic": (0.8050e9 * (M * N * K) / 16384 ** 3) if args.variant == "tc_fp4" else None,
                         "traffic_unit": "bytes per launch",
                         "kernel": "gemm_tc_pair_kernel", "kernel_ms": round(kern_avg, 4),
                         "peak_source": ("2 x dense INT8 measured in this run (cuBLASLt int8 GEMM 8192^3 "
                                         "via torch._int_mm, best of 10): the FP4 rate is twice the INT8 "
                                         "rate" if args.variant == "tc_fp4" else
                                         "dense INT8 measured in this run: cuBLASLt int8 GEMM 8192^3 "
                                         "via torch._int_mm, best of 10 (int8 ops as FLOPs)"),
                         "nominal": 9000.0 if args.variant == "tc_fp4" else 4500.0,
                         "frac_of_nominal": round(achieved / (9000.0 if args.variant == "tc_fp4" else 4500.0), 4)},
            "cpu_baseline": {"value": round(cpu_rate, 4) if cpu_rate else None, "unit": "Tbitop/s",
                             "cores": threads, "kind": "reference",
                             "sample": f"reference mela_matmul_gf2 ({isa}) on A * B[:, :{ns_}] "
                                       f"({ms_}x{ks_} * {ks_}x{ns_} logical), one call"},
            "e2e": e2e,
            "gpu_launches": 3 * args.steps,  # expand A, transposing expand of B, product
            "forms": forms,
            "clocks": clk,
            "device_error_flags": flags,
        }
        line.update(extras)
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0 if ok else 1


def elim_only():
    """Three ranks and three RREFs (first call, graph capture, replay) of the 16384 x 32768 rank-12000 configuration by the
    tensor-core elimination form (the dense section's inputs), for profiling."""
    import torch
    from mex_linear_algebra_b200 import device as D, gen, _lib
    from mex_linear_algebra_b200._lib import check, lib
    m, r0, n = 16384, 12000, 32768
    A = D.matmul(D.rand_dense(2, 0, m, r0), D.rand_dense(2, 1, r0, n), m, r0, n, variant="tc")
    for (i, a, b) in gen.replacement_triples(m, 164):
        A[i] = A[a] ^ A[b]
    L = lib()
    s = torch.cuda.current_stream().cuda_stream
    wc = n // 64
    wsb = L.mela_elim_workspace_size(m, n)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    dr = torch.zeros(1, dtype=torch.int64, device="cuda")
    dpv = torch.empty(m, dtype=torch.int64, device="cuda")
    dpr = torch.empty(m, dtype=torch.int64, device="cuda")
    out = {}
    for name, fn in (("rank", L.mela_dev_rank), ("rref", L.mela_dev_rref)):
        Mx = A.clone()
        calls = []
        for _ in range(3):  # first call, graph capture, replay
            Mx.copy_(A)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record()
            check(fn(_lib.ELIM_TC, Mx.data_ptr(), wc, m, n, dr.data_ptr(), dpv.data_ptr(), dpr.data_ptr(),
                     ws.data_ptr(), wsb, s))
            e1.record()
            e1.synchronize()
            calls.append((round(e0.elapsed_time(e1), 3), round((time.perf_counter() - t0) * 1e3, 3)))
        out[name + "_ms"] = calls[-1][0]
        out[name + "_calls_device_host_ms"] = calls
        out[name] = int(dr.item())
    print(json.dumps(out))


def batch_only(lo: int, hi: int, logical: bool = False, reps: int = 3):
    """Profiling aid: the parity-check batch (seed 3) restricted to the matrices
    with lo <= m < hi, packed (or, with `logical`, MATLAB logical) input
    resident in HBM, launched without a graph; prints the per-run time."""
    import numpy as np
    import torch
    from mex_linear_algebra_b200 import device as D, gen
    shapes, offsets, buf = gen.ldpc_batch(20000, 3)
    sel = (shapes[:, 0] >= lo) & (shapes[:, 0] < hi)
    idx = np.nonzero(sel)[0]
    sh = shapes[sel]
    wcs = (sh[:, 1] + 63) // 64
    packed = np.concatenate([buf[offsets[i]:offsets[i] + shapes[i, 0] * w] for i, w in zip(idx, wcs)])
    plan = D.BatchPlan(sh)
    d = torch.from_numpy(packed.view(np.int64)).cuda()
    ranks, zt = plan.outputs()
    if logical:
        d = plan.unpack_logical(d)
    run = plan.run_logical if logical else plan.run
    for _ in range(2):
        run(d, ranks, zt, use_graph=False)
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run(d, ranks, zt, use_graph=False)
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    print(json.dumps({"matrices": int(sel.sum()), "m_range": [lo, hi], "input": "logical" if logical else "packed",
                      "ms": round(min(times), 3),
                      "classes": plan.stats()}))
    plan.close()


def form_only(form: str, reps: int = 3):
    """Profiling aid: C = A*B at the --size cube (seed 1) by one product form,
    `reps` timed calls after a warm-up; prints the median time and rate."""
    import torch
    from mex_linear_algebra_b200 import _lib, device as D
    v = _lib.GEMM_VARIANTS[form]
    A = D.rand_dense(SEED, 0, M, K)
    B = D.rand_dense(SEED, 1, K, N)
    C = D.empty_packed(M, N)
    wsb = D.matmul_workspace(v, M, K, N)
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
    D.matmul(A, B, M, K, N, variant=v, out=C, workspace=ws)
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        D.matmul(A, B, M, K, N, variant=v, out=C, workspace=ws)
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    ts.sort()
    ms = ts[len(ts) // 2]
    print(json.dumps({"form": form, "size": M, "ms": round(ms, 3), "tbitops": round(BITOPS / (ms * 1e-3) / 1e12, 1)}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["mela", "reference"], default="mela")
    ap.add_argument("--size", type=int, default=32768,
                    help="square product size (32768 is the benchmark; smaller sizes are for profiling)")
    ap.add_argument("--quick", action="store_true",
                    help="device timing only: no e2e, CPU baseline, peak, forms or extras")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched / dense-rank / dispatch sections")
    ap.add_argument("--variant", choices=["tc", "tc_fp4"], default="tc_fp4",
                    help="tensor-core form timed as the headline (both are reported)")
    ap.add_argument("--elim-only", action="store_true",
                    help="profiling aid: build the dense rank configuration and run one rank and one "
                         "RREF with the tensor-core elimination form, print their times, nothing else")
    ap.add_argument("--batch-only", nargs=2, type=int, metavar=("M_LO", "M_HI"),
                    help="profiling aid: run the parity-check batch restricted to M_LO <= m < M_HI "
                         "(packed input, no graph) and print its time, nothing else")
    ap.add_argument("--batch-logical", action="store_true",
                    help="with --batch-only: start from the MATLAB logical input instead")
    ap.add_argument("--form-only", choices=["plain", "m4ri", "tc", "tc_fp4"],
                    help="profiling aid: time one product form at the --size cube, nothing else")
    args = ap.parse_args()
    set_size(args.size)
    if args.form_only:
        return form_only(args.form_only)
    if args.elim_only:
        return elim_only()
    if args.batch_only:
        return batch_only(*args.batch_only, logical=args.batch_logical)
    from mex_linear_algebra_b200 import parallel
    ws, rank, local = parallel.world()
    if args.impl == "reference":
        return run_reference(args, ws, rank)
    return run_mela(args, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
