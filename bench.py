#!/usr/bin/env python
"""Benchmark: GF(2) GEMM Tbitop/s at 32768^3 on B200.

Workload (one step): C = A*B over GF(2) with A, B 32768 x 32768, iid
Bernoulli(1/2) from seed 1, packed uint64 row-major, computed by the
tcgen05 kind::i8 tensor-core form (operand preparation -- transpose of B and
0/1 byte expansion -- plus the tensor-core kernel).  Bit-ops are counted as
2*m*n*k (one AND and one XOR per term), the analogue of 2mnk FLOPs.

  value  -- device-timed (CUDA events, max over ranks) with packed inputs
            resident in HBM; inputs are 256 MiB packed + 2 GiB of expanded
            operands per step, all larger than L2 (126 MB).
  e2e    -- the same product through the C ABI host entry point
            mela_matmul_packed_host with pinned host buffers: the host->device
            copy of A and B and the device->host copy of C are inside the
            timed region of every step (host-timed around the blocking call).
  roofline -- the tensor-core kernel alone, timed live with CUDA events on its
            stream, against a dense INT8 peak measured in the same run
            (cuBLASLt int8 GEMM through torch._int_mm).
  cpu_baseline -- the reference's own mela_matmul_gf2 (compiled from its
            sources with its AVX512/OpenMP flags) on the host cores, on a
            2048 x 32768 * 32768 x 2048 sub-block of the same product.

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


def set_size(size: int) -> None:
    global M, K, N, BITOPS
    M = K = N = size
    BITOPS = 2.0 * M * N * K
CPU_SAMPLE = (2048, 32768, 2048)  # rows of A, K, columns of B for the CPU legs


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
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ distributed
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, value: float) -> float:
    if ws == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------ CPU legs
def cpu_reference_sample(steps: int = 1):
    """Time the reference gateway mela_matmul_gf2 (oracle/_ref) on the
    CPU sample; returns (Tbitop/s, seconds per call, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle as O
    ms, ks, ns = CPU_SAMPLE
    A = O.unpack(O.rand_dense(SEED, 0, ms, ks), ms, ks)
    B = O.unpack(O.rand_dense(SEED, 1, ks, ns), ks, ns)
    O.ref_call("mela_matmul_gf2", A[:64], B)  # warm the code and pages
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
    sample = (f"reference mela_matmul_gf2 ({isa} build, OpenMP) on A {ms}x{ks} * B {ks}x{ns} "
              f"(logical), a sub-block of the 32768^3 product; median of {args.steps} calls")
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
        "config": {"workload": "gemm_gf2_32768^3_sample", "m": ms, "k": ks, "n": ns},
        "cpu_baseline": {"value": round(rate, 4), "unit": "Tbitop/s", "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": round(rate, 4), "unit": "Tbitop/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ GPU leg
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


def run_mela(args, ws, rank, local):
    import torch
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
    v = _lib.GEMM_TC
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
    barrier(ws)

    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
            torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier(ws)
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
    barrier(ws)
    clk = clocks.stop()
    total_ms = t_start.elapsed_time(t_end)
    kernel_ms = [e1.elapsed_time(e2) for (_, e1, e2) in evs]
    total_ms = max_over_ranks(ws, total_ms)
    ms_step = total_ms / args.steps
    value = ws * BITOPS / (ms_step * 1e-3) / 1e12
    kern_avg = sum(kernel_ms) / len(kernel_ms)

    # correctness guard on the timed result: a block of rows against the plain form
    ok = True
    if rank == 0:
        rows = 256
        Cp = D.matmul(A[:rows], B, rows, K, N, variant="plain")
        ok = bool(torch.equal(Cp, C[:rows]))
    flags = D.device_error_flags()

    # the same product through the CUDA-core forms (one timed call each)
    forms = {"tc_ms": round(ms_step, 3)}
    if not args.quick:
        for name, var in (("plain", _lib.GEMM_PLAIN), ("m4ri", _lib.GEMM_M4RI)):
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
        forms["tc_over_plain"] = round(forms["plain_ms"] / ms_step, 2)
        forms["tc_over_m4ri"] = round(forms["m4ri_ms"] / ms_step, 2)

    if args.quick:
        if rank == 0:
            print(json.dumps({"metric": "GF(2) GEMM Tbitop/s", "value": round(value, 3),
                              "unit": "Tbitop/s", "ms_per_step": round(ms_step, 4),
                              "kernel_ms": round(kern_avg, 4), "size": M, "result_check": ok}))
        return 0 if ok else 1

    # e2e through the C ABI with pinned host buffers
    e2e = None
    del work
    torch.cuda.empty_cache()
    hA = torch.empty((M, wk), dtype=torch.int64, pin_memory=True)
    hB = torch.empty((K, wn), dtype=torch.int64, pin_memory=True)
    hC = torch.empty((M, wn), dtype=torch.int64, pin_memory=True)
    hA.copy_(A)
    hB.copy_(B)
    del A, B, C
    torch.cuda.empty_cache()

    def e2e_step():
        check(L.mela_matmul_packed_host(hA.data_ptr(), wk, hB.data_ptr(), wn, hC.data_ptr(), wn,
                                        M, K, N, v))

    e2e_step()  # warm the stream-ordered pool
    barrier(ws)
    e2e_steps = max(1, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    dt_e2e = (time.perf_counter() - t0) / e2e_steps
    dt_e2e = max_over_ranks(ws, dt_e2e)
    e2e = {"value": round(ws * BITOPS / dt_e2e / 1e12, 3), "unit": "Tbitop/s",
           "h2d_bytes_per_step": int(hA.numel() * 8 + hB.numel() * 8),
           "d2h_bytes_per_step": int(hC.numel() * 8), "ms_per_step": round(dt_e2e * 1e3, 3),
           "timing": "host clock around the blocking mela_matmul_packed_host call"}
    del hA, hB, hC

    line = None
    if rank == 0:
        peak = measure_int8_peak(torch)
        achieved = BITOPS / (kern_avg * 1e-3) / 1e12  # 2 int8 ops per MAC
        cpu_rate, cpu_dt, threads, isa = (None, None, None, None)
        try:
            os.environ.setdefault("OMP_DYNAMIC", "FALSE")
            cpu_rate, cpu_dt, threads, isa = cpu_reference_sample(1)
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
            "dtype": "u8",
            "data": "synthetic (seeded splitmix64 Bernoulli(1/2), generated on device)",
            "config": {"workload": "gemm_gf2_32768^3_tensor_core", "m": M, "k": K, "n": N,
                       "variant": "tc (tcgen05 kind::i8)", "seed": SEED,
                       "l2": "inputs larger than L2 (256 MiB packed + 2 GiB expanded operands)",
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                       "result_check": "ok" if ok else "MISMATCH"},
            "roofline": {"bound": "tensor", "achieved": round(achieved, 1), "peak": round(peak, 1),
                         "unit": "TFLOP/s", "frac": round(achieved / peak, 4), "traffic": None,
                         "kernel": "gemm_tc_kernel", "kernel_ms": round(kern_avg, 4),
                         "peak_source": "dense INT8 measured in this run: cuBLASLt int8 GEMM "
                                        "8192^3 via torch._int_mm, best of 10 (int8 ops as FLOPs)"},
            "cpu_baseline": {"value": round(cpu_rate, 4) if cpu_rate else None, "unit": "Tbitop/s",
                             "cores": threads, "kind": "reference",
                             "sample": f"reference mela_matmul_gf2 ({isa}) on A {ms_}x{ks_} * B "
                                       f"{ks_}x{ns_}, one call"},
            "e2e": e2e,
            "gpu_launches": 4 * args.steps,
            "forms": forms,
            "clocks": clk,
            "device_error_flags": flags,
        }
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0 if ok else 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["mela", "reference"], default="mela")
    ap.add_argument("--size", type=int, default=32768,
                    help="square problem size (32768 is the benchmark; smaller sizes are for profiling)")
    ap.add_argument("--quick", action="store_true",
                    help="device timing only: no e2e, CPU baseline, peak or form comparison")
    args = ap.parse_args()
    set_size(args.size)
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference(args, ws, rank)
    return run_mela(args, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
