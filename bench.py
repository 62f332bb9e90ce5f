#!/usr/bin/env python
"""Benchmark: FP64-accurate solves per second on B200, mixed precision +
iterative refinement, batched and served forms against plain FP64.

Workloads (--workload; the default is the first):
  mixed    Mixed-precision Cholesky + IR, n = 16384, 32 RHS: A = Q diag(s) Q^T,
           Q the orthogonal factor of a seeded N(0,1) matrix, s log-spaced over
           [1, 1e6]; B ~ N(0,1).  One step = egpu_dposv_mixed (tcgen05 TF32 x 3
           trailing updates, FP64 refinement to backward error <= 1e-14).  The
           plain FP64 path (egpu_dposv: Cholesky + HPD solve) is timed on the
           same A and B in the same run and reported beside it.
  lu       Plain FP64 LU with partial pivoting + solve, n = 8192, 64 RHS,
           A ~ U[-1,1], B ~ N(0,1): egpu_dgetrf + egpu_dgetrs per step.
  chol     Plain FP64 Cholesky + HPD solve, n = 2048, 16 RHS, A = G G^T + n I.
  batched  4096 HPD + 4096 general systems, n ~ U{32..512}, 1-8 RHS, one
           persistent launch per kind, the step replayed from a CUDA graph.
  serve    Poisson request stream through the continuous-batching server.

  value      device-resident inputs (HBM), CUDA events on the library stream
  e2e        the same solves through the host-memory C ABI entry, pinned host
             inputs copied in and the solutions copied out every step
  roofline   the dominant kernel, from per-launch CUDA events recorded inside
             the timed region
  cpu_baseline  the CPU oracle (the reference's algorithm restated in C,
             OpenMP over all host cores), rank 0 only, on a bounded sample

--impl reference runs the oracle arm alone on the host cores.
Multi-GPU (torchrun, one rank per GPU): every rank solves its own
independently seeded problems; no data-path collective ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NB = 128
SEED = 20240
FP64_PEAK_TFLOPS = 37.15  # measured DMMA peak, profiles/fp64_peak.md
HBM_PEAK_GBS_FALLBACK = 6650.0

WORKLOADS = {
    "mixed": {"n": 16384, "nrhs": 32, "kappa": 1e6,
              "metric": "FP64-accurate solves/sec (HPD solve, n=16384, 32 RHS, kappa 1e6): mixed-precision+IR",
              "desc": "mixed-precision Cholesky (tcgen05 TF32x3 trailing updates) + FP64 iterative refinement to "
                      "backward error <= 1e-14, n=16384, nb=128, 32 RHS, A = Q diag(s) Q^T, s log-spaced [1, 1e6]"},
    "lu": {"n": 8192, "nrhs": 64,
           "metric": "FP64-accurate solves/sec (LU-PP factor + 64-RHS solve, n=8192)",
           "desc": "LU partial pivoting + solve, n=8192, nb=128, 64 RHS (plain FP64)"},
    "batched": {"count": 4096, "nmin": 32, "nmax": 512, "rmin": 1, "rmax": 8, "n": 512, "nrhs": 8,
                "metric": "FP64-accurate solves/sec (batched uneven: 4096 HPD + 4096 GE systems, n in [32, 512])",
                "desc": "batched uneven solves: 4096 HPD (G G^T + n I) and 4096 general (U[-1,1]) systems, n ~ U{32..512}, "
                        "1-8 RHS, FP64, one persistent launch per kind (autotuned grid), the step captured in a CUDA graph"},
    "serve": {"rate": 2000.0, "window_s": 2.0, "nmin": 64, "nmax": 8192, "kmin": 1e2, "kmax": 1e8, "rmin": 1,
              "rmax": 64, "pool": 48, "budget": 150 << 30, "slots": 4, "n": 8192, "nrhs": 64,
              "metric": "FP64-accurate solves/sec and p50/p99 latency (served stream, Poisson 2000 req/s): mixed+IR",
              "desc": "request server, continuous batching: Poisson arrivals (mean 2000 req/s, 2 s window), 50/50 "
                      "HPD/GE, n log-uniform [64, 8192], kappa log-uniform [1e2, 1e8] (Q diag(s) Q^T), 1-64 RHS, "
                      "150 GB HBM budget, 4 slots; served form: the pool's matrices resident on the device (registered "
                      "once, factors formed by the first request on each and reused), structure test for GE requests; "
                      "plain_fp64: every request a full FP64 factor-and-solve from its host A"},
    "chol": {"n": 2048, "nrhs": 16,
             "metric": "FP64-accurate solves/sec (Cholesky + 16-RHS HPD solve, n=2048)",
             "desc": "Cholesky + HPD solve, lower, n=2048, nb=128, 16 RHS (plain FP64)"},
}


def flops_lu_solve(n, nrhs):
    return 2.0 * n ** 3 / 3.0 + 2.0 * n * n * nrhs


def flops_chol_solve(n, nrhs):
    return n ** 3 / 3.0 + 2.0 * n * n * nrhs


def fp64_peak_probe():
    """FP64 DMMA throughput of the current GPU (TFLOP/s) from the
    benchmark-only library (elemental_b200/bench_csrc/fp64_peak.cu)."""
    import ctypes
    from elemental_b200 import build as _b
    L = ctypes.CDLL(_b.BENCH_LIB)
    v = ctypes.c_double()
    rc = L.egpu_bench_fp64_peak(ctypes.byref(v))
    if rc != 0:
        raise RuntimeError(f"FP64 peak probe failed (cudaError {rc})")
    return v.value


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE).  The
    process group is NCCL; EGPU_BENCH_BACKEND=gloo selects gloo for the
    host-side tests of this plumbing."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(os.environ.get("EGPU_BENCH_BACKEND", "nccl"), timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, x, device):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_of(ws, rank, sizes, kinds):
    """The systems this rank owns when `ws` ranks share one list of
    independent systems (egpu_partition_systems: largest first to the least
    loaded rank, cost n^3/3 HPD, 2n^3/3 GE).  Every rank computes the same
    partition; returns (owned indices in list order, per-rank loads)."""
    import elemental_b200 as eg
    owner, load = eg.partition_systems(sizes, kinds, ws)
    return [i for i in range(len(sizes)) if owner[i] == rank], load


def gather_to_host(ws, obj):
    """Every rank's `obj` on every rank (host-side exchange of statuses and
    results; the data path itself has no collective)."""
    if ws == 1:
        return [obj]
    import torch.distributed as dist
    out = [None] * ws
    dist.all_gather_object(out, obj)
    return out


def make_inputs(kind, n, nrhs, seed, device=None):
    """Seeded inputs of a workload (numpy, column-major; the mixed workload's
    A is built on the GPU when ``device`` is given)."""
    from elemental_b200 import inputs
    if kind == "lu":
        A = inputs.uniform(n, n, seed)
    elif kind == "chol":
        A = inputs.spd_ggt(n, seed)
    else:
        A = inputs.spd_spectrum(n, WORKLOADS["mixed"]["kappa"], seed, device=device)
    B = inputs.normal(n, nrhs, seed + 1)
    return A, B


def cpu_checker():
    """The CPU implementation timed beside the GPU: the reference's own code
    (oracle/_ref/libelemref.so: Elemental compiled from its sources, level-3
    flops in the scipy wheel's OpenBLAS on every host core) when it is built,
    else the C restatement (oracle/liboracle.so, OpenMP).  Returns (module,
    kind, description)."""
    from oracle import ref
    if ref.available():
        return ref, "reference", "Elemental's own code (oracle/_ref, OpenBLAS on all host cores)"
    from oracle import pyoracle as orc
    orc.set_threads(os.cpu_count() or 1)
    return orc, "port", "the C restatement of the reference (oracle/liboracle.so, OpenMP on all host cores)"


def cpu_solve(kind, n, nrhs, seed):
    """One FP64 factor + solve on the host cores by the CPU checker (Cholesky +
    HPDSolve for chol/mixed, LU + lu::SolveAfter for lu); returns seconds.
    The mixed workload's matrix is timed as G G^T + n I of the same order
    (the factorization's cost does not depend on the spectrum, and the
    Q diag(s) Q^T construction needs an n^3 QR on the host)."""
    M, _, _ = cpu_checker()
    A, B = make_inputs("lu" if kind == "lu" else "chol", n, nrhs, seed)
    t0 = time.perf_counter()
    if kind == "lu":
        F, p, st = M.lu(A, NB)
        X = M.lu_solve_after(F, p, B, 0)
    else:
        _, X, st = M.hpd_solve(A, B, 0, nb=NB)
    dt = time.perf_counter() - t0
    assert st == 0 and np.isfinite(X).all()
    return dt


def flops_of(kind, n, nrhs):
    return flops_lu_solve(n, nrhs) if kind == "lu" else flops_chol_solve(n, nrhs)


def cpu_sample(kind, n_full, nrhs, seed, budget_s, reps):
    """Time the CPU checker on the full-size solve when `reps` of them fit in
    about budget_s (estimated from one run at a quarter of the order), else on the largest
    n <= n_full (halving) that fits, flop-scaled and labelled so.  Returns
    (seconds per full-size solve, reps timed, sample description)."""
    n_probe = max(512, n_full // 4)
    t_probe = cpu_solve(kind, n_probe, nrhs, seed)
    est = t_probe * flops_of(kind, n_full, nrhs) / flops_of(kind, n_probe, nrhs)
    reps = max(1, min(reps, int(budget_s / max(est, 1e-9))))
    n_s = n_full
    while n_s > 1024 and est * flops_of(kind, n_s, nrhs) / flops_of(kind, n_full, nrhs) * reps > budget_s:
        n_s //= 2
    times = [cpu_solve(kind, n_s, nrhs, seed + 7 * i) for i in range(reps)]
    scale = flops_of(kind, n_s, nrhs) / flops_of(kind, n_full, nrhs)
    t_full = sum(times) / len(times) / scale
    what = "Cholesky + HPD solve" if kind != "lu" else "LU + solve"
    if n_s == n_full:
        return t_full, reps, f"{reps} full-size FP64 {what} runs at n={n_full}, {nrhs} RHS"
    return t_full, reps, f"{reps} FP64 {what} runs at n={n_s}, {nrhs} RHS (flop-scaled to n={n_full})"


def reference_record(args, workload):
    """The reference arm for one workload on the host cores: the reference's
    own code (oracle/_ref) with OpenBLAS on every core, or the restatement
    where the reference was not built.  The reference has no mixed-precision
    path: for the mixed workload its FP64 Cholesky + HPD solve is the
    baseline.  Each step is one full-size solve when `steps` of them fit in
    about two minutes, else the run is cut to what fits (at least one step;
    `steps` reports the number timed)."""
    W = WORKLOADS[workload]
    _, kind, what = cpu_checker()
    threads = os.cpu_count() or 1
    if workload == "batched":
        return reference_batched(args, W, kind, what, threads)
    if workload == "serve":
        return reference_serve(args, W, kind, what, threads)
    n, nrhs = W["n"], W["nrhs"]
    cpu_solve(workload, 512, nrhs, SEED)  # warm-up: library load, thread pool
    t_full, reps, sample = cpu_sample(workload, n, nrhs, SEED, 120.0, max(args.steps, 1))
    value = 1.0 / t_full
    return {
        "metric": W["metric"], "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": reps,
        "steps_requested": args.steps, "warmup": 1, "ms_per_step": t_full * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
        "config": {"workload": W["desc"], "n": n, "nrhs": nrhs, "nb": NB, "parallelism": f"{threads} host cores"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": kind,
                         "sample": sample + ", " + what},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def reference_batched(args, W, kind, what, threads):
    """The reference's HPD solves and GaussianEliminations (1 x 1 Grid form)
    on systems drawn from the batch (same sizes and right-hand-side counts),
    one after another, OpenBLAS on all host cores."""
    from elemental_b200 import inputs
    M, _, _ = cpu_checker()
    sizes, rhs = batched_sets(SEED, W)
    r = np.random.default_rng(SEED + 5)
    per_step = 16
    times = []
    steps = max(1, min(args.steps, 10))
    for s in range(1 + steps):
        idx = r.choice(W["count"], per_step, replace=False)
        mats = [(inputs.spd_ggt(sizes[0][i], int(i)), inputs.normal(sizes[0][i], rhs[0][i], int(i) + 1),
                 inputs.uniform(sizes[1][i], sizes[1][i], int(i) + 2), inputs.normal(sizes[1][i], rhs[1][i], int(i) + 3))
                for i in idx]
        t0 = time.perf_counter()
        for Ah, Bh, Ag, Bg in mats:
            M.hpd_solve(Ah, Bh, 0, nb=NB)
            M.gaussian_elimination(Ag, Bg, nb=NB)
        if s >= 1:
            times.append(time.perf_counter() - t0)
    value = 2 * per_step * len(times) / sum(times)
    return {
        "metric": W["metric"], "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": len(times),
        "steps_requested": args.steps, "warmup": 1, "ms_per_step": 1e3 * 2 * W["count"] / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "impl": "reference", "config": {"workload": W["desc"], "count_per_kind": W["count"],
                                        "parallelism": f"{threads} host cores"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": kind,
                         "sample": f"{per_step} HPD + {per_step} GE systems per step drawn from the batch, " + what},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def reference_serve(args, W, kind, what, threads):
    """The reference's FP64 rate on the served mix: Cholesky + solve and LU +
    solve timed at n = 2048 on all host cores, applied to the stream's mean
    work per request (E[n^3] of the log-uniform size law, 50/50 kinds, mean
    32 RHS); requests served one after another."""
    lo, hi = np.log(W["nmin"]), np.log(W["nmax"])
    en3 = (W["nmax"] ** 3 - W["nmin"] ** 3) / (3.0 * (hi - lo))
    en2 = (W["nmax"] ** 2 - W["nmin"] ** 2) / (2.0 * (hi - lo))
    k = 0.5 * (W["rmin"] + W["rmax"])
    work = 0.5 * (en3 / 3.0 + 2.0 * en2 * k) + 0.5 * (2.0 * en3 / 3.0 + 2.0 * en2 * k)
    ns = 2048
    cpu_solve("chol", 512, 32, SEED)
    tc = cpu_solve("chol", ns, 32, SEED)
    tl = cpu_solve("lu", ns, 32, SEED)
    rate = (flops_chol_solve(ns, 32) + flops_lu_solve(ns, 32)) / (tc + tl)  # FP64 flop/s on the host
    value = rate / work
    return {
        "metric": W["metric"], "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": 1,
        "warmup": 1, "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
        "config": {"workload": W["desc"], "parallelism": f"{threads} host cores"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": kind,
                         "sample": f"one Cholesky+solve and one LU+solve at n={ns}, 32 RHS ({what}); host flop rate "
                                   f"{rate / 1e9:.1f} GFLOP/s applied to the stream's mean work per request, each "
                                   f"request a full factor-and-solve (the reference keeps no state between calls)"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def timed(args, ws, dev, stream, h, step):
    """W warm-up steps, then K timed steps between barriers + syncs, with the
    launch trace and the clock sampler on; returns (ms over K, trace, launches, clocks)."""
    import torch
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize(dev)
        barrier(ws)
        torch.cuda.synchronize(dev)
        launches0 = h.launch_count()
        h.trace_enable(True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(dev.index) as clk:
            e0.record(stream)
            for _ in range(args.steps):
                step()
            e1.record(stream)
            torch.cuda.synchronize(dev)
        trace = h.trace_summary()
        trace["_busy_ms"] = h.trace_busy_ms()
        h.trace_enable(False)
        launches = h.launch_count() - launches0
        barrier(ws)
        ms = max_over_ranks(ws, e0.elapsed_time(e1), dev)
    return ms, trace, launches, clk.summary()


def backward_error(A, X, B):
    """max_j ||b_j - A x_j||_inf / (||A||_inf ||x_j||_inf + ||b_j||_inf) (torch, on the device)."""
    R = B - A @ X
    den = A.abs().sum(1).max() * X.abs().amax(0) + B.abs().amax(0)
    return float((R.abs().amax(0) / den).max())


# DRAM bytes (read + write) per algorithmic byte, from the committed ncu
# captures of the same kernels on smaller cases (traffic grows with the bytes
# the launch streams, so the ratio scales to the bench's launches)
TRAFFIC_RATIO = {
    "tc": (577.2 / 604.0, "profiles/tc_gemm_update_n12288.md: 330.6 + 246.6 MB of DRAM traffic for 604 MB of "
                          "algorithmic bytes, scaled to this run's bytes per launch"),
    "update": (429.1 / 352.0, "profiles/dgemm_update_k1024_n6144.md: 321.9 + 107.2 MB of DRAM traffic for 352 MB of "
                              "algorithmic bytes, scaled to this run's bytes per launch"),
}


def roofline_of(trace, kind, peaks, busy_total_ms):
    """Roofline line for one traced kernel class.  Its time is the class's
    busy time on the device (the union of its launches' intervals across the
    concurrent streams, egpu_trace_busy), not the sum of per-launch spans,
    which counts overlapped launches twice."""
    t = trace.get(kind, {})
    if not t or not t.get("launches") or t["busy_ms"] <= 0:
        return None
    ms = t["busy_ms"]
    ratio, source = TRAFFIC_RATIO.get(kind, (None, None))
    traffic = ratio * t["bytes"] / t["launches"] if ratio else None
    common = {"traffic_source": source, "algorithmic_bytes_per_launch": t["bytes"] / t["launches"],
              "launches": t["launches"], "time_ms": ms, "time_basis": "busy time of the kernel class (union of "
              "its launch intervals across streams, CUDA events on each launch's stream)",
              "share_of_busy_time": t["share_ms"] / busy_total_ms if busy_total_ms > 0 else None}
    if kind == "tc":  # FP32 C read-modify-write + split panels: HBM-bound at K = 128
        peak = peaks.get("hbm_gbs") or HBM_PEAK_GBS_FALLBACK
        achieved = t["bytes"] / (ms / 1e3) / 1e9
        return {"bound": "hbm", "kernel": "tc_gemm_kernel (tcgen05 TF32x3 trailing update)", "achieved": achieved,
                "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peaks.get("hbm_gbs") else "fallback",
                "tensor_tflops": t["flops"] / (ms / 1e3) / 1e12, "traffic": traffic, **common}
    achieved = t["flops"] / (ms / 1e3) / 1e12
    return {"bound": "tensor", "kernel": "dgemm_tma_kernel (FP64 DMMA trailing update)", "achieved": achieved,
            "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s", "frac": achieved / FP64_PEAK_TFLOPS, "traffic": traffic,
            "peak_source": "measured FP64 DMMA peak (profiles/fp64_peak.md); MEASURED_PEAKS.json has no FP64 entry",
            **common}


def kernel_table(trace, steps):
    """Per-class device time per step: busy (union across streams) and share
    (overlapped time split among the classes in flight; the shares add up to
    the traced busy time, which is at most the step time)."""
    return {k: {"busy_ms_per_step": v["busy_ms"] / steps, "share_ms_per_step": v["share_ms"] / steps,
                "launches_per_step": v["launches"] / steps}
            for k, v in trace.items() if v["launches"]}


def pinned_like(a):
    import torch
    t = torch.empty((a.size,), dtype=torch.float64, pin_memory=True).numpy().reshape(a.shape, order="F")
    np.copyto(t, a)
    return t


def our_arm(args, ws, rank, local, kind):
    import torch
    import elemental_b200 as eg

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    h = eg.Handle(local)
    h.set_blocksize(NB)
    stream = torch.cuda.Stream(device=dev)
    W = WORKLOADS[kind]
    n, nrhs = W["n"], W["nrhs"]
    seed = SEED + 1000 * rank
    A_host, B_host = make_inputs(kind, n, nrhs, seed, device=dev if kind == "mixed" else None)
    A0 = eg.colmajor_cuda(A_host, device=dev)
    B0 = eg.colmajor_cuda(B_host, device=dev)
    A = eg.empty_colmajor(n, n, device=dev)
    B = eg.empty_colmajor(n, nrhs, device=dev)
    p = torch.zeros(n, dtype=torch.int32, device=dev)
    info = {}

    # plain FP64 step (the drop-in path): restore A, B, factor, solve
    def plain_step():
        A.copy_(A0)
        B.copy_(B0)
        if kind == "lu":
            h.lu(A, p)
            h.lu_solve_after(A, p, B, eg.NORMAL)
        else:
            h.hpd_solve(A, B, eg.LOWER)

    def mixed_step():
        X, it, be = h.hpd_solve_mixed(A0, B0, eg.LOWER, 30, 1e-14)
        info["X"], info["iters"], info["berr"] = X, it, be

    step = mixed_step if kind == "mixed" else plain_step
    ms, trace, launches, clocks = timed(args, ws, dev, stream, h, step)
    ms_per_step = ms / args.steps
    value = ws * args.steps / (ms / 1e3)
    with torch.cuda.stream(stream):
        Xd = info["X"] if kind == "mixed" else B
        bwd = backward_error(A0, Xd, B0)
    plain = None
    if kind == "mixed":
        # the plain FP64 path on the same inputs, same timing rules
        pms, ptrace, plaunches, _ = timed(args, ws, dev, stream, h, plain_step)
        with torch.cuda.stream(stream):
            pbwd = backward_error(A0, B, B0)
        plain = {"value": ws * args.steps / (pms / 1e3), "unit": "solves/s", "ms_per_step": pms / args.steps,
                 "backward_error": pbwd, "api": "egpu_dposv (Cholesky + HPD solve, FP64)",
                 "roofline": roofline_of(ptrace, "update", measured_peaks(), ptrace.pop("_busy_ms")),
                 "kernels": kernel_table(ptrace, args.steps)}

    # ---- end to end through the host-memory C ABI, pinned host buffers
    Ah, Bh = pinned_like(A_host), pinned_like(B_host)
    Xh = pinned_like(np.zeros((n, nrhs), order="F"))
    h.set_stream(None)
    hs = torch.cuda.ExternalStream(eg.lib().egpu_get_stream(h.h), device=dev)
    e2e_ms = []
    for i in range(args.warmup + args.steps):
        if kind != "mixed":
            np.copyto(Ah, A_host)
            np.copyto(Bh, B_host)
        barrier(ws)
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(hs)
        if kind == "mixed":
            h.host_hpd_solve_mixed(Ah, Bh, Xh)
        elif kind == "lu":
            h.host_gaussian_elimination(Ah, Bh)
        else:
            h.host_hpd_solve(Ah, Bh)
        f1.record(hs)
        f1.synchronize()
        if i >= args.warmup:
            e2e_ms.append(max_over_ranks(ws, f0.elapsed_time(f1), dev))
    e2e_value = ws * len(e2e_ms) / (sum(e2e_ms) / 1e3)
    Xe = Xh if kind == "mixed" else Bh
    xref = (info["X"] if kind == "mixed" else B).cpu().numpy()
    xerr = float(np.max(np.abs(Xe - xref)) / max(1e-300, np.max(np.abs(xref))))
    in_bytes = 8 * (n * n + n * nrhs)
    out_bytes = 8 * n * nrhs + (0 if kind == "mixed" else 8 * n * n)

    if rank != 0:
        return
    peaks = measured_peaks()
    busy = trace.pop("_busy_ms")
    roof = roofline_of(trace, "tc" if kind == "mixed" else "update", peaks, busy)
    cpu = None
    if ws == 1 and not args.no_cpu:
        _, ckind, cwhat = cpu_checker()
        t_full, _, sample = cpu_sample(kind, n, nrhs, seed, 30.0, 1)
        cpu = {"value": 1.0 / t_full, "unit": "solves/s", "cores": os.cpu_count() or 1, "kind": ckind,
               "sample": sample + ", " + cwhat}
    f_useful = flops_of(kind, n, nrhs)
    line = {
        "metric": W["metric"], "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if kind != "mixed" else "f64 (tf32x3 trailing updates)",
        "data": "synthetic (seeded)",
        "config": {"workload": W["desc"], "n": n, "nrhs": nrhs, "nb": NB,
                   "parallelism": f"{ws} independent systems" if ws > 1 else "1 GPU",
                   "l2": f"inputs ({8 * n * n >> 20} MiB) larger than L2",
                   "step_includes": "device restore copy of A and B" if kind != "mixed"
                   else "FP32/FP64 working copies of A made inside egpu_dposv_mixed"},
        "equiv_fp64_tflops": f_useful / (ms_per_step / 1e3) / 1e12,
        "backward_error": bwd,
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": in_bytes,
                "d2h_bytes_per_step": out_bytes,
                "api": {"mixed": "egpu_host_dposv_mixed", "lu": "egpu_host_dgesv (GaussianElimination)",
                        "chol": "egpu_host_dposv (HPDSolve)"}[kind],
                "x_rel_diff_vs_device_path": xerr},
        "roofline": roof,
        "kernels": kernel_table(trace, args.steps),
        "traced_busy_ms_per_step": busy / args.steps,
        "gpu_launches": launches,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    if kind == "mixed":
        line["refinement"] = {"corrections": info["iters"], "berr": info["berr"], "tol": 1e-14}
        line["plain_fp64"] = plain
        line["speedup_vs_plain_fp64"] = value / plain["value"]
    return line


def batched_sets(seed, W):
    r = np.random.default_rng(seed)
    cnt = W["count"]
    sizes = [r.integers(W["nmin"], W["nmax"] + 1, cnt), r.integers(W["nmin"], W["nmax"] + 1, cnt)]
    rhs = [r.integers(W["rmin"], W["rmax"] + 1, cnt), r.integers(W["rmin"], W["rmax"] + 1, cnt)]
    return [[int(x) for x in s] for s in sizes], [[int(x) for x in s] for s in rhs]


def arm_batched(args, ws, rank, local):
    """C4: 4096 HPD + 4096 general systems of uneven order in one persistent
    launch per kind, the step (refill + both launches, the two kinds on two
    streams) captured once in a CUDA graph and replayed."""
    import torch
    import elemental_b200 as eg

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    W = WORKLOADS["batched"]
    h = eg.Handle(local)
    # one list of 2 x count systems shared by all ranks (multi-GPU: each rank
    # factors the systems the partition gives it; no data-path collective)
    seed = SEED
    sizes, rhs = batched_sets(seed, W)
    mine, shard_load = shard_of(ws, rank, sizes[0] + sizes[1], [0] * W["count"] + [1] * W["count"])
    own = [[i for i in mine if i < W["count"]], [i - W["count"] for i in mine if i >= W["count"]]]
    sizes = [[sizes[k][i] for i in own[k]] for k in (0, 1)]
    rhs = [[rhs[k][i] for i in own[k]] for k in (0, 1)]
    cnt = [len(sizes[0]), len(sizes[1])]
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed + rank)
    # one arena per kind for A and B (column-major, ld = n rounded up to even)
    arenas = []
    for kind in (0, 1):
        lds = [n + (n & 1) for n in sizes[kind]]
        offA = np.cumsum([0] + [ld * n for ld, n in zip(lds, sizes[kind])])
        offB = np.cumsum([0] + [ld * k for ld, k in zip(lds, rhs[kind])])
        A = torch.empty(int(offA[-1]), dtype=torch.float64, device=dev)
        B = torch.empty(int(offB[-1]), dtype=torch.float64, device=dev)
        views_A, views_B = [], []
        for i, n in enumerate(sizes[kind]):
            va = torch.as_strided(A, (n, n), (1, lds[i]), int(offA[i]))
            vb = torch.as_strided(B, (n, rhs[kind][i]), (1, lds[i]), int(offB[i]))
            if kind == 0:
                g = torch.randn(n, n, dtype=torch.float64, device=dev, generator=gen)
                va.copy_(g @ g.T + n * torch.eye(n, dtype=torch.float64, device=dev))
            else:
                va.copy_(torch.rand(n, n, dtype=torch.float64, device=dev, generator=gen) * 2 - 1)
            vb.copy_(torch.randn(n, rhs[kind][i], dtype=torch.float64, device=dev, generator=gen))
            views_A.append(va)
            views_B.append(vb)
        arenas.append({"A": A, "B": B, "A0": A.clone(), "B0": B.clone(), "vA": views_A, "vB": views_B,
                       "lds": lds, "offA": offA, "offB": offB})
    torch.cuda.synchronize()
    plans = [eg.BatchPlan(h, k, arenas[k]["vA"], arenas[k]["vB"]) for k in (0, 1)]
    s0, s1 = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    tuned = []
    with torch.cuda.stream(s0):
        for k in (0, 1):
            tuned.append(plans[k].autotune(reps=1, stream=s0))
    torch.cuda.synchronize()
    plans_shape = [p_.shape() for p_ in plans]

    def refill_and_run():
        cur = torch.cuda.current_stream()
        s1.wait_stream(cur)
        for k, s in ((0, cur), (1, s1)):
            with torch.cuda.stream(s):
                arenas[k]["A"].copy_(arenas[k]["A0"])
                arenas[k]["B"].copy_(arenas[k]["B0"])
                plans[k].run(s)
        cur.wait_stream(s1)

    graph = torch.cuda.CUDAGraph()
    s0.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s0):
        refill_and_run()  # untimed warm run outside capture
    torch.cuda.synchronize()
    with torch.cuda.graph(graph, stream=s0):
        refill_and_run()
    torch.cuda.synchronize()

    def step():
        graph.replay()

    ms, trace, launches, clocks = timed(args, ws, dev, s0, h, step)
    total = 2 * W["count"]  # the whole list, all ranks together
    value = total * args.steps / (ms / 1e3)
    # one traced (uncaptured) run for the kernel's own time
    with torch.cuda.stream(s0):
        for k in (0, 1):
            arenas[k]["A"].copy_(arenas[k]["A0"])
            arenas[k]["B"].copy_(arenas[k]["B0"])
        h.trace_enable(True)
        for k in (0, 1):
            plans[k].run(s0)
        torch.cuda.synchronize()
        ktrace = h.trace_summary()
        h.trace_enable(False)
    infos = [plans[k].info(s0) for k in (0, 1)]
    assert all(v == 0 for inf in infos for v in inf)
    # accuracy on a sample of systems (backward error, FP64)
    r = np.random.default_rng(seed + 5)
    berr = 0.0
    for k in (0, 1):
        for i in r.choice(cnt[k], min(32, cnt[k]), replace=False):
            a0 = torch.as_strided(arenas[k]["A0"], arenas[k]["vA"][i].shape, arenas[k]["vA"][i].stride(),
                                  arenas[k]["vA"][i].storage_offset())
            b0 = torch.as_strided(arenas[k]["B0"], arenas[k]["vB"][i].shape, arenas[k]["vB"][i].stride(),
                                  arenas[k]["vB"][i].storage_offset())
            berr = max(berr, backward_error(a0, arenas[k]["vB"][i], b0))
    # plain FP64 path (one egpu_dposv / egpu_dgesv call per system) on a sample
    samp = 128
    t_plain = 0.0
    with torch.cuda.stream(s0):
        for k in (0, 1):
            idx = r.choice(cnt[k], min(samp, cnt[k]), replace=False)
            work = [(torch.as_strided(arenas[k]["A0"], arenas[k]["vA"][i].shape, arenas[k]["vA"][i].stride(),
                                      arenas[k]["vA"][i].storage_offset()).clone(),
                     arenas[k]["vB"][i].clone()) for i in idx]
            work = [(a.t().contiguous().t(), b.t().contiguous().t()) for a, b in work]
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s0)
            for A_, B_ in work:
                if k == 0:
                    h.hpd_solve(A_, B_, eg.LOWER)
                else:
                    h.gaussian_elimination(A_, B_)
            e1.record(s0)
            torch.cuda.synchronize()
            t_plain += e0.elapsed_time(e1) / len(idx) * W["count"]
    plain_value = total / (t_plain / 1e3)
    # e2e: pinned host arenas in, both plans, solutions out, every step
    hostA = [arenas[k]["A0"].cpu().pin_memory() for k in (0, 1)]
    hostB = [arenas[k]["B0"].cpu().pin_memory() for k in (0, 1)]
    outB = [torch.empty_like(hostB[k]).pin_memory() for k in (0, 1)]
    e2e_ms = []
    with torch.cuda.stream(s0):
        for i in range(args.warmup + args.steps):
            barrier(ws)
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f0.record(s0)
            for k in (0, 1):
                arenas[k]["A"].copy_(hostA[k], non_blocking=True)
                arenas[k]["B"].copy_(hostB[k], non_blocking=True)
                plans[k].run(s0)
                outB[k].copy_(arenas[k]["B"], non_blocking=True)
            f1.record(s0)
            f1.synchronize()
            if i >= args.warmup:
                e2e_ms.append(max_over_ranks(ws, f0.elapsed_time(f1), dev))
    e2e_value = total * len(e2e_ms) / (sum(e2e_ms) / 1e3)
    h2d = sum(int(hostA[k].numel() + hostB[k].numel()) * 8 for k in (0, 1))
    d2h = sum(int(outB[k].numel()) * 8 for k in (0, 1))
    for p_ in plans:
        p_.close()
    refined = batched_refined(args, ws, dev, h, arenas, cnt, total, ms, r)
    if rank != 0:
        return
    flops = sum(n ** 3 / 3.0 for n in sizes[0]) + sum(2.0 * n ** 3 / 3.0 for n in sizes[1])
    t = ktrace.get("other", {})
    achieved = t["flops"] / (t["ms"] / 1e3) / 1e12 if t.get("ms") else None
    cpu = None
    if ws == 1 and not args.no_cpu:
        M, ckind, cwhat = cpu_checker()
        idx = r.choice(min(cnt), 24, replace=False)
        mats = []
        for i in idx:
            for k in (0, 1):
                n = sizes[k][i]
                a = arenas[k]["A0"][int(arenas[k]["offA"][i]):int(arenas[k]["offA"][i]) + arenas[k]["lds"][i] * n]
                b = arenas[k]["B0"][int(arenas[k]["offB"][i]):int(arenas[k]["offB"][i]) + arenas[k]["lds"][i] * rhs[k][i]]
                Ah_ = np.asfortranarray(a.cpu().numpy().reshape((arenas[k]["lds"][i], n), order="F")[:n])
                Bh_ = np.asfortranarray(b.cpu().numpy().reshape((arenas[k]["lds"][i], rhs[k][i]), order="F")[:n])
                mats.append((k, Ah_, Bh_))
        M.hpd_solve(mats[0][1], mats[0][2], 0, nb=NB)  # warm-up
        t0 = time.perf_counter()
        for k, Ah_, Bh_ in mats:
            if k == 0:
                M.hpd_solve(Ah_, Bh_, 0, nb=NB)
            else:
                M.gaussian_elimination(Ah_, Bh_, nb=NB)
        dt = time.perf_counter() - t0
        cpu = {"value": len(mats) / dt, "unit": "solves/s", "cores": os.cpu_count() or 1, "kind": ckind,
               "sample": "24 HPD + 24 GE systems drawn from the batch, one after another, " + cwhat}
    line = {
        "metric": W["metric"], "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, generated on the device)",
        "config": {"workload": W["desc"], "count_per_kind": W["count"], "n_range": [W["nmin"], W["nmax"]],
                   "rhs_range": [W["rmin"], W["rmax"]], "parallelism": "1 GPU" if ws == 1 else f"{ws} GPUs, one list sharded by egpu_partition_systems (greedy n^3 balance)",
                   "l2": f"arenas ({sum(int(a['A'].numel()) for a in arenas) * 8 >> 20} MiB) larger than L2",
                   "step_includes": "device refill of every matrix and right-hand side, both batched launches"},
        "equiv_fp64_tflops": flops / (ms / args.steps / 1e3) / 1e12,
        "backward_error": berr,
        "autotuned_grid": {"hpd": tuned[0][1], "ge": tuned[1][1]},
        "autotuned_shapes": {"hpd": plans_shape[0], "ge": plans_shape[1]},
        "fp32_ir": refined,
        "shard": {"systems_per_rank": cnt, "load_balance": float(max(shard_load) / (sum(shard_load) / ws))}
        if ws > 1 else None,
        "plain_fp64": {"value": plain_value, "unit": "solves/s",
                       "api": "egpu_dposv / egpu_dgesv, one call per system (sampled, 128 per kind)"},
        "speedup_vs_plain_fp64": value / plain_value,
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "api": "egpu_batch_plan_run with pinned host arenas copied in and solutions copied out"},
        "roofline": {"bound": "tensor", "kernel": "chol_batched_kernel + lu_batched_kernel (FP64 DMMA)",
                     "achieved": achieved, "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s",
                     "frac": achieved / FP64_PEAK_TFLOPS if achieved else None,
                     "peak_source": "measured FP64 DMMA peak (profiles/fp64_peak.md)",
                     # profiles/batched_kernel_512.md: 1.66 + 1.43 GB of DRAM traffic for 512 GE systems of
                     # these shapes; the step's GE launch has W["count"] of them
                     "traffic": 3.09e9 * W["count"] / 512,
                     "traffic_source": "profiles/batched_kernel_512.md (the GE launch; scaled by the system count)"},
        "kernels": {k: {"ms": v["ms"], "launches": v["launches"]} for k, v in ktrace.items() if v["launches"]},
        "gpu_launches": launches + 2 * args.steps,
        "gpu_launches_note": "2 persistent batched kernels per step, replayed from the CUDA graph",
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    return line


def batched_refined(args, ws, dev, h, arenas, cnt, total, fp64_ms, r):
    """C4's FP32+IR variant on the same systems: refined batch plans (FP32
    working copies, FP64 iterative refinement to backward error <= 1e-14,
    an FP64 re-solve in the same launch for a system whose refinement
    stalls), autotuned, the step (refill of the right-hand sides + both
    launches) captured in a CUDA graph and timed like the FP64 plans.  The
    refined plans leave A unchanged, so the step refills only B."""
    import torch
    import elemental_b200 as eg

    s0, s1 = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    for k in (0, 1):
        arenas[k]["A"].copy_(arenas[k]["A0"])
        arenas[k]["B"].copy_(arenas[k]["B0"])
    torch.cuda.synchronize()
    plans = [eg.BatchPlan(h, k, arenas[k]["vA"], arenas[k]["vB"], precision=1) for k in (0, 1)]
    tuned = []
    with torch.cuda.stream(s0):
        for k in (0, 1):
            tuned.append(plans[k].autotune(reps=1, stream=s0))
    torch.cuda.synchronize()
    shapes = [p_.shape() for p_ in plans]

    def refill_and_run():
        cur = torch.cuda.current_stream()
        s1.wait_stream(cur)
        for k, s in ((0, cur), (1, s1)):
            with torch.cuda.stream(s):
                arenas[k]["B"].copy_(arenas[k]["B0"])
                plans[k].run(s)
        cur.wait_stream(s1)

    graph = torch.cuda.CUDAGraph()
    s0.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s0):
        refill_and_run()
    torch.cuda.synchronize()
    with torch.cuda.graph(graph, stream=s0):
        refill_and_run()
    torch.cuda.synchronize()
    ms, _, launches, clocks = timed(args, ws, dev, s0, h, graph.replay)
    infos = [plans[k].info(s0) for k in (0, 1)]
    iters = [plans[k].iters(s0) for k in (0, 1)]
    torch.cuda.synchronize()
    berr = 0.0
    for k in (0, 1):
        for i in r.choice(cnt[k], min(32, cnt[k]), replace=False):
            b0 = torch.as_strided(arenas[k]["B0"], arenas[k]["vB"][i].shape, arenas[k]["vB"][i].stride(),
                                  arenas[k]["vB"][i].storage_offset())
            berr = max(berr, backward_error(arenas[k]["vA"][i], arenas[k]["vB"][i], b0))
    for p_ in plans:
        p_.close()
    del graph
    hist = {}
    for its in iters:
        for v in its:
            hist[str(v)] = hist.get(str(v), 0) + 1
    return {"value": total * args.steps / (ms / 1e3), "unit": "solves/s", "ms_per_step": ms / args.steps,
            "speedup_vs_fp64_batched": fp64_ms / ms, "backward_error": berr,
            "failed_systems": sum(1 for inf in infos for v in inf if v != 0),
            "corrections_histogram": hist,
            "corrections_note": "refinement corrections per system; -1 = re-solved in FP64 inside the launch "
                                "after the refinement stalled",
            "autotuned_grid": {"hpd": tuned[0][1], "ge": tuned[1][1]},
            "autotuned_shapes": {"hpd": shapes[0], "ge": shapes[1]},
            "step_includes": "device refill of every right-hand side (A is left unchanged), both refined launches",
            "gpu_launches": launches + 2 * args.steps, "clocks": clocks}


def serve_stream(seed, W, device):
    """The request stream: a pool of matrices (log-uniform n and kappa) in
    pinned host memory and a seeded Poisson arrival sequence over the pool."""
    import torch
    from elemental_b200 import inputs
    r = np.random.default_rng(seed)
    pool = []
    for i in range(W["pool"]):
        n = int(np.exp(r.uniform(np.log(W["nmin"]), np.log(W["nmax"]))))
        kappa = float(np.exp(r.uniform(np.log(W["kmin"]), np.log(W["kmax"]))))
        A = inputs.spd_spectrum_torch(n, kappa, seed + i, device)
        Ah = torch.empty((n * n,), dtype=torch.float64, pin_memory=True)
        Ah.copy_(A.t().reshape(-1))  # symmetric: column-major values
        Bh = torch.empty((n * W["rmax"],), dtype=torch.float64, pin_memory=True)
        Bh.copy_(torch.from_numpy(inputs.normal(n, W["rmax"], seed + 500 + i).ravel(order="F")))
        pool.append((n, kappa, Ah.numpy().reshape((n, n), order="F"), Bh.numpy().reshape((n, W["rmax"]), order="F")))
        del A
    torch.cuda.empty_cache()
    t, reqs = 0.0, []
    while True:
        t += r.exponential(1.0 / W["rate"])
        if t > W["window_s"]:
            break
        reqs.append((t, int(r.integers(0, W["pool"])), int(r.integers(W["rmin"], W["rmax"] + 1)), int(r.integers(0, 2))))
    return pool, reqs


def run_stream(eg, W, pool, reqs, mode, device_index, resident=False):
    """Replay the arrival sequence against a server; returns per-request
    records.  resident: the pool's matrices are registered with the server
    (copied to the device once, inside the timed region, for each kind the
    stream asks of them) and requests send only B; otherwise every request
    carries its A."""
    srv = eg.Server(device_index, hbm_budget_bytes=W["budget"], slots=W["slots"], mode=mode, tol=1e-14)
    ids, outs = [], []
    t0 = time.perf_counter()
    mids = {}
    if resident:
        for key in sorted({(pi, kind) for (_, pi, _, kind) in reqs}):
            mids[key] = srv.register(key[1], pool[key[0]][2])
    for (ta, pi, k, kind) in reqs:
        now = time.perf_counter() - t0
        if ta > now:
            time.sleep(ta - now)
        n, _, Ah, Bh = pool[pi]
        X = np.zeros((n, k), order="F")
        if resident:
            ids.append(srv.submit_resident(mids[(pi, kind)], Bh[:, :k], X))
        else:
            ids.append(srv.submit(kind, Ah, Bh[:, :k], X))
        outs.append(X)
    srv.drain()
    t_end = time.perf_counter() - t0
    recs = [srv.query(i) for i in ids]
    srv.close()
    return recs, outs, t_end


def arm_serve(args, ws, rank, local):
    """C5: the served stream through the request server, mixed mode (value)
    and FP64 mode (plain_fp64) on the same arrivals."""
    import torch
    import elemental_b200 as eg
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    W = WORKLOADS["serve"]
    seed = SEED + 1000 * rank
    pool, reqs = serve_stream(seed, W, dev)
    # warm-up: a few requests per mode (kernels loaded, workspaces sized)
    for mode in (1, 0):
        run_stream(eg, W, pool, [(0.0, i % len(pool), 4, i % 2) for i in range(max(args.warmup, 3))], mode, local)
    # the served form (mode 1, resident matrices and factors), the plain FP64
    # path (mode 0, every request a full factor-and-solve from its host A),
    # and for attribution mode 0 with residency and mode 1 without
    runs = {"served": (1, True), "plain": (0, False), "fp64_resident": (0, True), "mixed_nonresident": (1, False)}
    res = {}
    clocks = None
    for key, (mode, resident) in runs.items():
        barrier(ws)
        with ClockSampler(local) as clk:
            recs, outs, t_end = run_stream(eg, W, pool, reqs, mode, local, resident)
        if key == "served":
            clocks = clk.summary()
        ok = [i for i, r_ in enumerate(recs) if r_ and r_["status"] == 0]
        lat = np.array([recs[i]["latency_ms"] for i in ok])
        # backward error on a sample (host FP64)
        rs = np.random.default_rng(seed + 9)
        berr = 0.0
        for i in rs.choice(ok, min(24, len(ok)), replace=False):
            _, pi, k, _ = reqs[i]
            n, _, Ah, Bh = pool[pi]
            R = Bh[:, :k] - Ah @ outs[i]
            den = np.abs(Ah).sum(axis=1).max() * np.abs(outs[i]).max(axis=0) + np.abs(Bh[:, :k]).max(axis=0)
            berr = max(berr, float((np.abs(R).max(axis=0) / den).max()))
        paths = [recs[i]["path"] for i in ok]
        res[key] = {"value": len(ok) / t_end, "completed": len(ok), "submitted": len(reqs), "makespan_s": t_end,
                    "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                    "backward_error_sampled": berr, "mode": mode, "resident": resident,
                    "paths": {"fp64": paths.count(0), "mixed": paths.count(1), "batched": paths.count(2),
                              "mixed_fell_back": paths.count(3), "ge_as_hpd_fp64": paths.count(4),
                              "ge_as_hpd_mixed": paths.count(5), "resident_factored": paths.count(6),
                              "resident_factor_reused": paths.count(7)}}
    if rank != 0:
        return
    m, p = res["served"], res["plain"]
    line = {
        "metric": W["metric"], "value": m["value"], "unit": "solves/s", "n_gpus": ws, "steps": 1,
        "warmup": args.warmup, "ms_per_step": m["makespan_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (resident FP64 factors; mixed tf32x3 + IR for large one-off HPD requests)",
        "data": "synthetic (seeded pool of 48 matrices, seeded Poisson arrivals)",
        "config": {"workload": W["desc"], "requests": len(reqs), "parallelism": "1 GPU",
                   "l2": "pool matrices up to 512 MiB, larger than L2",
                   "step_includes": "the whole stream: host->device copies, solves, device->host copies"},
        "latency_ms": {"p50": m["p50_ms"], "p99": m["p99_ms"]},
        "served": m,
        "plain_fp64": p,
        "speedup_vs_plain_fp64": m["value"] / p["value"],
        "attribution": {"fp64_resident": res["fp64_resident"], "mixed_nonresident": res["mixed_nonresident"]},
        "e2e": {"value": m["value"], "unit": "solves/s",
                "h2d_bytes_per_step": int(sum(8 * pool[pi][0] ** 2 for pi, _ in {(pi, kd) for _, pi, _, kd in reqs})
                                          + sum(8 * pool[pi][0] * k for _, pi, k, _ in reqs)),
                "d2h_bytes_per_step": int(sum(8 * pool[pi][0] * k for _, pi, k, _ in reqs)),
                "api": "egpu_server_submit / egpu_server_query with pinned host buffers"},
        "roofline": None,
        "gpu_launches": None,
        "clocks": clocks,
        "cpu_baseline": None,
    }
    if ws == 1 and not args.no_cpu:
        _, ckind, cwhat = cpu_checker()
        rec = reference_serve(args, W, ckind, cwhat, os.cpu_count() or 1)
        line["cpu_baseline"] = rec["cpu_baseline"]
    return line


def kernel_case(args):
    """One launch of a single kernel class at a chosen size, for profiler
    captures (ncu -k ...): 'update' = one lower Herk trailing update
    (n x n, K = 128), 'gemm' = one Gemm trailing update, 'lu' = one LU with
    partial pivoting (warm-up call first), 'panel' = one LU panel (n x 128), 'diag' = one diagonal-block Cholesky (128 x 128), 'mixed' = one
    mixed-precision HPD solve, 'tc' = the tcgen05 trailing update alone,
    'chol' = one plain FP64 Cholesky (warm-up call first); 'inverse',
    'hpdinverse', 'trtri', 'ldl', 'revchol', 'det' time those entry points
    (best of three, flops: 2n^3, n^3, n^3/3, n^3/3, n^3/3, 2n^3/3); 'sweep32'
    = the FP32 solve sweeps alone; 'batched' = one launch of each batched
    kernel over n systems of the C4 shapes; 'mixed_lu' = one mixed-precision
    GaussianElimination.  --k sets the inner dimension of 'update' and 'gemm'
    (default 128)."""
    import torch
    import elemental_b200 as eg
    from elemental_b200 import inputs
    h = eg.Handle(0)
    n = args.n
    if args.case in ("update", "gemm"):
        A = eg.empty_colmajor(n, args.k).normal_()
        C = eg.empty_colmajor(n, n).normal_()
        if args.case == "update":
            h.herk(eg.LOWER, eg.NORMAL, -1.0, A, 1.0, C)
        else:
            Bm = eg.empty_colmajor(args.k, n).normal_()
            h.gemm(eg.NORMAL, eg.NORMAL, -1.0, A, Bm, 1.0, C)
    elif args.case == "chol":
        A0 = inputs.spd_spectrum_torch(n, 1e3, SEED, "cuda")
        A = A0.clone()
        h.cholesky(A)  # warm-up
        A.copy_(A0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        h.cholesky(A)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        print(json.dumps({"case": "chol", "n": n, "ms": ms, "tflops": n ** 3 / 3 / ms / 1e9}))
        return
    elif args.case == "lu":
        # LU with partial pivoting of a U[-1,1] matrix of order n: warm-up, timed
        A0 = eg.colmajor_cuda(torch.rand(n, n, dtype=torch.float64, device="cuda") * 2 - 1)
        A = A0.clone()
        p = torch.zeros(n, dtype=torch.int32, device="cuda")
        h.lu(A, p)
        A.copy_(A0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        h.lu(A, p)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        print(json.dumps({"case": "lu", "n": n, "ms": ms, "tflops": 2 * n ** 3 / 3 / ms / 1e9}))
        return
    elif args.case == "panel":
        A = eg.colmajor_cuda(inputs.uniform(n, NB, 1))
        p = torch.zeros(NB, dtype=torch.int32, device="cuda")
        h.lu(A, p)
    elif args.case == "peaks":
        # roofline denominators and vendor reference points on this GPU
        out = {"dmma_peak_tflops": fp64_peak_probe()}
        torch.backends.cuda.matmul.allow_tf32 = False
        for m in (4096, 8192):
            a = torch.randn(m, m, dtype=torch.float64, device="cuda")
            b_ = torch.randn(m, m, dtype=torch.float64, device="cuda")
            for _ in range(2):
                c = a @ b_
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(3):
                c = a @ b_
            e1.record()
            torch.cuda.synchronize()
            out[f"cublas_dgemm_{m}_tflops"] = 2 * m ** 3 * 3 / (e0.elapsed_time(e1) / 1e3) / 1e12
            del a, b_, c
        for m in (2048, 8192, 16384):
            g = torch.randn(m, m, dtype=torch.float64, device="cuda")
            spd = g @ g.T + m * torch.eye(m, dtype=torch.float64, device="cuda")
            torch.linalg.cholesky(spd)
            torch.linalg.lu_factor(g)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            torch.linalg.cholesky(spd)
            e1.record()
            torch.cuda.synchronize()
            out[f"cusolver_potrf_{m}_ms"] = e0.elapsed_time(e1)
            if m <= 8192:
                e0.record()
                torch.linalg.lu_factor(g)
                e1.record()
                torch.cuda.synchronize()
                out[f"cusolver_getrf_{m}_ms"] = e0.elapsed_time(e1)
            del g, spd
        print(json.dumps(out))
        return
    elif args.case == "mixed":
        # one mixed-precision HPD solve (kappa 1e6, 32 RHS) at order --n
        A = inputs.spd_spectrum_torch(n, 1e6, 7, "cuda")
        B = torch.randn(32, n, dtype=torch.float64, device="cuda").t()
        X, it, be = h.hpd_solve_mixed(A, B)
        assert be <= 1e-14
    elif args.case == "diag":
        A = eg.colmajor_cuda(inputs.spd_ggt(NB, 1))
        h.cholesky(A, eg.LOWER)
    elif args.case == "tc":
        # the mixed factorization's trailing update alone: C (n x n FP32, lower
        # triangle) -= L L^T with L n x 128, TF32 x 3 on tcgen05; three timed
        # launches (the trace separates the kernel from the operand splits)
        L = eg.empty_colmajor(n, NB).normal_()
        C = eg.empty_colmajor(n, n).normal_().float().t().contiguous().t()
        h.tc_gemm_split(L, L, C, alpha=-1.0, beta=1.0, lower=True, terms=3)
        torch.cuda.synchronize()
        h.trace_enable(True)
        for _ in range(3):
            h.tc_gemm_split(L, L, C, alpha=-1.0, beta=1.0, lower=True, terms=3)
        torch.cuda.synchronize()
        s = h.trace_summary()
        h.trace_enable(False)
        ms = s["tc"]["ms"] / max(1, s["tc"]["launches"])
        cbytes = 8.0 * n * (n + 1) / 2  # FP32 lower triangle read + written
        print(json.dumps({"case": "tc", "n": n, "ms_per_launch": ms, "c_gbs": cbytes / ms / 1e6,
                          "tf32_tflops": 3 * 2.0 * n * (n + 1) / 2 * NB / ms / 1e9}))
        return
    elif args.case == "sweep32":
        # the mixed solver's FP32 super-block sweeps alone at order n, 32 RHS:
        # one forward + backward launch, three timed repetitions (the trace
        # separates the super-block inverses ("other") from the sweeps)
        A = torch.randn(n, n, dtype=torch.float64, device="cuda")
        A = A @ A.T + n * torch.eye(n, dtype=torch.float64, device="cuda")
        L = torch.linalg.cholesky(A)
        del A
        ld = (n + 31) // 32 * 32
        store = torch.zeros((n, ld), dtype=torch.float32, device="cuda")
        L32 = torch.as_strided(store, (n, n), (1, ld))
        L32.copy_(L.float())
        del L
        X = eg.colmajor_cuda(torch.randn(n, 32, dtype=torch.float64, device="cuda"))
        h.sweep32_solve(L32, X, 2)  # warm-up
        torch.cuda.synchronize()
        h.trace_enable(True)
        for _ in range(3):
            h.sweep32_solve(L32, X, 2)  # forward + backward, one launch
        torch.cuda.synchronize()
        s = h.trace_summary()
        h.trace_enable(False)
        sw = s["solve"]
        ms = sw["busy_ms"] / sw["launches"]
        print(json.dumps({"case": "sweep32", "n": n, "nrhs": 32, "ms_per_solve": ms, "ms_per_sweep": ms / 2,
                          "triangle_gbs": 2 * 2.0 * n * n / ms / 1e6,
                          "prepare_ms": s["other"]["busy_ms"] / max(1, s["other"]["launches"])}))
        return
    elif args.case == "batched":
        # one launch of each batched kernel over --n systems of the C4 shapes
        # (n ~ U{32..512}, 8 RHS): HPD first, then GE; warm-up launch first
        r = np.random.default_rng(SEED)
        sizes = [int(x) for x in r.integers(32, 513, n)]
        def fresh(kind):
            As = [inputs.spd_spectrum_torch(m, 1e3, SEED + i, "cuda") if kind == 0 else
                  eg.colmajor_cuda(torch.rand(m, m, dtype=torch.float64, device="cuda") * 2 - 1)
                  for i, m in enumerate(sizes)]
            Bs = [eg.colmajor_cuda(torch.randn(m, 8, dtype=torch.float64, device="cuda")) for m in sizes]
            return As, Bs
        for kind, solve in ((0, h.hpd_solve_batched), (1, h.gaussian_elimination_batched)):
            solve(*fresh(kind))  # warm-up
            As, Bs = fresh(kind)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            info = solve(As, Bs)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            fl = sum((m ** 3 / 3 if kind == 0 else 2 * m ** 3 / 3) + 2 * m * m * 8 for m in sizes)
            print(json.dumps({"case": "batched", "kind": ["hpd", "ge"][kind], "count": n, "ms": ms,
                              "tflops": fl / ms / 1e9, "failed": int(sum(1 for v in info if v))}))
        return
    elif args.case == "mixed_lu":
        # one mixed-precision GaussianElimination at order n, 32 RHS, U[-1,1]
        A = eg.colmajor_cuda(inputs.uniform(n, n, SEED))
        B = eg.colmajor_cuda(inputs.normal(n, 32, SEED + 1))
        h.gaussian_elimination_mixed(A, B)  # warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        X, it, be = h.gaussian_elimination_mixed(A, B)
        e1.record()
        torch.cuda.synchronize()
        print(json.dumps({"case": "mixed_lu", "n": n, "ms": e0.elapsed_time(e1), "corrections": it, "berr": be,
                          "mode": h.mixed_mode()}))
        return
    elif args.case in ("inverse", "hpdinverse", "trtri", "ldl", "revchol", "det"):
        # the next rows (inverses, determinants, LDL, ReverseCholesky) at order
        # n: one warm-up call, then three timed calls on fresh copies of A
        if args.case in ("inverse", "det"):
            A0 = eg.colmajor_cuda(inputs.uniform(n, n, SEED))
        elif args.case == "trtri":
            rs = np.random.default_rng(SEED)
            A0 = eg.colmajor_cuda(rs.standard_normal((n, n)) * (0.5 / n) + np.diag(rs.uniform(1.0, 2.0, n)))
        else:
            A0 = inputs.spd_spectrum_torch(n, 1e3, SEED, "cuda")
        flops = {"inverse": 2.0 * n ** 3, "hpdinverse": 1.0 * n ** 3, "trtri": n ** 3 / 3.0, "ldl": n ** 3 / 3.0,
                 "revchol": n ** 3 / 3.0, "det": 2.0 * n ** 3 / 3.0}[args.case]
        call = {"inverse": lambda A: h.inverse(A), "hpdinverse": lambda A: h.hpd_inverse(A),
                "trtri": lambda A: h.triangular_inverse(A), "ldl": lambda A: h.ldl(A),
                "revchol": lambda A: h.reverse_cholesky(A), "det": lambda A: h.safe_determinant(A, overwrite=True)}
        A = A0.clone()
        call[args.case](A)
        times = []
        for _ in range(3):
            A.copy_(A0)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            call[args.case](A)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        ms = min(times)
        print(json.dumps({"case": args.case, "n": n, "ms": ms, "algorithmic_gflop": flops / 1e9,
                          "tflops": flops / ms / 1e9, "frac_of_dmma_peak": flops / ms / 1e9 / FP64_PEAK_TFLOPS}))
        return
    torch.cuda.synchronize()
    print(json.dumps({"case": args.case, "n": n, "ok": True}))


NESTED = {"chol": "C1", "lu": "C2", "mixed": "C3", "batched": "C4", "serve": "C5"}
NESTED_KEYS = ("metric", "value", "unit", "ms_per_step", "steps", "backward_error", "latency_ms", "roofline", "e2e",
               "cpu_baseline", "plain_fp64", "speedup_vs_plain_fp64", "refinement", "kernels", "gpu_launches",
               "clocks", "config", "impl", "steps_requested", "fp32_ir", "autotuned_grid", "autotuned_shapes",
               "equiv_fp64_tflops")


def run_workload(args, ws, rank, local, workload):
    if args.impl == "reference":
        return reference_record(args, workload) if rank == 0 else None
    if workload == "batched":
        return arm_batched(args, ws, rank, local)
    if workload == "serve":
        return arm_serve(args, ws, rank, local)
    return our_arm(args, ws, rank, local, workload)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mixed", choices=sorted(WORKLOADS), help="benchmark configuration")
    ap.add_argument("--no-nested", action="store_true",
                    help="time only --workload (by default the mixed line also carries the other configurations)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline legs")
    ap.add_argument("--case", choices=["update", "gemm", "lu", "panel", "diag", "peaks", "mixed", "tc", "chol", "inverse",
                                       "hpdinverse", "trtri", "ldl", "revchol", "det", "sweep32", "batched",
                                       "mixed_lu"],
                    default=None,
                    help="run one launch of one kernel class (profiling)")
    ap.add_argument("--n", type=int, default=6144, help="size for --case")
    ap.add_argument("--k", type=int, default=NB, help="inner dimension for --case update/gemm")
    args = ap.parse_args()
    if args.case:
        kernel_case(args)
        return
    ws, rank, local = dist_setup()
    try:
        if args.impl == "reference" and ws > 1 and rank != 0:
            return  # the reference arm runs on rank 0 alone
        line = run_workload(args, ws, rank, local, args.workload)
        if args.workload == "mixed" and not args.no_nested:
            # every other benchmark configuration, timed in the same run under
            # the same rules, as nested records (the top-level line stays the
            # mixed-precision headline)
            line_cfgs = {}
            for wl in ("chol", "lu", "batched", "serve"):
                rec = run_workload(args, ws, rank, local, wl)
                if rec is not None:
                    line_cfgs[NESTED[wl] + "_" + wl] = {k: rec[k] for k in NESTED_KEYS if k in rec}
            if line is not None:
                line["configs"] = line_cfgs
        if line is not None and rank == 0:
            if args.workload == "mixed":
                line["config"]["benchmark_config"] = "C3"
            print(json.dumps(line), flush=True)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
