#!/usr/bin/env python
"""Benchmark: FP64-accurate factor-and-solve throughput on B200.

Workload (default, one GPU): LU with partial pivoting + solve of one dense
system, n = 8192, block size 128, A ~ U[-1,1] (seeded), B = 64 right-hand
sides ~ N(0,1).  One "step" = restore A and B from pristine device copies,
factor (egpu_dgetrf), solve (egpu_dgetrs).  metric = solves per second
(systems factored and solved), whole job.

  value      device-resident inputs (HBM), CUDA events on the library stream
  e2e        the same factor-and-solve through the host-memory C ABI entry
             GaussianElimination (egpu_host_dgesv): pinned host A, B copied in,
             factored and solved, A and X copied back, every step
  roofline   the trailing-update kernel (FP64 DMMA GEMM), from per-launch CUDA
             events recorded inside the timed region
  cpu_baseline  the CPU oracle (the reference's algorithm restated in C,
             OpenMP over all host cores) on the same input, rank 0 only

--impl reference runs the oracle arm alone on the host cores.
Multi-GPU (torchrun, one rank per GPU): every rank factors its own
independently seeded system; no data-path collective ("scaling": "weak").
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

N = 8192
NRHS = 64
NB = 128
SEED = 20240
FP64_PEAK_TFLOPS = 37.15  # measured DMMA peak, profiles/fp64_peak.md
HBM_PEAK_GBS_FALLBACK = 6650.0


def flops_lu_solve(n, nrhs):
    return 2.0 * n ** 3 / 3.0 + 2.0 * n * n * nrhs


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
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
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
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
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


def cpu_oracle_solve(n, nrhs, seed, threads):
    """One LU + solve by the CPU oracle; returns seconds."""
    from elemental_b200 import inputs
    from oracle import pyoracle as orc
    orc.set_threads(threads)
    A = inputs.uniform(n, n, seed)
    B = inputs.normal(n, nrhs, seed + 1)
    t0 = time.perf_counter()
    F, p, st = orc.lu(A, NB)
    X = orc.lu_solve_after(F, p, B, orc.NORMAL)
    dt = time.perf_counter() - t0
    assert st == 0 and np.isfinite(X).all()
    return dt


def reference_arm(args, ws, rank):
    """CPU oracle timed on the host cores (the reference's own algorithm for
    this path, restated in C; the reference itself needs MPI + BLAS and is not
    built here)."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    # warm-up: small problems (thread pool, page faults)
    for _ in range(max(args.warmup, 0)):
        cpu_oracle_solve(512, NRHS, SEED, threads)
    # size the sample so that the K timed steps stay within ~150 s
    t_probe = cpu_oracle_solve(2048, NRHS, SEED, threads)
    est_full = t_probe * flops_lu_solve(N, NRHS) / flops_lu_solve(2048, NRHS)
    n_s = N
    while n_s > 1024 and est_full * (n_s / N) ** 3 * args.steps > 150.0:
        n_s //= 2
    times = [cpu_oracle_solve(n_s, NRHS, SEED + 7 * i, threads) for i in range(args.steps)]
    scale = flops_lu_solve(n_s, NRHS) / flops_lu_solve(N, NRHS)
    t_step = sum(times) / len(times) / scale  # seconds per full-size solve
    value = 1.0 / t_step
    line = {
        "metric": "FP64-accurate solves/sec (LU-PP factor + 64-RHS solve, n=8192)",
        "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded U[-1,1] A, N(0,1) B)", "impl": "reference",
        "config": {"workload": "LU partial pivoting + solve, n=8192, nb=128, 64 RHS", "n": N, "nrhs": NRHS,
                   "nb": NB, "parallelism": "host cores"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} LU+solve runs at n={n_s} (flop-scaled to n={N})"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def our_arm(args, ws, rank, local):
    import torch
    import elemental_b200 as eg
    from elemental_b200 import inputs

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    h = eg.Handle(local)
    h.set_blocksize(NB)
    stream = torch.cuda.Stream(device=dev)
    seed = SEED + 1000 * rank
    A_host = inputs.uniform(N, N, seed)
    B_host = inputs.normal(N, NRHS, seed + 1)
    A0 = eg.colmajor_cuda(A_host, device=dev)
    B0 = eg.colmajor_cuda(B_host, device=dev)
    A = eg.empty_colmajor(N, N, device=dev)
    B = eg.empty_colmajor(N, NRHS, device=dev)
    p = torch.zeros(N, dtype=torch.int32, device=dev)

    def step():
        A.copy_(A0)
        B.copy_(B0)
        h.lu(A, p)
        h.lu_solve_after(A, p, B, eg.NORMAL)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize(dev)
        # accuracy of the last solve (checked, reported)
        X = B.double()
        R = torch.from_numpy(B_host).to(dev) - torch.from_numpy(A_host).to(dev) @ X
        bwd = float(R.abs().sum(0).max() / (torch.from_numpy(A_host).to(dev).abs().sum(0).max() *
                                            X.abs().sum(0).max() * N * np.finfo(np.float64).eps))
        del R, X
        barrier(ws)
        torch.cuda.synchronize(dev)
        launches0 = h.launch_count()
        h.trace_enable(True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            e0.record(stream)
            for _ in range(args.steps):
                step()
            e1.record(stream)
            torch.cuda.synchronize(dev)
        trace = h.trace_summary()
        h.trace_enable(False)
        launches = h.launch_count() - launches0
        barrier(ws)
        ms = max_over_ranks(ws, e0.elapsed_time(e1), dev)

    ms_per_step = ms / args.steps
    value = ws * args.steps / (ms / 1e3)

    # ---- end to end through the host-memory C ABI (GaussianElimination)
    Ah = torch.empty((N * N,), dtype=torch.float64, pin_memory=True).numpy().reshape((N, N), order="F")
    Bh = torch.empty((N * NRHS,), dtype=torch.float64, pin_memory=True).numpy().reshape((N, NRHS), order="F")
    e2e_ms = []
    hs = torch.cuda.ExternalStream(eg.lib().egpu_get_stream(h.h) or 0, device=dev)
    h.set_stream(None)
    hs = torch.cuda.ExternalStream(eg.lib().egpu_get_stream(h.h), device=dev)
    for i in range(args.warmup + args.steps):
        np.copyto(Ah, A_host)
        np.copyto(Bh, B_host)
        barrier(ws)
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(hs)
        h.host_gaussian_elimination(Ah, Bh)
        f1.record(hs)
        f1.synchronize()
        if i >= args.warmup:
            e2e_ms.append(max_over_ranks(ws, f0.elapsed_time(f1), dev))
    e2e_value = ws * len(e2e_ms) / (sum(e2e_ms) / 1e3)
    xerr = float(np.max(np.abs(Bh - np.asarray(B.cpu().numpy()))) / max(1e-300, np.max(np.abs(Bh))))

    if rank != 0:
        return
    # ---- roofline of the dominant kernel (trailing-update DMMA GEMM)
    try:
        live_peak = h.measure_fp64_peak()
    except Exception:
        live_peak = None
    upd = trace["update"]
    achieved = upd["flops"] / (upd["ms"] / 1e3) / 1e12 if upd["ms"] > 0 else None
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            traffic = json.load(f).get("dgemm_update_bytes_per_launch")
    except Exception:
        pass
    total_ms = sum(v["ms"] for v in trace.values())
    # ---- CPU baseline (oracle on the host cores, same seeded input)
    cpu = None
    if ws == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        t = cpu_oracle_solve(N, NRHS, seed, threads)
        cpu = {"value": 1.0 / t, "unit": "solves/s", "cores": threads, "kind": "port",
               "sample": f"one LU+solve at n={N} (the full workload), oracle in C with OpenMP"}
    clocks = clk.summary()
    line = {
        "metric": "FP64-accurate solves/sec (LU-PP factor + 64-RHS solve, n=8192)",
        "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded U[-1,1] A, N(0,1) B)",
        "config": {"workload": "LU partial pivoting + solve, n=8192, nb=128, 64 RHS (plain FP64)", "n": N,
                   "nrhs": NRHS, "nb": NB, "parallelism": f"{ws} independent systems" if ws > 1 else "1 GPU",
                   "l2": "inputs (512 MiB) larger than L2", "step_includes": "device restore copy of A and B"},
        "tflops": flops_lu_solve(N, NRHS) / (ms_per_step / 1e3) / 1e12,
        "backward_error": bwd,
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": 8 * (N * N + N * NRHS),
                "d2h_bytes_per_step": 8 * (N * N + N * NRHS), "api": "egpu_host_dgesv (GaussianElimination)",
                "x_rel_diff_vs_device_path": xerr},
        "roofline": {"bound": "tensor", "kernel": "dgemm_tma_kernel (trailing update)",
                     "achieved": achieved, "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s",
                     "frac": (achieved / FP64_PEAK_TFLOPS) if achieved else None,
                     "peak_source": "measured FP64 DMMA peak (profiles/fp64_peak.md); MEASURED_PEAKS.json has no FP64 entry",
                     "peak_live_tflops": live_peak,
                     "traffic": traffic, "launches": upd["launches"],
                     "share_of_traced_time": upd["ms"] / total_ms if total_ms else None},
        "kernels": {k: {"ms": v["ms"], "launches": v["launches"]} for k, v in trace.items() if v["launches"]},
        "gpu_launches": launches,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def kernel_case(args):
    """One launch of a single kernel class at a chosen size, for profiler
    captures (ncu -k ...): 'update' = one lower Herk trailing update
    (n x n, K = 128), 'gemm' = one Gemm trailing update, 'panel' = one LU panel
    (n x 128), 'diag' = one diagonal-block Cholesky (128 x 128)."""
    import torch
    import elemental_b200 as eg
    from elemental_b200 import inputs
    h = eg.Handle(0)
    n = args.n
    if args.case in ("update", "gemm"):
        A = eg.empty_colmajor(n, NB).normal_()
        C = eg.empty_colmajor(n, n).normal_()
        if args.case == "update":
            h.herk(eg.LOWER, eg.NORMAL, -1.0, A, 1.0, C)
        else:
            Bm = eg.empty_colmajor(NB, n).normal_()
            h.gemm(eg.NORMAL, eg.NORMAL, -1.0, A, Bm, 1.0, C)
    elif args.case == "panel":
        A = eg.colmajor_cuda(inputs.uniform(n, NB, 1))
        p = torch.zeros(NB, dtype=torch.int32, device="cuda")
        h.lu(A, p)
    elif args.case == "peaks":
        # roofline denominators and vendor reference points on this GPU
        out = {"dmma_peak_tflops": h.measure_fp64_peak()}
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
    elif args.case == "diag":
        A = eg.colmajor_cuda(inputs.spd_ggt(NB, 1))
        h.cholesky(A, eg.LOWER)
    torch.cuda.synchronize()
    print(json.dumps({"case": args.case, "n": n, "ok": True}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--case", choices=["update", "gemm", "panel", "diag", "peaks"], default=None,
                    help="run one launch of one kernel class (profiling)")
    ap.add_argument("--n", type=int, default=6144, help="size for --case")
    args = ap.parse_args()
    if args.case:
        kernel_case(args)
        return
    ws, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            reference_arm(args, ws, rank)
        else:
            our_arm(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
