#!/usr/bin/env python
"""bench.py -- throughput of the hcBLAS GEMM drop-in on B200.

Workload (one "step"): DGEMM, column-major, transA = N, transB = T,
M = N = K = 4096, alpha = 1, beta = 0, entries i.i.d. N(0,1) from seed 1 --
one hcblasDgemm call through the library's C ABI (libhcblas.so) on inputs
already resident in HBM.  A, B, C take 3 x 128 MiB > the 126 MB L2, so
consecutive steps do not hit in L2.

Printed (rank 0, one JSON line):
  value       whole-job TFLOPS (2*M*N*K per step per GPU / max-over-ranks time)
  e2e         the same metric through hcblasSetMatrix (H2D from pinned host
              memory) + hcblasDgemm + hcblasGetMatrix (D2H) per step
  roofline    the dominant kernel's achieved rate (CUDA events around each of
              its launches) against its peak, plus ncu DRAM traffic when a
              capture summary is committed under profiles/
  cpu_baseline  host CBLAS (OpenBLAS's cblas_dgemm, all host threads) on a
              bounded column sample of the same problem
  accuracy    normwise error of the GPU result against the double-double oracle
              on sampled columns, and against the CPU CBLAS result

Multi-GPU: GEMM calls are independent problems here (replicas only): every rank
runs the same workload on its own GPU; no collective is in the data path.

`--impl reference` times the reference's CPU GEMM path (host CBLAS) instead.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

M = N = K = 4096
ALPHA, BETA = 1.0, 0.0
FLOP = 2.0 * M * N * K
WORKLOAD = "dgemm_colmajor_NT_4096^3_alpha1_beta0_N01_seed1"
FP64_PEAK_NOMINAL_TFLOPS = 37.0  # B200 datasheet FP64 (no measured FP64 peak on this pool)


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


# ------------------------------------------------------------------ clocks --

class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)], stdout=self.fh,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for i, n in enumerate(names):
                if r[5 + i].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ------------------------------------------------------------ CPU baseline --

def cpu_cblas_sample(A, B, target_s=8.0, threads=None):
    """Time OpenBLAS cblas_dgemm (the reference's host CBLAS path) on a column
    sample C[:, :nb] of the same NT problem; returns (TFLOPS, nb, threads, C_sample)."""
    from oracle import cblas_ref
    threads = threads or os.cpu_count() or 1
    cblas_ref.set_threads(threads)
    Af = A  # column-major M x K, lda = M
    # op(B) = B^T with B column-major N x K (ldb = N): sample rows 0..nb-1 of B
    nb = 64
    while True:
        Bs = np.ascontiguousarray(B.reshape(K, N)[:, :nb]).reshape(-1)  # N x K sample, ld = nb
        Cs = np.zeros(M * nb)
        t0 = time.perf_counter()
        cblas_ref.gemm(1, 0, 1, M, nb, K, ALPHA, Af, M, Bs, nb, BETA, Cs, M)
        dt = time.perf_counter() - t0
        if dt * 4 > target_s or nb >= N:
            break
        nb = min(N, nb * 4)
    reps = max(1, int(target_s / max(dt, 1e-3) / 2))
    t0 = time.perf_counter()
    for _ in range(reps):
        cblas_ref.gemm(1, 0, 1, M, nb, K, ALPHA, Af, M, Bs, nb, BETA, Cs, M)
    dt = (time.perf_counter() - t0) / reps
    return 2.0 * M * nb * K / dt / 1e12, nb, threads, Cs, dt * reps


def run_reference_arm(args, rank):
    if rank != 0:
        return 0
    rng = np.random.default_rng(1)
    A = rng.standard_normal(M * K)
    B = rng.standard_normal(N * K)
    from oracle import cblas_ref
    threads = os.cpu_count() or 1
    cblas_ref.set_threads(threads)
    # size the per-step sample so that warmup + steps stay within ~2 minutes
    tf_est, nb, _, _, _ = cpu_cblas_sample(A, B, target_s=2.0, threads=threads)
    per_full = FLOP / (tf_est * 1e12)
    budget = 90.0 / max(args.steps + args.warmup, 1)
    nb = N if per_full <= budget else max(64, int(N * budget / per_full) // 64 * 64)
    Bs = np.ascontiguousarray(B.reshape(K, N)[:, :nb]).reshape(-1)
    Cs = np.zeros(M * nb)
    for _ in range(args.warmup):
        cblas_ref.gemm(1, 0, 1, M, nb, K, ALPHA, A, M, Bs, nb, BETA, Cs, M)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cblas_ref.gemm(1, 0, 1, M, nb, K, ALPHA, A, M, Bs, nb, BETA, Cs, M)
    dt = (time.perf_counter() - t0) / args.steps
    tflops = 2.0 * M * nb * K / dt / 1e12
    sample = ("full 4096^3 per step" if nb == N else
              f"C[:, :{nb}] column sample per step ({nb}/{N} of the flops)")
    line = {
        "impl": "reference", "metric": "dgemm_tflops", "value": round(tflops, 4),
        "unit": "TFLOPS", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dt * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic N(0,1) seed 1",
        "config": {"workload": WORKLOAD, "parallelism": "host threads"},
        "cpu_baseline": {"value": round(tflops, 4), "unit": "TFLOPS", "cores": threads,
                         "kind": "reference",
                         "sample": f"host CBLAS cblas_dgemm (OpenBLAS {cblas_ref.config().split()[1] if len(cblas_ref.config().split()) > 1 else ''}, "
                                   f"the CBLAS hcBLAS's tests link); {sample}"},
        "e2e": {"value": round(tflops, 4), "unit": "TFLOPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------- main --

def load_traffic(kernel):
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d.get(kernel)
    except Exception:
        return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    local = env_int("LOCAL_RANK", 0)

    if args.impl == "reference":
        return run_reference_arm(args, rank)

    import torch
    import hcblas_b200 as hb

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    stream = torch.cuda.Stream()
    s, h = hb.hcblasCreate(local, stream.cuda_stream)
    assert s == 0, f"hcblasCreate: {s}"

    rng = np.random.default_rng(1)
    A = rng.standard_normal(M * K)  # column-major M x K, lda = M
    B = rng.standard_normal(N * K)  # column-major N x K (op = T), ldb = N
    dA, dB = hb.DeviceArray(h, A), hb.DeviceArray(h, B)
    dC = hb.DeviceArray(h, nbytes=8 * M * N, dtype=np.float64)
    L = hb.lib()
    one = np.array([ALPHA])
    zero = np.array([BETA])

    def step():
        st = L.hcblasDgemm(h, hb.HCBLAS_OP_N, hb.HCBLAS_OP_T, M, N, K, one.ctypes.data, dA.ptr, M,
                           dB.ptr, N, zero.ctypes.data, dC.ptr, M)
        if st != 0:
            raise RuntimeError(f"hcblasDgemm status {st}")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    path = hb.hcblasGetLastPath(h)

    # ---- timed region (device-resident inputs) ----
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    hb.set_profiling(h, True)
    launches0 = hb.kernel_launch_count()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = hb.kernel_launch_count() - launches0
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1) / args.steps
    prof = hb.get_profile(h)
    hb.set_profiling(h, False)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * FLOP / (ms * 1e-3) / 1e12

    # dominant kernel: the one with the largest total time
    dom, (cnt, tot) = max(prof.items(), key=lambda kv: kv[1][1])
    kernel_ms = tot / cnt
    achieved = FLOP / (kernel_ms * 1e-3) / 1e12

    # ---- end to end through the C ABI with host buffers ----
    pin = lambda n: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    hA, hB, hC = pin(M * K), pin(N * K), pin(M * N)
    hA[:] = A
    hB[:] = B
    e2e_steps = max(1, min(args.steps, 5))
    for _ in range(1):
        hb.hcblasSetMatrix(h, M, K, 8, hA.ctypes.data, M, dA.ptr, M)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        assert hb.hcblasSetMatrix(h, M, K, 8, hA.ctypes.data, M, dA.ptr, M) == 0
        assert hb.hcblasSetMatrix(h, N, K, 8, hB.ctypes.data, N, dB.ptr, N) == 0
        step()
        assert hb.hcblasGetMatrix(h, M, N, 8, dC.ptr, M, hC.ctypes.data, M) == 0
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    if dist:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = world * FLOP / (e2e_ms * 1e-3) / 1e12

    # ---- accuracy (rank 0) and CPU baseline (rank 0, N = 1) ----
    line = None
    if rank == 0:
        from oracle import oracle as O
        Cg = hC.reshape(N, M).T  # (M, N) view of the column-major result
        cols = np.random.default_rng(5).choice(N, 8, replace=False)
        Bsamp = np.ascontiguousarray(B.reshape(K, N)[:, cols]).reshape(-1)
        _, ref = O.gemm(O.COL, 0, 1, M, len(cols), K, ALPHA, A, M, Bsamp, len(cols), BETA,
                        np.zeros(M * len(cols)), M)
        err_dd = O.normwise_rel_error(Cg[:, cols], ref)
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            tf, nb, thr, Cs, secs = cpu_cblas_sample(A, B, target_s=8.0)
            err_cpu = O.normwise_rel_error(Cg[:, :nb], Cs.reshape(nb, M).T)
            cpu = {"value": round(tf, 4), "unit": "TFLOPS", "cores": thr, "kind": "reference",
                   "sample": f"host CBLAS cblas_dgemm (OpenBLAS in the scipy wheel, the CBLAS "
                             f"hcBLAS's tests link) on C[:, :{nb}] of the same problem, "
                             f"{secs:.1f} s of CPU work",
                   "gpu_vs_cpu_normwise_err": err_cpu}
        traffic = load_traffic(dom)
        line = {
            "metric": "dgemm_tflops", "value": round(value, 3), "unit": "TFLOPS",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic N(0,1) seed 1",
            "config": {"workload": WORKLOAD, "M": M, "N": N, "K": K, "transA": "N",
                       "transB": "T", "order": "col", "alpha": ALPHA, "beta": BETA,
                       "path": path, "l2": "inputs 384 MiB exceed the 126 MB L2; no flush",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": round(e2e, 3), "unit": "TFLOPS",
                    "h2d_bytes_per_step": 8 * (M * K + N * K),
                    "d2h_bytes_per_step": 8 * M * N, "ms_per_step": round(e2e_ms, 3)},
            "roofline": {"kernel": dom, "bound": "fp64", "achieved": round(achieved, 3),
                         "peak": FP64_PEAK_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                         "frac": round(achieved / FP64_PEAK_NOMINAL_TFLOPS, 4),
                         "peak_source": "B200 nominal FP64 (no measured FP64 peak)",
                         "traffic": traffic, "kernel_ms": round(kernel_ms, 4),
                         "algorithmic_flop_per_launch": FLOP},
            "cpu_baseline": cpu,
            "accuracy": {"normwise_err_vs_double_double_oracle": err_dd,
                         "oracle_columns": len(cols)},
            "clocks": clocks,
            "gpu_launches": int(launches),
        }
    hb.hcblasDestroy(h)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
