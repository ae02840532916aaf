#!/usr/bin/env python3
"""Benchmark: FP64-accurate SPD solve (tile Cholesky + forward/backward solves).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload fp64|mixed]

One step = one SPD solve A x = b of the workload (factor + both triangular
solves, plus refinement for the mixed workload) on one batch of synthetic
input already resident in HBM.  The metric is TFLOP/s with the FP64-equivalent
flop count n^3/3 + 2 n^2 nrhs (the same count for plain and mixed solves).

Workloads (synthetic, seeded, shapes and distributions of the reference
configurations):
  fp64  : n = 16384, tile b = 512, 1 rhs, A = G G^T / n + 1e-2 I, G ~ N(0,1)
          (plain FP64 tile Cholesky with DMMA updates)
Inputs are 2 GiB (> L2), and the factor runs in place, so A is restored from a
pristine copy before every step, outside the timed events (which also flushes
L2 between steps).

Multi-GPU: a single SPD system does not shard (the tile Cholesky exchanges a
panel at every k-step), so N GPUs run N independent replicas, one rank per
GPU, and value = N * flops / max-over-ranks time ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64-accurate SPD solve TFLOP/s (FP64-equivalent n^3/3+2n^2*nrhs)"
UNIT = "TFLOP/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="fp64", choices=["fp64"])
    p.add_argument("--n", type=int, default=16384)
    p.add_argument("--b", type=int, default=512)
    p.add_argument("--nrhs", type=int, default=1)
    p.add_argument("--e2e-steps", type=int, default=None)
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def flops_of(n, nrhs):
    return n ** 3 / 3.0 + 2.0 * n * n * nrhs


# ----------------------------------------------------------------------------
# distributed plumbing
# ----------------------------------------------------------------------------
def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(world, v):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------------------
# clocks sampled during the timed region
# ----------------------------------------------------------------------------
class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev_index):
        self.dev = dev_index
        self.proc = None
        self.path = os.path.join("/tmp", f"lnb_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------
# workload generation (device, seeded)
# ----------------------------------------------------------------------------
def make_spd(n, delta, seed, device):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    G = torch.randn(n, n, dtype=torch.float64, device=device, generator=g)
    A = torch.mm(G, G.t()).div_(n)
    del G
    A.diagonal().add_(delta)
    return A  # symmetric: row-major == column-major


def measure_fp64_peak(device):
    """cuBLAS dgemm throughput on this GPU (denominator of the DMMA roofline)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    torch.mm(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.mm(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


# ----------------------------------------------------------------------------
# CPU: the reference (oracle/_ref) or the oracle port, bounded sample
# ----------------------------------------------------------------------------
def cpu_run(n, b, nrhs, steps, warmup, A_host=None):
    """Times dspdsolv_main of the reference build (OpenBLAS, all host threads)
    on an n x n sample; returns (TFLOP/s, kind, cores, seconds per step)."""
    import numpy as np
    cores = os.cpu_count() or 1
    os.environ["OPENBLAS_NUM_THREADS"] = str(cores)
    from oracle import oracle as O
    kind = "reference" if O.ref_available() else "port"
    if A_host is None:
        rng = np.random.default_rng(0)
        G = rng.standard_normal((n, n))
        A_host = G @ G.T / n + 1e-2 * np.eye(n)
    A0 = np.asfortranarray(A_host)
    B0 = np.asfortranarray(np.ones((n, nrhs)))
    times = []
    for i in range(warmup + steps):
        A = A0.copy(order="F")
        B = B0.copy(order="F")
        t0 = time.perf_counter()
        if kind == "reference":
            O.ref_spdsolv(A, B, b)
        else:
            O.spdsolv(A, B, b)
        t1 = time.perf_counter()
        if i >= warmup:
            times.append(t1 - t0)
    sec = statistics.median(times)
    return flops_of(n, nrhs) / sec / 1e12, kind, (cores if kind == "reference" else 1), sec


def reference_arm(args, world, rank):
    if rank != 0:
        return
    # bounded sample of the workload: the same distribution at n = 8192
    n = min(args.n, 8192)
    try:
        import torch
        if torch.cuda.is_available():
            A = make_spd(n, 1e-2, 0, "cuda").cpu().numpy()
        else:
            A = None
    except Exception:
        A = None
    v, kind, cores, sec = cpu_run(n, args.b, args.nrhs, args.steps, args.warmup, A)
    line = {"metric": METRIC, "value": round(v, 6), "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(sec * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": f"spd_fp64_n{n}_b{args.b}_rhs{args.nrhs}", "n": n, "b": args.b,
                       "nrhs": args.nrhs, "sample_of": f"n={args.n}"},
            "cpu_baseline": {"value": round(v, 6), "unit": UNIT, "cores": cores, "kind": kind,
                             "sample": f"dspdsolv_main n={n} b={args.b} nrhs={args.nrhs}, "
                                       f"OpenBLAS threads={cores}, median of {args.steps}"},
            "e2e": {"value": round(v, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------
def ours_arm(args, world, rank, local):
    import numpy as np
    import torch

    import linompss_b200 as lnb

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L = lnb.lib()
    n, b, nrhs = args.n, args.b, args.nrhs
    fl = flops_of(n, nrhs)

    peak_fp64 = measure_fp64_peak(dev)

    A0 = make_spd(n, 1e-2, 1234 + rank, dev)
    g = torch.Generator(device=dev)
    g.manual_seed(99 + rank)
    B0 = torch.randn(nrhs, n, dtype=torch.float64, device=dev, generator=g)  # column-major (nrhs, ld=n)
    A = torch.empty_like(A0)
    B = torch.empty_like(B0)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    s = torch.cuda.current_stream()

    def one_step(timed):
        A.copy_(A0)
        B.copy_(B0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        lnb.dposv_dev(A, B, n, nrhs, b, info=info, stream=s)
        e1.record(s)
        return e0, e1

    for _ in range(args.warmup):
        one_step(False)
    torch.cuda.synchronize()
    assert int(info.item()) == 0, "warm-up factorization failed"

    barrier(world)
    torch.cuda.synchronize()
    L.lnb_prof_reset()
    L.lnb_prof_enable(1)
    evs = []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            evs.append(one_step(True))
        torch.cuda.synchronize()
    barrier(world)
    L.lnb_prof_enable(0)
    prof = lnb_prof(L)
    total_ms = sum(e0.elapsed_time(e1) for e0, e1 in evs)
    ms_step = allmax(world, total_ms / args.steps)
    value = world * fl / (ms_step * 1e-3) / 1e12

    # correctness of the timed result (last step)
    X = B.double()
    bw = backward_error_dev(A0, X, B0)
    assert int(info.item()) == 0 and bw <= 10 * n * np.finfo(float).eps, f"backward error {bw}"

    # e2e: the host entry point dspdsolv_main on pinned host buffers
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else max(1, min(args.steps, 3))
    Ah0 = A0.cpu().pin_memory()
    Bh0 = B0.cpu().pin_memory()
    Ah = torch.empty_like(Ah0).pin_memory()
    Bh = torch.empty_like(Bh0).pin_memory()
    e2e_t = []
    for i in range(e2e_steps + 1):
        Ah.copy_(Ah0)
        Bh.copy_(Bh0)
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        rc = lnb.dspdsolv_main(n, nrhs, b, Ah.numpy().T, Bh.numpy().T)  # column-major views
        t1 = time.perf_counter()
        assert rc == 0
        if i > 0:  # first call warms the pinned-path
            e2e_t.append(t1 - t0)
    e2e_sec = allmax(world, statistics.mean(e2e_t))
    Xh = Bh.numpy().T
    bw_e2e = backward_error_dev(A0, torch.from_numpy(np.ascontiguousarray(Xh.T)).to(dev), B0)
    assert bw_e2e <= 10 * n * np.finfo(float).eps
    nblk = (n + b - 1) // b
    lower_elems = sum((n - j * b) * min(b, n - j * b) for j in range(nblk))
    h2d = 8 * (lower_elems + n * nrhs)
    d2h = 8 * (lower_elems + n * nrhs)

    roof = None
    if prof["update_ms"] > 0:
        per_launch_flops = prof["update_flops"] / prof["update_launches"]
        per_launch_ms = prof["update_ms"] / prof["update_launches"]
        ach = per_launch_flops / (per_launch_ms * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": round(ach, 3), "peak": round(peak_fp64, 3), "unit": "TFLOP/s",
                "frac": round(ach / peak_fp64, 4), "traffic": traffic_from_profiles("syrk_lower_f64", n, b),
                "kernel": "k_syrk_lower_f64 (DMMA trailing update)",
                "peak_source": "cuBLAS dgemm 8192^3 measured in this run (FP64 has no entry in "
                               "MEASURED_PEAKS.json)",
                "update_share_of_step": round(prof["update_ms"] / total_ms, 4)}

    line = {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"spd_fp64_n{n}_b{b}_rhs{nrhs}", "n": n, "b": b, "nrhs": nrhs,
                       "matrix": "G G^T/n + 1e-2 I, G~N(0,1)", "factor": "fp64 (DMMA)",
                       "l2": "inputs (2 GiB) larger than L2; A restored between steps",
                       "parallelism": f"replicas x{world}", "backward_error": bw},
            "e2e": {"value": round(world * fl / e2e_sec / 1e12, 4), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": round(e2e_sec * 1e3, 3),
                    "api": "dspdsolv_main (host pointers, pinned), wall clock"},
            "roofline": roof,
            "gpu_launches": prof["launches"],
            "clocks": clk.summary()}

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ns = min(n, 8192)
        Asample = make_spd(ns, 1e-2, 0, dev).cpu().numpy()
        v, kind, cores, sec = cpu_run(ns, b, nrhs, 2, 1, Asample)
        line["cpu_baseline"] = {"value": round(v, 6), "unit": UNIT, "cores": cores, "kind": kind,
                                "sample": f"dspdsolv_main n={ns} b={b} nrhs={nrhs} (reference build, "
                                          f"OpenBLAS {cores} threads), median of 2 after 1 warm-up, "
                                          f"{sec:.2f} s each"}
    if rank == 0:
        print(json.dumps(line), flush=True)


def backward_error_dev(A, X, B):
    """||B - A X||_inf / (||A||_inf ||X||_inf + ||B||_inf); X, B as (nrhs, n) column-major rows."""
    import torch
    R = B.t() - A @ X.t()
    an = A.abs().sum(dim=1).max()
    return float(R.abs().max() / (an * X.abs().max() + B.abs().max()))


def lnb_prof(L):
    class P(C.Structure):
        _fields_ = [("launches", C.c_longlong), ("update_launches", C.c_longlong), ("update_ms", C.c_double),
                    ("update_flops", C.c_double), ("update_bytes", C.c_double)]
    p = P()
    L.lnb_prof_read(C.byref(p))
    return {k: getattr(p, k) for k, _ in P._fields_}


def traffic_from_profiles(kernel, n, b):
    """DRAM bytes per launch of `kernel` from a committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        d = json.load(open(path))
        return d.get(kernel, {}).get("dram_bytes_per_launch")
    except Exception:
        return None


def main():
    args = parse()
    world, rank, local = dist_init()
    try:
        if args.impl == "reference":
            reference_arm(args, world, rank)
        else:
            ours_arm(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
