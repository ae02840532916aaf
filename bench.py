#!/usr/bin/env python3
"""Benchmark: FP64-accurate SPD solve, mixed-precision refinement vs plain FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload mixed|fp64|bf16]

One step = one solve A X = B to FP64 backward error (<= 10 n eps) on one batch
of synthetic input already resident in HBM.  The metric is TFLOP/s with the
FP64-equivalent flop count n^3/3 + 2 n^2 nrhs, the same count for plain and
mixed solves, so the values compare time to solution directly.

Workloads (seeded synthetic inputs with the reference configurations' shapes
and distributions):
  mixed (default): n = 32768, b = 512, 1 rhs, A = G G^T/n + 1e-3 I, G ~ N(0,1):
        TF32x3 tensor-core factor in FP32 storage + FP64 refinement.  The plain
        FP64 tile Cholesky of the same matrix is timed in the same run
        ("fp64_plain") so the line carries the mixed / plain speed-up.
  fp64: n = 16384, b = 512, 1 rhs, A = G G^T/n + 1e-2 I: plain FP64 factor
        (DMMA) + triangular solves.
  bf16: n = 49152, b = 1024, 8 rhs, A = D (G G^T/n + 1e-2 I) D, D = diag(10^u),
        u ~ U[-2,2]: per-block-scaled BF16 factor, equilibration, refinement
        with PCG fallback.
Inputs are larger than L2 (126 MB); the plain FP64 factor runs in place, so its
A is restored from a pristine copy before every step outside the timed events.

Multi-GPU: one SPD system does not shard (the tile Cholesky exchanges a panel
at every k-step), so N GPUs run N independent replicas, one rank per GPU, and
value = N * flops / max-over-ranks time ("scaling": "weak").
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

METRIC = "FP64-accurate SPD solve TFLOP/s (FP64-equivalent n^3/3+2n^2*nrhs): mixed-prec IR vs plain FP64"
UNIT = "TFLOP/s"

WORKLOADS = {
    "mixed": dict(n=32768, b=512, nrhs=1, delta=1e-3, scaled=False, factor="TF32X3"),
    "fp64": dict(n=16384, b=512, nrhs=1, delta=1e-2, scaled=False, factor="FP64"),
    "bf16": dict(n=49152, b=1024, nrhs=8, delta=1e-2, scaled=True, factor="BF16"),
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="mixed", choices=sorted(WORKLOADS))
    p.add_argument("--n", type=int, default=None)
    p.add_argument("--b", type=int, default=None)
    p.add_argument("--nrhs", type=int, default=None)
    p.add_argument("--e2e-steps", type=int, default=None)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-plain", action="store_true", help="skip the plain-FP64 comparison (mixed/bf16)")
    p.add_argument("--no-batched", action="store_true", help="skip the batched uneven-systems measurement")
    p.add_argument("--batch-count", type=int, default=10000)
    p.add_argument("--no-configs", action="store_true", help="skip the other configurations' records")
    p.add_argument("--case", default=None, choices=sorted(CASES),
                   help="run one small single-kernel case (for ncu captures) and exit")
    p.add_argument("--ref-budget-s", type=float, default=150.0,
                   help="reference arm: stop timing full-size calls once their total passes this")
    a = p.parse_args()
    w = dict(WORKLOADS[a.workload])
    for k in ("n", "b", "nrhs"):
        if getattr(a, k) is not None:
            w[k] = getattr(a, k)
    a.w = w
    return a


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

        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _coll_device():
    """tensors for collectives live where the process group's backend wants them"""
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def allmax(world, v):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=_coll_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allgather_vec(world, vals):
    """every rank's list of floats (same length on all ranks), as a world x k array"""
    import numpy as np
    if world == 1:
        return np.asarray([vals], dtype=np.float64)
    import torch
    import torch.distributed as dist
    t = torch.tensor(vals, dtype=torch.float64, device=_coll_device())
    out = torch.empty(world * t.numel(), dtype=torch.float64, device=t.device)
    dist.all_gather_into_tensor(out, t)
    return out.cpu().numpy().reshape(world, -1)


def batch_shape(count, seed):
    """orders and right-hand-side counts of the uneven batch: n ~ U{16..512}, nrhs ~ U{1..8}"""
    import numpy as np
    rng = np.random.default_rng(seed)
    return rng.integers(16, 513, count), rng.integers(1, 9, count)


def shard_batch(ns, rs, world, rank):
    """this rank's systems of the batch: longest-processing-time split by estimated
    cost (lnb_batched_partition), the same on every rank"""
    import numpy as np

    import linompss_b200 as lnb
    owner, load = lnb.batched_partition(ns, rs, world)
    return np.nonzero(owner == rank)[0], load


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
def make_spd(n, delta, seed, device, scaled=False):
    """A = G G^T/n + delta I (symmetric, so row- and column-major agree);
    scaled: A = D A D with D = diag(10^u), u ~ U[-2, 2]."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    A = torch.empty(n, n, dtype=torch.float64, device=device)
    chunk = 8192
    G = torch.randn(n, n, dtype=torch.float64, device=device, generator=g)
    for r0 in range(0, n, chunk):          # blockwise product keeps the peak memory at 2 n^2
        A[r0:r0 + chunk] = G[r0:r0 + chunk] @ G.t()
    del G
    A.div_(n)
    A.diagonal().add_(delta)
    if scaled:
        d = torch.pow(10.0, torch.rand(n, dtype=torch.float64, device=device, generator=g) * 4.0 - 2.0)
        A.mul_(d[:, None]).mul_(d[None, :])
    torch.cuda.empty_cache()
    return A


def measure_peaks(device):
    """cuBLAS throughput on this GPU for the roofline denominators: FP64 dgemm
    (the DMMA path has no entry in MEASURED_PEAKS.json) and TF32 sgemm."""
    import torch
    out = {}
    n = 8192
    for name, dt, tf32 in (("fp64", torch.float64, False), ("tf32", torch.float32, True)):
        torch.backends.cuda.matmul.allow_tf32 = tf32
        a = torch.randn(n, n, dtype=dt, device=device)
        b = torch.randn(n, n, dtype=dt, device=device)
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
        out[name] = best
        del a, b
    torch.backends.cuda.matmul.allow_tf32 = False
    torch.cuda.empty_cache()
    try:
        out["bf16"] = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"]
        out["hbm_gbs"] = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
    except Exception:
        out["bf16"], out["hbm_gbs"] = 1590.0, 6650.0
    return out


# ----------------------------------------------------------------------------
# CPU: the reference build (oracle/_ref) or the oracle port, bounded sample
# ----------------------------------------------------------------------------
# The reference's external BLAS (the OpenBLAS 0.3.15 build it links here) picks
# its kernels by CPU; on the benchmark host its default choice ran dspdsolv_main
# at n = 32768 in 53.4 s and the Haswell kernels in 32.9 s, with the same
# backward error (1.9e-17 / 2.0e-17).  The baseline runs the faster one.
OPENBLAS_CORETYPE = "Haswell"


def cpu_run(n, b, nrhs, steps, warmup, A_host=None):
    """Times dspdsolv_main of the reference build (OpenBLAS, all host threads)
    on an n x n sample; returns (TFLOP/s, kind, cores, seconds per step)."""
    import numpy as np
    cores = os.cpu_count() or 1
    os.environ["OPENBLAS_NUM_THREADS"] = str(cores)
    os.environ.setdefault("OPENBLAS_CORETYPE", OPENBLAS_CORETYPE)
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


def workload_inputs(w, rank, device):
    """The seeded inputs of a workload: A (n x n, symmetric) and B (nrhs x n,
    i.e. the n x nrhs right-hand sides column-major), on `device`."""
    import torch
    A0 = make_spd(w["n"], w["delta"], 1234 + rank, device, w["scaled"])
    g = torch.Generator(device=device)
    g.manual_seed(99 + rank)
    B0 = torch.randn(w["nrhs"], w["n"], dtype=torch.float64, device=device, generator=g)
    return A0, B0


def workload_config(args, w, world):
    """`config` of the JSON line: the workload, identical for both arms"""
    return {"workload": f"spd_{args.workload}_n{w['n']}_b{w['b']}_rhs{w['nrhs']}", "n": w["n"], "b": w["b"],
            "nrhs": w["nrhs"],
            "matrix": ("D (G G^T/n + %g I) D" if w["scaled"] else "G G^T/n + %g I") % w["delta"],
            "inputs": "A: G ~ N(0,1) seed 1234 (torch generator on the device); B ~ N(0,1) seed 99",
            "l2": "inputs larger than L2 (126 MB); plain-FP64 A restored between steps",
            "parallelism": f"replicas x{world}"}


def reference_arm(args, world, rank):
    """The reference's own FP64-accurate solve, dspdsolv_main (spdsolv_main.c:10-20:
    tile Cholesky + two blocked triangular solves), compiled from its sources
    (oracle/_ref/libref.so, OpenBLAS on every host thread), on the SAME seeded
    inputs and size as this workload.  One full-size call takes tens of seconds
    on the host, so the warm-up calls run an n = 4096 slice of the same matrix
    and the timed steps stop once their total passes --ref-budget-s (at least
    one full-size call); `steps` reports the calls actually timed."""
    if rank != 0:
        return
    import numpy as np
    w = args.w
    n, b, nrhs = w["n"], w["b"], w["nrhs"]
    cores = os.cpu_count() or 1
    os.environ["OPENBLAS_NUM_THREADS"] = str(cores)
    os.environ.setdefault("OPENBLAS_CORETYPE", OPENBLAS_CORETYPE)
    from oracle import oracle as O
    kind = "reference" if O.ref_available() else "port"
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    A0d, B0d = workload_inputs(w, 0, dev)
    A0 = A0d.cpu().numpy().T                          # symmetric: the transposed view is column-major
    B0 = np.asfortranarray(B0d.cpu().numpy().T)
    solve = O.ref_spdsolv if kind == "reference" else O.spdsolv
    nw = min(n, 4096)
    for _ in range(args.warmup):
        # copies: asfortranarray of B0[:nw] (n x 1, already Fortran-ordered) would be a view,
        # and the warm-up solve would overwrite the timed call's right-hand side
        A = np.array(A0[:nw, :nw], order="F")
        B = np.array(B0[:nw], order="F")
        solve(A, B, min(b, nw))
    times = []
    A = np.empty_like(A0, order="F")
    B = np.empty_like(B0, order="F")
    for i in range(args.steps):
        A[...] = A0
        B[...] = B0
        t0 = time.perf_counter()
        rc = solve(A, B, b)
        t1 = time.perf_counter()
        assert rc == 0, rc
        times.append(t1 - t0)
        if sum(times) >= args.ref_budget_s:
            break
    sec = statistics.mean(times)
    v = flops_of(n, nrhs) / sec / 1e12
    # accuracy of the reference's solution, checked in FP64 on the device
    be = None
    if dev == "cuda":
        X = torch.tensor(np.ascontiguousarray(B.T), device=dev)
        be = backward_error_dev(A0d, X, B0d)
    line = {"metric": METRIC, "value": round(v, 6), "unit": UNIT, "n_gpus": args.gpus, "steps": len(times),
            "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": round(sec * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": workload_config(args, w, world),
            "result": {"backward_error": be},
            "cpu_baseline": {"value": round(v, 6), "unit": UNIT, "cores": cores, "kind": kind,
                             "sample": f"the full workload: dspdsolv_main n={n} b={b} nrhs={nrhs} on the same "
                                       f"seeded inputs, OpenBLAS threads={cores} "
                                       f"({os.environ.get('OPENBLAS_CORETYPE')} kernels), mean of {len(times)} "
                                       f"call(s); warm-up on the leading {nw} x {nw} block"},
            "e2e": {"value": round(v, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------
def backward_error_dev(A, X, B):
    """max over columns of ||B - A X||_inf / (||A||_inf ||X||_inf + ||B||_inf);
    X, B as (nrhs, n) tensors (rows = columns of the column-major matrices)."""
    an = A.abs().sum(dim=1).max()
    worst = 0.0
    for q in range(X.shape[0]):
        r = B[q] - A @ X[q]
        worst = max(worst, float(r.abs().max() / (an * X[q].abs().max() + B[q].abs().max())))
    return worst


def lnb_prof(L):
    class P(C.Structure):
        _fields_ = [("launches", C.c_longlong), ("update_launches", C.c_longlong), ("update_ms", C.c_double),
                    ("update_flops", C.c_double), ("update_bytes", C.c_double)]
    p = P()
    L.lnb_prof_read(C.byref(p))
    return {k: getattr(p, k) for k, _ in P._fields_}


def traffic_from_profiles(kernel, alg_bytes_per_launch):
    """DRAM bytes per launch of `kernel`: the DRAM / algorithmic byte ratio of
    one committed ncu capture of that kernel (profiles/traffic.json), scaled to
    this run's average algorithmic bytes per launch; None without a capture."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        ratio = d[kernel]["dram_per_algorithmic_byte"]
    except Exception:
        return None
    return int(ratio * alg_bytes_per_launch)


def make_batch(ns, rs, seed, device):
    """Systems of orders ns and right-hand-side counts rs, A_i = G G^T/n_i + 1e-2 I,
    packed column-major in one flat FP64 buffer (and B_i ~ N(0,1) likewise)."""
    import numpy as np
    import torch
    ns = np.asarray(ns)
    rs = np.asarray(rs)
    a_off = np.concatenate([[0], np.cumsum(ns.astype(np.int64) ** 2)[:-1]])
    b_off = np.concatenate([[0], np.cumsum(ns.astype(np.int64) * rs)[:-1]])
    A = torch.empty(int((ns.astype(np.int64) ** 2).sum()), dtype=torch.float64, device=device)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    for n in np.unique(ns):
        idx = np.nonzero(ns == n)[0]
        G = torch.randn(len(idx), n, n, dtype=torch.float64, device=device, generator=g)
        Ai = torch.bmm(G, G.transpose(1, 2)).div_(float(n))
        Ai.diagonal(dim1=1, dim2=2).add_(1e-2)
        flat = (torch.tensor(a_off[idx], device=device)[:, None] +
                torch.arange(n * n, device=device)[None, :]).reshape(-1)
        A.index_copy_(0, flat, Ai.reshape(-1))          # symmetric: row- and column-major agree
        del G, Ai, flat
    B = torch.randn(int((ns.astype(np.int64) * rs).sum()), dtype=torch.float64, device=device, generator=g)
    t = lambda x, dt: torch.tensor(x, dtype=dt, device=device)
    return (ns, rs, a_off, b_off, t(ns, torch.int32), t(rs, torch.int32), t(a_off, torch.int64),
            t(b_off, torch.int64), A, B)


def batched_arm(args, world, rank, local, peaks):
    """Batched uneven solves: one persistent launch (autotuned launch shape,
    captured in a CUDA graph) against a loop of per-system plain FP64 solves.
    With N GPUs the one batch is split across them (longest processing time
    first on the estimated cost); the batch time is the slowest rank's."""
    import numpy as np
    import torch

    import linompss_b200 as lnb
    dev = torch.device("cuda", local)
    L = lnb.lib()
    ns_all, rs_all = batch_shape(args.batch_count, 4321)
    mine, load = shard_batch(ns_all, rs_all, world, rank)
    flops = float(sum(n ** 3 / 3.0 + 2.0 * n * n * r for n, r in zip(ns_all.astype(float), rs_all.astype(float))))
    ns, rs, a_off, b_off, nd, rd, ao, bo, dA, dB = make_batch(ns_all[mine], rs_all[mine], 4321 + 17 * rank, dev)
    count = len(ns)
    dX = torch.zeros_like(dB)
    info = torch.zeros(count, dtype=torch.int32, device=dev)
    iters = torch.zeros(count, dtype=torch.int32, device=dev)
    s = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(s):
        pw = lnb.batched_autotune(nd, rd, ao, bo, dA, dB, dX, lnb.FACTOR_FP32, 10, stream=s)
        lnb.batched_posv_dev(nd, rd, ao, bo, dA, dB, dX, lnb.FACTOR_FP32, 10, info, iters, stream=s)
        torch.cuda.synchronize()
        gr = torch.cuda.CUDAGraph()
        with torch.cuda.graph(gr, stream=s):
            lnb.batched_posv_dev(nd, rd, ao, bo, dA, dB, dX, lnb.FACTOR_FP32, 10, info, iters, stream=s)
        for _ in range(2):
            gr.replay()
        torch.cuda.synchronize()
        reps = max(3, min(args.steps, 10))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        dX.zero_()
        e0.record(s)
        for _ in range(reps):
            gr.replay()
        e1.record(s)
        torch.cuda.synchronize()
    t_batch = allmax(world, e0.elapsed_time(e1) / reps)
    assert int((info != 0).sum().item()) == 0, "batched: non-SPD report"
    # backward error of EVERY system, FP64 on the device: systems of one order n are
    # stacked (right-hand sides padded to 8 with zeros) and checked in one batched product
    eps = np.finfo(float).eps / 2
    worst = 0.0
    for n in np.unique(ns):
        idx = np.nonzero(ns == n)[0]
        n = int(n)
        As_ = torch.stack([dA[a_off[k]:a_off[k] + n * n].view(n, n) for k in idx])
        Xs_ = torch.zeros(len(idx), n, 8, dtype=torch.float64, device=dev)
        Bs_ = torch.zeros_like(Xs_)
        for j, k in enumerate(idx):
            r = int(rs[k])
            Xs_[j, :, :r] = dX[b_off[k]:b_off[k] + n * r].view(r, n).t()
            Bs_[j, :, :r] = dB[b_off[k]:b_off[k] + n * r].view(r, n).t()
        R = Bs_ - torch.bmm(As_, Xs_)
        den = As_.abs().sum(2).amax(1) * Xs_.abs().amax((1, 2)) + Bs_.abs().amax((1, 2))
        be = (R.abs().amax((1, 2)) / den).max().item()
        worst = max(worst, be / (n * eps))
        del As_, Xs_, Bs_, R
    assert worst <= 10.0, f"batched backward error {worst} n eps"
    it = iters.cpu().numpy()
    # the whole batch's refinement counts and worst error: one all-gather of
    # per-rank summaries (the only collective of the batched arm)
    g = allgather_vec(world, [float(count), float(it.sum()), float(it.min()), float(it.max()), worst])
    del gr
    # per-system plain FP64 launches on a copy (dposv factors A in place)
    Aw = dA.clone()
    Bw = dB.clone()
    infop = torch.zeros(1, dtype=torch.int32, device=dev)
    f = L.lnb_dposv_dev
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    pa, pb, sp = Aw.data_ptr(), Bw.data_ptr(), C.c_void_p(s.cuda_stream)
    with torch.cuda.stream(s):
        for k in range(min(count, 50)):     # warm-up: workspace and first-launch costs
            n, r = int(ns[k]), int(rs[k])
            f(n, r, 128, C.c_void_p(pa + 8 * int(a_off[k])), n, C.c_void_p(pb + 8 * int(b_off[k])), n,
              C.c_void_p(infop.data_ptr()), sp)
        Aw.copy_(dA)
        Bw.copy_(dB)
        torch.cuda.synchronize()
        e0.record(s)
        for k in range(count):
            n, r = int(ns[k]), int(rs[k])
            rc = f(n, r, 128, C.c_void_p(pa + 8 * int(a_off[k])), n, C.c_void_p(pb + 8 * int(b_off[k])), n,
                   C.c_void_p(infop.data_ptr()), sp)
            assert rc == 0, lnb.last_error()
        e1.record(s)
        torch.cuda.synchronize()
    t_loop = allmax(world, e0.elapsed_time(e1))
    del Aw, Bw, dA, dB, dX
    torch.cuda.empty_cache()
    tf = flops / (t_batch * 1e-3) / 1e12
    total = int(g[:, 0].sum())
    return {"systems": total, "n_range": [16, 512], "nrhs_range": [1, 8], "factor": "fp32 + fp64 refinement",
            "split": f"one batch over {world} GPU(s), longest processing time first (lnb_batched_partition)",
            "scaling": "strong", "est_load_max_over_mean": round(float(load.max() / load.mean()), 4),
            "ms_per_batch": round(t_batch, 3), "value": round(tf, 4), "unit": UNIT,
            "solves_per_s": round(total / (t_batch * 1e-3), 1),
            "frac_of_fp64_dgemm_peak": round(tf / peaks["fp64"], 4),
            "frac_of_tf32_peak": round(tf / peaks["tf32"], 4),
            "per_system_loop_ms": round(t_loop, 3), "speedup_vs_per_system_launches": round(t_loop / t_batch, 2),
            "per_system_loop": "lnb_dposv_dev (plain FP64, b=128) once per system, same stream",
            "launch": "one persistent launch in a CUDA graph, replayed",
            "autotuned_shape": lnb.batched_config(lnb.FACTOR_FP32),
            "max_backward_error_over_n_eps_all_systems": round(float(g[:, 4].max()), 4),
            "refinement_iterations": {"min": int(g[:, 2].min()), "max": int(g[:, 3].max()),
                                      "mean": round(float(g[:, 1].sum() / total), 2)}}


def fp64_oracle_solve(A, B):
    """X (nrhs x n) solving A X^T = B^T in FP64 by an independent algorithm:
    cuSOLVER's potrf + potrs (LAPACK's blocked Cholesky), through torch.  A
    checker only; the library never calls it."""
    import torch
    Lc = torch.linalg.cholesky(A)
    X = torch.cholesky_solve(B.t().contiguous(), Lc).t().contiguous()
    del Lc
    torch.cuda.empty_cache()
    return X


def fwd_err(X, Xref):
    """normwise forward error max|X - Xref| / max|Xref|"""
    return float((X - Xref).abs().max() / Xref.abs().max())


def factor_residual_dev(A, L):
    """||A - L L^T||_inf / (n eps ||A||_inf), the bar of potrf_test.c:31-36,
    in FP64 on the device; L is the column-major lower factor stored as a
    (cols, ld) tensor (so L.t() is the matrix), A symmetric."""
    import numpy as np
    import torch
    n = A.shape[0]
    Lm = torch.tril(L.t())
    R = Lm @ Lm.t()
    del Lm
    R.sub_(A)
    num = R.abs().sum(dim=1).max()
    del R
    torch.cuda.empty_cache()
    return float(num / (n * np.finfo(float).eps / 2 * A.abs().sum(dim=1).max()))


def time_events(fn, reps, s, prep=None):
    """mean device time (ms) of reps calls of fn on stream s (prep outside the events)"""
    import torch
    evs = []
    for _ in range(reps):
        if prep is not None:
            prep()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        fn()
        e1.record(s)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    return statistics.mean(a.elapsed_time(b) for a, b in evs)


def config_records(args, world, rank, dev, peaks):
    """The other reference configurations, each at its full stated size and input
    distribution, timed on the device (mean of a few calls after one warm-up)
    with its accuracy checked:
      fp64_n16384 : plain FP64 factor + solves, b = 512, 1 and 64 rhs, with the
                    factor residual ||A - L L^T||_inf/(n eps ||A||_inf)
      tf32x3_delta: the headline workload's matrix family at delta 1e-1 and 1e-5
      bf16_n49152 : per-tile-scaled BF16 factor + FP64 refinement / PCG, b = 1024,
                    8 rhs, D-scaled, delta 1e-2 and 1e-4, beside the plain FP64 solve
    Each mixed record carries iterations, PCG use, refactored tiles, backward
    error and the forward error against an FP64 cuSOLVER solve."""
    import numpy as np
    import torch

    import linompss_b200 as lnb
    eps = np.finfo(float).eps / 2
    s = torch.cuda.current_stream()
    reps = max(1, min(args.steps, 3))
    out = {}

    def plain(A0, B0, n, b, nrhs, resid):
        A = torch.empty_like(A0)
        B = torch.empty_like(B0)
        info = torch.zeros(1, dtype=torch.int32, device=dev)

        def prep():
            A.copy_(A0)
            B.copy_(B0)
        run = lambda: lnb.dposv_dev(A, B, n, nrhs, b, info=info, stream=s)
        time_events(run, 1, s, prep)
        ms = allmax(world, time_events(run, reps, s, prep))
        assert int(info.item()) == 0
        rec = {"ms": round(ms, 3), "value": round(world * flops_of(n, nrhs) / ms / 1e9, 4),
               "backward_error": backward_error_dev(A0, B, B0)}
        assert rec["backward_error"] <= 10 * n * eps, rec
        if resid:
            rec["factor_residual"] = factor_residual_dev(A0, A)
            assert rec["factor_residual"] <= 10.0, rec
        X = B.clone()
        del A, B
        torch.cuda.empty_cache()
        return rec, X

    def mixed(A0, B0, n, b, nrhs, factor):
        X = torch.zeros_like(B0)
        opts = lnb.ir_opts(factor=getattr(lnb, "FACTOR_" + factor), max_iter=40, pcg_max_iter=400)
        res = {}

        def run():
            rc, r = lnb.dsposv_ir_dev(A0, B0, X, n, nrhs, b, opts, stream=s)
            assert rc == 0, (rc, r, lnb.last_error())
            res.update(r)
        time_events(run, 1, s)
        ms = allmax(world, time_events(run, reps, s))
        rec = {"ms": round(ms, 3), "value": round(world * flops_of(n, nrhs) / ms / 1e9, 4),
               "backward_error": backward_error_dev(A0, X, B0)}
        assert rec["backward_error"] <= 10 * n * eps, rec
        rec.update({k: res.get(k) for k in ("iterations", "used_pcg", "pcg_iterations", "refactored_tiles",
                                            "factor_ms", "solve_ms")})
        return rec, X

    def schedules(A0, B0, n, b, nrhs):
        """plain FP64 factor + solves under each FP64 schedule (device DAG vs
        host-issued streams), same inputs; the library's default picks by n"""
        rec = {}
        try:
            for name, sched in (("dag", lnb.SCHED_DAG), ("streams", lnb.SCHED_STREAMS)):
                lnb.set_chol_schedule(sched)
                r, X = plain(A0, B0, n, b, nrhs, resid=False)
                rec[name + "_ms"] = r["ms"]
                rec[name + "_backward_error"] = r["backward_error"]
                del X
        finally:
            lnb.set_chol_schedule(lnb.SCHED_AUTO)
        rec["dag_speedup"] = round(rec["streams_ms"] / rec["dag_ms"], 3)
        return rec

    # configuration 1: plain FP64, n = 2048, b = 256, 1 rhs, (R + R^T)/2 + n I
    n, b = 2048, 256
    gr = torch.Generator(device=dev)
    gr.manual_seed(rank)
    R = torch.rand(n, n, dtype=torch.float64, device=dev, generator=gr)
    A0 = (R + R.t()) / 2
    A0.diagonal().add_(float(n))
    del R
    xt = torch.rand(1, n, dtype=torch.float64, device=dev, generator=gr) * 2 - 1
    B0 = (A0 @ xt.t()).t().contiguous()
    r, X = plain(A0, B0, n, b, 1, resid=True)
    r["forward_error_vs_x_true"] = fwd_err(X, xt)
    r["forward_error_vs_fp64_oracle"] = fwd_err(X, fp64_oracle_solve(A0, B0))
    r["schedule"] = "dag" if n <= 16384 else "streams"      # the library's automatic choice
    r["schedules"] = schedules(A0, B0, n, b, 1)
    out["fp64_n2048_b256"] = r
    del A0, B0, X, xt

    # configuration 2: plain FP64, n = 16384, b = 512, 1 and 64 right-hand sides
    n, b = 16384, 512
    A0 = make_spd(n, 1e-2, 2024 + rank, dev)
    g = torch.Generator(device=dev)
    g.manual_seed(7 + rank)
    rec2 = {"n": n, "b": b, "matrix": "G G^T/n + 0.01 I", "bound": "fp64 DMMA tensor"}
    for nrhs in (1, 64):
        B0 = torch.randn(nrhs, n, dtype=torch.float64, device=dev, generator=g)
        r, X = plain(A0, B0, n, b, nrhs, resid=(nrhs == 1))
        r["forward_error_vs_fp64_oracle"] = fwd_err(X, fp64_oracle_solve(A0, B0))
        r["frac_of_fp64_dgemm_peak"] = round(r["value"] / peaks["fp64"], 4)
        if nrhs == 1:
            r["schedules"] = schedules(A0, B0, n, b, nrhs)
        rec2[f"rhs{nrhs}"] = r
        del B0, X
    out["fp64_n16384_b512"] = rec2
    del A0
    torch.cuda.empty_cache()

    # configuration 3: the delta sweep of the headline matrix family
    n, b = 32768, 512
    A0 = make_spd(n, 0.0, 1234 + rank, dev)        # G G^T / n; delta added below
    g.manual_seed(99 + rank)
    B0 = torch.randn(1, n, dtype=torch.float64, device=dev, generator=g)
    rec3 = {"n": n, "b": b, "factor": "tf32x3"}
    cur = 0.0
    for delta in (1e-1, 1e-5):
        A0.diagonal().add_(delta - cur)
        cur = delta
        r, X = mixed(A0, B0, n, b, 1, "TF32X3")
        r["forward_error_vs_fp64_oracle"] = fwd_err(X, fp64_oracle_solve(A0, B0))
        rec3[f"delta_{delta:g}"] = r
        del X
    out["tf32x3_n32768_delta_sweep"] = rec3
    del A0, B0
    torch.cuda.empty_cache()

    # configuration 4: BF16 per-tile-scaled factor, n = 49152, b = 1024, 8 rhs, D-scaled
    n, b, nrhs = 49152, 1024, 8
    A0 = make_spd(n, 0.0, 4900 + rank, dev)
    gd = torch.Generator(device=dev)
    gd.manual_seed(4901 + rank)
    d = torch.pow(10.0, torch.rand(n, dtype=torch.float64, device=dev, generator=gd) * 4.0 - 2.0)
    A0.mul_(d[:, None]).mul_(d[None, :])
    B0 = torch.randn(nrhs, n, dtype=torch.float64, device=dev, generator=gd)
    rec4 = {"n": n, "b": b, "nrhs": nrhs, "matrix": "D (G G^T/n + delta I) D, D = diag(10^u), u ~ U[-2,2]",
            "factor": "bf16 (per-tile power-of-two scales), equilibrated, PCG fallback"}
    cur = 0.0
    for delta in (1e-2, 1e-4):
        A0.diagonal().add_((delta - cur) * d * d)
        cur = delta
        r, X = mixed(A0, B0, n, b, nrhs, "BF16")
        r["forward_error_vs_fp64_oracle"] = fwd_err(X, fp64_oracle_solve(A0, B0))
        del X
        p, Xp = plain(A0, B0, n, b, nrhs, resid=False)
        r["fp64_plain_ms"] = p["ms"]
        r["speedup_vs_fp64_plain"] = round(p["ms"] / r["ms"], 3)
        del Xp
        rec4[f"delta_{delta:g}"] = r
    out["bf16_n49152_b1024_rhs8"] = rec4
    del A0, B0, d
    torch.cuda.empty_cache()
    return out


def blas_records(args, world, rank, dev, peaks):
    """The stand-alone BLAS-3 drivers and the LU / general solve at the reference's own chart sizes
    (tests/dsyrk.cfg: lower, transposed, n = k = 16000, alpha 13.44, beta
    -9.877, b in {550, 1032, 2898, 5988}; tests/dtrsm.cfg: left lower, no
    transpose, m = n = 1500, alpha 13.44, b in {121, 256, 350, 550}), each timed
    on the device (DMMA kernels), end to end through the reference-named host
    entry point (host arrays in, result back), and, on rank 0 of a 1-GPU run,
    the reference build's own call on the same arrays (OpenBLAS on every host
    thread; b only changes the reference's tiling)."""
    import numpy as np
    import torch

    import linompss_b200 as lnb
    cores = os.cpu_count() or 1
    os.environ["OPENBLAS_NUM_THREADS"] = str(cores)
    os.environ.setdefault("OPENBLAS_CORETYPE", OPENBLAS_CORETYPE)
    s = torch.cuda.current_stream()
    reps = max(1, min(args.steps, 3))
    out = {}
    with_ref = rank == 0 and world == 1 and not args.no_cpu_baseline
    if with_ref:
        from oracle import oracle as O
        with_ref = O.ref_available()

    # ---- dsyrk ----
    n = k = 16000
    alpha, beta = 13.44, -9.877
    g = torch.Generator(device=dev)
    g.manual_seed(16000 + rank)
    At = torch.randn(n, k, dtype=torch.float64, device=dev, generator=g)    # A stored k x n (trans = 'T')
    C0 = torch.randn(n, n, dtype=torch.float64, device=dev, generator=g)
    Ct = torch.empty_like(C0)
    run = lambda: lnb.dsyrk_dev("L", "T", n, k, alpha, At, beta, Ct, stream=s)
    prep = lambda: Ct.copy_(C0)
    time_events(run, 1, s, prep)
    ms = allmax(world, time_events(run, reps, s, prep))
    fl = float(n) * (n + 1) * k
    ref = torch.addmm(C0.t(), At, At.t(), beta=beta, alpha=alpha)          # cuBLAS FP64, full matrix
    got = Ct.t()
    lo = torch.tril(torch.ones(n, n, dtype=torch.bool, device=dev))
    err = float(((got - ref).abs() * lo).max() / ref.abs().max())
    assert err < 1e-12, err
    rec = {"n": n, "k": k, "uplo": "L", "trans": "T", "alpha": alpha, "beta": beta,
           "device_ms": round(ms, 3), "device_tflops": round(world * fl / ms / 1e9, 3),
           "frac_of_fp64_dgemm_peak": round(fl / ms / 1e9 / peaks["fp64"], 4),
           "max_rel_err_vs_cublas_dgemm": err, "kernel": "k_gemm_dmma (DMMA, 64x64 tiles, lower tiles only)"}
    del ref, got, lo
    Ah = torch.empty((n, k), dtype=torch.float64, pin_memory=True)
    Ah.copy_(At)
    Ch0 = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
    Ch0.copy_(C0)
    del At, C0, Ct
    torch.cuda.empty_cache()
    A_np = Ah.numpy().T          # column-major k x n view
    Ch = torch.empty_like(Ch0, pin_memory=True)
    times = []
    for i in range(2):
        Ch.copy_(Ch0)
        C_np = Ch.numpy().T
        t0 = time.perf_counter()
        lnb.ompss_dsyrk("L", "T", 550, n, k, alpha, A_np, k, C_np, n, beta=beta)
        times.append(time.perf_counter() - t0)
    rec["e2e_ms"] = round(allmax(world, times[-1]) * 1e3, 3)
    rec["e2e_tflops"] = round(world * fl / (rec["e2e_ms"] / 1e3) / 1e12, 3)
    rec["e2e_api"] = "ompss_dsyrk (host arrays, pinned): A and C in, C out (6.1 GB over PCIe)"
    if with_ref:
        rref = {}
        for bb in (550, 5988):
            Ch.copy_(Ch0)
            C_np = Ch.numpy().T
            t0 = time.perf_counter()
            O.ref_dsyrk("L", "T", bb, n, k, alpha, A_np, k, beta, C_np, n)
            rref[f"b{bb}_s"] = round(time.perf_counter() - t0, 3)
        rref["cores"] = cores
        rref["tflops_best"] = round(fl / min(v for kk, v in rref.items() if kk.endswith("_s")) / 1e12, 4)
        rec["reference"] = rref
        rec["e2e_speedup_vs_reference_best"] = round(min(rref["b550_s"], rref["b5988_s"]) / (rec["e2e_ms"] / 1e3), 2)
    out["dsyrk_n16000_k16000"] = rec
    del Ah, Ch0, Ch
    # ---- dtrsm ----
    m = nn = 1500
    alpha = 13.44
    rng = np.random.default_rng(1500 + rank)
    Lm = np.tril(rng.standard_normal((m, m))) + m * np.eye(m)
    Lm = np.asfortranarray(Lm)
    B0 = np.asfortranarray(rng.standard_normal((m, nn)))
    Ld = torch.tensor(np.ascontiguousarray(Lm.T), device=dev)
    Bd0 = torch.tensor(np.ascontiguousarray(B0.T), device=dev)
    Bd = torch.empty_like(Bd0)
    run = lambda: lnb.dtrsm_dev("L", "N", "N", m, nn, alpha, Ld, Bd, stream=s)
    prep = lambda: Bd.copy_(Bd0)
    time_events(run, 1, s, prep)
    ms = allmax(world, time_events(run, reps, s, prep))
    fl = float(m) * m * nn
    X = Bd.cpu().numpy().T
    err = float(np.abs(Lm @ X - alpha * B0).max() / (np.abs(Lm).sum(1).max() * np.abs(X).max()))
    rec = {"m": m, "n": nn, "side": "L", "uplo": "L", "trans": "N", "diag": "N", "alpha": alpha,
           "device_ms": round(ms, 4), "device_tflops": round(world * fl / ms / 1e9, 4), "backward_error": err}
    assert err < 10 * m * np.finfo(float).eps, err
    e2e = {}
    for bb in (121, 256, 350, 550):
        t = []
        for _ in range(3):
            B = B0.copy(order="F")
            t0 = time.perf_counter()
            lnb.ompss_dtrsm("L", "L", "N", "N", m, nn, bb, alpha, Lm, m, B, m)
            t.append(time.perf_counter() - t0)
        e2e[f"b{bb}_ms"] = round(min(t) * 1e3, 3)
    rec["e2e"] = e2e
    rec["e2e_api"] = "ompss_dtrsm (host arrays): L and B in, X out"
    if with_ref:
        rref = {}
        for bb in (121, 256, 350, 550):
            t = []
            for _ in range(3):
                B = B0.copy(order="F")
                t0 = time.perf_counter()
                O.ref_dtrsm("L", "L", "N", "N", m, nn, bb, alpha, Lm, m, B, m)
                t.append(time.perf_counter() - t0)
            rref[f"b{bb}_ms"] = round(min(t) * 1e3, 3)
        rref["cores"] = cores
        rec["reference"] = rref
    out["dtrsm_m1500_n1500"] = rec
    del Ld, Bd0, Bd
    torch.cuda.empty_cache()
    # ---- LU and the general solve (tests/dlu.cfg, tests/dgensolv.cfg: m = n = 1500) ----
    m = 1500
    bs = (121, 256, 350, 550, 1000)
    gA = np.random.default_rng(1501 + rank).random((m, m))
    gA[np.arange(m), np.arange(m)] += 100.0                 # GENMAT_IP: U[0,1) + 100 on the diagonal
    A0 = np.asfortranarray(gA)
    B0 = np.asfortranarray(np.random.default_rng(1502 + rank).random((m, m)))
    fl_lu = 2.0 * m ** 3 / 3.0
    fl_gs = fl_lu + 2.0 * m * m * m
    Ad = torch.tensor(np.ascontiguousarray(A0.T), device=dev)
    Aw = torch.empty_like(Ad)
    piv = torch.zeros(m, dtype=torch.int32, device=dev)
    run = lambda: lnb.dgetrf_dev(Aw, m, m, piv, stream=s)
    prep = lambda: Aw.copy_(Ad)
    time_events(run, 1, s, prep)
    ms = allmax(world, time_events(run, reps, s, prep))
    rec = {"m": m, "n": m, "matrix": "U[0,1) + 100 I (the reference's GENMAT_IP)", "device_ms": round(ms, 3),
           "device_tflops": round(world * fl_lu / ms / 1e9, 4)}
    e2e, e2e_gs = {}, {}
    for bb in bs:
        t, tg = [], []
        for _ in range(2):
            A = A0.copy(order="F")
            t0 = time.perf_counter()
            lnb.ompss_getrf(A, bb)
            t.append(time.perf_counter() - t0)
            A, B = A0.copy(order="F"), B0.copy(order="F")
            t0 = time.perf_counter()
            lnb.gensolv(A, B, bb)
            tg.append(time.perf_counter() - t0)
        e2e[f"b{bb}_ms"] = round(min(t) * 1e3, 3)
        e2e_gs[f"b{bb}_ms"] = round(min(tg) * 1e3, 3)
    berr = float(np.abs(A0 @ B - B0).max() / (np.abs(A0).sum(1).max() * np.abs(B).max() + np.abs(B0).max()))
    assert berr < 10 * m * np.finfo(float).eps, berr
    rec["getrf_e2e"] = e2e
    rec["gensolv_e2e"] = e2e_gs
    rec["gensolv_backward_error"] = berr
    rec["e2e_api"] = "ompss_dgetrf / dgensolv_main (host arrays in and out)"
    if with_ref:
        rref, rgs = {}, {}
        for bb in bs:
            A = A0.copy(order="F")
            t0 = time.perf_counter()
            ip = O.ref_getrf(A, bb)
            rref[f"b{bb}_ms"] = round((time.perf_counter() - t0) * 1e3, 3)
            if bb == bs[0]:
                Ag = A0.copy(order="F")
                _, ipg = lnb.ompss_getrf(Ag, bb)
                rec["factor_max_rel_diff_vs_reference"] = float(np.abs(Ag - A).max() / np.abs(A).max())
                rec["pivots_equal_reference"] = bool((ipg == ip).all())
            A, B = A0.copy(order="F"), B0.copy(order="F")
            t0 = time.perf_counter()
            O.ref_gensolv(A, B, bb)
            rgs[f"b{bb}_ms"] = round((time.perf_counter() - t0) * 1e3, 3)
        rec["reference_getrf"] = rref
        rec["reference_gensolv"] = rgs
        rec["reference_cores"] = cores
        rec["gensolv_e2e_speedup_vs_reference_best"] = round(min(rgs.values()) / min(e2e_gs.values()), 2)
    out["lu_gensolv_m1500"] = rec
    del Ad, Aw, piv
    torch.cuda.empty_cache()
    return out


def ours_arm(args, world, rank, local):
    import numpy as np
    import torch

    import linompss_b200 as lnb

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L = lnb.lib()
    w = args.w
    n, b, nrhs = w["n"], w["b"], w["nrhs"]
    fl = flops_of(n, nrhs)
    eps = np.finfo(float).eps / 2
    peaks = measure_peaks(dev)

    A0, B0 = workload_inputs(w, rank, dev)        # B0: column-major (nrhs, ld=n)
    s = torch.cuda.current_stream()
    mixed = w["factor"] != "FP64"

    if mixed:
        X = torch.zeros_like(B0)
        opts = lnb.ir_opts(factor=getattr(lnb, "FACTOR_" + w["factor"]), max_iter=40, pcg_max_iter=400)
        last = {}

        def run_step():
            rc, res = lnb.dsposv_ir_dev(A0, B0, X, n, nrhs, b, opts, stream=s)
            assert rc == 0, (rc, res, lnb.last_error())
            last.update(res)
    else:
        A = torch.empty_like(A0)
        B = torch.empty_like(B0)
        info = torch.zeros(1, dtype=torch.int32, device=dev)

        def prep():
            A.copy_(A0)
            B.copy_(B0)

        def run_step():
            lnb.dposv_dev(A, B, n, nrhs, b, info=info, stream=s)

    def timed_steps(k, prof):
        evs = []
        for _ in range(k):
            if not mixed:
                prep()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            run_step()
            e1.record(s)
            evs.append((e0, e1))
        torch.cuda.synchronize()
        return sum(a.elapsed_time(bb) for a, bb in evs)

    timed_steps(args.warmup, False)
    barrier(world)
    torch.cuda.synchronize()
    L.lnb_prof_reset()
    L.lnb_prof_enable(1)
    with Clocks(local) as clk:
        total_ms = timed_steps(args.steps, True)
    barrier(world)
    L.lnb_prof_enable(0)
    prof = lnb_prof(L)
    ms_step = allmax(world, total_ms / args.steps)
    value = world * fl / (ms_step * 1e-3) / 1e12

    Xres = X if mixed else B
    bw = backward_error_dev(A0, Xres, B0)
    assert bw <= 10 * n * eps, f"backward error {bw}"
    if not mixed:
        assert int(info.item()) == 0

    line = {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if not mixed else "f64 (factor " +
            w["factor"].lower() + ")", "data": "synthetic",
            "config": workload_config(args, w, world),
            "gpu_launches": prof["launches"]}
    # accuracy: backward error, and forward error against an independent FP64
    # solve of the same A and B (LAPACK's potrf/potrs algorithm, cuSOLVER)
    Xo = fp64_oracle_solve(A0, B0)
    line["result"] = {"factor": w["factor"].lower(), "backward_error": bw,
                      "backward_error_bar": 10 * n * eps, "forward_error_vs_fp64_oracle": fwd_err(Xres, Xo),
                      "fp64_oracle": "cuSOLVER potrf + potrs in FP64 (torch.linalg) on the same A, B"}
    del Xo
    if mixed:
        line["result"]["ir"] = {k: last.get(k) for k in ("iterations", "used_pcg", "pcg_iterations",
                                                         "refactored_tiles", "factor_ms", "solve_ms",
                                                         "backward_error")}

    # roofline of the dominant kernel (the trailing update), timed live
    if prof["update_ms"] > 0:
        per_flops = prof["update_flops"] / prof["update_launches"]
        per_ms = prof["update_ms"] / prof["update_launches"]
        ach = per_flops / (per_ms * 1e-3) / 1e12
        if w["factor"] == "FP64":
            peak, src, kern = peaks["fp64"], "cuBLAS dgemm 8192^3 measured in this run", "k_syrk_lower_f64 (DMMA)"
        else:
            # the library runs the update on CTA pairs unless LNB_TC_PAIR=0
            pair = os.environ.get("LNB_TC_PAIR", "1") != "0"
            name = "k_tc2_syrk_lower" if pair else "k_tc_syrk_lower"
            how = "(tcgen05, CTA pairs)" if pair else "(tcgen05)"
            if w["factor"] == "TF32X3":
                peak, src = peaks["tf32"] / 3.0, "cuBLAS TF32 GEMM 8192^3 measured in this run, / 3 products"
                kern = f"{name}<TF32X3> {how}"
            elif w["factor"] == "BF16":
                peak, src, kern = peaks["bf16"], "MEASURED_PEAKS.json bf16_tflops", f"{name}<BF16> {how}"
            else:
                peak, src, kern = peaks["tf32"], "cuBLAS TF32 GEMM measured in this run", f"{name}<TF32> {how}"
        line["roofline"] = {"bound": "tensor", "achieved": round(ach, 3), "peak": round(peak, 3),
                            "unit": "TFLOP/s", "frac": round(ach / peak, 4),
                            "traffic": traffic_from_profiles(kern.split()[0],
                                                             prof["update_bytes"] / prof["update_launches"]),
                            "traffic_note": "DRAM bytes per launch scaled from one ncu capture (profiles/)",
                            "kernel": kern, "peak_source": src,
                            "update_share_of_step": round(prof["update_ms"] / total_ms, 4),
                            "flops_note": "algorithmic flops per launch: 2 k per updated lower-triangle element"}

    # plain FP64 on the same matrix, same run: the comparison the metric names
    if mixed and not args.no_plain:
        Ap = torch.empty_like(A0)
        Bp = torch.empty_like(B0)
        infop = torch.zeros(1, dtype=torch.int32, device=dev)
        tp = []
        for i in range(2 + max(1, min(args.steps, 3))):
            Ap.copy_(A0)
            Bp.copy_(B0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            lnb.dposv_dev(Ap, Bp, n, nrhs, b, info=infop, stream=s)
            e1.record(s)
            torch.cuda.synchronize()
            if i >= 2:
                tp.append(e0.elapsed_time(e1))
        plain_ms = allmax(world, statistics.mean(tp))
        bwp = backward_error_dev(A0, Bp, B0)
        # forward error of the mixed solution against the plain FP64 one
        fwd = ((X - Bp).abs().max() / Bp.abs().max()).item()
        line["fp64_plain"] = {"ms_per_step": round(plain_ms, 3), "value": round(world * fl / plain_ms / 1e9, 4),
                              "backward_error": bwp, "speedup_mixed_vs_plain": round(plain_ms / ms_step, 3),
                              "forward_error_mixed_vs_plain": fwd}
        del Ap, Bp
        torch.cuda.empty_cache()

    # e2e through the host entry point, pinned host buffers, copies inside
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else max(1, min(args.steps, 3))
    if e2e_steps > 0:
        Ah = A0.cpu().pin_memory()
        Bh = B0.cpu().pin_memory()
        nblk = (n + b - 1) // b
        lower_elems = sum((n - j * b) * min(b, n - j * b) for j in range(nblk))
        e2e_t = []
        if mixed:
            Xh = torch.zeros_like(Bh).pin_memory()
            res = lnb.IrResult()
            lower512 = sum((n - c0) * min(512, n - c0) for c0 in range(0, n, 512))
            for i in range(e2e_steps + 1):
                barrier(world)
                t0 = time.perf_counter()
                rc = L.lnb_dsposv_ir(C.c_int(n), C.c_int(nrhs), C.c_int(b), C.c_void_p(Ah.data_ptr()), C.c_int(n),
                                     C.c_void_p(Bh.data_ptr()), C.c_int(n), C.c_void_p(Xh.data_ptr()), C.c_int(n),
                                     C.byref(opts), C.byref(res))
                t1 = time.perf_counter()
                assert rc == 0, lnb.last_error()
                if i > 0:
                    e2e_t.append(t1 - t0)
            bw_e2e = backward_error_dev(A0, Xh.to(dev), B0)
            h2d, d2h = 8 * (lower512 + n * nrhs), 8 * n * nrhs
            api = "lnb_dsposv_ir (host pointers, pinned), wall clock"
        else:
            Ahw = torch.empty_like(Ah).pin_memory()
            Bhw = torch.empty_like(Bh).pin_memory()
            for i in range(e2e_steps + 1):
                Ahw.copy_(Ah)
                Bhw.copy_(Bh)
                barrier(world)
                t0 = time.perf_counter()
                rc = lnb.dspdsolv_main(n, nrhs, b, Ahw.numpy().T, Bhw.numpy().T)
                t1 = time.perf_counter()
                assert rc == 0
                if i > 0:
                    e2e_t.append(t1 - t0)
            bw_e2e = backward_error_dev(A0, Bhw.to(dev), B0)
            h2d, d2h = 8 * (lower_elems + n * nrhs), 8 * (lower_elems + n * nrhs)
            api = "dspdsolv_main (host pointers, pinned), wall clock"
        assert bw_e2e <= 10 * n * eps, bw_e2e
        e2e_sec = allmax(world, statistics.mean(e2e_t))
        line["e2e"] = {"value": round(world * fl / e2e_sec / 1e12, 4), "unit": UNIT, "h2d_bytes_per_step": h2d,
                       "d2h_bytes_per_step": d2h, "ms_per_step": round(e2e_sec * 1e3, 3), "api": api}
    line["clocks"] = clk.summary()
    if not args.no_batched:
        line["batched"] = batched_arm(args, world, rank, local, peaks)
    if args.workload == "mixed" and not args.no_configs:
        del A0, B0, X
        torch.cuda.empty_cache()
        line["configs"] = config_records(args, world, rank, dev, peaks)
        line["blas"] = blas_records(args, world, rank, dev, peaks)

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ns = min(n, 8192)
        bs = min(b, 512)
        Asample = make_spd(ns, w["delta"], 0, dev, w["scaled"]).cpu().numpy()
        v, kind, cores, sec = cpu_run(ns, bs, nrhs, 2, 1, Asample)
        line["cpu_baseline"] = {"value": round(v, 6), "unit": UNIT, "cores": cores, "kind": kind,
                                "sample": f"dspdsolv_main n={ns} b={bs} nrhs={nrhs} (reference build, "
                                          f"OpenBLAS {cores} threads), median of 2 after 1 warm-up, "
                                          f"{sec:.2f} s each"}
    if rank == 0:
        print(json.dumps(line), flush=True)


def case_symv8(n):
    """k_symv_tc: Y = A X from the lower triangle, n x n FP64 (2 GB at n = 16384), 8 columns, 3 calls"""
    import torch
    import linompss_b200 as lnb
    A = torch.randn(n, n, dtype=torch.float64, device="cuda")
    X = torch.randn(8, n, dtype=torch.float64, device="cuda")
    Y = torch.empty_like(X)
    for _ in range(3):
        lnb.dsymv_dev(A, X, Y, n, 8)


def case_syrk(n):
    """k_gemm_dmma: C = A^T A + C on the lower triangle, n = k (FP64), 2 calls"""
    import torch
    import linompss_b200 as lnb
    A = torch.randn(n, n, dtype=torch.float64, device="cuda")
    C = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        lnb.dsyrk_dev("L", "T", n, n, 1.0, A, 1.0, C)


def case_dag(n):
    """k_chol_dag_f64: the FP64 factorization on the device DAG walk, b = 512, 2 calls"""
    import linompss_b200 as lnb
    A0 = make_spd(n, 1e-2, 3, "cuda")
    lnb.set_chol_schedule(lnb.SCHED_DAG)
    for _ in range(2):
        A = A0.clone()
        lnb.dchol_dev(A, n, 512)


def case_bf16(n):
    """configuration 4's solver at order n: BF16 factor, 8 right-hand sides, delta 1e-4 (PCG: k_trsm_blk with 8
    columns, k_symv_tc), one call"""
    import torch
    import linompss_b200 as lnb
    A = make_spd(n, 1e-4, 7, "cuda", scaled=True)
    B = torch.randn(8, n, dtype=torch.float64, device="cuda")
    X = torch.zeros_like(B)
    rc, res = lnb.dsposv_ir_dev(A, B, X, n, 8, 1024, lnb.ir_opts(factor=lnb.FACTOR_BF16, max_iter=40,
                                                                 pcg_max_iter=400))
    assert rc == 0, (rc, res)


def case_lu(n):
    """the LU with partial pivoting on device memory (lnb_dgetrf_dev), n x n N(0,1), 2 calls"""
    import torch
    import linompss_b200 as lnb
    A0 = torch.randn(n, n, dtype=torch.float64, device="cuda")
    A = torch.empty_like(A0)
    piv = torch.zeros(n, dtype=torch.int32, device="cuda")
    for _ in range(2):
        A.copy_(A0)
        lnb.dgetrf_dev(A, n, n, piv)


def case_batched(count):
    """the batched solver (configuration 5's distribution, `count` systems), autotuned, then 2 calls"""
    import torch
    import linompss_b200 as lnb
    ns, rs = batch_shape(count, 4321)
    ns, rs, a_off, b_off, nd, rd, ao, bo, dA, dB = make_batch(ns, rs, 4321, torch.device("cuda", 0))
    dX = torch.zeros_like(dB)
    lnb.batched_autotune(nd, rd, ao, bo, dA, dB, dX, lnb.FACTOR_FP32, 10)
    for _ in range(2):
        lnb.batched_posv_dev(nd, rd, ao, bo, dA, dB, dX, lnb.FACTOR_FP32, 10)


CASES = {"symv8": (case_symv8, 16384), "syrk": (case_syrk, 8192), "dag": (case_dag, 4096),
         "bf16": (case_bf16, 16384), "lu": (case_lu, 1500), "batched": (case_batched, 2000)}


def main():
    args = parse()
    if args.case:
        import torch
        fn, n = CASES[args.case]
        fn(args.n or n)
        torch.cuda.synchronize()
        print(json.dumps({"case": args.case, "n": args.n or n, "ok": True}))
        return
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
