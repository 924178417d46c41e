#!/usr/bin/env python
"""rskelf factor + solve throughput (DOF/s) on B200.

Workload (one "step"): build the tree, factor, and solve 256 right-hand sides
for N = 262144 points on the star curve r(t) = 1 + 0.3 cos 5t with t drawn
from Beta(1/2, 1/2) (clustered, uneven boxes), second-kind log-kernel matrix
A = I + K diag(w) with arc-length weights, occ 64, tol 1e-10, symm 'n',
64-point two-sided ring proxy.  Synthetic, seeded; each rank factors its own
instance (seed = rank), so per-GPU work is fixed as the GPU count grows.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl flam|reference]

``value``: DOF/s with the inputs resident in HBM (CUDA events on the launch
stream, max over ranks).  ``e2e``: the same through the public API with host
buffers (pinned), host<->device copies inside the timed region.
``--impl reference`` times the CPU restatement of the reference algorithm
(the reference itself is MATLAB and does not run here) on a bounded sample.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "rskelf factor+solve DOF/s at 1e-10 rel. err: chosen form vs plain FP64, 1 B200"
UNIT = "DOF/s"
N_DEF, NRHS_DEF, OCC, TOL = 262144, 256, 64, 1e-10
CPU_SAMPLE_N = 16384
# DRAM bytes (read + write) per compress step of the N=262144 workload: one ncu capture
# of every k_compress_tc launch of an N=65536 factorization (156.4 MB over its level
# steps; profiles/k_compress_tc_star65536_top.md) scaled by the box count (x4) and
# divided by this workload's 23 steps.
COMPRESS_TRAFFIC_PER_STEP = 4 * 156.4e6 / 23


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="flam", choices=["flam", "reference"])
    ap.add_argument("--n", type=int, default=N_DEF)
    ap.add_argument("--nrhs", type=int, default=NRHS_DEF)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def config(args, world):
    return {"workload": f"rskelf star curve N={args.n} Beta(1/2,1/2)-clustered, occ {OCC}, tol {TOL:g}, "
                        f"{args.nrhs} RHS, symm n, factor+solve per step",
            "N_per_gpu": args.n, "nrhs": args.nrhs, "occ": OCC, "tol": TOL, "symm": "n",
            "parallelism": f"instances x{world} (one independent problem per rank)",
            "l2": "flushed between timed steps (256 MiB write); B (N x 256 FP64) is larger than L2"}


# --------------------------------------------------------------------- CPU (oracle) timing
def cpu_sample(n, nrhs, seed=0):
    """Oracle factor + solve on a bounded sample of the workload; returns (seconds, N)."""
    from oracle import configs
    from oracle.rskelf import rskelf, rskelf_sv
    x, A, pxy = configs.star(n, seed=seed)
    B = np.random.default_rng(seed).standard_normal((n, nrhs))
    t0 = time.perf_counter()
    F = rskelf(A, x, OCC, TOL, pxy, dict(symm="n"), order="reference")
    rskelf_sv(F, B)
    return time.perf_counter() - t0, n


def run_reference(args, rank, world):
    if rank != 0:
        return
    for _ in range(max(args.warmup, 0)):
        cpu_sample(4096, args.nrhs)
    ts = [cpu_sample(CPU_SAMPLE_N, args.nrhs, seed=s)[0] for s in range(args.steps)]
    t = statistics.mean(ts)
    v = CPU_SAMPLE_N / t
    cores = os.cpu_count()
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
           "config": config(args, 1),
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                            "sample": f"N={CPU_SAMPLE_N} instance of the same workload (NumPy/SciPy restatement of "
                                      f"the MATLAB reference, reference box order, {args.nrhs} RHS)"},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# --------------------------------------------------------------------- helpers
def start_clocks(path):
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    try:
        return subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "100"],
                                stdout=open(path, "w"), stderr=subprocess.DEVNULL)
    except Exception:
        return None


def read_clocks(path, dev):
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    try:
        for line in open(path):
            f = [v.strip() for v in line.split(",")]
            if len(f) < 9 or f[0] != str(dev):
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
    except OSError:
        pass
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
            "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def dgemm_peak(torch, dev):
    """FP64 dense peak of this GPU measured with cuBLAS DGEMM (8192^3, best of 5)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2 * n ** 3 / (e0.elapsed_time(e1) * 1e-3))
    del a, b
    return best / 1e12


def sampled_residual(x, w, X, B, rows):
    """max over columns of ||A X - B|| / ||B|| on sampled rows, FP64 on the host."""
    xs = x[:, rows]
    d = xs[:, :, None] - x[:, None, :]
    r2 = np.sum(d * d, axis=0)
    with np.errstate(divide="ignore"):
        K = -np.log(r2) / (4 * math.pi) * w[None, :]
    K[np.arange(len(rows)), rows] = 1.0
    R = K @ X - B[rows]
    return float(np.max(np.linalg.norm(R, axis=0) / np.linalg.norm(B[rows], axis=0)))


# --------------------------------------------------------------------- main
def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch
    import torch.distributed as dist
    import flam_b200 as fb
    from flam_b200 import problems

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    N, nrhs = args.n, args.nrhs
    x, A, pxy = problems.star(N, seed=rank)
    gen = torch.Generator(device="cpu").manual_seed(1234 + rank)
    B_host = torch.randn(N, nrhs, dtype=torch.float64, generator=gen)
    stream = torch.cuda.current_stream()
    # device-resident inputs
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).to(dev).t()
    Ad = fb.Kernel("laplace2d", scale=A.scale, dval=A.dval, weights=torch.from_numpy(A.weights).to(dev))
    Bd = B_host.to(dev).t().contiguous().t()
    Xd = torch.empty_like(Bd)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    opts = dict(symm="n", stream=stream.cuda_stream, profile=True)

    def step_dev():
        F = fb.rskelf(Ad, xd, OCC, TOL, pxy, opts)
        Xd.copy_(Bd)
        F.sv_(Xd)
        return F

    peak_fp64 = dgemm_peak(torch, dev)
    for _ in range(args.warmup):
        step_dev().free()
    clk_path = os.path.join(ROOT, f".clocks_rank{rank}.csv")
    clk = start_clocks(clk_path)
    times, F = [], None
    for _ in range(args.steps):
        flush.fill_(float(len(times)))
        if F is not None:
            F.free()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        F = step_dev()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) * 1e-3)
    barrier()
    if clk:
        clk.terminate()
        clk.wait()
    clocks = read_clocks(clk_path, local)
    try:
        os.remove(clk_path)
    except OSError:
        pass
    t_step = max_over_ranks(statistics.mean(times))
    prof = F.profile()
    info = F.info()
    # accuracy against FP64 on sampled rows (not timed)
    rows = np.random.default_rng(7).choice(N, 64, replace=False)
    Xh = Xd.cpu().numpy()
    resid = sampled_residual(x, A.weights, Xh, B_host.numpy(), rows)
    F.free()

    # ---- end to end through the public API with pinned host buffers
    xp = torch.from_numpy(np.ascontiguousarray(x.T)).pin_memory()
    wp = torch.from_numpy(A.weights.copy()).pin_memory()
    Bp = B_host.t().contiguous().t().pin_memory()          # column-major, pinned
    Wp = torch.empty_like(Bp).pin_memory()
    xnp = xp.numpy().T                                      # d x N view, Fortran order
    Ah = fb.Kernel("laplace2d", scale=A.scale, dval=A.dval, weights=wp.numpy())
    opts_h = dict(symm="n", stream=stream.cuda_stream)
    Wnp = Wp.numpy()

    def step_e2e():
        F = fb.rskelf(Ah, xnp, OCC, TOL, pxy, opts_h)
        F.sv_(Wnp)
        return F

    for _ in range(max(1, args.warmup // 2)):
        Wp.copy_(Bp)
        step_e2e().free()
    et = []
    for _ in range(args.steps):
        Wp.copy_(Bp)
        flush.fill_(1.0)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        Fe = step_e2e()
        e1.record(stream)
        e1.synchronize()
        et.append(e0.elapsed_time(e1) * 1e-3)
        Fe.free()
    t_e2e = max_over_ranks(statistics.mean(et))

    # ---- roofline of the dominant kernel (FP64 compute bound)
    fam = {"compress": (prof["t_compress"], prof["flop_compress"], prof["n_compress"]),
           "elim": (prof["t_elim"], prof["flop_elim"], prof["n_elim"]),
           "sweep": (prof["t_sweep"], prof["flop_sweep"], prof["n_sweep"])}
    top = max(fam, key=lambda k: fam[k][0])
    t_k, f_k, n_k = fam[top]
    achieved = f_k / t_k / 1e12 if t_k > 0 else 0.0
    kernel_name = {"compress": "k_compress (fused proxy filter + assembly + TSQR + CPQR + RRQR)",
                   "elim": "k_eliminate", "sweep": "k_sweep"}[top]
    roofline = {"kernel": kernel_name, "bound": "fp64", "achieved": achieved, "peak": peak_fp64,
                "unit": "TFLOP/s", "frac": achieved / peak_fp64 if peak_fp64 else None,
                "traffic": COMPRESS_TRAFFIC_PER_STEP if top == "compress" and args.n == N_DEF else None,
                "traffic_unit": "bytes per step launch group (ncu capture at N=65536 scaled x4)",
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 figure)",
                "launches": n_k, "avg_launch_ms": t_k / max(n_k, 1) * 1e3,
                "algorithmic_flop_per_launch": f_k / max(n_k, 1),
                "kernel_share_of_step": t_k / t_step,
                "by_kernel_ms": {k: v[0] * 1e3 for k, v in fam.items()},
                "by_kernel_tflops": {k: (v[1] / v[0] / 1e12 if v[0] > 0 else 0) for k, v in fam.items()}}

    out = None
    if rank == 0:
        value = N * world / t_step
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            ts = [cpu_sample(CPU_SAMPLE_N, nrhs, seed=s)[0] for s in range(2)]
            tc = statistics.mean(ts)
            cpu = {"value": CPU_SAMPLE_N / tc, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                   "sample": f"N={CPU_SAMPLE_N} instance of the same workload, oracle (NumPy/SciPy restatement of "
                             f"the reference, reference box order), {nrhs} RHS, mean of 2 runs"}
        h2d = N * 2 * 8 + N * 8 + N * nrhs * 8
        d2h = N * nrhs * 8
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded star curve, Beta-clustered)",
               "config": config(args, world),
               "e2e": {"value": N * world / t_e2e, "unit": UNIT, "h2d_bytes_per_step": h2d,
                       "d2h_bytes_per_step": d2h, "ms_per_step": t_e2e * 1e3},
               "gpu_launches": int(prof["launches"]),
               "roofline": roofline,
               "cpu_baseline": cpu,
               "clocks": clocks,
               "accuracy": {"rel_residual_fp64_sampled_rows": resid, "rows": 64,
                            "note": "max over the 256 RHS of ||(A X - B)_rows|| / ||B_rows||, FP64 on the host"},
               "breakdown_ms": {"tree": info["t_tree"] * 1e3, "factor": info["t_factor"] * 1e3},
               "factor": {"nbox": info["nbox"], "nfactor": info["nfactor"], "levels": info["nstep"],
                          "device_bytes": info["bytes"]},
               "peaks": {k: measured_peaks().get(k) for k in ("hbm_gbs", "bf16_tflops")}}
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
