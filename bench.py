#!/usr/bin/env python
"""rskelf factor+solve throughput (DOF/s) on B200 to 1e-10: the chosen form and plain FP64.

Workload (one "step"): build the tree, factor, and solve 256 right-hand sides
for N = 262144 points on the star curve r(t) = 1 + 0.3 cos 5t with t drawn
from Beta(1/2, 1/2) (clustered, uneven boxes), second-kind log-kernel matrix
A = I + K diag(w) with arc-length weights, occ 64, tol 1e-10, symm 'n',
64-point two-sided ring proxy.  Synthetic, seeded; each rank factors its own
instance (seed = rank), so per-GPU work is fixed as the GPU count grows.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl flam|reference]

value       DOF/s of the chosen form (flam_b200/chosen.py picks it per problem: here
            FP64 row sketches on the FP64 tensor path with learned widths, the
            factorization at 1e-10 and one rskelf_sv) with the inputs resident in HBM
            (CUDA events on the launch stream, max over ranks).
plain_fp64  the same workload with the reference's exact ID (plain FP64), timed the
            same way; vs_baseline = value / plain_fp64.value.
e2e         the chosen form through the public API with pinned host buffers, the
            host<->device copies inside the timed region.
accuracy    the FP64 relative residual of all 256 solutions, from the library's
            on-the-fly FP64 matvec (not timed).
value_excluding_tree  `value` with the tree construction's device time taken out.
chosen_form_other_problems (rank 0)  the same comparison on the 3D sphere of the
            mixed-precision configuration at N = 16384 (plain FP64 against both forms:
            the TF32 tensor-core sketch at 1e-6 refined in FP64 to 1e-10, and the FP64
            sketch at 1e-10), and the chosen form alone at that configuration's full size
            (N = 131072, 64 RHS), each with its FP64 error.
--impl reference  times the CPU restatement of the reference algorithm (the
            reference is MATLAB and does not run here) on a bounded sample.
"""
import argparse
import json
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
SPHERE_NRHS = 64
CONFIG2_N = 131072


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="flam", choices=["flam", "reference"])
    ap.add_argument("--n", type=int, default=N_DEF)
    ap.add_argument("--nrhs", type=int, default=NRHS_DEF)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-chosen", action="store_true", help="skip the chosen-form comparison")
    ap.add_argument("--sphere-n", type=int, default=16384, help="points of the 3D sphere comparison")
    ap.add_argument("--no-config2", action="store_true", help="skip the full-size config-2 run of the chosen form")
    return ap.parse_args()


def config(args, world, n=None):
    n = args.n if n is None else n
    return {"workload": f"rskelf star curve N={n} Beta(1/2,1/2)-clustered, occ {OCC}, tol {TOL:g}, "
                        f"{args.nrhs} RHS, symm n, factor+solve per step",
            "N_per_gpu": n, "nrhs": args.nrhs, "occ": OCC, "tol": TOL, "symm": "n",
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


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


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
           "config": config(args, 1, CPU_SAMPLE_N),
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "cpu": cpu_model(),
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


def relres(F, X, B):
    """max over columns of ||B - A X|| / ||B||, FP64, with the library's on-the-fly matvec."""
    import torch
    R = torch.empty_like(B)
    F.matvec_(X, R, B)
    return float((R.norm(dim=0) / B.norm(dim=0)).max().item())


def event_time(torch, stream, fn):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) * 1e-3, out


# --------------------------------------------------------------------- chosen form
def chosen_vs_plain(torch, fb, chosen, stream, name, Ad, xd, pxy, symm, Bd, plain_reps, chosen_reps, predictor, flush,
                    forms=None):
    """One problem: plain FP64 at TOL (factor + rskelf_sv) against the chosen form (and any
    other forms listed), each timed on the device from the inputs in HBM, with its FP64
    residual."""
    N, nrhs = Bd.shape
    d = xd.shape[0]
    Xd = torch.empty_like(Bd)

    def plain():
        F = fb.rskelf(Ad, xd, OCC, TOL, pxy, dict(symm=symm, stream=stream.cuda_stream))
        Xd.copy_(Bd)
        F.sv_(Xd)
        return F

    res = {"problem": name}
    if plain_reps >= 0:
        tp = []
        for rep in range(plain_reps + 1):          # one untimed warm-up
            flush.fill_(float(rep))
            t, F = event_time(torch, stream, plain)
            if rep > 0 or plain_reps == 0:
                tp.append(t)
            if rep < plain_reps:
                F.free()
        res["plain"] = {"dofs": N / statistics.mean(tp), "ms": 1e3 * statistics.mean(tp), "steps": len(tp),
                        "tol": TOL, "rel_residual_fp64": relres(F, Xd, Bd), "nfactor": F.info()["nfactor"]}
        F.free()
    pick = chosen.choose(d, N, nrhs, TOL, symm)
    for form in forms or [pick]:
        tc = []
        for rep in range(chosen_reps + 1):
            flush.fill_(float(rep))
            t, (F, _, it, rel) = event_time(torch, stream, lambda: chosen.solve(
                Ad, xd, OCC, pxy, Bd, Xd, TOL, symm, predictor, form, stream.cuda_stream, True))
            if rep > 0 or chosen_reps == 0:
                tc.append(t)
            if rep < chosen_reps:
                F.free()
        prof = F.profile()
        key = "chosen" if form == pick else form
        res[key] = {"form": form, "dofs": N / statistics.mean(tc), "ms": 1e3 * statistics.mean(tc), "steps": len(tc),
                    "factor_tol": chosen.factor_tol(form, TOL), "refinement_steps": it,
                    "rel_residual_fp64": relres(F, Xd, Bd),
                    "rel_residual_reported": None if rel is None else float(np.max(rel)),
                    "sketched_boxes": prof["n_sketch"], "exact_redo_boxes": prof["n_sketch_redo"],
                    "sketch_rows": prof["sketch_rows"], "rows_of_K": prof["sketch_rows_k"],
                    "learned_widths": predictor is not None, "nfactor": F.info()["nfactor"]}
        F.free()
    if "plain" in res:
        res["ratio_chosen_over_plain"] = res["chosen"]["dofs"] / res["plain"]["dofs"]
    return res


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
    from flam_b200 import chosen, problems

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
    pred = chosen.load_predictor()
    form = chosen.choose(2, N, nrhs, TOL, "n")

    def plain_dev():
        F = fb.rskelf(Ad, xd, OCC, TOL, pxy, dict(symm="n", stream=stream.cuda_stream, profile=True))
        Xd.copy_(Bd)
        F.sv_(Xd)
        return F

    def chosen_dev():
        return chosen.solve(Ad, xd, OCC, pxy, Bd, Xd, TOL, "n", pred, form, stream.cuda_stream, True)[0]

    def timed(step):
        for _ in range(args.warmup):
            step().free()
        ts, F = [], None
        for _ in range(args.steps):
            flush.fill_(float(len(ts)))
            if F is not None:
                F.free()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            F = step()
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) * 1e-3)
        barrier()
        return max_over_ranks(statistics.mean(ts)), F

    peak_fp64 = dgemm_peak(torch, dev)
    clk_path = os.path.join(ROOT, f".clocks_rank{rank}.csv")
    clk = start_clocks(clk_path)
    t_plain, Fp = timed(plain_dev)
    resid_plain = relres(Fp, Xd, Bd)     # accuracy against FP64, every column (not timed)
    prof_plain = Fp.profile()
    Fp.free()
    t_step, F = timed(chosen_dev)
    if clk:
        clk.terminate()
        clk.wait()
    clocks = read_clocks(clk_path, local)
    try:
        os.remove(clk_path)
    except OSError:
        pass
    prof = F.profile()
    info = F.info()
    resid = relres(F, Xd, Bd)
    F.free()

    # ---- end to end through the public API with pinned host buffers
    xp = torch.from_numpy(np.ascontiguousarray(x.T)).pin_memory()
    wp = torch.from_numpy(A.weights.copy()).pin_memory()
    Bp = B_host.t().contiguous().t().pin_memory()          # column-major, pinned
    Wp = torch.empty_like(Bp).pin_memory()
    xnp = xp.numpy().T                                      # d x N view, Fortran order
    Ah = fb.Kernel("laplace2d", scale=A.scale, dval=A.dval, weights=wp.numpy())
    Wnp = Wp.numpy()

    def e2e(opts, tol):
        def step():
            F = fb.rskelf(Ah, xnp, OCC, tol, pxy, opts)
            F.sv_(Wnp)
            return F
        for _ in range(max(1, args.warmup // 2)):
            Wp.copy_(Bp)
            step().free()
        et = []
        for _ in range(args.steps):
            Wp.copy_(Bp)
            flush.fill_(1.0)
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            Fe = step()
            e1.record(stream)
            e1.synchronize()
            et.append(e0.elapsed_time(e1) * 1e-3)
            Fe.free()
        return max_over_ranks(statistics.mean(et))

    t_e2e = e2e(chosen.factor_opts(form, "n", pred, stream.cuda_stream), chosen.factor_tol(form, TOL))
    t_e2e_plain = e2e(dict(symm="n", stream=stream.cuda_stream), TOL)

    # ---- roofline of the chosen form's dominant kernel family (FP64: the FP64 tensor path)
    fam = {"sketch": (prof["t_sketch"], prof["flop_sketch"]),
           "id": (prof["t_compress"] - prof["t_sketch"], prof["flop_id"]),
           "elim": (prof["t_elim"], prof["flop_elim"]),
           "sweep": (prof["t_sweep"], prof["flop_sweep"])}
    launches = {"sketch": None, "id": prof["n_compress"], "elim": prof["n_elim"], "sweep": prof["n_sweep"]}
    top = max(fam, key=lambda k: fam[k][0])
    t_k, f_k = fam[top]
    achieved = f_k / t_k / 1e12 if t_k > 0 else 0.0
    kernel_name = {"sketch": "k_sketch_f64 (FP64 row sketch, DMMA)",
                   "id": "k_compress_tc / k_cpqr_wide (pivoted QR + R11\\R12 of the sketches, exact ID elsewhere)",
                   "elim": "k_eliminate / k_eliminate_big (LU + Schur updates, DMMA tile)",
                   "sweep": "k_sweep (solve sweeps)"}[top]
    roofline = {"kernel": kernel_name, "bound": "fp64", "achieved": achieved, "peak": peak_fp64,
                "unit": "TFLOP/s", "frac": achieved / peak_fp64 if peak_fp64 else None, "traffic": None,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 figure)",
                "flop_basis": "executed FP64 work: sketch products 2 w rows(K) n; ID on the rows it folds; "
                              "elimination and sweeps as the reference's dense operations",
                "step_groups": launches[top], "kernel_share_of_step": t_k / t_step,
                "by_family_ms": {k: v[0] * 1e3 for k, v in fam.items()},
                "by_family_tflops": {k: (v[1] / v[0] / 1e12 if v[0] > 0 else 0) for k, v in fam.items()},
                "plain_fp64_by_family_ms": {"compress": prof_plain["t_compress"] * 1e3,
                                            "elim": prof_plain["t_elim"] * 1e3, "sweep": prof_plain["t_sweep"] * 1e3}}

    out = None
    if rank == 0:
        value = N * world / t_step
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            ts = [cpu_sample(CPU_SAMPLE_N, nrhs, seed=s)[0] for s in range(2)]
            tc = statistics.mean(ts)
            cpu = {"value": CPU_SAMPLE_N / tc, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                   "cpu": cpu_model(),
                   "sample": f"N={CPU_SAMPLE_N} instance of the same workload, oracle (NumPy/SciPy restatement of "
                             f"the reference, reference box order, plain FP64), {nrhs} RHS, mean of 2 runs"}
        others = None
        if not args.no_chosen:
            Ns = args.sphere_n
            xs, As, ps = problems.sphere(Ns, p=256, seed=0)
            xsd = torch.from_numpy(np.ascontiguousarray(xs.T)).to(dev).t()
            Bs = torch.randn(Ns, SPHERE_NRHS, dtype=torch.float64, generator=gen).to(dev).t().contiguous().t()
            # plain FP64 takes about a minute here: one timed run, no warm-up
            others = {"sphere": chosen_vs_plain(torch, fb, chosen, stream, f"3D sphere N={Ns}, p=256, "
                                                f"{SPHERE_NRHS} RHS (config 2 geometry)", As, xsd, ps, "n", Bs, 0, 2,
                                                pred, flush, forms=["tf32-refine", "fp64-sketch"])}
            if not args.no_config2:
                # config 2 at full size: the chosen form alone (plain FP64's exact IDs of its
                # top boxes run for hours on this implementation)
                N2 = CONFIG2_N
                x2, A2, p2 = problems.sphere(N2, p=256, seed=0)
                x2d = torch.from_numpy(np.ascontiguousarray(x2.T)).to(dev).t()
                B2 = torch.randn(N2, SPHERE_NRHS, dtype=torch.float64, generator=gen).to(dev).t().contiguous().t()
                others["config2"] = chosen_vs_plain(torch, fb, chosen, stream, f"config 2: 3D sphere N={N2}, p=256, "
                                                    f"{SPHERE_NRHS} RHS", A2, x2d, p2, "n", B2, -1, 1, pred, flush)
        h2d = N * 2 * 8 + N * 8 + N * nrhs * 8
        d2h = N * nrhs * 8
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": (N * world / t_step) / (N * world / t_plain),
               "vs_baseline_note": "chosen form over plain FP64 on the same workload, both measured in this run "
                                   "(BASELINE.md publishes no number for this metric)",
               "dtype": "f64", "data": "synthetic (seeded star curve, Beta-clustered)",
               "config": config(args, world),
               "form": {"chosen": form, "factor_tol": chosen.factor_tol(form, TOL),
                        "note": "FP64 row sketches on the FP64 tensor path with learned widths (rank predictor), "
                                "FP64 pivoted QR / rank / R11\\R12 on the sketches, factorization at 1e-10, one "
                                "rskelf_sv; rule in flam_b200/chosen.py"},
               "plain_fp64": {"value": N * world / t_plain, "ms_per_step": t_plain * 1e3,
                              "rel_residual_fp64": resid_plain,
                              "e2e": {"value": N * world / t_e2e_plain, "ms_per_step": t_e2e_plain * 1e3}},
               "e2e": {"value": N * world / t_e2e, "unit": UNIT, "h2d_bytes_per_step": h2d,
                       "d2h_bytes_per_step": d2h, "ms_per_step": t_e2e * 1e3},
               "gpu_launches": int(prof["launches"]),
               "roofline": roofline,
               "cpu_baseline": cpu,
               "clocks": clocks,
               "accuracy": {"rel_residual_fp64": resid,
                            "note": f"max over the {nrhs} RHS of ||B - A X|| / ||B||, every row, FP64 on-the-fly "
                                    f"matvec (flam_matvec)"},
               "chosen_form_other_problems": others,
               "breakdown_ms": {"tree": info["t_tree"] * 1e3, "factor": info["t_factor"] * 1e3},
               "value_excluding_tree": N * world / max(t_step - info["t_tree"], 1e-9),
               "factor": {"nbox": info["nbox"], "nfactor": info["nfactor"], "levels": info["nstep"],
                          "device_bytes": info["bytes"], "sketched_boxes": prof["n_sketch"],
                          "exact_redo_boxes": prof["n_sketch_redo"]},
               "peaks": {k: measured_peaks().get(k) for k in ("hbm_gbs", "bf16_tflops")}}
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
