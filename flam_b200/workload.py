"""One factor + solve of the star-curve workload, for profilers.

    python -m flam_b200.workload [--n 65536] [--nrhs 16] [--reps 1] [--symm n]

Runs ``reps`` factorizations and solves of the Beta-clustered star curve
(the benchmark's geometry and matrix at a chosen size) on cuda:0 with no
warm-up and nothing else launched, so a kernel profiler sees only the
factorization's and the sweeps' kernels.
"""
import argparse

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=65536)
    ap.add_argument("--nrhs", type=int, default=16)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--symm", default="n")
    ap.add_argument("--tol", type=float, default=1e-10)
    args = ap.parse_args()
    import torch

    import flam_b200 as fb
    from flam_b200 import problems

    x, A, pxy = problems.star(args.n, seed=0)
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda().t()
    Ad = fb.Kernel(A.kind, scale=A.scale, dval=A.dval, weights=torch.from_numpy(A.weights).cuda())
    B = torch.randn(args.n, args.nrhs, dtype=torch.float64, device="cuda").t().contiguous().t()
    for _ in range(args.reps):
        F = fb.rskelf(Ad, xd, 64, args.tol, pxy, dict(symm=args.symm))
        X = B.clone()
        F.sv_(X)
        torch.cuda.synchronize()
        F.free()
    print("ok", args.n, args.nrhs, args.reps)


if __name__ == "__main__":
    main()
