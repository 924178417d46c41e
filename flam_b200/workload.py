"""One factor + solve of a benchmark workload, for kernel profilers.

    python -m flam_b200.workload [--cfg star|sphere] [--n 65536] [--nrhs 16] [--reps 1]
                                 [--form plain|chosen] [--symm n] [--tol 1e-10]

Runs ``reps`` factorizations and solves on cuda:0 with no warm-up and nothing else
launched, so a kernel profiler sees only the library's kernels:

* ``--form plain``: the exact ID at ``--tol`` and rskelf_sv;
* ``--form chosen``: the form flam_b200/chosen.py picks for the problem at ``--tol``
  (with the trained rank predictor): the FP64-sketched factorization at ``--tol`` and
  one rskelf_sv, or the TF32-sketched factorization at 1e-6 refined in FP64 to
  ``--tol`` against the on-the-fly FP64 matvec;
* ``--form fp64-sketch`` / ``--form tf32-refine``: that form, whatever the rule picks.

``--cfg star`` is the Beta-clustered star curve of the benchmark (2D log kernel);
``--cfg sphere`` the Fibonacci sphere of the mixed-precision configuration (3D Laplace,
256-point proxy sphere).  This is the entry point the committed ncu summaries name.
"""
import argparse

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cfg", default="star", choices=["star", "sphere"])
    ap.add_argument("--n", type=int, default=65536)
    ap.add_argument("--nrhs", type=int, default=16)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--symm", default="n")
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--form", default="plain", choices=["plain", "chosen", "fp64-sketch", "tf32-refine"])
    args = ap.parse_args()
    import torch

    import flam_b200 as fb
    from flam_b200 import problems

    if args.cfg == "star":
        x, A, pxy = problems.star(args.n, seed=0)
    else:
        x, A, pxy = problems.sphere(args.n, p=256, seed=0)
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda().t()
    w = None if A.weights is None else torch.from_numpy(A.weights).cuda()
    Ad = fb.Kernel(A.kind, scale=A.scale, dval=A.dval, param=A.param, weights=w)
    B = torch.randn(args.n, args.nrhs, dtype=torch.float64, device="cuda").t().contiguous().t()
    pred = None
    if args.form != "plain":
        from flam_b200 import chosen
        pred = chosen.load_predictor()
    for _ in range(args.reps):
        if args.form == "plain":
            F = fb.rskelf(Ad, xd, 64, args.tol, pxy, dict(symm=args.symm))
            X = B.clone()
            F.sv_(X)
            extra = ""
        else:
            X = torch.empty_like(B)
            F, form, it, rel = chosen.solve(Ad, xd, 64, pxy, B, X, args.tol, args.symm, pred,
                                            None if args.form == "chosen" else args.form)
            extra = f" form {form} refinement steps {it}" + ("" if rel is None else f" relres {float(np.max(rel)):.2e}")
        torch.cuda.synchronize()
        F.free()
    print("ok", args.cfg, args.form, args.n, args.nrhs, args.reps, extra)


if __name__ == "__main__":
    main()
