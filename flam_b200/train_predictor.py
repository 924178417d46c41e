"""Train the rank predictor on ranks logged by the exact ID and save its weights.

    python -m flam_b200.train_predictor [--geometries 200] [--out flam_b200/predictor_weights.npz]

Training data: every compressed box of 200 seeded random geometries, factored on the
GPU by the exact (reference) ID with ``rank_log``: the box's 16 features and its rank
as a fraction of its point count.  The geometries cycle through the survey's problem
families at sizes whose factorizations take a fraction of a second -- Matern-3/2 GP
covariance on uniform points in the unit cube (the learned-rank configuration), the
3D Laplace second-kind operator on a randomly rotated Fibonacci sphere, and the 2D
log kernel on seeded star curves -- each at a tolerance drawn from {1e-5, 1e-6, 1e-8, 1e-10}.
The network is trained on the GPU by the library's own kernels (flam_predictor_train)
and checked on 10% of the geometries held out.
"""
import argparse
import math
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "predictor_weights.npz")


def geometry(i):
    """Problem i of the training set: (x, A, pxy, symm, tol)."""
    from . import problems
    rng = np.random.default_rng(1000 + i)
    tol = float(rng.choice([1e-5, 1e-6, 1e-8, 1e-10]))
    fam = i % 3
    if fam == 0:
        N = int(rng.integers(2000, 6000))
        x, A, pxy = problems.matern_cube(N, seed=10_000 + i, p=64, p_rad=6)
        return x, A, pxy, "p", tol
    if fam == 1:
        N = int(rng.integers(2000, 6000))
        x, A, pxy = problems.sphere(N, p=256, seed=10_000 + i)
        return x, A, pxy, "n", tol
    N = int(rng.integers(4000, 16000))
    theta = 2 * math.pi * np.sort(rng.beta(0.5, 0.5, size=N))
    x, w = problems.star_points(N, float(rng.uniform(0.1, 0.4)), int(rng.integers(3, 10)), theta)
    from .registry import Kernel, Proxy
    return x, Kernel("laplace2d", scale=1.0, dval=1.0, weights=w), Proxy("ring", 64, "laplace2d", two_sided=True), \
        "n", tol


def collect(indices):
    import flam_b200 as fb
    Xs, ys = [], []
    for i in indices:
        x, A, pxy, symm, tol = geometry(i)
        F = fb.rskelf(A, x, 64, tol, pxy, dict(symm=symm, rank_log=1))
        X, y = F.rank_log()
        F.free()
        Xs.append(X)
        ys.append(y)
    return np.concatenate(Xs), np.concatenate(ys)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--geometries", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--out", default=DEFAULT_OUT)
    args = ap.parse_args()
    import flam_b200 as fb
    t0 = time.time()
    n = args.geometries
    held = set(range(0, n, 10))
    X, y = collect([i for i in range(n) if i not in held])
    Xh, yh = collect(sorted(held))
    t1 = time.time()
    P = fb.Predictor(seed=0)
    base = float(np.mean((P.predict(Xh) - yh) ** 2))
    loss = P.train(X, y, epochs=args.epochs, batch=256, lr=2e-3)
    t2 = time.time()
    held_mse = float(np.mean((P.predict(Xh) - yh) ** 2))
    P.save(args.out)
    print(f"samples {len(y)} (held out {len(yh)}) from {n} geometries in {t1 - t0:.1f} s; "
          f"trained {args.epochs} epochs in {t2 - t1:.1f} s: train mse {loss:.2e}, held-out mse {held_mse:.2e} "
          f"(untrained {base:.2e}); weights -> {args.out}")


if __name__ == "__main__":
    main()
